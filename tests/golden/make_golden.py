"""Generate the golden fixtures in this directory from the reference solver's
own code (oracle/_ref/ref_f64 = the reference promoted to double, ref_f32 =
as shipped), run with one OpenMP thread so every reduction is sequential.

Run from the repository root where the reference sources are available:
    make -C oracle ref REF=<reference checkout> && python tests/golden/make_golden.py
The fixtures are committed; tests read them without the reference present.

`python tests/golden/make_golden.py NAME ...` writes only the named flow
fixtures; `python tests/golden/make_golden.py thermal` writes only the thermal_asm_*
fixtures: the CSR matrix and right-hand side that the reference's own
ThermalSolver3D::solve assembles (oracle/_ref/thermal_asm, the solver class
compiled with its AMGCL solve cut out) for seeded inputs, with those inputs.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from coldplate_solver_b200 import geometry as g  # noqa: E402
from oracle import reference  # noqa: E402

DESIGN_KEYS = ("M", "N", "hx", "hy", "inletVelocity", "convectionScheme", "enableTwoPointFiveD",
               "enableConvectionScaling", "Ht_channel", "twoPointFiveDSinkMultiplier", "uvAlpha", "pAlpha", "rho",
               "eta", "pTol", "maxPressureIter", "momentumTol", "maxMomentumIter")


def cases():
    yield "straight_11x13", g.straight_channel(M=11, N=13, band=(3, 8)), 40, None
    yield "network_30x48_sou25d", g.channel_network(M=30, N=48, h=20e-6, wmin=3, wmax=6, seed=3), 25, None
    yield "density_13x27_sou", g.density_field(Nx=27, seed=9, sigma=2.0, plenum=3, twoFiveD=False), 25, None
    d = g.density_field(Nx=40, seed=5, sigma=3.0, plenum=4)
    rng = np.random.default_rng(11)
    init = {"u": rng.normal(0, 0.05, (d.M + 1, d.N)), "v": rng.normal(0, 0.02, (d.M, d.N + 1)),
            "p": rng.normal(0, 10.0, (d.M + 1, d.N + 1))}
    yield "density_20x40_random_state", d, 3, init
    yield "minimal_3x3", g.straight_channel(M=3, N=3, band=(1, 2)), 5, None
    d = g.straight_channel(M=9, N=17, band=(2, 7)).replace(maxMomentumIter=3, maxPressureIter=2, pTol=1e-12,
                                                            momentumTol=1e-12)
    yield "capped_9x17", d, 6, None
    # a channel one cell wide
    yield "single_row_channel_9x21", g.straight_channel(M=9, N=21, band=(4, 5)), 30, None
    # the band blocked by a solid column except for a one-cell gap, SOU
    d = g.straight_channel(M=12, N=24, band=(3, 9))
    gm = d.gamma.copy()
    gm[3:8, 12] = 0.0
    a, gm = g.alpha_ramp_reference(gm)
    yield "gap_12x24_sou", d.replace(gamma=gm, alpha=a, convectionScheme=1), 25, None
    # odd sizes, SOU
    yield "odd_7x13_sou", g.straight_channel(M=7, N=13, band=(2, 5)).replace(convectionScheme=1), 20, None


def main(selected=()) -> None:
    for name, d, n, init in cases():
        if selected and name not in selected:
            continue
        rec = {k: np.asarray(getattr(d, k)) for k in DESIGN_KEYS}
        rec.update(gamma=d.gamma, alpha=d.alpha, n_outer=np.asarray(n))
        if init is not None:
            rec.update(u0=init["u"], v0=init["v"], p0=init["p"])
        for prec in ("f64", "f32"):
            out = reference.run(d, n, precision=prec, threads=1, init=init)
            for k in ("residU", "residV", "residMass", "residMassDof", "err", "pIters", "uSweeps", "vSweeps",
                      "u", "v", "p", "pStar", "uStar", "vStar", "dE", "dN", "planes"):
                rec[f"{prec}_{k}"] = out[k]
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **rec)
        print("wrote", name)
    if selected:
        return
    gm = np.random.default_rng(0).random((17, 23))
    rec = {"gamma_in": gm}
    for prec in ("f64", "f32"):
        a, gg = reference.build_alpha(gm, 1e-14, 1.0, precision=prec)
        rec[f"{prec}_alpha"], rec[f"{prec}_gamma"] = a, gg
    np.savez_compressed(os.path.join(HERE, "alpha_ramp_17x23.npz"), **rec)
    print("wrote alpha_ramp_17x23")


THERMAL_PARAMS = ("dx", "dy", "H_b", "H_t", "k_s", "k_f", "rho", "Cp", "T_inlet", "qk")


def thermal_cases():
    # name, Nx, Ny, seed, k_interp_mode, H_t, qk, nz_solid, nz_fluid
    yield "thermal_asm_13x9_mode0", 13, 9, 1, 0, 4e-4, 1.0, 2, 7
    yield "thermal_asm_13x9_mode1", 13, 9, 2, 1, 4e-4, 3.0, 2, 7
    yield "thermal_asm_13x9_mode2", 13, 9, 3, 2, 4e-4, 3.0, 2, 7
    yield "thermal_asm_21x11_mode1_h3", 21, 11, 4, 1, 3e-3, 10.0, 3, 5


def thermal_main() -> None:
    for name, Nx, Ny, seed, mode, Ht, qk, nzs, nzf in thermal_cases():
        rng = np.random.default_rng(seed)
        gamma = (rng.random((Ny, Nx)) > 0.4).astype(float)
        gamma[rng.random((Ny, Nx)) > 0.85] = 0.37
        gamma[:, 0] = 1.0
        u = np.abs(rng.normal(0.2, 0.15, (Ny, Nx))) * gamma
        v = rng.normal(0.0, 0.05, (Ny, Nx)) * gamma
        q0 = rng.uniform(5e5, 1.5e6, (Ny, Nx)) if mode != 0 else np.full((Ny, Nx), 8e5)
        dx = dy = 20e-6
        ref = reference.run_thermal_assembly(Nx, Ny, dx, dy, gamma, u, v, q0, nz_solid=nzs, nz_fluid=nzf, H_t=Ht,
                                             qk=qk, k_interp_mode=mode)
        p = dict(dx=float(ref["dxdy"][0]), dy=float(ref["dxdy"][1]), H_b=0.0005, H_t=Ht, k_s=400.0, k_f=0.6,
                 rho=998.0, Cp=4180.0, T_inlet=30.0, qk=qk)
        rec = dict(ints=np.array([Nx, Ny, nzs, nzf, mode], dtype=np.int64),
                   reals=np.array([p[k] for k in THERMAL_PARAMS]), gamma=gamma, u=u, v=v, q0=q0,
                   row_ptr=np.asarray(ref["row_ptr"], dtype=np.int64), col_idx=np.asarray(ref["col_idx"], dtype=np.int64),
                   values=np.asarray(ref["values"]), b=np.asarray(ref["b"]))
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **rec)
        print("wrote", name)


if __name__ == "__main__":
    if sys.argv[1:] == ["thermal"]:
        thermal_main()
    else:
        main(tuple(sys.argv[1:]))
