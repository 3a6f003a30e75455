"""CPU restatement of the reference's 3-D conjugate-heat-transfer solve
(ThermalSolver/thermal_solver.cpp) — TEST INFRASTRUCTURE ONLY: the oracle the
CUDA thermal path is checked against; no product code calls it (tests use
it, and bench.py's CPU-baseline leg times mg_bicgstab_cpu).

Parity: the assembly is pinned against the reference's own code.  The
reference's thermal solver includes AMGCL, whose headers are absent from the
reference tree (ThermalSolver/amgcl/ is empty and no version is pinned), so it
cannot be built whole; oracle/thermal_asm_harness.cpp compiles it with the
AMGCL solve cut out, and the matrix and right-hand side it assembles equal
this module's bit for bit (live, and through the committed fixtures
tests/golden/thermal_asm_*).  The linear solve here is a direct sparse LU
(scipy), i.e. the exact solution of the system the reference's AMGCL solve
approximates to a relative residual of rtol; that solve itself stays unpinned.

Index space: T[k, j, i] with P = k*Nx*Ny + j*Nx + i (thermal_solver.cpp:241);
2-D inputs (gamma, u, v, q0) are (Ny, Nx), gamma = 1 fluid, 0 solid
(thermal_solver.cpp:740-746).
"""
from __future__ import annotations

import dataclasses
from typing import Dict, Optional, Tuple

import numpy as np

PLANES = ("cW", "cE", "cS", "cN", "cB", "cT", "diag")


@dataclasses.dataclass
class ThermalParams:
    """Params (thermal_solver.cpp:147-193), reference member names."""

    Nx: int
    Ny: int
    dx: float
    dy: float
    nz_solid: int = 2
    nz_fluid: int = 7
    H_b: float = 0.0005
    H_t: float = 0.004
    k_s: float = 400.0
    k_f: float = 0.6
    rho: float = 998.0
    Cp: float = 4180.0
    T_inlet: float = 30.0
    rtol: float = 1e-6
    maxiter: int = 1000
    k_interp_mode: int = 1
    qk: float = 1.0

    @property
    def Nz(self) -> int:
        return self.nz_solid + self.nz_fluid

    @property
    def n(self) -> int:
        return self.Nx * self.Ny * self.Nz

    def dz_cells(self) -> np.ndarray:
        """thermal_solver.cpp:189-190, 237-239."""
        dz_s = self.H_b / self.nz_solid
        dz_f = self.H_t / self.nz_fluid
        return np.array([dz_s] * self.nz_solid + [dz_f] * self.nz_fluid, dtype=np.float64)


def kval_layer(p: ThermalParams, gamma: np.ndarray, k: int) -> np.ndarray:
    """kval (thermal_solver.cpp:283-312) for every cell of layer k."""
    if k < p.nz_solid:
        return np.full(gamma.shape, p.k_s)
    g = np.maximum(0.0, np.minimum(1.0, gamma))
    if p.k_interp_mode == 1:
        num = 1.0 - g
        den = 1.0 + p.qk * g
        return p.k_f + (p.k_s - p.k_f) * num / den
    if p.k_interp_mode == 2:
        return p.k_s * p.k_f / ((1.0 - g) * p.k_f + g * p.k_s + 1e-30)
    return p.k_s * (1.0 - g) + p.k_f * g


def pois(p: ThermalParams, k: int) -> float:
    """thermal_solver.cpp:336-340."""
    if k < p.nz_solid:
        return 0.0
    z = (k - p.nz_solid + 0.5) * (p.H_t / p.nz_fluid) / p.H_t
    return 4.0 * z * (1 - z)


def harm(a, b):
    """thermal_solver.cpp:242."""
    return 2 * a * b / (a + b + 1e-30)


def region_layer(p: ThermalParams, gamma: np.ndarray, k: int) -> np.ndarray:
    """region (thermal_solver.cpp:246-250): 1 = fluid."""
    if k < p.nz_solid:
        return np.zeros(gamma.shape, dtype=bool)
    return gamma > 0.01


def assemble(p: ThermalParams, gamma: np.ndarray, u: np.ndarray, v: np.ndarray,
             q0: np.ndarray) -> Tuple[Dict[str, np.ndarray], np.ndarray]:
    """The matrix and right-hand side of ThermalSolver3D::solve
    (thermal_solver.cpp:420-517), vectorised per layer in the reference's
    operation order: returns the seven coefficient planes (cW, cE, cS, cN, cB,
    cT: the merged off-diagonal CSR entries, 0 where absent; diag: the diagonal
    with its 1e-12) as (Nz, Ny, Nx) arrays, and b."""
    Nx, Ny, Nz = p.Nx, p.Ny, p.Nz
    dx, dy = p.dx, p.dy
    rhoCp, T_in = p.rho * p.Cp, p.T_inlet
    dz = p.dz_cells()
    planes = {k: np.zeros((Nz, Ny, Nx)) for k in PLANES}
    b = np.zeros((Nz, Ny, Nx))
    I = np.broadcast_to(np.arange(Nx)[None, :], (Ny, Nx))
    J = np.broadcast_to(np.arange(Ny)[:, None], (Ny, Nx))
    Az_cell = dx * dy
    for k in range(Nz):
        dz_k = dz[k]
        Ax, Ay = dy * dz_k, dx * dz_k
        kP = kval_layer(p, gamma, k)
        po = pois(p, k)
        g = np.zeros((Ny, Nx)) if k < p.nz_solid else gamma
        g = np.maximum(0.0, np.minimum(1.0, g))
        uP = np.where(g > 0.01, u * po, 0.0)
        vP = np.where(g > 0.01, v * po, 0.0)
        reg = region_layer(p, gamma, k)
        diag = np.zeros((Ny, Nx))
        bk = np.zeros((Ny, Nx))

        def shifted(a, di, dj, fill=0.0):
            out = np.full_like(a, fill)
            src = a[max(0, dj):Ny + min(0, dj), max(0, di):Nx + min(0, di)]
            out[max(0, -dj):Ny + min(0, -dj), max(0, -di):Nx + min(0, -di)] = src
            return out

        # X faces (thermal_solver.cpp:465-482)
        m = I > 0
        D = harm(kP, shifted(kP, -1, 0, 1.0)) * Ax / dx
        diag = np.where(m, diag + D, diag)
        cW = np.where(m, -D, 0.0)
        adv = m & reg & shifted(reg, -1, 0, False)
        uW = shifted(u, -1, 0) * po
        F = rhoCp * 0.5 * (uP + uW) * Ax
        diag = np.where(adv, diag + np.maximum(-F, 0.0), diag)
        cW = np.where(adv, cW + -np.maximum(F, 0.0), cW)
        bc = (I == 0) & reg
        D_bc = 2.0 * kP * Ax / dx
        F_bc = rhoCp * uP * Ax
        diag = np.where(bc, diag + D_bc, diag)
        bk = np.where(bc, bk + D_bc * T_in, bk)
        bk = np.where(bc & (F_bc > 0), bk + F_bc * T_in, bk)
        diag = np.where(bc & ~(F_bc > 0), diag + -F_bc, diag)
        m = I < Nx - 1
        D = harm(kP, shifted(kP, 1, 0, 1.0)) * Ax / dx
        diag = np.where(m, diag + D, diag)
        cE = np.where(m, -D, 0.0)
        adv = m & reg & shifted(reg, 1, 0, False)
        uE = shifted(u, 1, 0) * po
        F = rhoCp * 0.5 * (uP + uE) * Ax
        diag = np.where(adv, diag + np.maximum(F, 0.0), diag)
        cE = np.where(adv, cE + -np.maximum(-F, 0.0), cE)
        out = (I == Nx - 1) & reg & (uP > 0)
        diag = np.where(out, diag + rhoCp * uP * Ax, diag)
        # Y faces (:485-502)
        m = J > 0
        D = harm(kP, shifted(kP, 0, -1, 1.0)) * Ay / dy
        diag = np.where(m, diag + D, diag)
        cS = np.where(m, -D, 0.0)
        adv = m & reg & shifted(reg, 0, -1, False)
        vS = shifted(v, 0, -1) * po
        F = rhoCp * 0.5 * (vP + vS) * Ay
        diag = np.where(adv, diag + np.maximum(-F, 0.0), diag)
        cS = np.where(adv, cS + -np.maximum(F, 0.0), cS)
        m = J < Ny - 1
        D = harm(kP, shifted(kP, 0, 1, 1.0)) * Ay / dy
        diag = np.where(m, diag + D, diag)
        cN = np.where(m, -D, 0.0)
        adv = m & reg & shifted(reg, 0, 1, False)
        vN = shifted(v, 0, 1) * po
        F = rhoCp * 0.5 * (vP + vN) * Ay
        diag = np.where(adv, diag + np.maximum(F, 0.0), diag)
        cN = np.where(adv, cN + -np.maximum(-F, 0.0), cN)
        out = (J == Ny - 1) & reg & (vP > 0)
        diag = np.where(out, diag + rhoCp * vP * Ay, diag)
        # Z faces (:505-516)
        cB = np.zeros((Ny, Nx))
        cT = np.zeros((Ny, Nx))
        if k > 0:
            kN = kval_layer(p, gamma, k - 1)
            dz_P, dz_N = dz[k], dz[k - 1]
            kf = (dz_P + dz_N) / (dz_P / kP + dz_N / kN)
            D = kf * Az_cell / (0.5 * (dz_P + dz_N))
            diag = diag + D
            cB = -D
        else:
            bk = bk + q0 * Az_cell
        if k < Nz - 1:
            kN = kval_layer(p, gamma, k + 1)
            dz_P, dz_N = dz[k], dz[k + 1]
            kf = (dz_P + dz_N) / (dz_P / kP + dz_N / kN)
            D = kf * Az_cell / (0.5 * (dz_P + dz_N))
            diag = diag + D
            cT = -D
        for name, a in (("cW", cW), ("cE", cE), ("cS", cS), ("cN", cN), ("cB", cB), ("cT", cT)):
            planes[name][k] = a
        planes["diag"][k] = diag + 1e-12
        b[k] = bk
    return planes, b


def assemble_loops(p: ThermalParams, gamma: np.ndarray, u: np.ndarray, v: np.ndarray, q0: np.ndarray):
    """The same assembly cell by cell in the reference's own loop structure
    (pure Python, small grids only): COO triplets merged as SparseMatrix::
    from_coo does (thermal_solver.cpp:82-120).  Returns (planes, b)."""
    Nx, Ny, Nz = p.Nx, p.Ny, p.Nz
    dx, dy = p.dx, p.dy
    rhoCp, T_in = p.rho * p.Cp, p.T_inlet
    dz = p.dz_cells()
    g2 = gamma

    def kval(i, j, k):
        if k < p.nz_solid:
            return p.k_s
        g = max(0.0, min(1.0, g2[j, i]))
        if p.k_interp_mode == 1:
            return p.k_f + (p.k_s - p.k_f) * (1.0 - g) / (1.0 + p.qk * g)
        if p.k_interp_mode == 2:
            return p.k_s * p.k_f / ((1.0 - g) * p.k_f + g * p.k_s + 1e-30)
        return p.k_s * (1.0 - g) + p.k_f * g

    def region(i, j, k):
        return 0 if k < p.nz_solid else (1 if g2[j, i] > 0.01 else 0)

    coo = {}
    b = np.zeros((Nz, Ny, Nx))

    def add(r, c, val):
        coo.setdefault((r, c), []).append(val)

    def idx(i, j, k):
        return k * Nx * Ny + j * Nx + i

    for k in range(Nz):
        dz_k = dz[k]
        Ax, Ay, Az_cell = dy * dz_k, dx * dz_k, dx * dy
        for j in range(Ny):
            for i in range(Nx):
                P = idx(i, j, k)
                diag, kP, po = 0.0, kval(i, j, k), pois(p, k)
                g = 0.0 if k < p.nz_solid else g2[j, i]
                g = max(0.0, min(1.0, g))
                uP = u[j, i] * po if g > 0.01 else 0.0
                vP = v[j, i] * po if g > 0.01 else 0.0
                if i > 0:
                    D = harm(kP, kval(i - 1, j, k)) * Ax / dx
                    diag += D
                    add(P, idx(i - 1, j, k), -D)
                    if region(i, j, k) == 1 and region(i - 1, j, k) == 1:
                        F = rhoCp * 0.5 * (uP + u[j, i - 1] * po) * Ax
                        diag += max(-F, 0.0)
                        add(P, idx(i - 1, j, k), -max(F, 0.0))
                elif region(i, j, k) == 1:
                    D_bc, F_bc = 2.0 * kP * Ax / dx, rhoCp * uP * Ax
                    diag += D_bc
                    b[k, j, i] += D_bc * T_in
                    if F_bc > 0:
                        b[k, j, i] += F_bc * T_in
                    else:
                        diag += -F_bc
                if i < Nx - 1:
                    D = harm(kP, kval(i + 1, j, k)) * Ax / dx
                    diag += D
                    add(P, idx(i + 1, j, k), -D)
                    if region(i, j, k) == 1 and region(i + 1, j, k) == 1:
                        F = rhoCp * 0.5 * (uP + u[j, i + 1] * po) * Ax
                        diag += max(F, 0.0)
                        add(P, idx(i + 1, j, k), -max(-F, 0.0))
                elif region(i, j, k) == 1 and uP > 0:
                    diag += rhoCp * uP * Ax
                if j > 0:
                    D = harm(kP, kval(i, j - 1, k)) * Ay / dy
                    diag += D
                    add(P, idx(i, j - 1, k), -D)
                    if region(i, j, k) == 1 and region(i, j - 1, k) == 1:
                        F = rhoCp * 0.5 * (vP + v[j - 1, i] * po) * Ay
                        diag += max(-F, 0.0)
                        add(P, idx(i, j - 1, k), -max(F, 0.0))
                if j < Ny - 1:
                    D = harm(kP, kval(i, j + 1, k)) * Ay / dy
                    diag += D
                    add(P, idx(i, j + 1, k), -D)
                    if region(i, j, k) == 1 and region(i, j + 1, k) == 1:
                        F = rhoCp * 0.5 * (vP + v[j + 1, i] * po) * Ay
                        diag += max(F, 0.0)
                        add(P, idx(i, j + 1, k), -max(-F, 0.0))
                elif region(i, j, k) == 1 and vP > 0:
                    diag += rhoCp * vP * Ay
                if k > 0:
                    kN, dz_P, dz_N = kval(i, j, k - 1), dz[k], dz[k - 1]
                    kf = (dz_P + dz_N) / (dz_P / kP + dz_N / kN)
                    D = kf * Az_cell / (0.5 * (dz_P + dz_N))
                    diag += D
                    add(P, idx(i, j, k - 1), -D)
                else:
                    b[k, j, i] += q0[j, i] * Az_cell
                if k < Nz - 1:
                    kN, dz_P, dz_N = kval(i, j, k + 1), dz[k], dz[k + 1]
                    kf = (dz_P + dz_N) / (dz_P / kP + dz_N / kN)
                    D = kf * Az_cell / (0.5 * (dz_P + dz_N))
                    diag += D
                    add(P, idx(i, j, k + 1), -D)
                add(P, P, diag + 1e-12)
    planes = {k: np.zeros((Nz, Ny, Nx)) for k in PLANES}
    offs = {-1: "cW", 1: "cE", -Nx: "cS", Nx: "cN", -Nx * Ny: "cB", Nx * Ny: "cT", 0: "diag"}
    for (r, c), vals in coo.items():
        s = 0.0
        for x in sorted(vals):  # from_coo: sorted triplets, duplicates summed in order
            s += x
        k, rem = divmod(r, Nx * Ny)
        j, i = divmod(rem, Nx)
        planes[offs[c - r]][k, j, i] = s
    return planes, b


def to_csr(p: ThermalParams, planes: Dict[str, np.ndarray]):
    import scipy.sparse as sp
    Nx, Ny, Nz = p.Nx, p.Ny, p.Nz
    n = p.n
    P = np.arange(n).reshape(Nz, Ny, Nx)
    rows, cols, vals = [], [], []
    for name, off, mask in (("cW", -1, P % Nx > 0), ("cE", 1, P % Nx < Nx - 1),
                            ("cS", -Nx, (P // Nx) % Ny > 0), ("cN", Nx, (P // Nx) % Ny < Ny - 1),
                            ("cB", -Nx * Ny, P // (Nx * Ny) > 0), ("cT", Nx * Ny, P // (Nx * Ny) < Nz - 1),
                            ("diag", 0, np.ones_like(P, dtype=bool))):
        rows.append(P[mask])
        cols.append(P[mask] + off)
        vals.append(planes[name][mask])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))


def solve_direct(p: ThermalParams, gamma, u, v, q0) -> np.ndarray:
    """The exact solution of the assembled system (sparse LU), (Nz, Ny, Nx)."""
    import scipy.sparse.linalg as spl
    planes, b = assemble(p, gamma, u, v, q0)
    A = to_csr(p, planes)
    return spl.spsolve(A.tocsc(), b.ravel()).reshape(p.Nz, p.Ny, p.Nx)


def relative_residual(p: ThermalParams, planes, b: np.ndarray, T: np.ndarray) -> float:
    A = to_csr(p, planes)
    r = b.ravel() - A @ T.ravel()
    return float(np.linalg.norm(r) / np.linalg.norm(b.ravel()))


def stats(p: ThermalParams, gamma: np.ndarray, u: np.ndarray, T: np.ndarray) -> Dict[str, float]:
    """The temperature ranges and energy balance the reference prints after
    its solve (thermal_solver.cpp:567-619); q0 uniform is not assumed: Q_in
    is summed by the caller's q0 in thermal_stats."""
    Nz = p.Nz
    out = {}
    base = T[:p.nz_solid]
    fluid_mask = np.zeros(T.shape, dtype=bool)
    for k in range(p.nz_solid, Nz):
        fluid_mask[k] = region_layer(p, gamma, k)
    fin_mask = np.ones(T.shape, dtype=bool)
    fin_mask[:p.nz_solid] = False
    fin_mask &= ~fluid_mask
    out["T_base_min"], out["T_base_max"] = float(base.min()), float(base.max())
    out["T_fluid_min"] = float(T[fluid_mask].min()) if fluid_mask.any() else 1e30
    out["T_fluid_max"] = float(T[fluid_mask].max()) if fluid_mask.any() else -1e30
    out["T_fin_min"] = float(T[fin_mask].min()) if fin_mask.any() else 1e30
    out["T_fin_max"] = float(T[fin_mask].max()) if fin_mask.any() else -1e30
    dz = p.dz_cells()
    mdot = mdotT = 0.0
    for k in range(p.nz_solid, Nz):
        A = p.dy * dz[k]
        po = pois(p, k)
        for j in range(p.Ny):
            i = p.Nx - 1
            if gamma[j, i] > 0.01:
                uu = u[j, i] * po
                if uu > 0:
                    m = p.rho * uu * A
                    mdot += m
                    mdotT += m * T[k, j, i]
    out["mdot"] = mdot
    out["T_out"] = mdotT / mdot if mdot > 0 else p.T_inlet
    return out


def energy_balance(p: ThermalParams, gamma, u, q0, T) -> Dict[str, float]:
    """Q_in, T_out, Q_out and the imbalance in % (thermal_solver.cpp:588-619)."""
    s = stats(p, gamma, u, T)
    Q_in = 0.0
    for j in range(p.Ny):
        for i in range(p.Nx):
            Q_in += q0[j, i] * p.dx * p.dy
    Q_out = s["mdot"] * p.Cp * (s["T_out"] - p.T_inlet)
    s.update(Q_in=Q_in, Q_out=Q_out, imbalance=100 * (Q_in - Q_out) / (Q_in + 1e-30))
    return s


def mg_bicgstab_cpu(p: ThermalParams, gamma, u, v, q0, sweeps: int = 2, omega: float = 0.8, alpha: float = 1.7,
                    time_cap: float = 1e30):
    """CPU port (scipy, single process) of the GPU solve's algorithm: the
    assembly above, the 2 x 2 aggregation hierarchy with exact Galerkin
    coarse operators, BiCGStab right-preconditioned by the same V-cycle, from
    T = T_inlet to ||b - A T|| <= rtol ||b||.  Used only as the CPU baseline of
    the thermal benchmark (the reference's own solve needs the absent AMGCL).
    Returns (T, iterations, seconds, finished)."""
    import time

    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    t0 = time.perf_counter()
    planes, b3 = assemble(p, gamma, u, v, q0)
    A = to_csr(p, planes)
    b = b3.ravel()
    levels = []
    nx, ny, Nz = p.Nx, p.Ny, p.Nz
    Al = A
    while True:
        levels.append({"A": Al, "dinv": 1.0 / Al.diagonal()})
        if nx == 1 and ny == 1:
            break
        cx, cy = (nx + 1) // 2, (ny + 1) // 2
        k, j, i = np.meshgrid(np.arange(Nz), np.arange(ny), np.arange(nx), indexing="ij")
        P = sp.csr_matrix((np.ones(k.size), ((k * ny * nx + j * nx + i).ravel(), (k * cy * cx + (j // 2) * cx + i // 2).ravel())),
                          shape=(nx * ny * Nz, cx * cy * Nz))
        levels[-1]["P"] = P
        Al = (P.T @ Al @ P).tocsr()
        nx, ny = cx, cy
    levels[-1]["lu"] = spl.splu(levels[-1]["A"].tocsc())

    def vcycle(l, rhs):
        L = levels[l]
        if "lu" in L:
            return L["lu"].solve(rhs)
        A_, dinv = L["A"], L["dinv"]
        x = omega * dinv * rhs
        for _ in range(sweeps - 1):
            x = x + omega * dinv * (rhs - A_ @ x)
        e = vcycle(l + 1, L["P"].T @ (rhs - A_ @ x))
        x = x + alpha * (L["P"] @ e)
        for _ in range(sweeps):
            x = x + omega * dinv * (rhs - A_ @ x)
        return x

    T = np.full(p.n, p.T_inlet)
    r = b - A @ T
    rhat = r.copy()
    pv = np.zeros_like(r)
    vv = np.zeros_like(r)
    bnorm = np.linalg.norm(b) or 1.0
    rho = al = om = 1.0
    rho_new = float(r @ r)
    it = 0
    while np.linalg.norm(r) > p.rtol * bnorm and it < p.maxiter:
        if time.perf_counter() - t0 > time_cap:
            return T.reshape(Nz, p.Ny, p.Nx), it, time.perf_counter() - t0, False
        beta = (rho_new / rho) * (al / om)
        pv = r + beta * (pv - om * vv)
        ph = vcycle(0, pv)
        vv = A @ ph
        al = rho_new / float(rhat @ vv)
        s = r - al * vv
        if np.linalg.norm(s) <= p.rtol * bnorm:
            T = T + al * ph
            it += 1
            break
        sh = vcycle(0, s)
        t = A @ sh
        om = float(t @ s) / float(t @ t)
        T = T + al * ph + om * sh
        r = s - om * t
        rho, rho_new = rho_new, float(rhat @ r)
        it += 1
    return T.reshape(Nz, p.Ny, p.Nx), it, time.perf_counter() - t0, True


def load_assembly_fixture(path: str):
    """A thermal_asm_* golden fixture (tests/golden/make_golden.py): the
    ThermalParams, the inputs (gamma, u, v, q0) and the reference's own CSR
    matrix (scipy, sorted indices) and right-hand side for them."""
    import scipy.sparse as sp
    z = np.load(path)
    Nx, Ny, nzs, nzf, mode = (int(x) for x in z["ints"])
    dx, dy, H_b, H_t, k_s, k_f, rho, Cp, T_inlet, qk = (float(x) for x in z["reals"])
    p = ThermalParams(Nx=Nx, Ny=Ny, dx=dx, dy=dy, nz_solid=nzs, nz_fluid=nzf, H_b=H_b, H_t=H_t, k_s=k_s, k_f=k_f,
                      rho=rho, Cp=Cp, T_inlet=T_inlet, k_interp_mode=mode, qk=qk)
    A = sp.csr_matrix((z["values"], z["col_idx"], z["row_ptr"]), shape=(p.n, p.n))
    inputs = {k: np.asarray(z[k]) for k in ("gamma", "u", "v", "q0")}
    return p, inputs, A, np.asarray(z["b"])


def same_csr(A, B) -> bool:
    """Bit-identical sparsity structure and values (both sorted)."""
    return (A.shape == B.shape and np.array_equal(A.indptr, B.indptr) and np.array_equal(A.indices, B.indices)
            and np.array_equal(A.data.view(np.uint64), B.data.view(np.uint64)))
