"""Design descriptions and seeded synthetic geometry generators.

A :class:`Design` carries everything one SIMPLE solve needs: the grid, the
physical and solver parameters under the reference's own member names
(``SIMPLE.h:68-358``), and the cell fields ``gamma`` (density, 1 = fluid) and
``alpha`` (Brinkman drag) of shape ``(M, N)``, row-major, in the reference's
cell index space (cell (i, j) is row i, column j; ``SIMPLE.cpp:199-201``).

Grid naming follows the reference: ``M`` rows (y), ``N`` columns (x, the flow
direction).  A "P-grid Nx x Ny" in a workload description is ``N = Nx``,
``M = Ny``.

The generators are this project's own seeded stand-ins for the reference's
Python geometry scripts (which need matplotlib and write text files); they
produce the workloads named in the benchmark description:

* :func:`straight_channel`  -- 2-D straight channel, centred fluid band, FOU.
* :func:`channel_network`   -- seeded Manhattan random-walk channel network,
  SOU, 2.5-D.
* :func:`density_field`     -- smoothed, tanh-projected random density field,
  SOU, 2.5-D, RAMP Brinkman alpha.
* :func:`batch_mix`         -- many density-field designs of log-uniform size.
* :func:`served_stream`     -- Poisson arrivals of density-field designs.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Tuple

import numpy as np

__all__ = [
    "Design",
    "alpha_ramp_reference",
    "alpha_ramp_q",
    "straight_channel",
    "channel_network",
    "density_field",
    "batch_mix",
    "served_stream",
]

RHO = 997.0  # SIMPLE.h:334
ETA = 0.00089  # SIMPLE.h:335
K_MIN = 1e-14  # SIMPLE.h:242 brinkmanKMin


@dataclasses.dataclass
class Design:
    """One solve's inputs (reference member names, SIMPLE.h)."""

    M: int
    N: int
    hx: float
    hy: float
    inletVelocity: float
    gamma: np.ndarray
    alpha: np.ndarray
    convectionScheme: int = 0  # SIMPLE.h:193 (0 FOU, 1 SOU)
    enableTwoPointFiveD: bool = False  # SIMPLE.h:205
    enableConvectionScaling: bool = False  # SIMPLE.h:206
    Ht_channel: float = 0.0  # SIMPLE.h:207
    twoPointFiveDSinkMultiplier: float = 4.8  # SIMPLE.h:208
    uvAlpha: float = 0.7  # SIMPLE.h:357
    pAlpha: float = 0.2  # SIMPLE.h:358
    rho: float = RHO
    eta: float = ETA
    pTol: float = 1e-4  # SIMPLE.h:153
    maxPressureIter: int = 20  # SIMPLE.h:152
    momentumTol: float = 1e-5  # SIMPLE.h:176
    maxMomentumIter: int = 200  # SIMPLE.h:177
    momentumSolverType: int = 1  # SIMPLE.h:172 (0 explicit point update, 1 implicit Jacobi)
    name: str = "design"
    # Pseudo-transient term and its CFL controllers (SIMPLE.h:255-313; all off by default).
    enablePseudoTimeStepping: bool = False
    useLocalPseudoTime: bool = True
    timeStepMultiplier: float = 0.01  # timeStep = multiplier * N hx / max(inletVelocity, 1e-6)
    minPseudoSpeed: float = 0.05
    pseudoCFL: float = 0.1  # the CFL number when the ramp does not set it
    enableSER: bool = True
    serCFLMin: float = 0.1
    serCFLMax: float = 5.0
    serSmooth: float = 0.5
    serMinIter: int = 10
    serMaxIncrease: float = 1.1
    serMaxDecrease: float = 0.7
    serUseMaxResid: bool = False
    enableLineSearch: bool = True
    lsAlphaMin: float = 0.1
    lsAlphaReduce: float = 0.3
    lsMaxTries: int = 4
    lsResidIncreaseTol: float = 1.01
    enableCflRamp: bool = True
    pseudoCFLInitial: float = 0.1
    pseudoCFLMax: float = 30.0
    cflRampStartRes: float = 1e-4
    cflRampExponent: float = 0.8
    cflRampSmooth: float = 0.1
    # Inlet velocity ramp of the outer loop (SIMPLE.h:345-346, SIMPLE.cpp:303-307): for the first
    # rampSteps iterations the inlet velocity is (iter + 1) / rampSteps of inletVelocity.
    enableInletRamp: bool = False
    rampSteps: int = 1000

    def __post_init__(self) -> None:
        self.gamma = np.ascontiguousarray(self.gamma, dtype=np.float64)
        self.alpha = np.ascontiguousarray(self.alpha, dtype=np.float64)
        if self.M < 3 or self.N < 3:
            raise ValueError(f"grid {self.M}x{self.N} too small: need M >= 3 and N >= 3")
        if self.gamma.shape != (self.M, self.N) or self.alpha.shape != (self.M, self.N):
            raise ValueError("gamma and alpha must have shape (M, N)")

    @property
    def cells(self) -> int:
        return self.M * self.N

    # Unknown counts (momentum_solver.cpp:52-74, pressure_solver.cpp:438-458).
    @property
    def nU(self) -> int:
        return (self.M - 1) * (self.N - 2)

    @property
    def nV(self) -> int:
        return (self.M - 2) * (self.N - 1)

    @property
    def nP(self) -> int:
        return (self.M - 1) * (self.N - 2)

    def pseudo_cfl_start(self) -> float:
        """The CFL number of the first step: the constructor starts the ramp
        at pseudoCFLInitial when enableCflRamp (SIMPLE.cpp:78-82)."""
        return self.pseudoCFLInitial if self.enableCflRamp else self.pseudoCFL

    def int_params(self) -> np.ndarray:
        return np.array([self.M, self.N, self.convectionScheme, int(self.enableTwoPointFiveD),
                         int(self.enableConvectionScaling), self.maxPressureIter, self.maxMomentumIter,
                         self.momentumSolverType, int(self.enablePseudoTimeStepping), int(self.useLocalPseudoTime),
                         int(self.enableSER), int(self.enableLineSearch), int(self.enableCflRamp),
                         int(self.serUseMaxResid), self.serMinIter, self.lsMaxTries, int(self.enableInletRamp),
                         self.rampSteps], dtype=np.int32)

    def real_params(self, pseudo_cfl: Optional[float] = None) -> np.ndarray:
        """dp[27] is the CFL number the step uses (default: the first step's)."""
        return np.array([self.hx, self.hy, self.rho, self.eta, self.uvAlpha, self.pAlpha, self.inletVelocity,
                         self.Ht_channel, self.twoPointFiveDSinkMultiplier, self.pTol, self.momentumTol,
                         self.timeStepMultiplier, self.minPseudoSpeed, self.pseudoCFLInitial, self.pseudoCFLMax,
                         self.cflRampStartRes, self.cflRampExponent, self.cflRampSmooth, self.serCFLMin,
                         self.serCFLMax, self.serSmooth, self.serMaxIncrease, self.serMaxDecrease, self.lsAlphaMin,
                         self.lsAlphaReduce, self.lsResidIncreaseTol, self.inletVelocity,
                         self.pseudo_cfl_start() if pseudo_cfl is None else pseudo_cfl], dtype=np.float64)

    def replace(self, **kw) -> "Design":
        return dataclasses.replace(self, **kw)


def alpha_ramp_reference(gamma: np.ndarray, alpha_max: float = ETA / K_MIN, q: float = 1.0) -> Tuple[np.ndarray, np.ndarray]:
    """Brinkman alpha exactly as the reference builds it (SIMPLE.cpp:589-630).

    alpha = alpha_max (1 - g) / (1 + q g + 1e-10), evaluated in that operation
    order in float64, then rows 0 and M-2 forced to a solid wall
    (alpha = alpha_max, gamma = 0).  Returns (alpha, gamma_after_forcing).
    """
    g = np.array(gamma, dtype=np.float64, copy=True)
    alpha = alpha_max * (1.0 - g) / (1.0 + q * g + 1e-10)
    _force_walls(alpha, g, alpha_max)
    return alpha, g


def alpha_ramp_q(gamma: np.ndarray, alpha_max: float = 1e9, q: float = 0.1) -> Tuple[np.ndarray, np.ndarray]:
    """The density-field workload's RAMP form alpha = alpha_max q (1-g) / (q+g),
    with the reference's wall-row forcing (SIMPLE.cpp:616-625) applied after."""
    g = np.array(gamma, dtype=np.float64, copy=True)
    alpha = alpha_max * q * (1.0 - g) / (q + g)
    _force_walls(alpha, g, alpha_max)
    return alpha, g


def _force_walls(alpha: np.ndarray, gamma: np.ndarray, alpha_max: float) -> None:
    M = alpha.shape[0]
    if M >= 2:
        for r in (0, M - 2):
            alpha[r, :] = alpha_max
            gamma[r, :] = 0.0


def straight_channel(M: int = 100, N: int = 200, h: float = 50e-6, band: Optional[Tuple[int, int]] = None,
                     U: float = 0.1, pAlpha: float = 0.3, name: str = "straight_channel") -> Design:
    """2-D straight channel: cellType = 1 (solid) except a centred fluid band
    (rows 30..69 for the 100-row grid), FOU, no 2.5-D, reference Brinkman
    defaults (alpha_max = mu/1e-14, q = 1)."""
    if band is None:
        half = max(1, (2 * M) // 10)
        band = (M // 2 - half, M // 2 + half)
    cell_type = np.ones((M, N))
    cell_type[band[0]:band[1], :] = 0.0
    gamma = 1.0 - cell_type  # SIMPLE.cpp:569
    alpha, gamma = alpha_ramp_reference(gamma)
    return Design(M=M, N=N, hx=h, hy=h, inletVelocity=U, gamma=gamma, alpha=alpha, convectionScheme=0,
                  pAlpha=pAlpha, name=name)


def channel_network(M: int = 250, N: int = 500, h: float = 20e-6, n_paths: int = 6, wmin: int = 6, wmax: int = 12,
                    seed: int = 42, U: float = 0.2, Ht: float = 500e-6, uvAlpha: float = 0.3, pAlpha: float = 0.1,
                    name: str = "channel_network") -> Design:
    """Seeded Manhattan random-walk network: ``n_paths`` paths run from the
    inlet column to the outlet column in horizontal runs joined by vertical
    moves; each path is a band of width U[wmin, wmax] cells; crossing paths
    merge (union).  SOU, 2.5-D sink and 6/7 scaling on, sink multiplier 1
    (the literal -(5 mu / 2 Ht^2)).

    Relaxation uvAlpha 0.3 / pAlpha 0.1: with SOU the reference algorithm
    stalls near a 3e-3 residual at 0.7 / 0.3 and near 3e-5 at 0.5 / 0.2 on
    this geometry, and converges to 1e-6 at 0.3 / 0.1."""
    rng = np.random.default_rng(seed)
    fluid = np.zeros((M, N), dtype=bool)
    for _ in range(n_paths):
        w = int(rng.integers(wmin, wmax + 1))
        lo = 2 + w // 2
        hi = max(lo, M - 4 - (w - w // 2))
        row = int(rng.integers(lo, hi + 1))
        col = 0
        while col < N:
            run = int(rng.integers(max(2, N // 20), max(3, N // 5)))
            c1 = min(N, col + run)
            fluid[max(0, row - w // 2):row - w // 2 + w, col:min(N, c1 + w // 2)] = True
            col = c1
            if col >= N:
                break
            new_row = int(rng.integers(lo, hi + 1))
            r0, r1 = min(row, new_row), max(row, new_row)
            fluid[max(0, r0 - w // 2):r1 - w // 2 + w, max(0, col - w // 2):min(N, col - w // 2 + w)] = True
            row = new_row
    gamma = fluid.astype(np.float64)
    alpha, gamma = alpha_ramp_reference(gamma)
    return Design(M=M, N=N, hx=h, hy=h, inletVelocity=U, gamma=gamma, alpha=alpha, convectionScheme=1,
                  enableTwoPointFiveD=True, enableConvectionScaling=True, Ht_channel=Ht,
                  twoPointFiveDSinkMultiplier=1.0, uvAlpha=uvAlpha, pAlpha=pAlpha, name=name)


def _smooth(field: np.ndarray, sigma: float) -> np.ndarray:
    """Separable Gaussian blur with reflected edges (numpy only)."""
    radius = int(math.ceil(4 * sigma))
    x = np.arange(-radius, radius + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    out = field
    for axis in (0, 1):
        pad = [(0, 0), (0, 0)]
        pad[axis] = (radius, radius)
        padded = np.pad(out, pad, mode="symmetric")
        out = np.apply_along_axis(lambda s: np.convolve(s, k, mode="valid"), axis, padded)
    return out


def density_field(Nx: int = 1000, h: float = 10e-6, seed: int = 0, sigma: float = 8.0, beta: float = 8.0,
                  eta_p: float = 0.5, plenum: int = 8, U: float = 0.1, Ht: float = 300e-6,
                  twoFiveD: bool = True, alpha_max: float = 1e9, q: float = 0.1, uvAlpha: float = 0.3,
                  pAlpha: float = 0.1, maxPressureIter: int = 200, name: Optional[str] = None) -> Design:
    """Density-based gamma field on an ``Nx x Nx/2`` P-grid.

    gamma = tanh-projection(beta, eta) of seeded U[0,1] noise blurred with a
    Gaussian of ``sigma`` cells and rescaled to [0, 1] (without the rescale the
    blurred noise is ~0.5 +- 0.01 everywhere and the projection is uniformly
    grey).  gamma = 1 is pinned in the first and last ``plenum`` columns of
    rows 1..M-3 so that the reference's pure-fluid plane sampling
    (postprocessing.cpp:145-148) sees open inlet and outlet planes.  Brinkman
    alpha = alpha_max q (1-gamma)/(q+gamma), walls forced; SOU; 2.5-D with
    sink multiplier 1.

    Solver settings uvAlpha 0.3 / pAlpha 0.1 / maxPressureIter 200 (the
    reference's comment at SIMPLE.h:152 gives 200 for PCG): with 20 PCG
    iterations or with 0.5 / 0.2 relaxation the 256- to 1000-column fields
    stall between 1e-5 and 1e-4; with these settings they converge to 1e-6 in
    9k-17k outer iterations.
    """
    N = int(Nx)
    M = max(3, N // 2)
    rng = np.random.default_rng(seed)
    noise = rng.random((M, N))
    sm = _smooth(noise, sigma)
    lo, hi = sm.min(), sm.max()
    sm = (sm - lo) / (hi - lo) if hi > lo else np.full_like(sm, 0.5)
    t = math.tanh(beta * eta_p)
    gamma = (t + np.tanh(beta * (sm - eta_p))) / (t + math.tanh(beta * (1.0 - eta_p)))
    gamma = np.clip(gamma, 0.0, 1.0)
    p = min(plenum, N // 4)
    if M > 3 and p > 0:
        gamma[1:M - 2, :p] = 1.0
        gamma[1:M - 2, N - p:] = 1.0
    alpha, gamma = alpha_ramp_q(gamma, alpha_max, q)
    return Design(M=M, N=N, hx=h, hy=h, inletVelocity=U, gamma=gamma, alpha=alpha, convectionScheme=1,
                  enableTwoPointFiveD=twoFiveD, enableConvectionScaling=twoFiveD, Ht_channel=Ht if twoFiveD else 0.0,
                  twoPointFiveDSinkMultiplier=1.0, uvAlpha=uvAlpha, pAlpha=pAlpha, maxPressureIter=maxPressureIter,
                  name=name or f"density_{N}x{M}_s{seed}")


def batch_mix(n: int = 64, nx_range: Tuple[int, int] = (256, 1024), h: float = 10e-6, seed: int = 1234,
              U: float = 0.2, Ht: float = 500e-6) -> List[Design]:
    """``n`` density-field designs, Nx log-uniform in ``nx_range`` (Ny = Nx/2),
    independent seeds, SOU + 2.5-D (Ht = 500 um) as in the channel-network
    workload."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nx = int(round(math.exp(rng.uniform(math.log(nx_range[0]), math.log(nx_range[1])))))
        out.append(density_field(Nx=nx, h=h, seed=int(rng.integers(1 << 30)), U=U, Ht=Ht, name=f"mix{k}_{nx}"))
    return out


def served_stream(n: int, rate: float = 20.0, nx_range: Tuple[int, int] = (128, 2048), h: float = 10e-6,
                  seed: int = 777) -> List[Tuple[float, Design]]:
    """Poisson arrivals (``rate`` per second) of density-field designs: Nx
    log-uniform in ``nx_range`` (Ny = Nx/2), inlet U[0.05, 0.3] m/s, half with
    2.5-D on (Ht U[200, 600] um).  Returns (arrival_time_s, design) pairs."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += float(rng.exponential(1.0 / rate))
        nx = int(round(math.exp(rng.uniform(math.log(nx_range[0]), math.log(nx_range[1])))))
        two = bool(rng.random() < 0.5)
        d = density_field(Nx=nx, h=h, seed=int(rng.integers(1 << 30)), U=float(rng.uniform(0.05, 0.3)),
                          Ht=float(rng.uniform(200e-6, 600e-6)), twoFiveD=two, name=f"req{k}_{nx}")
        out.append((t, d))
    return out



def pressure_determined_mask(design: Design, u: np.ndarray, v: np.ndarray) -> np.ndarray:
    """p points (on p's (M+1) x (N+1) index space) whose pressure a state
    (u, v) determines: those joined to the outlet column (where p is fixed)
    through faces whose velocity is not at the outer iteration's clamp
    |vel| = 3 max(|U|, 0.1) (iterations.cpp:104).  A clamped face passes no
    pressure information (its velocity does not respond to the pressure
    difference across it), so cells enclosed by clamped faces keep whatever
    pressure level they had: two states whose outer residual is below 1e-12
    differ there by up to ~1e-5 of the pressure scale (measured on the
    500 x 250 density design: 213 such fluid cells, 99 % of the difference).
    Pressure comparisons between solves use this mask."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    M, N = design.M, design.N
    vmax = 3.0 * max(abs(design.inletVelocity), 0.1) * (1.0 - 1e-6)
    idx = np.arange((M + 1) * (N + 1)).reshape(M + 1, N + 1)
    fu = np.abs(u) < vmax  # u(i, j): between p(i, j) and p(i, j + 1)
    fv = np.abs(v) < vmax  # v(i, j): between p(i, j) and p(i + 1, j)
    rows = np.concatenate([idx[:, :N][fu], idx[:M, :][fv]])
    cols = np.concatenate([idx[:, 1:][fu], idx[1:, :][fv]])
    graph = coo_matrix((np.ones(len(rows)), (rows, cols)), shape=(idx.size, idx.size))
    _, lab = connected_components(graph, directed=False)
    lab = lab.reshape(M + 1, N + 1)
    return np.isin(lab, np.unique(lab[1:M, N]))
