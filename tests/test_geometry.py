import numpy as np

from coldplate_solver_b200 import geometry as g


def test_straight_channel_config():
    d = g.straight_channel()
    assert (d.M, d.N) == (100, 200) and d.hx == d.hy == 50e-6
    assert d.convectionScheme == 0 and not d.enableTwoPointFiveD
    # fluid band rows 30..69 (cellType 0), walls forced at rows 0 and M-2 (SIMPLE.cpp:616-625)
    assert (d.gamma[30:70] == 1).all() and (d.gamma[1:30] == 0).all() and (d.gamma[70:] == 0).all()
    assert (d.alpha[0] == d.alpha.max()).all() and (d.alpha[d.M - 2] == d.alpha.max()).all()
    assert d.nU == 99 * 198 and d.nV == 98 * 199 and d.nP == 99 * 198


def test_generators_are_seeded():
    a = g.channel_network(M=60, N=120, seed=5)
    b = g.channel_network(M=60, N=120, seed=5)
    c = g.channel_network(M=60, N=120, seed=6)
    assert np.array_equal(a.gamma, b.gamma) and not np.array_equal(a.gamma, c.gamma)
    d1 = g.density_field(Nx=64, seed=1)
    d2 = g.density_field(Nx=64, seed=1)
    assert np.array_equal(d1.alpha, d2.alpha)


def test_network_connects_inlet_to_outlet():
    d = g.channel_network()
    assert d.gamma[:, 0].sum() > 0 and d.gamma[:, -1].sum() > 0
    assert d.enableTwoPointFiveD and d.enableConvectionScaling and d.convectionScheme == 1
    assert d.twoPointFiveDSinkMultiplier == 1.0 and d.Ht_channel == 500e-6


def test_density_field_plenum_and_range():
    d = g.density_field(Nx=200, seed=3)
    assert (d.M, d.N) == (100, 200)
    assert (d.gamma[1:d.M - 2, :8] == 1).all() and (d.gamma[1:d.M - 2, -8:] == 1).all()
    assert d.gamma.min() >= 0 and d.gamma.max() <= 1
    interior = d.gamma[1:d.M - 2, 8:-8]
    assert interior.min() < 0.2 and interior.max() > 0.8  # projected, not uniformly grey


def test_batch_mix_sizes():
    mix = g.batch_mix(n=16)
    assert len(mix) == 16
    for d in mix:
        assert 256 <= d.N <= 1024 and d.M == d.N // 2


def test_served_stream_arrivals():
    s = g.served_stream(12, rate=20.0)
    t = [a for a, _ in s]
    assert all(b > a for a, b in zip(t, t[1:]))
    assert all(0.05 <= d.inletVelocity <= 0.3 for _, d in s)


def test_pressure_determined_mask_leaves_out_cells_behind_clamped_faces():
    """p points cut off from the outlet by faces at the velocity clamp
    (3 max(|U|, 0.1), iterations.cpp:104) are not determined by a state."""
    d = g.straight_channel(M=10, N=20)
    u = np.zeros((d.M + 1, d.N))
    v = np.zeros((d.M, d.N + 1))
    assert g.pressure_determined_mask(d, u, v).all()
    vmax = 3.0 * max(abs(d.inletVelocity), 0.1)
    i, j = 5, 8  # the four faces of p(5, 8) at the clamp
    u[i, j - 1] = vmax
    u[i, j] = -vmax
    v[i - 1, j] = vmax
    v[i, j] = vmax
    m = g.pressure_determined_mask(d, u, v)
    assert not m[i, j] and m.sum() == m.size - 1
    u[i, j] = 0.999 * vmax  # one face below the clamp joins it again
    assert g.pressure_determined_mask(d, u, v).all()
