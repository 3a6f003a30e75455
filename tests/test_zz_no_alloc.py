"""cps_solve_noalloc: the allocation-free solve for callers that cannot call
cudaMalloc (they hand the library device buffers and a stream; the library's
scratch is a static device array).  Checked through the C ABI against the
ordinary entry point (cps_create + cps_solve) on two calls in a row, with the
parity tests' per-step tolerance: 1e-10 relative L2 per field and identical
inner iteration counts.  This file is collected last."""
import ctypes

import numpy as np
import pytest

from coldplate_solver_b200 import cps, geometry

pytestmark = pytest.mark.gpu

REL_STEP = 1e-10
OUT_FIELDS = ("u", "v", "p", "pStar", "uStar", "vStar", "dE", "dN")


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


class CallerBuffers:
    """Device buffers the caller owns (allocated here by the test, as the
    caller's own pool would), all with one row pitch."""

    def __init__(self, design, pitch, init, pad=0.0):
        """``pad``: the value of every element outside the logical matrices
        (the columns past each matrix's width, row M of the v plane), as a
        pool allocator may leave it."""
        import torch
        self.torch = torch
        M, N = design.M, design.N
        self.design, self.pitch = design, pitch
        dev = torch.device("cuda", 0)

        def plane(rows, host=None):
            t = torch.full((rows, pitch), pad, dtype=torch.float64, device=dev)
            if host is not None:
                t[:host.shape[0], :host.shape[1]] = torch.from_numpy(np.ascontiguousarray(host)).to(dev)
            return t
        self.alpha = plane(M, design.alpha)
        self.gamma = plane(M, design.gamma)
        self.u = plane(M + 1, init["u"])
        self.v = plane(M + 1, init["v"])
        self.p = plane(M + 1, init["p"])
        self.out = {k: plane(M + 1) for k in ("pStar", "uStar", "vStar", "dE", "dN")}

    def ptr(self, t):
        return ctypes.c_void_p(t.data_ptr())

    def fields(self):
        M, N = self.design.M, self.design.N
        cols = {"u": N, "v": N + 1, "p": N + 1, "pStar": N + 1, "uStar": N, "vStar": N + 1, "dE": N, "dN": N + 1}
        rows = {"v": M, "vStar": M, "dN": M}
        src = {"u": self.u, "v": self.v, "p": self.p, **self.out}
        return {k: src[k][:rows.get(k, M + 1), :cols[k]].cpu().numpy() for k in OUT_FIELDS}


def call_noalloc(lib, design, buf, n, eps=0.0, stream=None):
    """One call on ``stream`` (a torch stream; default: torch's current one),
    after the work already queued on torch's current stream."""
    desc, keep = cps.make_desc(design)
    hist = (cps.CpsStepOut * n)()
    nd = ctypes.c_int(0)
    torch = buf.torch
    if stream is not None:
        stream.wait_stream(torch.cuda.current_stream())
    stream = ctypes.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)
    st = lib.cps_solve_noalloc(ctypes.byref(desc), buf.pitch, buf.ptr(buf.alpha), buf.ptr(buf.gamma), buf.ptr(buf.u),
                               buf.ptr(buf.v), buf.ptr(buf.p), buf.ptr(buf.out["pStar"]), buf.ptr(buf.out["uStar"]),
                               buf.ptr(buf.out["vStar"]), buf.ptr(buf.out["dE"]), buf.ptr(buf.out["dN"]),
                               design.inletVelocity, n, eps, hist, ctypes.byref(nd), stream)
    assert st == cps.CPS_OK, st
    return cps.history_to_array(hist, nd.value)


@pytest.mark.parametrize("which,pitch_extra", [("network", 0), ("straight", 7)])
def test_noalloc_matches_allocating_entry_point_twice(which, pitch_extra):
    lib = cps.load_library()
    if which == "network":
        d = geometry.channel_network(M=64, N=130, h=20e-6, wmin=4, wmax=8, seed=3)
    else:
        d = geometry.straight_channel()
    rng = np.random.default_rng(4)
    init = {"u": rng.normal(0, 0.05, (d.M + 1, d.N)), "v": rng.normal(0, 0.02, (d.M, d.N + 1)),
            "p": rng.normal(0, 5.0, (d.M + 1, d.N + 1))}
    pitch = ((d.N + 1 + 31) // 32) * 32 + pitch_extra
    buf = CallerBuffers(d, pitch, init)
    with cps.Solver(d) as ref:
        ref.upload_fields(init["u"], init["v"], init["p"])
        for call in range(2):  # two calls in a row, each continuing from the last state
            h_ref = ref.solve(12, eps=0.0)
            f_ref = ref.download()
            h = call_noalloc(lib, d, buf, 12)
            f = buf.fields()
            assert h.shape == h_ref.shape
            assert np.array_equal(h[:, 5:], h_ref[:, 5:]), (call, h[:, 5:], h_ref[:, 5:])
            np.testing.assert_allclose(h[:, :5], h_ref[:, :5], rtol=1e-8, atol=1e-300)
            for k in OUT_FIELDS:
                assert rel(f[k], f_ref[k]) <= REL_STEP, (call, k, rel(f[k], f_ref[k]))


def test_noalloc_stops_at_convergence_like_cps_solve():
    lib = cps.load_library()
    d = geometry.straight_channel(M=20, N=40, band=(5, 15))
    zeros = {"u": np.zeros((d.M + 1, d.N)), "v": np.zeros((d.M, d.N + 1)), "p": np.zeros((d.M + 1, d.N + 1))}
    buf = CallerBuffers(d, 64, zeros)
    h = call_noalloc(lib, d, buf, 4000, eps=1e-6)
    with cps.Solver(d) as ref:
        h_ref = ref.solve(4000, eps=1e-6)
    assert len(h) == len(h_ref) < 4000


def test_noalloc_rejects_designs_beyond_the_static_scratch():
    lib = cps.load_library()
    d = geometry.straight_channel(M=600, N=300, band=(200, 400))
    desc, keep = cps.make_desc(d)
    nd = ctypes.c_int(-1)
    st = lib.cps_solve_noalloc(ctypes.byref(desc), 320, None, None, None, None, None, None, None, None, None, None,
                               0.1, 5, 0.0, None, ctypes.byref(nd), None)
    assert st == cps.CPS_ERR_ARG and nd.value == 0


def test_noalloc_ignores_padding_and_runs_on_the_callers_stream():
    """Caller buffers straight from a pool carry whatever the padding held
    before: with NaN in every element outside the logical matrices, on a
    non-default stream, two calls in a row still match cps_solve."""
    import torch
    lib = cps.load_library()
    d = geometry.channel_network(M=48, N=100, h=20e-6, wmin=4, wmax=8, seed=8)
    rng = np.random.default_rng(9)
    init = {"u": rng.normal(0, 0.05, (d.M + 1, d.N)), "v": rng.normal(0, 0.02, (d.M, d.N + 1)),
            "p": rng.normal(0, 5.0, (d.M + 1, d.N + 1))}
    pitch = ((d.N + 1 + 31) // 32) * 32 + 32
    buf = CallerBuffers(d, pitch, init, pad=float("nan"))
    side = torch.cuda.Stream()
    with cps.Solver(d) as ref:
        ref.upload_fields(init["u"], init["v"], init["p"])
        for call in range(2):
            h_ref = ref.solve(10, eps=0.0)
            f_ref = ref.download()
            h = call_noalloc(lib, d, buf, 10, stream=side)
            f = buf.fields()
            assert np.array_equal(h[:, 5:], h_ref[:, 5:]), (call, h[:, 5:], h_ref[:, 5:])
            np.testing.assert_allclose(h[:, :5], h_ref[:, :5], rtol=1e-8, atol=1e-300)
            for k in OUT_FIELDS:
                assert np.isfinite(f[k]).all(), (call, k)
                assert rel(f[k], f_ref[k]) <= REL_STEP, (call, k, rel(f[k], f_ref[k]))
