"""Allocation-free divergence (cfsa_ns_compute_divergence_noalloc) against the regular
computeDivergence entry point.

The no-alloc variant exists for callers that cannot allocate device memory when they call it:
hosts whose pool allocator has already reserved the whole device, and coupling loops where
cudaMalloc/cudaFree would synchronise the device on every call. It takes the caller's device
arrays and keeps its per-tet intermediate in a static device array; these checks call it through
the C ABI twice in a row (different inputs) and require the same bits as the regular operator,
whose own parity with the oracle is bit-exact. The call runs on the handle's stream, so the test
finishes writing the input (synchronize) before each call.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_TETS = 1 << 20


def make_solver(cf, rings, layers):
    m = cf.Mesh.cylinder(30.0, 2.0, rings, layers)
    m.setupBoundaryConditions((1.0, 0.0, 0.0), 1.0)
    s = cf.NavierStokesSolver()
    s.setDt(0.01)
    s.initialize(m, cf.Fluid(1060.0, 0.004))
    return s


def test_noalloc_divergence_matches_regular_entry_point(cf):
    import torch

    torch.cuda.set_device(0)
    s = make_solver(cf, 4, 20)
    lib = cf.load_library()
    rng = np.random.default_rng(7)
    for call in range(2):  # two calls in a row share the static scratch
        u = rng.standard_normal((s.N2, 3))
        expected = s.computeDivergence(u)
        u_dev = torch.tensor(np.ascontiguousarray(u.T), dtype=torch.float64, device="cuda")
        div_dev = torch.full((s.nv,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        code = lib.cfsa_ns_compute_divergence_noalloc(s._h, ctypes.c_void_p(u_dev.data_ptr()),
                                                      ctypes.c_void_p(div_dev.data_ptr()))
        assert code == cf.OK, lib.cfsa_ns_last_error(s._h).decode()
        got = div_dev.cpu().numpy()
        assert np.array_equal(got, expected), call


def test_noalloc_divergence_rejects_meshes_above_the_scratch_size(cf):
    import torch

    torch.cuda.set_device(0)
    s = make_solver(cf, 16, 228)  # 1,050,624 tets > 2^20
    assert s.nt > MAX_TETS
    lib = cf.load_library()
    u_dev = torch.zeros((3, s.N2), dtype=torch.float64, device="cuda")
    div_dev = torch.zeros(s.nv, dtype=torch.float64, device="cuda")
    code = lib.cfsa_ns_compute_divergence_noalloc(s._h, ctypes.c_void_p(u_dev.data_ptr()),
                                                  ctypes.c_void_p(div_dev.data_ptr()))
    assert code == cf.BAD_ARG
    assert "static scratch" in lib.cfsa_ns_last_error(s._h).decode()
