"""The allocation-free eigensolver entry point, tb_sygvd_noalloc.

It exists for callers that cannot let a library allocate device memory (for
example a framework that owns all GPU memory through its own pool, or a
latency-critical loop where cudaMalloc would synchronise the device).  The
test allocates the caller-owned device buffers itself (with torch), calls the
entry point through the C ABI twice in a row on different problems, and checks
each result against the allocating entry point tb_sygvd_batch within the
eigensolver tolerance used by the other GPU tests (1e-10)."""
import ctypes as C

import numpy as np
import pytest

from tblite_b200 import capi

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _problem(n, seed):
    rng = np.random.default_rng(seed)
    M = rng.normal(size=(n, n))
    R = rng.normal(size=(n, n))
    return 0.5 * (M + M.T), R @ R.T / n + np.eye(n)


def _noalloc(torch, H, S):
    L = capi.load_library()
    n = H.shape[0]
    dH = torch.tensor(H, dtype=torch.float64, device="cuda").contiguous()
    dS = torch.tensor(S, dtype=torch.float64, device="cuda").contiguous()
    dw = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    dC = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = L.tb_sygvd_noalloc(C.c_int32(n), C.c_void_p(dH.data_ptr()), C.c_void_p(dS.data_ptr()),
                            C.c_void_p(dw.data_ptr()), C.c_void_p(dC.data_ptr()), C.c_void_p(stream))
    torch.cuda.synchronize()
    return st, dw.cpu().numpy(), dC.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    for n, seed in ((200, 1), (37, 2)):  # two calls in a row, different sizes
        H, S = _problem(n, seed)
        st, w, Cm = _noalloc(torch, H, S)
        assert st == capi.TB_OK, capi.last_error()
        rst, ref = capi.sygvd_batch([H], [S])
        assert rst == capi.TB_OK
        np.testing.assert_allclose(w, ref[0][0], atol=TOL)
        np.testing.assert_allclose(Cm, ref[0][1], atol=TOL)
        np.testing.assert_allclose(Cm.T @ S @ Cm, np.eye(n), atol=TOL)


def test_noalloc_rejects_sizes_beyond_the_static_limit():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = capi.load_library()
    st = L.tb_sygvd_noalloc(C.c_int32(257), C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                            C.c_void_p(0))
    assert st == capi.TB_CAPACITY_EXCEEDED
    assert "1..256" in capi.last_error()
