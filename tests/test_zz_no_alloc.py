"""The allocation-free eigensolver entry point, tb_sygvd_noalloc.

It exists for callers that cannot let a library allocate device memory (for
example a framework that owns all GPU memory through its own pool, or a
latency-critical loop where cudaMalloc would synchronise the device).  The
tests allocate the caller-owned device buffers themselves (with torch) and call
the entry point through the C ABI:

* in this process, on three problems in a row, each result checked against the
  allocating entry point tb_sygvd_batch within the eigensolver tolerance of the
  other GPU tests (1e-10), and against numpy;
* in fresh processes whose first library call is tb_sygvd_noalloc (n = 1, 64,
  200 and 256; from n = 237 on the eigensolver needs more than the default
  48 KiB of shared memory, which the first call's set-up provides), two calls in
  a row each, checked against numpy's eigenvalues of S^-1/2 H S^-1/2 and
  against C^T S C = I and H C = S C diag(w).

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from tblite_b200 import capi

pytestmark = pytest.mark.gpu

TOL = 1e-10
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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


def _numpy_check(H, S, w, Cm):
    """Largest deviations from numpy's eigenvalues, from S-orthonormality and
    from the eigen-equation."""
    n = H.shape[0]
    e, U = np.linalg.eigh(S)
    Sih = (U / np.sqrt(e)) @ U.T
    ref = np.linalg.eigvalsh(Sih @ H @ Sih)
    return {"dw": float(np.max(np.abs(w - ref))),
            "orth": float(np.max(np.abs(Cm.T @ S @ Cm - np.eye(n)))),
            "resid": float(np.max(np.abs(H @ Cm - S @ Cm * w[None, :])))}


def test_noalloc_matches_allocating_entry_point_in_a_row():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    for n, seed in ((256, 3), (200, 1), (37, 2)):  # calls in a row, different sizes
        H, S = _problem(n, seed)
        st, w, Cm = _noalloc(torch, H, S)
        assert st == capi.TB_OK, capi.last_error()
        rst, ref = capi.sygvd_batch([H], [S])
        assert rst == capi.TB_OK
        np.testing.assert_allclose(w, ref[0][0], atol=TOL)
        np.testing.assert_allclose(Cm, ref[0][1], atol=TOL)
        chk = _numpy_check(H, S, w, Cm)
        assert max(chk.values()) < TOL, chk


_CHILD = r"""
import json, sys
import torch
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[2])
from tblite_b200 import capi
import test_zz_no_alloc as t
n = int(sys.argv[3])
out = []
for seed in (11, 12):  # the first tblite-b200 call of this process, then a second one
    H, S = t._problem(n, seed)
    st, w, Cm = t._noalloc(torch, H, S)
    rec = {"status": int(st), "error": capi.last_error() if st else ""}
    if st == 0:
        rec.update(t._numpy_check(H, S, w, Cm))
    out.append(rec)
print("RESULT " + json.dumps(out))
"""


@pytest.mark.parametrize("n", [1, 64, 200, 256])
def test_noalloc_first_call_in_a_fresh_process(n):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pkg = os.path.join(ROOT, "tblite-cuda_b200")
    here = os.path.join(ROOT, "tests")
    p = subprocess.run([sys.executable, "-c", _CHILD, pkg, here, str(n)], capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    line = [s for s in p.stdout.splitlines() if s.startswith("RESULT ")]
    assert line, p.stdout[-2000:] + p.stderr[-2000:]
    for rec in json.loads(line[-1][len("RESULT "):]):
        assert rec["status"] == capi.TB_OK, rec
        assert max(rec["dw"], rec["orth"], rec["resid"]) < TOL, rec


def test_noalloc_rejects_sizes_beyond_the_static_limit():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = capi.load_library()
    st = L.tb_sygvd_noalloc(C.c_int32(257), C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                            C.c_void_p(0))
    assert st == capi.TB_CAPACITY_EXCEEDED
    assert "1..256" in capi.last_error()
