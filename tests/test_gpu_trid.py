"""GPU: the Householder tridiagonalisation held in the shared memory of a
thread block cluster (k_trid_smem, clusters of 1, 2, 3, 4, 6 and 8 CTAs by
size, 64-560 AOs), ahead of k_syev.  Generalized eigenproblems at the sizes
around every class boundary against numpy (tb_sygvd_batch always uses it),
and singlepoints with it (tb_calculator_set_smem_tridiag, off by default)
against the one-CTA reduction of the same structures."""
import numpy as np
import pytest

from tblite_b200 import capi, geometry as g

pytestmark = pytest.mark.gpu

# the largest order of each cluster class and the first order of the next
BOUNDARY_SIZES = [64, 100, 208, 209, 288, 289, 352, 353, 400, 401, 480, 481, 560, 561]


def test_sygvd_across_cluster_classes():
    rng = np.random.default_rng(21)
    Hs, Ss = [], []
    for k, n in enumerate(BOUNDARY_SIZES):
        M = rng.normal(size=(n, n))
        Hs.append(0.5 * (M + M.T))
        if k % 2:
            R = rng.normal(size=(n, n))
            Ss.append(R @ R.T / n + np.eye(n))
        else:
            Ss.append(np.eye(n))
    st, out = capi.sygvd_batch(Hs, Ss)
    assert st == capi.TB_OK
    for H, S, (w, C) in zip(Hs, Ss, out):
        n = len(w)
        ref = np.linalg.eigvalsh(np.linalg.solve(np.linalg.cholesky(S), np.linalg.solve(np.linalg.cholesky(S), H).T))
        scale = max(1.0, np.max(np.abs(ref)))
        np.testing.assert_allclose(w, ref, atol=1e-12 * scale * n ** 0.5, err_msg=f"n={n}")
        np.testing.assert_allclose(C.T @ S @ C, np.eye(n), atol=1e-11, err_msg=f"n={n}")
        np.testing.assert_allclose(H @ C, S @ C * w, atol=1e-11 * scale * n ** 0.5, err_msg=f"n={n}")


def test_sygvd_degenerate_and_decoupled_in_clusters():
    # an 8-fold degenerate spectrum (zero sigma steps appear late) and a
    # block-diagonal matrix (zero columns below the band from the start) in
    # the 2- and 4-CTA classes, and a multiple of the identity (every
    # reflector trivial) in the 3-CTA class
    rng = np.random.default_rng(23)
    n = 264
    Qm, _ = np.linalg.qr(rng.normal(size=(n, n)))
    Hs = [Qm @ np.diag(np.repeat(np.arange(n // 8, dtype=float), 8)) @ Qm.T]
    blocks = [rng.normal(size=(96, 96)) for _ in range(4)]
    Bd = np.zeros((384, 384))
    for i, b in enumerate(blocks):
        Bd[96 * i:96 * i + 96, 96 * i:96 * i + 96] = b + b.T
    Hs.append(Bd)
    Hs.append(-0.75 * np.eye(320))
    st, out = capi.sygvd_batch(Hs, [np.eye(len(H)) for H in Hs])
    assert st == capi.TB_OK
    for H, (w, C) in zip(Hs, out):
        nn = len(w)
        scale = max(1.0, np.max(np.abs(H)))
        np.testing.assert_allclose(w, np.linalg.eigvalsh(H), atol=1e-12 * scale * nn ** 0.5)
        np.testing.assert_allclose(C.T @ C, np.eye(nn), atol=1e-12)
        np.testing.assert_allclose(H @ C, C * w, atol=1e-12 * scale * nn ** 0.5)


def _mols():
    rng = np.random.default_rng(31)
    mols = g.water_clusters(12, seed=1001, nmin=8, nmax=64)        # 48-384 AOs: classes 1-4
    mols += [g.alkane(n, rng) for n in (72, 78, 90)]              # 434, 470, 542 AOs: classes 6, 8
    mols += [g.water_cluster(n, rng) for n in (10, 35, 47, 59)]   # 60, 210, 282, 354 AOs
    return mols


def test_singlepoints_equal_the_one_cta_reduction(gpu_calc):
    mols = _mols()
    tun = gpu_calc.tuning()["smem_tridiag"]
    assert tun["min_n"] == 0 and [c["cluster"] for c in tun["classes"]] == [1, 2, 3, 4, 6, 8]
    assert max(c["smem_bytes"] for c in tun["classes"]) <= 227 * 1024
    slow = gpu_calc.singlepoint_batch(mols, solver=1)
    gpu_calc.set_smem_tridiag(True)
    try:
        assert gpu_calc.tuning()["smem_tridiag"]["min_n"] == 64
        fast = gpu_calc.singlepoint_batch(mols, solver=1)
    finally:
        gpu_calc.set_smem_tridiag(False)
    # the two reductions differ by rounding only: the plain form's parity bar
    for a, b in zip(fast, slow):
        assert a["status"] == b["status"] == 0
        assert abs(a["energy"] - b["energy"]) < 1e-9
        np.testing.assert_allclose(a["qat"], b["qat"], atol=1e-7)
        np.testing.assert_allclose(a["dipole"], b["dipole"], atol=1e-7)


def test_size_threshold(gpu_calc):
    # min_n = 353: only the 4-, 6- and 8-CTA classes take the cluster
    # reduction, the smaller structures the one-CTA kernel, in one batch
    mols = _mols()
    ref = gpu_calc.singlepoint_batch(mols, solver=1)
    gpu_calc.set_smem_tridiag(353)
    try:
        got = gpu_calc.singlepoint_batch(mols, solver=1)
    finally:
        gpu_calc.set_smem_tridiag(0)
    for a, b, m in zip(got, ref, mols):
        assert a["status"] == b["status"] == 0
        assert abs(a["energy"] - b["energy"]) < 1e-9
        if gpu_calc.basis_size(m)[1] < 353:  # reduced by the same kernel: the same bits
            assert a["energy"] == b["energy"]


def test_alone_equals_in_batch_with_clusters(gpu_calc):
    # the class (cluster size) of a structure depends on its size only
    mols = _mols()
    gpu_calc.set_smem_tridiag(True)
    try:
        batch = gpu_calc.singlepoint_batch(mols, solver=1)
        for m, r in zip(mols[-5:], batch[-5:]):
            alone = gpu_calc.singlepoint_batch([m], solver=1)[0]
            assert alone["energy"] == r["energy"] and alone["iterations"] == r["iterations"]
            np.testing.assert_array_equal(alone["qat"], r["qat"])
    finally:
        gpu_calc.set_smem_tridiag(False)
