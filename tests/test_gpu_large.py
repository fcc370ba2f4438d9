"""GPU: the library (cuSOLVER) path for structures above the in-house
eigensolver's size bound (1216 AOs).

The path is pinned against the FP64 oracle by forcing it for small structures
(tb_options.solver = 2), where the oracle finishes in seconds; at the 6000-AO
water box, where it does not, the checks are size-independent: SCF
convergence, charge conservation and agreement of the two solver paths on the
quantities they share.  Tolerances as in test_gpu_parity (1e-9 Eh, 1e-7 e)."""
import numpy as np
import pytest

from tblite_b200 import capi, geometry as g

pytestmark = pytest.mark.gpu

E_TOL, Q_TOL, MU_TOL = 1e-9, 1e-7, 1e-7


def _check(r, o):
    assert r["status"] == 0, capi.STATUS_NAMES.get(r["status"])
    assert abs(r["energy"] - o["energy"]) < E_TOL, (r["energy"], o["energy"])
    np.testing.assert_allclose(r["qat"], o["qat"], atol=Q_TOL)
    np.testing.assert_allclose(r["dipole"], o["dipole"], atol=MU_TOL)


def test_library_solver_matches_oracle(gpu_calc, oracle):
    mols = [g.octane()] + g.water_clusters(3, seed=21, nmin=2, nmax=12)
    res = gpu_calc.singlepoint_batch(mols, accuracy=1e-4, solver=2)
    for m, r in zip(mols, res):
        o = oracle.singlepoint(m, accuracy=1e-4)
        _check(r, o)
        assert r["iterations"] == o["iterations"]


def test_library_and_inhouse_agree(gpu_calc):
    mols = g.water_clusters(6, seed=22, nmin=4, nmax=30)
    a = gpu_calc.singlepoint_batch(mols, solver=1)
    b = gpu_calc.singlepoint_batch(mols, solver=2)
    for ra, rb in zip(a, b):
        assert ra["status"] == rb["status"] == 0
        assert abs(ra["energy"] - rb["energy"]) < E_TOL
        np.testing.assert_allclose(ra["qat"], rb["qat"], atol=Q_TOL)


def test_inhouse_only_rejects_above_bound(gpu_calc):
    box = g.water_box()
    with pytest.raises(capi.TBError) as e:
        gpu_calc.singlepoint_batch([box], solver=1)
    assert e.value.status == capi.TB_CAPACITY_EXCEEDED
    with pytest.raises(capi.TBError) as e:
        gpu_calc.singlepoint_batch([g.octane()], solver=7)
    assert e.value.status == capi.TB_BAD_INPUT


def test_sygvd_above_bound_mixed_batch():
    rng = np.random.default_rng(5)
    sizes = [1300, 40]  # one matrix on the library path, one on the in-house kernels
    Hs, Ss = [], []
    for n in sizes:
        M = rng.normal(size=(n, n))
        R = rng.normal(size=(n, n))
        Hs.append(0.5 * (M + M.T))
        Ss.append(R @ R.T / n + np.eye(n))
    st, out = capi.sygvd_batch(Hs, Ss)
    assert st == capi.TB_OK
    for H, S, (w, C) in zip(Hs, Ss, out):
        assert np.all(np.diff(w) >= 0)
        np.testing.assert_allclose(C.T @ S @ C, np.eye(len(w)), atol=1e-9)
        np.testing.assert_allclose(H @ C, S @ C * w, atol=1e-8)
        ref = np.linalg.eigvalsh(np.linalg.solve(np.linalg.cholesky(S), np.linalg.solve(np.linalg.cholesky(S), H).T))
        np.testing.assert_allclose(w, ref, atol=1e-9)


def test_sygvd_above_bound_not_spd():
    n = 1250
    st, _ = capi.sygvd_batch([np.eye(n)], [-np.eye(n)])
    assert st == capi.TB_NOT_SPD


def test_water_box_6000_aos(gpu_calc):
    box = g.water_box()
    nsh, nao = gpu_calc.basis_size(box)
    assert nao == 6000
    r = gpu_calc.singlepoint_batch([box])[0]
    assert r["status"] == 0, capi.STATUS_NAMES.get(r["status"])
    assert np.isfinite(r["energy"]) and 2 <= r["iterations"] < 32
    assert abs(r["qat"].sum() - box.charge) < 1e-8   # Mulliken charges conserve the total charge
    assert abs(r["qsh"].sum() - box.charge) < 1e-8
    # rigid, nearly neutral waters: each molecule's net charge stays small
    qmol = r["qat"].reshape(-1, 3).sum(axis=1)
    assert np.max(np.abs(qmol)) < 0.2


def test_automatic_solver_choice_matches_inhouse(gpu_calc):
    # a few large alkanes among small structures: the automatic choice (timed
    # cost models) may send the large ones to cuSOLVER; results must agree
    rng = np.random.default_rng(9)
    mols = [g.alkane(n, rng) for n in (140, 160)] + g.water_clusters(4, seed=31, nmin=4, nmax=12)
    auto = gpu_calc.singlepoint_batch(mols, solver=0)
    inhouse = gpu_calc.singlepoint_batch(mols, solver=1)
    for a, b in zip(auto, inhouse):
        assert a["status"] == b["status"] == 0
        assert abs(a["energy"] - b["energy"]) < E_TOL
        np.testing.assert_allclose(a["qat"], b["qat"], atol=Q_TOL)
