"""GPU parity at the benchmarked configurations, against committed FP64 oracle
singlepoints (tests/golden/parity_singlepoints.json, written by
make_parity_fixtures.py from oracle/liboracle.so).

* config-1 water clusters: the three largest (384 AOs) and five others;
* config-2 alkanes n = 20, 62, 120, 199 (122-1196 AOs) through the in-house
  batched eigensolver and with the automatic solver choice, in the plain FP64
  form and the mixed form;
* a 210-water cluster (1260 AOs), above the in-house bound: cuSOLVER path;
* an S-like element with s+p+d shells (test parameter file synthetic_hcos.tbp):
  integral matrices element-wise and full singlepoints, plus the reference's
  s-d transform0 known answer (src/test.old:152-176) on the GPU's on-site
  block.

Tolerances: plain FP64 form 1e-9 Eh, 1e-7 e, 1e-7 a.u. (and the oracle's SCF
iteration count); mixed form 1e-6 Eh at accuracy 1, charges and dipoles 1e-5 at
accuracy 0.01 (the charge spread of the default convergence threshold is
larger than the mixed form's tolerance, see test_gpu_mixed.py)."""
import os
import sys

import numpy as np
import pytest

from tblite_b200 import capi

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import make_parity_fixtures as fx  # noqa: E402

pytestmark = pytest.mark.gpu

E_TOL, Q_TOL, MU_TOL = 1e-9, 1e-7, 1e-7
E_TOL_MIXED, Q_TOL_MIXED, MU_TOL_MIXED = 1e-6, 1e-5, 1e-5

REC = fx.load()
CLUSTERS = [k for k in REC if k.startswith("water_clusters_1024")]
ALKANES = [k for k in REC if k.startswith("alkanes_256")]
S_SET = [k for k in REC if REC[k]["params"] == "hcos"]


@pytest.fixture(scope="module")
def calc_hcos():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return capi.Calculator(fx.PARAMS["hcos"])


@pytest.fixture(scope="module")
def oracle_hcos():
    import pyoracle
    return pyoracle.Oracle(fx.PARAMS["hcos"])


def _check(r, o, e_tol=E_TOL, q_tol=Q_TOL, mu_tol=MU_TOL, iterations=True):
    assert r["status"] == 0, capi.STATUS_NAMES.get(r["status"])
    assert abs(r["energy"] - o["energy"]) < e_tol, (r["energy"], o["energy"])
    np.testing.assert_allclose(r["qat"], o["qat"], atol=q_tol)
    np.testing.assert_allclose(r["dipole"], o["dipole"], atol=mu_tol)
    if iterations:
        assert r["iterations"] == o["iterations"]
    assert r["nao"] == o["nao"]


def _run(calc, names, **opts):
    mols = [fx.rebuild(REC[k]) for k in names]
    return calc.singlepoint_batch(mols, **opts)


def test_config1_clusters_fp64(gpu_calc):
    """Eight clusters of the benchmarked batch in one batch, largest 384 AOs."""
    for k, r in zip(CLUSTERS, _run(gpu_calc, CLUSTERS)):
        _check(r, REC[k]["acc1"])
        for c in ("e_rep", "e_band", "e_ts", "e_es2", "e_aes2", "e_es3"):
            assert abs(r[c] - REC[k]["acc1"][c]) < E_TOL, (k, c)


def test_config2_alkanes_fp64_inhouse(gpu_calc):
    """n = 20..199 (up to 1196 AOs) on the in-house eigensolver (solver = 1)."""
    for k, r in zip(ALKANES, _run(gpu_calc, ALKANES, solver=1)):
        _check(r, REC[k]["acc1"])


def test_config2_alkanes_fp64_automatic(gpu_calc):
    """The automatic per-size eigensolver choice gives the same results."""
    for k, r in zip(ALKANES, _run(gpu_calc, ALKANES)):
        _check(r, REC[k]["acc1"])


def test_above_inhouse_bound_cusolver_path(gpu_calc):
    """210 waters, 1260 AOs: above the in-house bound, so Xpotrf/Xtrtri/Xsyevd."""
    r = _run(gpu_calc, ["water_cluster_210"])[0]
    assert r["nao"] > 1216
    _check(r, REC["water_cluster_210"]["acc1"])


@pytest.mark.parametrize("which", ["clusters384", "alkanes"])
def test_mixed_energy_default_accuracy(gpu_calc, which):
    names = CLUSTERS[:3] if which == "clusters384" else ALKANES
    for k, r in zip(names, _run(gpu_calc, names, precision=1)):
        _check(r, REC[k]["acc1"], E_TOL_MIXED, 1e9, 1e9, iterations=False)


@pytest.mark.parametrize("which", ["clusters384", "alkanes"])
def test_mixed_charges_dipoles_accuracy_001(gpu_calc, which):
    names = CLUSTERS[:3] if which == "clusters384" else ALKANES
    for k, r in zip(names, _run(gpu_calc, names, precision=1, accuracy=0.01)):
        _check(r, REC[k]["acc001"], E_TOL_MIXED, Q_TOL_MIXED, MU_TOL_MIXED, iterations=False)


# ------------------------------------------------------------ d shells
@pytest.mark.parametrize("name", S_SET)
def test_d_shell_integrals(calc_hcos, oracle_hcos, name):
    """S, H0 (1e-12) and D, Q (1e-11) element-wise, every (l_i, l_j) pair up to d-d."""
    m = fx.rebuild(REC[name])
    S, H0, D, Q = capi.get_hamiltonian(calc_hcos, m)
    oS, oH0, oD, oQ = oracle_hcos.hamiltonian(m.id, m.xyz)
    np.testing.assert_allclose(S, oS, atol=1e-12)
    np.testing.assert_allclose(H0, oH0, atol=1e-12)
    np.testing.assert_allclose(D, oD, atol=1e-11)
    np.testing.assert_allclose(Q, oQ, atol=1e-11)


def test_d_shell_singlepoints(calc_hcos):
    for k, r in zip(S_SET, _run(calc_hcos, S_SET)):
        _check(r, REC[k]["acc1"])


def test_transform0_sd_known_answer_on_gpu(calc_hcos):
    """The reference's transform0 s-d case (src/test.old:152-176): an isotropic
    Cartesian d block (xx = yy = zz, mixed terms 0) transforms to a zero s-d
    spherical block.  On one atom with s and d shells that block is the on-site
    s-d overlap, which the GPU integrals must give as exactly zero (and the
    whole on-site overlap as the identity)."""
    from tblite_b200 import geometry as g
    atom = g.Molecule(np.array([fx.SPECIES_S], np.int32), np.zeros((1, 3)))
    S, H0, D, Q = capi.get_hamiltonian(calc_hcos, atom)
    assert S.shape == (9, 9)  # s (1) + p (3) + d (5)
    np.testing.assert_array_equal(S[0, 4:9], 0.0)
    np.testing.assert_array_equal(S[4:9, 0], 0.0)
    np.testing.assert_allclose(S, np.eye(9), atol=1e-14)
