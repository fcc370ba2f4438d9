"""GPU: the mixed-precision form (tb_options.precision = 1) against the FP64
oracle.  Tolerances of the mixed form: total energy 1e-6 Eh, atomic charges
1e-5 e, dipole 1e-5 a.u.  At the default accuracy the SCF stops once the RMS
charge change of an iteration is below 2e-5, so two correct FP64 runs that take
different paths to the fixed point (another mixer damping is enough) already
differ by up to ~1e-4 e in single charges while their energies agree to 1e-8
Eh.  Charges and dipoles are therefore compared at accuracy 0.01 (charge
threshold 2e-7), energies at both accuracies."""
import numpy as np
import pytest

from tblite_b200 import capi, geometry as g

pytestmark = pytest.mark.gpu

E_TOL, Q_TOL, MU_TOL = 1e-6, 1e-5, 1e-5


def _check(r, o):
    assert r["status"] == 0, capi.STATUS_NAMES.get(r["status"])
    assert abs(r["energy"] - o["energy"]) < E_TOL, (r["energy"], o["energy"])
    np.testing.assert_allclose(r["qat"], o["qat"], atol=Q_TOL)
    np.testing.assert_allclose(r["dipole"], o["dipole"], atol=MU_TOL)


def test_mixed_water_batch_energy_default_accuracy(gpu_calc, oracle):
    mols = g.water_clusters(12, seed=1001, nmin=2, nmax=24)
    res = gpu_calc.singlepoint_batch(mols, precision=1)
    for m, r in zip(mols, res):
        assert r["status"] == 0
        assert abs(r["energy"] - oracle.singlepoint(m)["energy"]) < E_TOL


def test_mixed_water_batch_vs_oracle(gpu_calc, oracle):
    mols = g.water_clusters(12, seed=1001, nmin=2, nmax=24)
    res = gpu_calc.singlepoint_batch(mols, precision=1, accuracy=0.01)
    for m, r in zip(mols, res):
        _check(r, oracle.singlepoint(m, accuracy=0.01))


def test_mixed_small_charged_open_shell(gpu_calc, oracle):
    m = g.octane()
    mols = [m, g.Molecule(m.id, m.xyz, charge=1.0, uhf=1),
            g.Molecule(np.array([0, 0], np.int32), np.array([[0, 0, 0], [0, 0, 1.4]], float)),
            g.alkane(1, np.random.default_rng(1))]
    res = gpu_calc.singlepoint_batch(mols, precision=1, accuracy=0.01)
    for mol, r in zip(mols, res):
        _check(r, oracle.singlepoint(mol, accuracy=0.01))


def test_mixed_agrees_with_plain(gpu_calc):
    mols = g.water_clusters(8, seed=33, nmin=8, nmax=40) + [g.alkane(12, np.random.default_rng(4))]
    a = gpu_calc.singlepoint_batch(mols, precision=0, accuracy=0.01)
    b = gpu_calc.singlepoint_batch(mols, precision=1, accuracy=0.01)
    for ra, rb in zip(a, b):
        assert ra["status"] == rb["status"] == 0
        assert abs(ra["energy"] - rb["energy"]) < E_TOL
        np.testing.assert_allclose(ra["qat"], rb["qat"], atol=Q_TOL)
        # the mixed phase is followed by at least two FP64 iterations
        assert rb["iterations"] >= 3


def test_mixed_library_fp32_path(gpu_calc, oracle):
    # solver = 2 sends every structure through cuSOLVER, here its FP32 eigensolver + refinement
    mols = g.water_clusters(3, seed=44, nmin=2, nmax=10)
    res = gpu_calc.singlepoint_batch(mols, precision=1, solver=2, accuracy=0.01)
    for m, r in zip(mols, res):
        _check(r, oracle.singlepoint(m, accuracy=0.01))


def test_mixed_alone_equals_in_batch(gpu_calc):
    mols = g.water_clusters(5, seed=55, nmin=3, nmax=16)
    batch = gpu_calc.singlepoint_batch(mols, precision=1)
    for m, rb in zip(mols, batch):
        ra = gpu_calc.singlepoint_batch([m], precision=1)[0]
        assert ra["energy"] == rb["energy"] and ra["iterations"] == rb["iterations"]
        np.testing.assert_array_equal(ra["qat"], rb["qat"])


def test_bad_precision_rejected(gpu_calc):
    with pytest.raises(capi.TBError) as e:
        gpu_calc.singlepoint_batch([g.octane()], precision=3)
    assert e.value.status == capi.TB_BAD_INPUT
