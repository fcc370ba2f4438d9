"""GPU: D4 dispersion (dispersion_get_engrad, src/xtb.cu:274-277) from the
synthetic D4 parameter block, through the C ABI against the FP64 oracle:
per-atom energies and gradient of tb_dispersion, the singlepoint energy and
its analytic gradient with the dispersion term, a structure alone and in a
batch (same bits), and no dispersion without a D4 block."""
import os

import numpy as np
import pytest

from tblite_b200 import capi, geometry as g

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
D4_PARAMS = os.path.join(ROOT, "tblite-cuda_b200", "params", "synthetic_hco_d4.tbp")


@pytest.fixture(scope="module")
def calc_d4():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return capi.Calculator(D4_PARAMS)


@pytest.fixture(scope="module")
def orc_d4():
    import pyoracle
    return pyoracle.Oracle(D4_PARAMS)


def _mols():
    rng = np.random.default_rng(51)
    mols = g.water_clusters(4, seed=52, nmin=2, nmax=24)
    mols += [g.alkane(n, rng) for n in (3, 12, 30)]
    mols.append(g.octane())
    return mols


def test_dispersion_stage_matches_oracle(calc_d4, orc_d4):
    for mol in _mols():
        e, grad, sigma = capi.dispersion(calc_d4, mol)
        oe, og, osig = orc_d4.dispersion(np.array(mol.id), np.array(mol.xyz))
        np.testing.assert_allclose(e, oe, rtol=1e-12, atol=1e-15, err_msg=mol.label)
        np.testing.assert_allclose(grad, og, rtol=1e-10, atol=1e-14, err_msg=mol.label)
        np.testing.assert_allclose(sigma, osig, rtol=1e-10, atol=1e-14, err_msg=mol.label)
        assert e.sum() < 0.0


def test_singlepoint_energy_and_gradient_with_dispersion(calc_d4, orc_d4):
    mols = _mols()
    res = calc_d4.singlepoint_batch(mols, gradient=True)
    for mol, r in zip(mols, res):
        o = orc_d4.singlepoint_gradient(mol)
        os_ = orc_d4.singlepoint(mol)
        assert r["status"] == 0
        assert abs(r["e_disp"] - os_["e_disp"]) < 1e-12
        assert abs(r["energy"] - o["energy"]) < 1e-9
        assert r["energy"] == r["e_elec"] + r["e_rep"] + r["e_disp"]
        np.testing.assert_allclose(r["gradient"], o["gradient"], atol=1e-9, err_msg=mol.label)


def test_alone_equals_in_batch_with_dispersion(calc_d4):
    mols = _mols()
    batch = calc_d4.singlepoint_batch(mols)
    for m, r in zip(mols[::3], batch[::3]):
        alone = calc_d4.singlepoint_batch([m])[0]
        assert alone["e_disp"] == r["e_disp"] and alone["energy"] == r["energy"]


def test_no_dispersion_without_d4_block(gpu_calc):
    mol = g.octane()
    e, grad, _ = capi.dispersion(gpu_calc, mol)
    assert not e.any() and not grad.any()
    assert gpu_calc.singlepoint_batch([mol])[0]["e_disp"] == 0.0
