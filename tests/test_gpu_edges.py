"""GPU: edge cases of the boundary -- empty and malformed inputs, a ragged
batch from one atom to hundreds of atoms, and the in-house eigensolver at its
largest accepted size -- through the C ABI."""
import numpy as np
import pytest

from tblite_b200 import capi, geometry as g

pytestmark = pytest.mark.gpu


def test_empty_and_malformed_inputs(gpu_calc):
    with pytest.raises(capi.TBError) as e:
        gpu_calc.singlepoint_batch([])
    assert e.value.status == capi.TB_BAD_INPUT
    with pytest.raises(capi.TBError) as e:  # a structure with no atoms
        gpu_calc.singlepoint_batch([g.Molecule(np.zeros(0, np.int32), np.zeros((0, 3)))])
    assert e.value.status == capi.TB_BAD_INPUT
    with pytest.raises(capi.TBError) as e:  # infinite coordinate
        gpu_calc.singlepoint_batch([g.Molecule(np.array([0, 0], np.int32), np.array([[0, 0, 0], [0, 0, np.inf]]))])
    assert e.value.status == capi.TB_BAD_INPUT


def test_ragged_batch_one_atom_to_hundreds(gpu_calc, oracle):
    """Sizes 1 to 302 atoms (1 to 602 AOs) in one batch: every structure at the
    plain bar against the oracle, each on its own size's eigensolver variant."""
    rng = np.random.default_rng(61)
    mols = [g.Molecule(np.array([0], np.int32), np.zeros((1, 3)), uhf=1),
            g.Molecule(np.array([2], np.int32), np.zeros((1, 3))),
            g.alkane(1, rng), g.water_cluster(3, rng), g.alkane(10, rng), g.water_cluster(40, rng),
            g.alkane(100, rng)]
    res = gpu_calc.singlepoint_batch(mols, accuracy=1e-4)
    for m, r in zip(mols, res):
        o = oracle.singlepoint(m, accuracy=1e-4)
        assert r["status"] == 0 and o["status"] == 0
        assert abs(r["energy"] - o["energy"]) < 1e-9
        np.testing.assert_allclose(r["qat"], o["qat"], atol=1e-7)
        assert r["iterations"] == o["iterations"]


def test_eigensolver_at_the_inhouse_limit():
    """n = 1216, the largest size of the in-house batched eigensolver, next to a
    small problem in the same batch: eigenvalues against numpy, S-orthonormal
    vectors and the eigen-equation."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(62)
    Hs, Ss = [], []
    for n in (1216, 17):
        M = rng.normal(size=(n, n))
        R = rng.normal(size=(n, n))
        Hs.append(0.5 * (M + M.T) / np.sqrt(n))
        Ss.append(R @ R.T / n + np.eye(n))
    st, res = capi.sygvd_batch(Hs, Ss)
    assert st == capi.TB_OK
    for H, S, (w, Cm) in zip(Hs, Ss, res):
        e, U = np.linalg.eigh(S)
        Sih = (U / np.sqrt(e)) @ U.T
        np.testing.assert_allclose(w, np.linalg.eigvalsh(Sih @ H @ Sih), atol=1e-10)
        np.testing.assert_allclose(Cm.T @ S @ Cm, np.eye(len(w)), atol=1e-9)
        np.testing.assert_allclose(H @ Cm, S @ Cm * w[None, :], atol=1e-9)
