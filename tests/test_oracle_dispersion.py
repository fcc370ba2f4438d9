"""CPU: the oracle's D4 dispersion (dispersion_get_engrad, src/xtb.cu:274-277,
a TODO in the reference; restated from the published D4 model at the neutral
reference charges) on the synthetic D4 parameter block: analytic gradient
against central finite differences of the energy, translational and
rotational invariance, the two-body limit at large separation, and the
singlepoint energy = electronic + repulsion + dispersion."""
import os

import numpy as np
import pytest

import pyoracle as po
from tblite_b200 import geometry as g

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
D4_PARAMS = os.path.join(ROOT, "tblite-cuda_b200", "params", "synthetic_hco_d4.tbp")


@pytest.fixture(scope="module")
def od4():
    return po.Oracle(D4_PARAMS)


def _mols():
    rng = np.random.default_rng(41)
    return [g.water_clusters(1, seed=42, nmin=5, nmax=5)[0], g.alkane(5, rng), g.octane()]


@pytest.mark.parametrize("k", [0, 1, 2])
def test_gradient_matches_finite_differences(od4, k):
    mol = _mols()[k]
    ids, xyz = np.array(mol.id), np.array(mol.xyz)
    e, grad, sigma = od4.dispersion(ids, xyz)
    h = 1e-4
    fd = np.zeros_like(grad)
    for a in range(len(ids)):
        for c in range(3):
            xp, xm = xyz.copy(), xyz.copy()
            xp[a, c] += h
            xm[a, c] -= h
            fd[a, c] = (od4.dispersion(ids, xp)[0].sum() - od4.dispersion(ids, xm)[0].sum()) / (2 * h)
    np.testing.assert_allclose(grad, fd, atol=2e-10)
    np.testing.assert_allclose(grad.sum(axis=0), 0.0, atol=1e-16)
    np.testing.assert_allclose(sigma, grad.T @ xyz, atol=1e-15)


def test_rotation_and_translation_invariance(od4):
    mol = _mols()[1]
    ids, xyz = np.array(mol.id), np.array(mol.xyz)
    e0 = od4.dispersion(ids, xyz)[0]
    q, _ = np.linalg.qr(np.random.default_rng(3).normal(size=(3, 3)))
    e1 = od4.dispersion(ids, xyz @ q.T + np.array([1.5, -2.0, 0.7]))[0]
    np.testing.assert_allclose(e1, e0, rtol=1e-12, atol=1e-16)
    assert e0.sum() < 0.0


def test_two_body_limit(od4):
    # two O atoms 30 Bohr apart (beyond the three-body and CN cutoffs' reach of
    # anything else): E = -C6 (s6 / (r^6 + R^6) + s8 q / (r^8 + R^8)) with the
    # CN = 0 reference weights, computed here from the file's data
    r = 30.0
    ids = np.array([2, 2], np.int32)
    xyz = np.array([[0.0, 0.0, 0.0], [r, 0.0, 0.0]])
    e = od4.dispersion(ids, xyz)[0].sum()
    lines = open(D4_PARAMS).read().splitlines()
    glob = {l.split()[1]: float(l.split()[2]) for l in lines if l.startswith("global d4_")}
    freq = np.array(next(l for l in lines if l.startswith("d4freq")).split()[2:], float)
    wts = np.array(next(l for l in lines if l.startswith("d4wts")).split()[2:], float)
    block = lines[lines.index("element O 8"):]  # the last element of the file
    refs = [np.array(l.split()[1:], float) for l in block if l.strip().startswith("d4_ref")]
    r4r2 = next(float(l.split()[1]) for l in block if l.strip().startswith("d4_r4r2"))
    cn_ref = np.array([x[0] for x in refs])
    # r is beyond the CN cutoff, so CN = 0 for both atoms
    w = np.exp(-glob["d4_wf"] * cn_ref ** 2)
    w /= w.sum()
    alpha = sum(wi * x[1:] for wi, x in zip(w, refs))
    c6 = 3.0 / np.pi * np.sum(wts * alpha * alpha)
    q = 3.0 * r4r2
    R = glob["d4_a1"] * np.sqrt(q) + glob["d4_a2"]
    ref = -c6 * (glob["d4_s6"] / (r ** 6 + R ** 6) + glob["d4_s8"] * q / (r ** 8 + R ** 8))
    assert abs(e - ref) < 1e-12 * abs(ref) + 1e-20


def test_singlepoint_includes_dispersion(od4):
    o0 = po.Oracle(os.path.join(ROOT, "tblite-cuda_b200", "params", "synthetic_hco.tbp"))
    mol = _mols()[0]
    a = od4.singlepoint(mol)
    b = o0.singlepoint(mol)
    e = od4.dispersion(np.array(mol.id), np.array(mol.xyz))[0].sum()
    assert od4.has_dispersion() and not o0.has_dispersion()
    assert b["e_disp"] == 0.0 and abs(a["e_disp"] - e) <= 1e-15 * abs(e)
    # the dispersion does not enter the SCF: everything else is the same bits
    assert a["e_elec"] == b["e_elec"] and a["iterations"] == b["iterations"]
    assert a["energy"] == a["e_elec"] + a["e_rep"] + a["e_disp"]
