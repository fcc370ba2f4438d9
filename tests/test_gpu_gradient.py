"""GPU: analytic nuclear gradient and virial (the gradient/sigma outputs of
xtb_singlepoint, src/xtb.cu:195-196), through the C ABI.

* against the oracle's analytic gradient on the same inputs, element-wise
  within 1e-9 Eh/Bohr (sigma 1e-8): water clusters, an open-shell cation, the
  s+p+d test element and a 384-AO cluster of the benchmarked batch;
* against central finite differences of the oracle energy (h = 1e-4 Bohr,
  SCF at accuracy 1e-7) within 1e-7 Eh/Bohr;
* translational invariance, the device-resident batch entry point, and the
  same bits alone and in a batch."""
import os
import sys

import numpy as np
import pytest

from tblite_b200 import capi, geometry as g

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import make_parity_fixtures as fx  # noqa: E402

pytestmark = pytest.mark.gpu

G_TOL, SIGMA_TOL = 1e-9, 1e-8


def _mols():
    rng = np.random.default_rng(31)
    o = g.octane()
    return [g.water_cluster(2, rng), g.water_cluster(12, rng), g.Molecule(o.id, o.xyz, charge=1.0, uhf=1),
            g.alkane(3, rng)]


def _check(r, o):
    assert r["status"] == 0 and o["status"] == 0
    assert abs(r["energy"] - o["energy"]) < 1e-9
    np.testing.assert_allclose(r["gradient"], o["gradient"], atol=G_TOL)
    np.testing.assert_allclose(r["sigma"], o["sigma"], atol=SIGMA_TOL)
    np.testing.assert_allclose(r["gradient"].sum(0), 0.0, atol=1e-10)


def test_gradient_matches_oracle(gpu_calc, oracle):
    mols = _mols()
    res = gpu_calc.singlepoint_batch(mols, accuracy=1e-4, gradient=True)
    for m, r in zip(mols, res):
        _check(r, oracle.singlepoint_gradient(m, accuracy=1e-4))


def test_gradient_d_shells():
    import pyoracle
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    calc = capi.Calculator(fx.PARAMS["hcos"])
    orc = pyoracle.Oracle(fx.PARAMS["hcos"])
    rec = fx.load()
    mols = [fx.rebuild(rec[k]) for k in ("dimethyl_sulfide", "water_cluster_8_h2s")]
    for m, r in zip(mols, calc.singlepoint_batch(mols, accuracy=1e-4, gradient=True)):
        _check(r, orc.singlepoint_gradient(m, accuracy=1e-4))


def test_gradient_benchmark_cluster(gpu_calc, oracle):
    m = fx.rebuild(fx.load()["water_clusters_1024[1019]"])  # 64 waters, 384 AOs
    r = gpu_calc.singlepoint_batch([m], gradient=True)[0]
    _check(r, oracle.singlepoint_gradient(m))


def test_gradient_finite_differences(gpu_calc, oracle):
    m = _mols()[0]
    r = gpu_calc.singlepoint_batch([m], accuracy=1e-7, gradient=True)[0]
    h, fd = 1e-4, np.zeros((m.nat, 3))
    for a in range(m.nat):
        for k in range(3):
            xp, xm = m.xyz.copy(), m.xyz.copy()
            xp[a, k] += h
            xm[a, k] -= h
            fd[a, k] = (oracle.singlepoint(g.Molecule(m.id, xp), accuracy=1e-7)["energy"] -
                        oracle.singlepoint(g.Molecule(m.id, xm), accuracy=1e-7)["energy"]) / (2 * h)
    np.testing.assert_allclose(r["gradient"], fd, atol=1e-7)


def test_gradient_alone_equals_in_batch_and_batch_api(gpu_calc):
    mols = g.water_clusters(5, seed=91, nmin=3, nmax=14)
    batch = gpu_calc.singlepoint_batch(mols, gradient=True)
    for m, rb in zip(mols, batch):
        ra = gpu_calc.singlepoint_batch([m], gradient=True)[0]
        np.testing.assert_array_equal(ra["gradient"], rb["gradient"])
        np.testing.assert_array_equal(ra["sigma"], rb["sigma"])
    b = capi.Batch(gpu_calc, mols)
    b.run()
    gg, sg = b.gradient()
    off = np.cumsum([0] + [m.nat for m in mols])
    for i, rb in enumerate(batch):
        np.testing.assert_array_equal(gg[off[i]:off[i + 1]], rb["gradient"])
        np.testing.assert_array_equal(sg[i], rb["sigma"])
