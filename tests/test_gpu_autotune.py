"""GPU: the per-size eigensolver variants and their measured choice.

Structures of at most 32 AOs may run on the one-warp Jacobi eigensolver
(k_syev_jacobi) instead of the one-CTA solver; the calculator measures both
once and picks per size.  Checked: the Jacobi variant forced on small
structures meets the plain FP64 bar against the oracle (1e-9 Eh, 1e-7 e, the
oracle's iteration count) and agrees with the one-CTA solver to 1e-10 Eh; the
measured mode records its table; results are the same bits alone and in a
batch mixing both variants; the mixed form's FP64 phase uses it too."""
import numpy as np
import pytest

from tblite_b200 import capi, geometry as g

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def calc():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return capi.Calculator(capi.DEFAULT_PARAMS)


def _small():
    rng = np.random.default_rng(41)
    o = g.octane()
    return [g.water_cluster(2, rng), g.water_cluster(5, rng), g.alkane(1, rng), g.alkane(2, rng),
            g.Molecule(np.array([0, 0], np.int32), np.array([[0, 0, 0], [0, 0, 1.4]], float)),
            g.Molecule(o.id[:8], o.xyz[:8], charge=1.0, uhf=1)]


def _check(r, o):
    assert r["status"] == 0, capi.STATUS_NAMES.get(r["status"])
    assert abs(r["energy"] - o["energy"]) < 1e-9
    np.testing.assert_allclose(r["qat"], o["qat"], atol=1e-7)
    assert r["iterations"] == o["iterations"]


def test_jacobi_variant_matches_oracle_and_cta_solver(calc, oracle):
    mols = _small()
    assert max(calc.basis_size(m)[1] for m in mols) <= 32
    calc.set_small_solver(32)
    jac = calc.singlepoint_batch(mols, accuracy=1e-4)
    calc.set_small_solver(0)
    cta = calc.singlepoint_batch(mols, accuracy=1e-4)
    for m, rj, rc in zip(mols, jac, cta):
        _check(rj, oracle.singlepoint(m, accuracy=1e-4))
        assert abs(rj["energy"] - rc["energy"]) < 1e-10
    calc.set_small_solver(-1)


def test_measured_choice_and_bits_alone_equal_in_batch(calc, oracle):
    calc.set_small_solver(-1)
    mols = _small() + g.water_clusters(3, seed=42, nmin=8, nmax=20)  # small and one-CTA structures
    batch = calc.singlepoint_batch(mols)
    t = calc.tuning()["small"]
    assert t["measured"] and [x["n"] for x in t["sizes"]] == [8, 12, 16, 20, 24, 28, 32]
    assert 0 <= t["jacobi_max"] <= 32
    assert all(x["s_per_structure_cta"] > 0 and x["s_per_structure_warp_jacobi"] > 0 for x in t["sizes"])
    for m, rb in zip(mols, batch):
        ra = calc.singlepoint_batch([m])[0]
        assert ra["energy"] == rb["energy"] and ra["iterations"] == rb["iterations"]
        np.testing.assert_array_equal(ra["qat"], rb["qat"])
        _check(rb, oracle.singlepoint(m))


def test_jacobi_in_mixed_form_fp64_phase(calc, oracle):
    calc.set_small_solver(32)
    mols = _small()
    for m, r in zip(mols, calc.singlepoint_batch(mols, precision=1, accuracy=0.01)):
        o = oracle.singlepoint(m, accuracy=0.01)
        assert r["status"] == 0 and abs(r["energy"] - o["energy"]) < 1e-6
        np.testing.assert_allclose(r["qat"], o["qat"], atol=1e-5)
    calc.set_small_solver(-1)


def test_bad_override_rejected(calc):
    with pytest.raises(capi.TBError):
        calc.set_small_solver(33)


# ---- FP64 GEMM tile shape (k_gemm 64 x 64 / k_gemm32 32 x 32)

def _tile_mols():
    rng = np.random.default_rng(43)
    mols = g.water_clusters(6, seed=44, nmin=2, nmax=40)  # 12..240 AOs
    mols += [g.alkane(n, rng) for n in (1, 5, 16, 40)]
    o = g.octane()
    mols.append(g.Molecule(o.id, o.xyz, charge=1.0, uhf=1))
    return mols


def _same(ra, rb):
    assert ra["status"] == rb["status"] == 0
    assert ra["energy"] == rb["energy"] and ra["iterations"] == rb["iterations"]
    np.testing.assert_array_equal(ra["qat"], rb["qat"])
    np.testing.assert_array_equal(ra["dipole"], rb["dipole"])


def test_gemm_tile_shapes_give_the_same_bits(calc, oracle):
    mols = _tile_mols()
    out = {}
    for shape, setting in (("64", 0), ("32", 100000)):
        calc.set_gemm_tiles(setting)
        out[shape] = (calc.singlepoint_batch(mols, gradient=True),
                      calc.singlepoint_batch(mols, precision=1, accuracy=0.01),
                      calc.singlepoint_batch(mols[-3:], nspin=2, wavefunction=True))
    calc.set_gemm_tiles(-1)
    for a, b in zip(out["64"][0], out["32"][0]):  # plain form with the gradient
        _same(a, b)
        np.testing.assert_array_equal(a["gradient"], b["gradient"])
    for a, b in zip(out["64"][1], out["32"][1]):  # mixed form: FP64 phase and refinement GEMMs
        _same(a, b)
    for a, b in zip(out["64"][2], out["32"][2]):  # open-shell density read-out
        np.testing.assert_array_equal(a["wfn"]["density"], b["wfn"]["density"])
    for m, r in zip(mols, out["32"][0]):
        o = oracle.singlepoint(m)
        assert abs(r["energy"] - o["energy"]) < 1e-9
        np.testing.assert_allclose(r["qat"], o["qat"], atol=1e-7)


def test_gemm_tile_measured_table_and_mixed_batch(calc):
    calc.set_gemm_tiles(-1)
    mols = _tile_mols()
    batch = calc.singlepoint_batch(mols)
    t = calc.tuning()["gemm_tiles"]
    assert t["measured"] and t["override"] == -1
    assert [x["n"] for x in t["sizes"]] == list(range(16, 385, 16))
    assert all(x["s_per_structure_64"] > 0 and x["s_per_structure_32"] > 0 for x in t["sizes"])
    assert all(x["tile"] == (32 if x["s_per_structure_32"] < x["s_per_structure_64"] else 64) for x in t["sizes"])
    # a threshold inside the batch splits it over both kernels: still the same bits
    calc.set_gemm_tiles(100)
    split = calc.singlepoint_batch(mols)
    calc.set_gemm_tiles(-1)
    for a, b in zip(batch, split):
        _same(a, b)


def test_bad_gemm_tile_override_rejected(calc):
    with pytest.raises(capi.TBError):
        calc.set_gemm_tiles(-2)
