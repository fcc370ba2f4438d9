"""GPU: the wavefunction half of the boundary (tb_wavefunction, the reference's
wavefunction_type& wfn argument of xtb_singlepoint, src/xtb.cu:188-197 and
src/wavefunction/type.h:81-99), through the C ABI.

* outputs against the FP64 oracle: orbital energies, occupations and density
  within 1e-9; the coefficients are not compared (their signs and rotations
  inside degenerate sets are arbitrary) but checked for C^T S C = I and
  C diag(f) C^T = P;
* warm start: a singlepoint started from the moments of an earlier result
  converges in fewer iterations to the same energy (1e-9 Eh) and charges
  (1e-7 e); structures without a guess in the same batch are unchanged."""
import numpy as np
import pytest

from tblite_b200 import capi, geometry as g

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _mols():
    rng = np.random.default_rng(21)
    o = g.octane()
    return [o, g.water_cluster(20, rng), g.Molecule(o.id, o.xyz, charge=1.0, uhf=1)]


@pytest.mark.parametrize("idx", range(3))
def test_wavefunction_outputs_match_oracle(gpu_calc, oracle, idx):
    m = _mols()[idx]
    r = gpu_calc.singlepoint_batch([m], accuracy=1e-4, wavefunction=True)[0]
    o = oracle.singlepoint(m, accuracy=1e-4)
    assert r["status"] == 0 and r["iterations"] == o["iterations"]
    w = r["wfn"]
    nsh, nao = gpu_calc.basis_size(m)
    assert (w["nspin"], w["nat"], w["nsh"], w["nao"]) == (1, m.nat, nsh, nao)
    np.testing.assert_allclose(w["emo"], o["emo"], atol=TOL)
    assert np.all(np.diff(w["emo"]) >= 0.0)
    np.testing.assert_allclose(w["density"], o["P"], atol=TOL)
    # occupations: the oracle's Fermi filling of the oracle's orbital energies, per channel
    focc = np.zeros(nao)
    for s in range(2):
        st, occ, _, _ = oracle.fermi(w["nel"][s], w["kt"], o["emo"])
        assert st == 0
        focc += occ
    np.testing.assert_allclose(w["focc"], focc, atol=TOL)
    assert abs(w["focc"].sum() - w["nocc"]) < 1e-9
    assert abs(w["nel"][0] - w["nel"][1] - w["nuhf"]) < 1e-12
    assert w["homo"] == [int(np.floor(x)) for x in w["nel"]]
    # moments and reference occupations
    np.testing.assert_array_equal(w["qat"], r["qat"])
    np.testing.assert_array_equal(w["qsh"], r["qsh"])
    np.testing.assert_array_equal(w["dpat"], r["dpat"])
    np.testing.assert_array_equal(w["qpat"], r["qpat"])
    assert abs(w["n0at"].sum() - m.charge - w["nocc"]) < 1e-12
    assert abs(w["n0at"].sum() - w["n0sh"].sum()) < 1e-12
    # coefficients: S-orthonormal, and they reproduce the density
    S = oracle.hamiltonian(m.id, m.xyz)[0]
    Cm = w["coeff"]
    np.testing.assert_allclose(Cm.T @ S @ Cm, np.eye(nao), atol=1e-10)
    np.testing.assert_allclose((Cm * w["focc"]) @ Cm.T, w["density"], atol=1e-10)


def test_warm_start_converges_faster_to_the_same_point(gpu_calc):
    # accuracy 1e-4: both runs stop within ~1e-8 e of the fixed point, so the
    # charges of the two paths agree far inside the 1e-7 tolerance
    mols = g.water_clusters(4, seed=77, nmin=6, nmax=24)
    cold = gpu_calc.singlepoint_batch(mols, accuracy=1e-4)
    guess = [dict(qsh=r["qsh"], dpat=r["dpat"], qpat=r["qpat"]) for r in cold]
    warm = gpu_calc.singlepoint_batch(mols, accuracy=1e-4, guess=guess)
    for c, w in zip(cold, warm):
        assert c["status"] == w["status"] == 0
        assert w["iterations"] < c["iterations"] and w["iterations"] <= 3, (w["iterations"], c["iterations"])
        assert abs(w["energy"] - c["energy"]) < TOL
        np.testing.assert_allclose(w["qat"], c["qat"], atol=1e-7)


def test_guess_only_where_given(gpu_calc):
    mols = g.water_clusters(3, seed=78, nmin=4, nmax=12)
    cold = gpu_calc.singlepoint_batch(mols)
    guess = [None, dict(qsh=cold[1]["qsh"], dpat=cold[1]["dpat"], qpat=cold[1]["qpat"]), None]
    mixed = gpu_calc.singlepoint_batch(mols, guess=guess, wavefunction=True)
    for i in (0, 2):  # no guess: bit-identical to the cold run
        assert mixed[i]["energy"] == cold[i]["energy"] and mixed[i]["iterations"] == cold[i]["iterations"]
        np.testing.assert_array_equal(mixed[i]["qat"], cold[i]["qat"])
    assert mixed[1]["iterations"] < cold[1]["iterations"]


def test_bad_guess_rejected(gpu_calc):
    m = g.octane()
    nsh, _ = gpu_calc.basis_size(m)
    bad = dict(qsh=np.full(nsh, np.nan), dpat=np.zeros((m.nat, 3)), qpat=np.zeros((m.nat, 6)))
    with pytest.raises(capi.TBError) as e:
        gpu_calc.singlepoint_batch([m], guess=[bad])
    assert e.value.status == capi.TB_BAD_INPUT


@pytest.mark.parametrize("idx", [0, 2])
def test_open_shell_representation_matches_oracle(gpu_calc, oracle, idx):
    """nspin = 2 (tblite's open-shell representation; the reference stops at
    "Unimplemented", src/scf/iterators.cu:247-248): per-channel occupations and
    densities within 1e-9 and the (total, up - down) moments within 1e-7 of the
    oracle; the total channel is the nspin = 1 result."""
    m = _mols()[idx]
    r = gpu_calc.singlepoint_batch([m], accuracy=1e-4, wavefunction=True, nspin=2)[0]
    o = oracle.singlepoint_spin(m, accuracy=1e-4)
    w = r["wfn"]
    assert r["status"] == 0 and w["nspin"] == 2
    np.testing.assert_allclose(w["focc"], o["focc"], atol=TOL)
    np.testing.assert_allclose(w["density"], o["density"], atol=TOL)
    for k in ("qat", "qsh", "dpat", "qpat"):
        np.testing.assert_allclose(w[k], o[k], atol=1e-7)
    np.testing.assert_array_equal(w["emo"][0], w["emo"][1])
    r1 = gpu_calc.singlepoint_batch([m], accuracy=1e-4, wavefunction=True)[0]
    assert r1["energy"] == r["energy"]
    np.testing.assert_allclose(w["density"].sum(0), r1["wfn"]["density"], atol=1e-12)
    np.testing.assert_array_equal(w["qat"][0], r1["qat"])
    for s in range(2):
        assert abs(w["focc"][s].sum() - w["nel"][s]) < 1e-9
    assert abs(w["qat"][1].sum() + (w["nel"][0] - w["nel"][1])) < 1e-9  # up - down = -(N_up - N_down)
