"""GPU parity: every stage of the CUDA path against the FP64 oracle on the same
inputs, through the C ABI.  Tolerances: bit-exact for the neighbour list;
1e-12 (absolute) for integral matrices and stage outputs; singlepoint total
energy 1e-9 Eh, atomic charges 1e-7 e, dipole 1e-7 a.u. (plain FP64 form)."""
import numpy as np
import pytest

from tblite_b200 import capi, geometry as g

pytestmark = pytest.mark.gpu

E_TOL, Q_TOL, MU_TOL = 1e-9, 1e-7, 1e-7


def _mols():
    rng = np.random.default_rng(7)
    return [g.octane(), g.water_cluster(8, rng), g.alkane(3, rng), g.water_cluster(20, rng)]


# ------------------------------------------------------------ stages
@pytest.mark.parametrize("idx", range(4))
def test_adjacency_list_bit_exact(gpu_calc, oracle, idx):
    m = _mols()[idx]
    cut = oracle.cutoff()
    assert gpu_calc.cutoff() == cut
    inl, nnl, nlat = capi.adjacency_list(gpu_calc, m, cut)
    oinl, onnl, onlat, _ = oracle.adjacency_list(m.xyz, cut)
    np.testing.assert_array_equal(nnl, onnl)
    np.testing.assert_array_equal(inl, oinl)
    np.testing.assert_array_equal(nlat, onlat)


def test_adjacency_list_edges(gpu_calc, oracle):
    # cutoff boundary cases: one atom, a pair beyond the cutoff, a pair exactly at it
    one = g.Molecule(np.array([0], np.int32), np.zeros((1, 3)))
    inl, nnl, nlat = capi.adjacency_list(gpu_calc, one, 10.0)
    assert nnl.tolist() == [0] and len(nlat) == 0
    far = g.Molecule(np.array([0, 2], np.int32), np.array([[0.0, 0, 0], [0.0, 0, 50.0]]))
    _, nnl, nlat = capi.adjacency_list(gpu_calc, far, 10.0)
    assert nnl.tolist() == [0, 0]
    at = g.Molecule(np.array([0, 0], np.int32), np.array([[0.0, 0, 0], [3.0, 0, 4.0]]))
    _, nnl, nlat = capi.adjacency_list(gpu_calc, at, 5.0)
    assert nnl.tolist() == [0, 1]  # r2 == cutoff^2 is kept
    rng = np.random.default_rng(11)
    cloud = g.Molecule(rng.integers(0, 3, 300).astype(np.int32), rng.uniform(-30, 30, (300, 3)))
    cut = oracle.cutoff()
    inl, nnl, nlat = capi.adjacency_list(gpu_calc, cloud, cut)
    oinl, onnl, onlat, _ = oracle.adjacency_list(cloud.xyz, cut)
    np.testing.assert_array_equal(nlat, onlat)
    np.testing.assert_array_equal(inl, oinl)


@pytest.mark.parametrize("idx", range(4))
def test_atomic_properties_and_repulsion(gpu_calc, oracle, idx):
    m = _mols()[idx]
    cn, mrad, se = capi.atomic_properties(gpu_calc, m)
    ocn = oracle.coordination_number(m.id, m.xyz)
    np.testing.assert_allclose(cn, ocn, rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(mrad, oracle.mrad(m.id, ocn), rtol=1e-12)
    np.testing.assert_allclose(se, oracle.selfenergy(m.id, ocn), rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(capi.repulsion(gpu_calc, m), oracle.repulsion(m.id, m.xyz), rtol=1e-11, atol=1e-15)


@pytest.mark.parametrize("idx", range(4))
def test_hamiltonian_integrals(gpu_calc, oracle, idx):
    m = _mols()[idx]
    S, H0, D, Q = capi.get_hamiltonian(gpu_calc, m)
    oS, oH0, oD, oQ = oracle.hamiltonian(m.id, m.xyz)
    np.testing.assert_allclose(S, oS, atol=1e-12)
    np.testing.assert_allclose(H0, oH0, atol=1e-12)
    np.testing.assert_allclose(D, oD, atol=1e-11)
    np.testing.assert_allclose(Q, oQ, atol=1e-11)


@pytest.mark.parametrize("idx", range(4))
def test_coulomb_potential(gpu_calc, oracle, idx):
    m = _mols()[idx]
    rng = np.random.default_rng(idx)
    nsh, _ = gpu_calc.basis_size(m)
    qsh = rng.normal(scale=0.2, size=nsh)
    dpat = rng.normal(scale=0.05, size=(m.nat, 3))
    qpat = rng.normal(scale=0.05, size=(m.nat, 6))
    qpat[:, 5] = -qpat[:, 0] - qpat[:, 2]
    got = capi.coulomb_potential(gpu_calc, m, qsh, dpat, qpat)
    ref = oracle.coulomb_potential(m.id, m.xyz, qsh, dpat, qpat)
    for a, b in zip(got, ref):
        np.testing.assert_allclose(a, b, rtol=1e-11, atol=1e-12)


def test_fock_build(gpu_calc, oracle):
    m = _mols()[1]
    S, H0, D, Q = oracle.hamiltonian(m.id, m.xyz)
    rng = np.random.default_rng(3)
    nsh, _ = gpu_calc.basis_size(m)
    v = (rng.normal(size=nsh), rng.normal(size=m.nat), rng.normal(size=(m.nat, 3)), rng.normal(size=(m.nat, 6)))
    F = capi.add_pot_to_h1(gpu_calc, m, S, H0, D, Q, *v)
    oF = oracle.fock(m.id, S, H0, D, Q, *v)
    np.testing.assert_allclose(F, oF, atol=1e-12)


def test_sygvd_batch_uneven(oracle):
    rng = np.random.default_rng(0)
    sizes = [1, 2, 5, 33, 64, 65, 130]
    Hs, Ss = [], []
    for n in sizes:
        M = rng.normal(size=(n, n))
        R = rng.normal(size=(n, n))
        Hs.append(0.5 * (M + M.T))
        Ss.append(R @ R.T / n + np.eye(n))
    st, out = capi.sygvd_batch(Hs, Ss)
    assert st == capi.TB_OK
    for H, S, (w, C) in zip(Hs, Ss, out):
        ost, ow, oC = oracle.sygvd(H, S)
        np.testing.assert_allclose(w, ow, atol=1e-10)
        np.testing.assert_allclose(C.T @ S @ C, np.eye(len(w)), atol=1e-10)
        np.testing.assert_allclose(H @ C, S @ C * w, atol=1e-9)


def test_sygvd_degenerate_and_kat():
    A = np.array([[4.0, 1.0], [1.0, 3.0]])
    B = np.array([[2.0, 0.5], [0.5, 1.5]])
    n = 12
    rng = np.random.default_rng(3)
    Qm, _ = np.linalg.qr(rng.normal(size=(n, n)))
    H = Qm @ np.diag(np.repeat([-1.0, 0.5, 2.0], 4)) @ Qm.T
    st, out = capi.sygvd_batch([A, H], [B, np.eye(n)])
    assert st == capi.TB_OK
    np.testing.assert_allclose(out[0][0], [2.0, 2.0], atol=1e-13)
    w, C = out[1]
    np.testing.assert_allclose(C[:, :4] @ C[:, :4].T, Qm[:, :4] @ Qm[:, :4].T, atol=1e-12)


def test_sygvd_tridiagonal_panel_sizes(oracle):
    # sizes around the FP64 panel width (8 reflectors) and its multiples
    rng = np.random.default_rng(5)
    sizes = [3, 4, 9, 10, 11, 17, 18, 19, 66, 67]
    Hs = []
    for n in sizes:
        M = rng.normal(size=(n, n))
        Hs.append(0.5 * (M + M.T))
    st, out = capi.sygvd_batch(Hs, [np.eye(n) for n in sizes])
    assert st == capi.TB_OK
    for H, (w, C) in zip(Hs, out):
        np.testing.assert_allclose(w, np.linalg.eigvalsh(H), atol=1e-12)
        np.testing.assert_allclose(C.T @ C, np.eye(len(w)), atol=1e-12)
        np.testing.assert_allclose(H @ C, C * w, atol=1e-11)


def test_sygvd_divide_and_conquer():
    # structures of 64 AOs and more take the divide-and-conquer tridiagonal
    # solver (from 128 on with the tensor-core Q formation): random spectra,
    # 8-fold degenerate ones, nearly decoupled blocks (every merge deflates)
    # and a multiple of the identity
    rng = np.random.default_rng(9)
    Hs = []
    for n in (64, 65, 97, 111, 127, 128, 129, 200, 256, 384):
        M = rng.normal(size=(n, n))
        Hs.append(0.5 * (M + M.T))
    n = 256
    Qm, _ = np.linalg.qr(rng.normal(size=(n, n)))
    Hs.append(Qm @ np.diag(np.repeat(np.arange(n // 8, dtype=float), 8)) @ Qm.T)
    blocks = [rng.normal(size=(40, 40)) for _ in range(4)]
    Bd = np.zeros((160, 160))
    for i, b in enumerate(blocks):
        Bd[40 * i:40 * i + 40, 40 * i:40 * i + 40] = b + b.T
    Bd += 1e-13 * rng.normal(size=(160, 160))
    Hs.append(0.5 * (Bd + Bd.T))
    Hs.append(2.5 * np.eye(140))
    Hs.append(-1.5 * np.eye(64))  # smallest divide-and-conquer size, fully degenerate
    b2 = [rng.normal(size=(40, 40)) for _ in range(2)]
    Bs = np.zeros((80, 80))
    Bs[:40, :40], Bs[40:, 40:] = b2[0] + b2[0].T, b2[1] + b2[1].T
    Hs.append(Bs)  # decoupled halves: the root merge deflates every entry
    st, out = capi.sygvd_batch(Hs, [np.eye(len(H)) for H in Hs])
    assert st == capi.TB_OK
    for H, (w, C) in zip(Hs, out):
        scale = max(1.0, np.max(np.abs(H)))
        np.testing.assert_allclose(w, np.linalg.eigvalsh(H), atol=1e-12 * scale * len(w) ** 0.5)
        np.testing.assert_allclose(C.T @ C, np.eye(len(w)), atol=1e-12)
        np.testing.assert_allclose(H @ C, C * w, atol=1e-12 * scale * len(w) ** 0.5)


def test_sygvd_not_spd_status():
    st, _ = capi.sygvd_batch([np.eye(3)], [-np.eye(3)])
    assert st == capi.TB_NOT_SPD


def test_fermi_filling(oracle):
    kt = 300 * 3.166811563455546e-6
    emo = np.linspace(-1.0, 1.0, 40)
    emo[10] = emo[9] + 1e-5
    for nel in (10.0, 10.5, 0.0, 3.0):
        st, occ, ef, ts = capi.fermi_filling(nel, kt, emo)
        ost, oocc, oef, ots = oracle.fermi(nel, kt, emo)
        assert st == ost == 0
        np.testing.assert_allclose(occ, oocc, atol=1e-12)
        assert abs(ts - ots) < 1e-13


# ------------------------------------------------------------ singlepoint
def _check(r, o):
    assert r["status"] == 0, capi.STATUS_NAMES.get(r["status"])
    assert abs(r["energy"] - o["energy"]) < E_TOL, (r["energy"], o["energy"])
    np.testing.assert_allclose(r["qat"], o["qat"], atol=Q_TOL)
    np.testing.assert_allclose(r["dipole"], o["dipole"], atol=MU_TOL)


def test_octane_singlepoint(gpu_calc, oracle):
    m = g.octane()
    r = gpu_calc.singlepoint_batch([m], accuracy=1e-4)[0]
    o = oracle.singlepoint(m, accuracy=1e-4)
    _check(r, o)
    assert r["iterations"] == o["iterations"]
    for k in ("e_rep", "e_band", "e_es2", "e_aes2", "e_es3", "e_ts"):
        assert abs(r[k] - o[k]) < 1e-9, k
    np.testing.assert_allclose(r["qsh"], o["qsh"], atol=Q_TOL)
    np.testing.assert_allclose(r["dpat"], o["dpat"], atol=1e-7)
    np.testing.assert_allclose(r["qpat"], o["qpat"], atol=1e-7)


def test_octane_default_accuracy(gpu_calc, oracle):
    m = g.octane()
    r = gpu_calc.singlepoint_batch([m])[0]
    o = oracle.singlepoint(m)
    _check(r, o)


def test_uneven_water_batch(gpu_calc, oracle):
    mols = g.water_clusters(12, seed=1001, nmin=2, nmax=24)
    res = gpu_calc.singlepoint_batch(mols, accuracy=1e-4)
    for m, r in zip(mols, res):
        _check(r, oracle.singlepoint(m, accuracy=1e-4))


def test_alone_equals_in_batch(gpu_calc):
    mols = g.water_clusters(6, seed=5, nmin=3, nmax=16)
    batch = gpu_calc.singlepoint_batch(mols)
    for m, rb in zip(mols, batch):
        ra = gpu_calc.singlepoint_batch([m])[0]
        assert ra["energy"] == rb["energy"] and ra["iterations"] == rb["iterations"]
        np.testing.assert_array_equal(ra["qat"], rb["qat"])


def test_charged_open_shell_and_small(gpu_calc, oracle):
    m = g.octane()
    mols = [g.Molecule(m.id, m.xyz, charge=1.0, uhf=1),
            g.Molecule(np.array([0, 0], np.int32), np.array([[0, 0, 0], [0, 0, 1.4]], float)),  # H2
            g.Molecule(np.array([0], np.int32), np.zeros((1, 3)), uhf=1),                         # H atom
            g.alkane(1, np.random.default_rng(1))]                                              # methane
    res = gpu_calc.singlepoint_batch(mols, accuracy=1e-4)
    for mol, r in zip(mols, res):
        _check(r, oracle.singlepoint(mol, accuracy=1e-4))


def test_status_reporting(gpu_calc):
    m = g.octane()
    r = gpu_calc.singlepoint_batch([m], max_iter=1)[0]
    assert r["status"] == capi.TB_SCF_NOT_CONVERGED and r["iterations"] == 1
    bad = g.Molecule(np.array([0, 7], np.int32), np.zeros((2, 3)))
    with pytest.raises(capi.TBError) as e:
        gpu_calc.singlepoint_batch([bad])
    assert e.value.status == capi.TB_BAD_INPUT
    nan = g.Molecule(np.array([0, 0], np.int32), np.array([[0, 0, 0], [0, 0, np.nan]]))
    with pytest.raises(capi.TBError):
        gpu_calc.singlepoint_batch([nan])


def test_device_batch_api(gpu_calc, oracle):
    mols = g.water_clusters(5, seed=9, nmin=2, nmax=10)
    b = capi.Batch(gpu_calc, mols, accuracy=1e-4)
    b.run()
    assert b.launches() > 10
    first = b.results()
    b.run()  # rerun on resident inputs gives identical results
    second = b.results()
    for m, r1, r2 in zip(mols, first, second):
        assert r1["energy"] == r2["energy"]
        _check(r1, oracle.singlepoint(m, accuracy=1e-4))


@pytest.mark.parametrize("precision", [0, 1])
def test_graph_replay_equals_eager(gpu_calc, precision):
    # use_graphs runs the whole SCF loop as one graph launch (a conditional
    # WHILE node over one captured iteration plus the loop-control kernel)
    mols = g.water_clusters(6, seed=13, nmin=2, nmax=20)
    eager = capi.Batch(gpu_calc, mols, precision=precision)
    eager.run()
    graph = capi.Batch(gpu_calc, mols, precision=precision, use_graphs=1)
    graph.run()
    graph.run()  # second run replays the instantiated graph
    res = graph.results()
    iters = max(r["iterations"] for r in res)
    assert graph.launches() == eager.launches() + iters  # one loop-control kernel per iteration
    for a, b in zip(eager.results(), res):
        assert a["energy"] == b["energy"] and a["iterations"] == b["iterations"]
        np.testing.assert_array_equal(a["qat"], b["qat"])


def test_graph_loop_stops_at_max_iter(gpu_calc):
    m = g.octane()
    r = gpu_calc.singlepoint_batch([m], max_iter=2, use_graphs=1)[0]
    assert r["status"] == capi.TB_SCF_NOT_CONVERGED and r["iterations"] == 2
    b = capi.Batch(gpu_calc, [m], max_iter=2, use_graphs=1)
    b.run()
    e = capi.Batch(gpu_calc, [m], max_iter=2)
    e.run()
    assert b.launches() == e.launches() + 2
