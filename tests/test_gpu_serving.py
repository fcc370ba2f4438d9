"""GPU: the continuous-batching request loop (tb_server).  Requests of mixed
sizes arrive while others are on the device; every result must equal the
singlepoint of the same structure alone (bit for bit: each kernel treats a
structure independently of its batch), and the resident workspace must stay
within the budget."""
import time

import numpy as np
import pytest

from tblite_b200 import capi, geometry as g

pytestmark = pytest.mark.gpu


def _requests():
    rng = np.random.default_rng(77)
    mols = g.water_clusters(6, seed=78, nmin=2, nmax=30)
    mols += [g.alkane(n, rng) for n in (3, 11, 24)]
    mols += [g.octane()]
    order = rng.permutation(len(mols))
    return [mols[i] for i in order]


def _serve(calc, mols, budget, max_batch, per_step=2, **opts):
    srv = capi.Server(calc, budget, max_batch=max_batch, **opts)
    tickets, got, peak = {}, {}, 0
    pending = list(mols)
    steps = 0
    while pending or len(got) < len(mols):
        for _ in range(min(per_step, len(pending))):  # staggered arrivals
            m = pending.pop(0)
            tickets[srv.submit(m)] = m
        resident, queued, nbytes = srv.step()
        peak = max(peak, nbytes)
        for t, r in srv.poll():
            got[t] = r
        time.sleep(0.0005)  # step() only polls the micro-batches' streams
        steps += 1
        assert steps < 200000
    return tickets, got, peak


@pytest.mark.parametrize("precision", [0, 1])
def test_serving_results_equal_alone(gpu_calc, precision):
    mols = _requests()
    tickets, got, peak = _serve(gpu_calc, mols, budget=8 << 30, max_batch=4, precision=precision)
    assert sorted(got) == sorted(tickets)
    for t, m in tickets.items():
        alone = gpu_calc.singlepoint_batch([m], precision=precision)[0]
        r = got[t]
        assert r["status"] == alone["status"] == 0
        assert r["energy"] == alone["energy"] and r["iterations"] == alone["iterations"]
        np.testing.assert_array_equal(r["qat"], alone["qat"])


def test_serving_budget_limits_residency(gpu_calc):
    mols = _requests()
    budget = 12 << 20  # two or three of these structures at a time
    tickets, got, peak = _serve(gpu_calc, mols, budget=budget, max_batch=8, per_step=4)
    assert len(got) == len(mols)
    assert 0 < peak <= budget


def test_serving_rejects_structure_above_budget(gpu_calc):
    srv = capi.Server(gpu_calc, 1 << 20)
    with pytest.raises(capi.TBError) as e:
        srv.submit(g.water_cluster(30, np.random.default_rng(1)))
    assert e.value.status == capi.TB_CAPACITY_EXCEEDED


@pytest.mark.parametrize("precision", [0, 1])
def test_serving_compaction_keeps_results(gpu_calc, precision):
    """One micro-batch of 8: six alkanes (about 6 SCF iterations) and two water
    clusters (about 8): once the alkanes are done, the two clusters move to a
    compacted micro-batch with their SCF state; every result still equals the
    structure alone, bit for bit, and the old workspace returned to the pool."""
    rng = np.random.default_rng(91)
    mols = [g.alkane(n, rng) for n in (4, 6, 8, 10, 12, 14)] + g.water_clusters(2, seed=92, nmin=10, nmax=16)
    srv = capi.Server(gpu_calc, 8 << 30, max_batch=8, precision=precision)
    tickets = {srv.submit(m): m for m in mols}
    got, steps = {}, 0
    while len(got) < len(mols):
        srv.step()
        for t, r in srv.poll():
            got[t] = r
        time.sleep(0.0005)
        steps += 1
        assert steps < 200000
    assert srv.compactions() >= 1
    for t, m in tickets.items():
        alone = gpu_calc.singlepoint_batch([m], precision=precision)[0]
        r = got[t]
        assert r["status"] == alone["status"] == 0
        assert r["energy"] == alone["energy"] and r["iterations"] == alone["iterations"]
        np.testing.assert_array_equal(r["qat"], alone["qat"])


@pytest.mark.parametrize("precision,solver,graphs", [(0, 0, 1), (1, 0, 1), (1, 2, 0), (1, 2, 1)])
def test_serving_compaction_graphs_and_library(gpu_calc, precision, solver, graphs):
    """The same compaction with the iteration replayed as a graph and/or every
    eigensolve on the library path (solver = 2): the compacted micro-batch's
    host copies of the flags (the mixed form's library path picks its FP32 or
    FP64 solver by the phase) and its occupied-orbital counts are those of its
    structures, so every result still equals the structure alone, bit for bit."""
    rng = np.random.default_rng(91)
    mols = [g.alkane(n, rng) for n in (4, 6, 8, 10, 12, 14)] + g.water_clusters(2, seed=92, nmin=10, nmax=16)
    opts = dict(precision=precision, solver=solver, use_graphs=graphs)
    srv = capi.Server(gpu_calc, 8 << 30, max_batch=8, **opts)
    tickets = {srv.submit(m): m for m in mols}
    got, steps = {}, 0
    while len(got) < len(mols):
        srv.step()
        for t, r in srv.poll():
            got[t] = r
        time.sleep(0.0005)
        steps += 1
        assert steps < 200000
    assert srv.compactions() >= 1
    for t, m in tickets.items():
        alone = gpu_calc.singlepoint_batch([m], precision=precision, solver=solver)[0]
        r = got[t]
        assert r["status"] == alone["status"] == 0
        assert r["energy"] == alone["energy"] and r["iterations"] == alone["iterations"]
        np.testing.assert_array_equal(r["qat"], alone["qat"])
