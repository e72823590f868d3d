"""Batched Bloch-periodic sweeps (``lightsmith_b200.batch.BlochBatch``): the persistent kernel against
lightsmith's own engine (the golden oblique-incidence case) and against the same runs stepped one by one by
their own engines, with runs of uneven size and uneven step counts."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"double": 1e-9, "single": 3e-4}  # against lightsmith's float64 engine, as the single-run tests
SAME = {"double": 1e-11, "single": 2e-5}  # batched against sequential kernels of this library


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("precision", ["double", "single"])
def test_batch_matches_lightsmith_bloch_column(precision, golden):
    from lightsmith_b200.batch import BlochBatch
    from lightsmith_b200.engine import Engine

    d = golden("engine_bloch_column")
    plan, out = d["plan"], d["out"]
    eng = Engine.from_plan(plan, precision=precision)
    last = out["n_chunks"] * plan["stride"]
    batch = BlochBatch([eng], last)
    batch.run_to_end(steps_per_launch=7)  # launches end mid-chunk: sampling follows the step count
    assert eng.n_host == last == int(eng.n.item())
    tol = TOL[precision]
    assert _rel(eng.E.cpu().numpy(), out["E"]) < tol
    assert _rel(eng.H.cpu().numpy(), out["H"]) < tol
    for k in range(len(eng.monitors)):
        e, h = eng.results(k)
        assert _rel(e, out["acc_e"][k]) < tol, k
        if h is not None:
            assert _rel(h, out["acc_h"][k]) < tol, k
    col = eng.source_arrays(0)["col"]
    assert _rel(col.E.cpu().numpy(), out["col_E"]) < tol
    assert _rel(col.H.cpu().numpy(), out["col_H"]) < tol
    batch.close()
    eng.close()


def _small_runs(precision, n=5, steps=240):
    from lightsmith_b200.workloads import metasurface_run

    rng = np.random.default_rng(11)
    plans = []
    for i in range(n):
        period = float(rng.uniform(60, 140))  # 6 to 14 cells: uneven sizes
        plans.append(metasurface_run(period, float(rng.uniform(5, 60)), float(rng.uniform(0, 90)),
                                     float(rng.uniform(450, 750)), "s" if i % 2 else "p", nz=90, pml=10,
                                     height=200.0, steps=steps, single=precision == "single"))
    return plans


# launch shapes: the default (groups of half the resident CTAs), clusters of 8 CTAs per run (as many as fit),
# and groups of 24 CTAs per run (two in flight) that meet at barriers in global memory
@pytest.mark.parametrize("shape", [(0, 0), (8, 0), (24, 2)])
@pytest.mark.parametrize("precision", ["double", "single"])
def test_batch_equals_sequential_runs(precision, shape):
    from lightsmith_b200.batch import BlochBatch
    from lightsmith_b200.engine import Engine

    plans = _small_runs(precision)
    lasts = [(200 // p["stride"]) * p["stride"] for p in plans]  # whole chunks, uneven per run
    batched = [Engine.from_plan(p, precision=precision) for p in plans]
    batch = BlochBatch(batched, lasts, cluster_ctas=shape[0], max_clusters=shape[1])
    batch.run_to_end(steps_per_launch=64)
    tol = SAME[precision]
    for p, eb, last in zip(plans, batched, lasts):
        es = Engine.from_plan(p, precision=precision)
        es.chunk(last // p["stride"], use_graph=True)
        assert eb.n_host == es.n_host == last
        assert np.abs(es.E.cpu().numpy()).max() > 0
        assert _rel(eb.E.cpu().numpy(), es.E.cpu().numpy()) < tol
        assert _rel(eb.H.cpu().numpy(), es.H.cpu().numpy()) < tol
        for k in range(len(es.monitors)):
            e_b, h_b = eb.results(k)
            e_s, h_s = es.results(k)
            assert np.abs(e_s).max() > 0
            assert _rel(e_b, e_s) < tol, k
            if h_s is not None:
                assert _rel(h_b, h_s) < tol, k
        es.close()
    batch.close()
    for e in batched:
        e.close()


def test_batch_in_pieces_equals_one_launch():
    """Launches of a few steps each reach the state one long launch does, bit for bit (the same kernel)."""
    from lightsmith_b200.batch import BlochBatch
    from lightsmith_b200.engine import Engine

    plans = _small_runs("single", n=3)
    last = 3 * max(p["stride"] for p in plans) + 5
    a = [Engine.from_plan(p) for p in plans]
    b = [Engine.from_plan(p) for p in plans]
    ba, bb = BlochBatch(a, last), BlochBatch(b, last)
    ba.run(last, 1, use_graph=False)
    bb.run(5, -(-last // 5), use_graph=True)
    for ea, eb in zip(a, b):
        assert ea.n_host == eb.n_host == last
        assert np.array_equal(ea.E.cpu().numpy(), eb.E.cpu().numpy())
        assert np.array_equal(ea.results(0)[0], eb.results(0)[0])
    for x in (ba, bb):
        x.close()
    for e in a + b:
        e.close()


def test_batch_rejects_runs_it_cannot_batch(golden):
    from lightsmith_b200._abi import LsfdtdError
    from lightsmith_b200.batch import BlochBatch
    from lightsmith_b200.engine import Engine

    eng = Engine.from_plan(golden("engine_line_periodic")["plan"], precision="single")  # real fields, 1D feed
    with pytest.raises(LsfdtdError, match="complex"):
        BlochBatch([eng], 10)
    col = Engine.from_plan(golden("engine_bloch_column")["plan"], precision="single")
    with pytest.raises(LsfdtdError, match="waveform"):
        BlochBatch([col], 10 ** 7)
    eng.close()
    col.close()


def test_a_run_turning_non_finite_retires_alone():
    """A NaN written from the host into one run's E between launches: that run's status word reports it and it
    stops stepping, while the other runs of the batch finish with the values of a batch without the NaN."""
    import torch

    from lightsmith_b200 import _abi
    from lightsmith_b200.batch import BlochBatch
    from lightsmith_b200.engine import Engine

    plans = _small_runs("double", n=3, steps=240)
    last = [p["stride"] * (240 // p["stride"]) for p in plans]
    ref = [Engine.from_plan(p) for p in plans]
    b_ref = BlochBatch(ref, last)
    b_ref.run_to_end(steps_per_launch=30)
    engs = [Engine.from_plan(p) for p in plans]
    batch = BlochBatch(engs, last)
    batch.run(30, 2)
    torch.cuda.synchronize()
    n0, n1, n2 = engs[1].shape
    node = ((1 * n0 + n0 // 2) * n1 + n1 // 2) * n2 + n2 // 2  # E_y at the middle node (ghost planes are never read)
    engs[1].E_flat[node] = float("nan")
    batch.run_to_end(steps_per_launch=30)
    assert batch.diverged() == [1] and b_ref.diverged() == []
    n1 = int(engs[1].n.item())
    assert 60 < n1 < last[1], (n1, last[1])
    with pytest.raises(_abi.LsfdtdError, match="non-finite"):
        engs[1].check_status()
    for i in (0, 2):
        assert int(engs[i].n.item()) == last[i]
        for k in range(len(engs[i].monitors)):
            assert np.array_equal(engs[i].results(k)[0], ref[i].results(k)[0])
    for x in (batch, b_ref):
        x.close()
    for e in engs + ref:
        e.close()


def test_batch_depth_tuner():
    """tune.tune_batch_depth times the batched kernel at each steps-per-visit depth on the runs it is given
    (which advance by the steps it runs: two timed launches and a capture per depth) and returns the fastest."""
    from lightsmith_b200.engine import Engine
    from lightsmith_b200.tune import tune_batch_depth

    plans = _small_runs("single")
    lasts = [(200 // p["stride"]) * p["stride"] for p in plans]  # the runs' waveforms cover 240 steps
    engines = [Engine.from_plan(p) for p in plans]
    depths = (7, 21)
    best, res = tune_batch_depth(engines, lasts, depths=depths, launches=2)
    assert best in depths and sorted(res) == sorted(depths) and all(v > 0 for v in res.values())
    for e, last in zip(engines, lasts):
        assert e.n_host == min(last, 3 * sum(depths))
        e.close()
