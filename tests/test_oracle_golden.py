"""The CPU oracle against golden vectors from lightsmith's own engine (float64): fields after the recorded
chunks, DFT accumulators and the decay-energy proxy."""

import numpy as np
import pytest

from conftest import golden_cases
from oracle.engine import OracleEngine

RTOL = 1e-11  # float64 restatement: only the summation order of a few shared nodes differs


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_matches_reference_engine(case, golden):
    d = golden("engine_" + case)
    plan, out = d["plan"], d["out"]
    eng = OracleEngine(plan)
    for i in range(out["n_chunks"]):
        eng.chunk()
        if i + 1 == out["snap"]:
            assert _rel(eng.E, out["E_snap"]) < RTOL and _rel(eng.H, out["H_snap"]) < RTOL
    assert eng.n == out["n"]
    assert _rel(eng.E, out["E"]) < RTOL, case
    assert _rel(eng.H, out["H"]) < RTOL, case
    for k, m in enumerate(eng.monitors):
        assert _rel(m["acc_e"], out["acc_e"][k]) < RTOL, (case, k)
        if m["acc_h"] is not None:
            assert _rel(m["acc_h"], out["acc_h"][k]) < RTOL, (case, k)
    np.testing.assert_allclose(eng.energy, out["energy"], rtol=1e-10, atol=0)
    if "col_E" in out:
        col = eng.sources[0].col
        assert _rel(col.E, out["col_E"]) < RTOL and _rel(col.H, out["col_H"]) < RTOL
    if "line_E" in out:
        s = eng.sources[0]
        assert _rel(s.E_flat, out["line_E"]) < RTOL and _rel(s.H_flat, out["line_H"]) < RTOL


@pytest.mark.parametrize("case", ["yee_cpml_dipole", "ade_groups"])
def test_oracle_threads_do_not_change_results(case, golden):
    plan = golden("engine_" + case)["plan"]
    a, b = OracleEngine(plan), OracleEngine(plan, threads=3)
    for _ in range(3):
        a.chunk()
        b.chunk()
    b.close()
    assert np.array_equal(a.E, b.E) and np.array_equal(a.H, b.H)


def test_oracle_detects_a_planted_mistake(golden):
    """A wrong CPML coefficient in the oracle must fail the golden comparison (the check has teeth)."""
    d = golden("engine_yee_cpml_dipole")
    eng = OracleEngine(d["plan"])
    eng.pml["H"][0]["cp"] *= 1.01
    for _ in range(d["out"]["n_chunks"]):
        eng.chunk()
    assert _rel(eng.H, d["out"]["H"]) > 1e-6


def sparse_operator(e, h, w):
    """The gather tables (targets, H indices, weights) as a merged sparse operator: keys target * 2^32 + H node
    and their summed weights, padding and other zero entries dropped."""
    e, h, w = np.asarray(e), np.asarray(h), np.asarray(w)
    key = np.repeat(e.astype(np.int64), h.shape[1]) * (1 << 32) + h.ravel()
    key, inv = np.unique(key, return_inverse=True)
    val = np.bincount(inv, w.ravel().real, len(key)) + 1j * np.bincount(inv, w.ravel().imag, len(key))
    nz = val != 0
    return key[nz], val[nz]


@pytest.mark.parametrize("case", ["offdiag", "offdiag_mirror"])
def test_offdiag_gather_tables_equal_the_reference_operator(case, golden):
    """The plan builder's conformal off-diagonal tables, rebuilt here from the fixture's rows, against the ones
    lightsmith's engine built from the same rows (engine.py:421-518), mirror planes and a dispersive group
    included: the same operator (every (target, H node) weight, to rounding), in a merged layout of its own."""
    from lightsmith_b200.plan import offdiag_tables

    d = golden("engine_" + case)
    plan, out = d["plan"], d["out"]
    rows = out["od_rows"]

    class Rows:
        idx3, comp, coef = rows["idx3"], rows["comp"], rows["coef"]
    gidx = np.concatenate([np.asarray(g["idx"]) for g in plan["groups"]]) if plan["groups"] else np.zeros(0, int)
    e, h, w = offdiag_tables(Rows, plan["shape"], plan["spacing"], plan["dt"], plan["periodic"], plan["bloch"],
                             plan.get("mirror", (0, 0, 0)), gidx, plan["complex"])
    for x, y in zip((e, h, w), (plan["offdiag"]["e"], plan["offdiag"]["h"], plan["offdiag"]["w"])):
        assert np.array_equal(x, y)  # the fixture's plan holds this builder's tables
    ka, va = sparse_operator(e, h, w)
    kb, vb = sparse_operator(out["od_e"], out["od_h"], out["od_w"])
    keys = np.union1d(ka, kb)  # an entry one side sums to exactly zero may be a rounding residue on the other
    dense_a, dense_b = np.zeros(len(keys), complex), np.zeros(len(keys), complex)
    dense_a[np.searchsorted(keys, ka)], dense_b[np.searchsorted(keys, kb)] = va, vb
    np.testing.assert_allclose(dense_a, dense_b, rtol=0, atol=1e-14 * np.abs(vb).max())
    assert len(np.setdiff1d(ka, kb)) < 0.01 * len(kb)
    assert h.shape[1] < np.asarray(out["od_h"]).shape[1]  # merged: fewer taps per target than lightsmith's
