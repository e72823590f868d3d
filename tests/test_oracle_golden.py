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


@pytest.mark.parametrize("case", ["offdiag", "offdiag_mirror"])
def test_offdiag_gather_tables_equal_the_reference(case, golden):
    """The plan builder's conformal off-diagonal gather tables (targets, H indices, weights) against the ones
    lightsmith's engine built from the same rows (engine.py:421-518), mirror planes and a dispersive group
    included."""
    d = golden("engine_" + case)
    od, out = d["plan"]["offdiag"], d["out"]
    assert np.array_equal(od["e"], out["od_e"])
    assert np.array_equal(od["h"], out["od_h"])
    assert np.array_equal(od["w"], out["od_w"])
