"""The CUDA engine (through the C ABI) against lightsmith's own engine: golden fields, DFT accumulators and
decay energy, in float64 and float32, eager and replayed as a CUDA graph."""

import numpy as np
import pytest

from conftest import golden_cases

pytestmark = pytest.mark.gpu

# float64 kernels differ from the reference only by fused multiply-adds and summation order; float32 is the
# reference GPU precision (lightsmith runs float32 on GPUs), compared with its float64 CPU run
TOL = {"double": 1e-9, "single": 3e-4}


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _engine(plan, precision):
    from lightsmith_b200.engine import Engine

    return Engine.from_plan(plan, precision=precision)


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("case", golden_cases())
def test_cuda_engine_matches_reference(case, precision, golden):
    d = golden("engine_" + case)
    plan, out = d["plan"], d["out"]
    eng = _engine(plan, precision)
    tol = TOL[precision]
    for i in range(out["n_chunks"]):
        eng.chunk(1)
        if i + 1 == out["snap"]:
            assert _rel(eng.E.cpu().numpy(), out["E_snap"]) < tol, (case, "E after first chunks")
    assert int(eng.n.item()) == out["n"] == eng.n_host
    assert _rel(eng.E.cpu().numpy(), out["E"]) < tol, case
    assert _rel(eng.H.cpu().numpy(), out["H"]) < tol, case
    for k in range(len(eng.monitors)):
        e, h = eng.results(k)
        assert _rel(e, out["acc_e"][k]) < tol, (case, k, "acc_e")
        if h is not None:
            assert _rel(h, out["acc_h"][k]) < tol, (case, k, "acc_h")
    np.testing.assert_allclose(eng.energy.cpu().numpy(), out["energy"], rtol=10 * tol, atol=0)
    for i, s in enumerate(eng._src_state):
        if s["kind"] == "column":
            assert _rel(s["col"].E.cpu().numpy(), out["col_E"]) < tol
        if s["kind"] == "line":
            assert _rel(s["E"].cpu().numpy(), out["line_E"]) < tol
    eng.close()


@pytest.mark.parametrize("case", ["tfsf_table", "bloch_column", "ade_groups"])
def test_cuda_graph_replay_is_bit_identical(case, golden):
    plan = golden("engine_" + case)["plan"]
    a, b = _engine(plan, "single"), _engine(plan, "single")
    for _ in range(4):
        a.chunk(1, use_graph=False)
        b.chunk(1, use_graph=True)
    assert np.array_equal(a.E.cpu().numpy(), b.E.cpu().numpy())
    assert np.array_equal(a.results(0)[0], b.results(0)[0])
    a.close()
    b.close()


def test_source_waveform_end_raises(golden):
    from lightsmith_b200._abi import LsfdtdError

    plan = golden("engine_yee_cpml_dipole")["plan"]
    eng = _engine(plan, "single")
    n_wave = len(plan["sources"][0].wave)
    with pytest.raises(LsfdtdError, match="waveform"):
        eng.step(n_wave + 1)
    eng.close()
