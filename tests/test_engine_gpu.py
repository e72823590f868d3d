"""The CUDA engine (through the C ABI) against lightsmith's own engine: golden fields, DFT accumulators and
decay energy, in float64 and float32, eager and replayed as a CUDA graph."""

import numpy as np
import pytest

from conftest import golden_cases

pytestmark = pytest.mark.gpu

# float64 kernels differ from the reference only by fused multiply-adds and summation order; float32 is the
# reference GPU precision (lightsmith runs float32 on GPUs), compared with its float64 CPU run
TOL = {"double": 1e-9, "single": 3e-4}
# two kernel paths of this library with the same arithmetic per value (fused multiply-adds may differ)
SAME_ARITHMETIC = {"double": 1e-13, "single": 2e-6}


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


# cases the fused single pass serves (no periodic axis, point-dipole sources)
FUSED_CASES = ["yee_cpml_dipole", "kappa_noncubic", "ade_groups", "offdiag"]


@pytest.mark.parametrize("variant,tile_y,planes,stages", [(1, 8, 3, 4), (1, 16, 5, 6), (1, 16, 128, 8), (1, 8, 2, 8),
                                                          (3, 8, 3, 4), (3, 16, 5, 6), (3, 8, 1, 8),
                                                          (4, 8, 3, 4), (4, 16, 5, 6), (4, 8, 1, 8)])
@pytest.mark.parametrize("case", FUSED_CASES)
def test_fused_pass_any_launch_shape(case, variant, tile_y, planes, stages, golden):
    """The fused pass under launch shapes that split x into several segments (each CTA then recomputes the
    H plane before its segment) still matches lightsmith's engine."""
    d = golden("engine_" + case)
    plan, out = d["plan"], d["out"]
    eng = _engine(plan, "double")
    eng.set_tuning(variant, tile_y, planes, stages)
    assert eng.fused
    for _ in range(out["n_chunks"]):
        eng.chunk(1, use_graph=True)
    assert _rel(eng.E.cpu().numpy(), out["E"]) < TOL["double"]
    assert _rel(eng.H.cpu().numpy(), out["H"]) < TOL["double"]
    assert _rel(eng.results(0)[1], out["acc_h"][0]) < TOL["double"]
    eng.close()


@pytest.mark.parametrize("case", FUSED_CASES)
def test_fused_pass_equals_in_place_kernels(case, golden):
    from lightsmith_b200.engine import Engine

    plan = golden("engine_" + case)["plan"]
    a = Engine.from_plan(plan, precision="single")
    b = Engine.from_plan(plan, precision="single", fused=False)
    a.set_tuning(1, 8, 4, 4)
    assert a.fused and not b.fused
    for _ in range(5):
        a.chunk(1, use_graph=True)
        b.chunk(1, use_graph=True)
    assert _rel(a.E.cpu().numpy(), b.E.cpu().numpy()) < 1e-6
    assert _rel(a.H.cpu().numpy(), b.H.cpu().numpy()) < 1e-6
    a.close()
    b.close()


@pytest.mark.parametrize("variant", [3, 4])
@pytest.mark.parametrize("precision", ["single", "double"])
def test_split_and_lean_passes_equal_fused_pass(variant, precision, golden):
    """The split step (interior box without region or CPML code, then the shell H and E kernels) and the
    lean-CPML pass give the fused pass's values: the same arithmetic per value, in separately compiled
    kernels (which may contract a multiply and an add into one fused multiply-add differently), so equal to
    the last bits."""
    from lightsmith_b200.engine import Engine

    plan = golden("engine_yee_cpml_dipole")["plan"]
    a = Engine.from_plan(plan, precision=precision)
    b = Engine.from_plan(plan, precision=precision)
    a.set_tuning(1, 8, 4, 4)
    b.set_tuning(variant, 8, 4, 4)
    assert a.uses_tma and b.uses_tma
    extra = 2 if variant == 3 else 0  # the shell H and E kernels of the split step
    assert b.launches_per_chunk() == a.launches_per_chunk() + extra * plan["stride"]
    for _ in range(5):
        a.chunk(1, use_graph=True)
        b.chunk(1, use_graph=True)
    b.check_status()
    assert np.abs(a.E.cpu().numpy()).max() > 0
    tol = SAME_ARITHMETIC[precision]
    assert _rel(b.E.cpu().numpy(), a.E.cpu().numpy()) < tol
    assert _rel(b.H.cpu().numpy(), a.H.cpu().numpy()) < tol
    assert _rel(b.results(0)[0], a.results(0)[0]) < tol
    a.close()
    b.close()


@pytest.mark.parametrize("case", ["yee_cpml_dipole", "ade_groups"])
def test_tma_and_cp_async_rings_agree_bit_for_bit(case, golden):
    """The two copy engines of the fused pass deliver the same values, so the steps are identical."""
    from lightsmith_b200.engine import Engine

    plan = golden("engine_" + case)["plan"]
    a = Engine.from_plan(plan, precision="double")
    b = Engine.from_plan(plan, precision="double")
    b.set_copy_engine(False)
    a.set_tuning(1, 8, 6, 4)
    b.set_tuning(1, 8, 6, 4)
    for _ in range(4):
        a.chunk(1, use_graph=True)
        b.chunk(1, use_graph=True)
    assert a.uses_tma and not b.uses_tma
    a.check_status()
    assert np.array_equal(a.E.cpu().numpy(), b.E.cpu().numpy())
    assert np.array_equal(a.H.cpu().numpy(), b.H.cpu().numpy())
    a.close()
    b.close()


@pytest.mark.parametrize("case", ["yee_cpml_dipole", "line_periodic"])
def test_vector_kernels_equal_per_node_kernels(case, golden):
    """The four-node vector kernels (rows of a multiple of four nodes) give the per-node kernels' values."""
    from lightsmith_b200.engine import Engine

    plan = golden("engine_" + case)["plan"]
    assert plan["shape"][2] % 4 == 0
    a = Engine.from_plan(plan, precision="single", fused=False)
    b = Engine.from_plan(plan, precision="single", fused=False)
    a.set_tuning(2, 8, 32, 4)
    for _ in range(5):
        a.chunk(1, use_graph=True)
        b.chunk(1, use_graph=True)
    assert _rel(a.E.cpu().numpy(), b.E.cpu().numpy()) < 1e-6
    assert _rel(a.H.cpu().numpy(), b.H.cpu().numpy()) < 1e-6
    a.close()
    b.close()


def test_rows_without_tensor_copies_step_in_place_by_default():
    """Rows of 30 FP32 nodes (120 bytes, not a multiple of 16): the engine's default steps in place (faster
    there than the fused pass's cp.async ring), and an explicit kernel choice keeps the fused pass; the two give
    the same values up to fused multiply-add contraction."""
    from lightsmith_b200.engine import Engine
    from lightsmith_b200.workloads import throughput_plan

    plan = throughput_plan(30, pml=4, max_steps=600, seed=4)
    w = plan["sources"][0].wave
    first = int(np.nonzero(np.abs(w) > 1e-3 * np.abs(w).max())[0][0])
    plan["sources"][0].wave = np.concatenate([w[first:], np.zeros(first)])
    a = Engine.from_plan(plan)
    b = Engine.from_plan(plan)
    b.set_tuning(1, 8, 4, 4)
    assert not a.fused and b.fused and not b.uses_tma
    for _ in range(4):
        a.chunk(1, use_graph=True)
        b.chunk(1, use_graph=True)
    assert np.abs(a.E.cpu().numpy()).max() > 0
    assert _rel(b.E.cpu().numpy(), a.E.cpu().numpy()) < SAME_ARITHMETIC["single"]
    assert _rel(b.results(0)[0], a.results(0)[0]) < SAME_ARITHMETIC["single"]
    a.close()
    b.close()
