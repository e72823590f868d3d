"""The throughput workload (random eps, CPML 16, centre dipole, 16-frequency DFT plane) on the GPU: against
the oracle at 128^3, and through size-independent properties at the full 640^3 size."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def test_throughput_case_matches_oracle_at_128():
    from lightsmith_b200.engine import Engine
    from lightsmith_b200.workloads import throughput_plan
    from oracle.engine import OracleEngine

    plan = throughput_plan(128, max_steps=4000, seed=3, single=False)
    ref = OracleEngine(plan, threads=8)
    gpu64 = Engine.from_plan(plan, precision="double")
    gpu32 = Engine.from_plan(plan, precision="single")
    gpu64.set_tuning(1, 8, 40, 4)  # the fused pass, several x segments per tile column
    gpu32.set_tuning(0, 8, 32, 4)  # float32 here: the in-place kernels
    assert gpu64.fused and not gpu32.fused
    for _ in range(3):
        ref.chunk()
        gpu64.chunk(1, use_graph=True)
        gpu32.chunk(1, use_graph=True)
    ref.close()
    assert np.abs(ref.E).max() > 0
    assert _rel(gpu64.E.cpu().numpy(), ref.E) < 1e-9
    assert _rel(gpu64.results(0)[0], ref.monitors[0]["acc_e"]) < 1e-9
    # float32 fields against the float64 oracle
    assert _rel(gpu32.E.cpu().numpy(), ref.E) < 3e-4
    assert _rel(gpu32.results(0)[1], ref.monitors[0]["acc_h"]) < 3e-4
    np.testing.assert_allclose(gpu32.energy.cpu().numpy()[0], ref.energy[0], rtol=1e-3)


# (72, 200, 64) with CPML 8 has no clean interior of whole 32-node z tiles: both engines take the lean kernel
@pytest.mark.parametrize("shape,pml,interior", [((128, 128, 128), 16, True), ((100, 90, 136), 12, True),
                                                ((72, 200, 64), 8, False), ((64, 64, 96), 0, True)])
@pytest.mark.parametrize("precision", ["single", "double"])
def test_clean_interior_split_gives_the_lean_kernels_values(shape, pml, interior, precision):
    """Variant 4 with one kernel per class of CTA box (the clean interior compiled without region or CPML
    code, the boxes beside it with one axis's slab code each, the edges and corners with all of it; all but
    the interior's on a second stream) against the lean kernel on every tile:
    the same fields and DFT accumulators bit for bit, on grids whose sides are and are not whole tiles,
    with CPML slabs of several widths and with walls only."""
    from lightsmith_b200.engine import Engine
    from lightsmith_b200.workloads import throughput_plan

    plan = throughput_plan(shape, pml=pml, max_steps=4000, seed=11, single=precision == "single")
    split, whole = Engine.from_plan(plan, precision=precision), Engine.from_plan(plan, precision=precision)
    for e in (split, whole):
        e.set_tuning(4, 8, 0, 4)
    whole.set_clean_split(False)
    assert split.fused and split.uses_tma and whole.fused
    # where the grid has a clean interior the step takes five launches, one per class of CTA box (the clean
    # interior, the boxes beside it along x, y and z, the edges and corners), in place of one
    assert split.launches_per_chunk() == whole.launches_per_chunk() + (4 * split.stride if interior else 0)
    for _ in range(4):
        split.chunk(1, use_graph=True)
        whole.chunk(1, use_graph=True)
    assert np.abs(whole.E.cpu().numpy()).max() > 0
    assert np.array_equal(split.E.cpu().numpy(), whole.E.cpu().numpy())
    assert np.array_equal(split.H.cpu().numpy(), whole.H.cpu().numpy())
    for a, b in zip(split.results(0), whole.results(0)):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision,tol", [("double", 1e-9), ("single", 3e-4)])
def test_bench_kernel_matches_oracle_at_128(precision, tol):
    """The bench's own kernel and launch shape (the lean fused pass, variant 4, x planes chosen per grid, TMA
    copies) in both precisions against the float64 oracle on the throughput case at 128^3 (CPML 16), over six
    chunks (186 steps): fields, both DFT accumulators and the decay-energy proxy."""
    from lightsmith_b200.engine import Engine
    from lightsmith_b200.workloads import throughput_plan
    from oracle.engine import OracleEngine

    plan = throughput_plan(128, max_steps=4000, seed=5, single=False)
    ref = OracleEngine(plan, threads=8)
    eng = Engine.from_plan(plan, precision=precision)
    eng.set_tuning(4, 8, 0, 4)
    assert eng.fused and eng.uses_tma
    for _ in range(6):
        ref.chunk()
        eng.chunk(1, use_graph=True)
    ref.close()
    assert np.abs(ref.E).max() > 0
    assert _rel(eng.E.cpu().numpy(), ref.E) < tol
    assert _rel(eng.H.cpu().numpy(), ref.H) < tol
    assert _rel(eng.results(0)[0], ref.monitors[0]["acc_e"]) < tol
    assert _rel(eng.results(0)[1], ref.monitors[0]["acc_h"]) < tol
    np.testing.assert_allclose(eng.energy.cpu().numpy()[0], ref.energy[0], rtol=10 * tol)
    eng.close()


@pytest.mark.parametrize("variant", [3, 4])
@pytest.mark.parametrize("n,pml", [(128, 16), (100, 10), (72, 12)])
def test_split_and_lean_passes_equal_fused_pass_on_the_throughput_case(n, pml, variant):
    """Interior box plus shell (3) and the lean-CPML pass (4) against the one-kernel fused pass, on grids
    whose box and slab edges fall inside tiles and x segments (n = 100, 72) and where they do not (128): the
    same arithmetic per value, equal to the last bits (the kernels may contract multiply-adds differently)."""
    from lightsmith_b200.engine import Engine
    from lightsmith_b200.workloads import throughput_plan

    plan = throughput_plan(n, pml=pml, max_steps=2000, seed=5)
    w = plan["sources"][0].wave
    first = int(np.nonzero(np.abs(w) > 1e-3 * np.abs(w).max())[0][0])
    plan["sources"][0].wave = np.concatenate([w[first:], np.zeros(first)])
    a = Engine.from_plan(plan)
    b = Engine.from_plan(plan)
    a.set_tuning(1, 8, 24, 4)
    b.set_tuning(variant, 8, 24, 4)
    assert a.uses_tma and b.uses_tma
    for _ in range(3):
        a.chunk(1, use_graph=True)
        b.chunk(1, use_graph=True)
    b.check_status()
    ea, eb = a.E.cpu().numpy(), b.E.cpu().numpy()
    assert np.abs(ea).max() > 0
    assert _rel(eb, ea) < 2e-6
    assert _rel(b.H.cpu().numpy(), a.H.cpu().numpy()) < 2e-6
    assert _rel(b.results(0)[0], a.results(0)[0]) < 2e-6
    a.close()
    b.close()


@pytest.mark.slow
def test_full_size_run_is_linear_in_the_source_bit_for_bit():
    """Every update is linear in the fields, and scaling by 2 is exact in binary floating point (away from
    subnormal numbers, which the wavefront's far tail reaches): doubling the source current must double every
    normal-range field value exactly, at the full 640^3 size."""
    import torch

    from lightsmith_b200.engine import Engine
    from lightsmith_b200.workloads import throughput_plan

    n = 640
    gen = torch.Generator(device="cuda").manual_seed(7)
    inv = 1.0 / (torch.rand((n, n, n), generator=gen, device="cuda", dtype=torch.float32) * 11.25 + 1.0)
    plan = throughput_plan(n, inv_eps=inv, max_steps=3000)
    # start the pulse early so that a short run carries a sizeable field
    w = plan["sources"][0].wave
    first = int(np.nonzero(np.abs(w) > 1e-3 * np.abs(w).max())[0][0])
    plan["sources"][0].wave = np.concatenate([w[first:], np.zeros(first)])
    a = Engine.from_plan(plan)
    a.chunk(2, use_graph=True)
    e1 = a.E[:, ::7, ::5, ::3].clone()
    h1 = a.H[:, ::5, ::7, ::3].clone()
    acc1 = a.monitors[0]["acc_e"].clone()
    a.close()
    del a
    plan["sources"][0].coef = 2 * plan["sources"][0].coef
    b = Engine.from_plan(plan)
    b.chunk(2, use_graph=True)
    def same(x, ref):
        normal = ref.abs() > 1e-30
        assert int(normal.sum()) > 1000
        assert torch.equal(x[normal], ref[normal])
        assert float((x - ref)[~normal].abs().max()) < 1e-30

    assert float(e1.abs().max()) > 0
    same(b.E[:, ::7, ::5, ::3], 2 * e1)
    same(b.H[:, ::5, ::7, ::3], 2 * h1)
    same(torch.view_as_real(b.monitors[0]["acc_e"]), torch.view_as_real(2 * acc1))
    b.close()
