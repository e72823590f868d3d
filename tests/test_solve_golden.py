"""Whole-solve parity: the dispersive-sphere scattering run that ``ls.solve(sim, "fdtd", "cpu")`` made.

Each ``solve_sphere_*.npz`` fixture holds the plan lightsmith's scattering driver handed to its engine (a
16 nm Drude-Lorentz sphere in n = 1.33, 49^3 cells at 4 nm, CPML 8, table-fed TF/SF, two flux boxes and the
incident reference view; staircase and subpixel meshing, and with symmetry="auto" a quarter grid of 26 x 26 x 49
cells between a PEC and a PMC mirror plane; a non-dispersive n = 2 sphere with conformal interfaces, whose
off-diagonal 1/eps terms the plan carries as gather tables; the metal sphere with conformal interfaces (the
vertex-tensor ADE), and with lightsmith's default options, conformal and symmetry="auto" together), the
driver's post-processing inputs, and lightsmith's own accumulators and cross sections (float64). The run is replayed for the recorded number of steps, and
C_ext, C_sca and C_abs are formed by the oracle's restatement of the driver's post-processing.
"""

import numpy as np
import pytest

from oracle.post import cross_sections

CASES = ["sphere_staircase", "sphere_subpixel", "sphere_symmetric", "dielectric_conformal", "sphere_conformal",
         "sphere_defaults"]
RTOL_F64 = 1e-9  # float64 on the GPU: the same arithmetic, a different summation order at shared nodes
RTOL_F32 = 1e-4  # float32 on the GPU against lightsmith's float64 CPU run (lightsmith's own GPU-vs-CPU bar)


def _accumulators(eng, n_mon):
    es, hs = [], []
    for k in range(n_mon):
        e, h = eng.results(k)
        es.append(np.asarray(e))
        hs.append(None if h is None else np.asarray(h))
    return es, hs


@pytest.mark.parametrize("case", CASES)
def test_post_processing_reproduces_lightsmith(case, golden):
    d = golden("solve_" + case)
    out = d["out"]
    cs = cross_sections(out["acc_e"], out["acc_h"], d["post"])
    for k in ("c_ext", "c_sca", "c_abs"):
        np.testing.assert_allclose(cs[k], out[k], rtol=1e-13, atol=0)


@pytest.mark.slow
@pytest.mark.parametrize("case", CASES)
def test_oracle_replays_the_solve(case, golden):
    from oracle.engine import OracleEngine

    d = golden("solve_" + case)
    plan, out, post = d["plan"], d["out"], d["post"]
    eng = OracleEngine(plan, threads=4)
    for _ in range(post["steps"] // plan["stride"]):
        eng.chunk()
    eng.close()
    assert eng.n == out["n"]
    es, hs = _accumulators(eng, len(plan["monitors"]))
    cs = cross_sections(es, hs, post)
    for k in ("c_ext", "c_sca", "c_abs"):
        np.testing.assert_allclose(cs[k], out[k], rtol=1e-10, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("case", CASES)
def test_cuda_engine_replays_the_solve(case, precision, golden):
    from lightsmith_b200.engine import Engine

    d = golden("solve_" + case)
    plan, out, post = d["plan"], d["out"], d["post"]
    eng = Engine.from_plan(plan, precision=precision)
    run, used = eng.make_runner(True)
    assert used
    for _ in range(post["steps"] // plan["stride"]):
        run()
    assert eng.n_host == out["n"]
    es, hs = _accumulators(eng, len(plan["monitors"]))
    eng.close()
    cs = cross_sections(es, hs, post)
    rtol = RTOL_F64 if precision == "double" else RTOL_F32
    for k in ("c_ext", "c_sca", "c_abs"):
        np.testing.assert_allclose(cs[k], out[k], rtol=rtol, atol=0, err_msg=f"{case} {precision} {k}")
