"""Driver-level parity: every engine lightsmith's periodic and emission drivers build inside
``ls.solve(problem, "fdtd", "cpu")``, replayed from the plan the driver handed its engine.

Each ``driver_*.npz`` fixture (``tests/golden/make_fixtures.py:driver_case``) holds, per engine the driver built,
that plan, the number of steps the run took and lightsmith's own DFT accumulators (float64):

* ``periodic_normal``: a square lattice (300 nm) of n = 2 pillars on glass at normal incidence, s polarisation,
  one real-valued run (22 x 22 x 78 cells at 15 nm, periodic x and y, CPML in z, the Bloch plane source);
* ``periodic_oblique``: the same lattice at theta = 30, phi = 10 degrees, p polarisation, one complex-valued
  Bloch-periodic run per wavelength (22 x 22 x 90 cells);
* ``emission``: a dipole 15 nm off an n = 2 sphere, the scene run and the run in the medium alone
  (69 x 69 x 75 cells at 4 nm, the point-dipole current source, flux box and far-field monitors);
* ``device_2d``, ``device_3d``: a silicon waveguide width step (500 -> 700 nm) in silica between two ports, one
  run per port with its mode source; 2D TE at 25 nm (123 x 139 x 3 cells) and a 220 nm wire in 3D at 40 nm
  (73 x 83 x 73 cells).

Each run is replayed for its recorded number of steps and every monitor's accumulators are compared with
lightsmith's, norm-wise per monitor.
"""

import numpy as np
import pytest

CASES = [("periodic_normal", 0), ("periodic_oblique", 0), ("periodic_oblique", 1), ("emission", 0),
         ("emission", 1), ("device_2d", 0), ("device_2d", 1), ("device_3d", 0), ("device_3d", 1)]
RTOL_F64 = 1e-9  # float64 on the GPU: the same arithmetic, a different summation order at shared nodes
RTOL_F32 = 2e-4  # float32 on the GPU against lightsmith's float64 CPU run


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def _check(eng_results, run, rtol, label):
    for k, (ref_e, ref_h) in enumerate(zip(run["acc_e"], run["acc_h"])):
        e, h = eng_results(k)
        assert _rel(e, ref_e) <= rtol, f"{label} monitor {k} E: {_rel(e, ref_e):.3e}"
        if ref_h.size:
            assert _rel(h, ref_h) <= rtol, f"{label} monitor {k} H: {_rel(h, ref_h):.3e}"


def test_driver_fixtures_cover_the_drivers(golden):
    for name, runs in (("periodic_normal", 1), ("periodic_oblique", 2), ("emission", 2), ("device_2d", 2),
                       ("device_3d", 2)):
        d = golden("driver_" + name)
        assert len(d["runs"]) == runs
        for run in d["runs"]:
            plan = run["plan"]
            assert run["n"] > 0 and run["n"] % plan["stride"] == 0
            assert len(run["acc_e"]) == len(plan["monitors"]) > 0
    oblique = golden("driver_periodic_oblique")["runs"][0]["plan"]
    assert oblique["complex"] and any(oblique["periodic"])
    emission = golden("driver_emission")["runs"][0]["plan"]
    assert type(emission["sources"][0]).__name__ == "DipoleSource"
    for name in ("device_2d", "device_3d"):
        assert type(golden("driver_" + name)["runs"][0]["plan"]["sources"][0]).__name__ == "ModeSource"


@pytest.mark.slow
@pytest.mark.parametrize("case,run", CASES)
def test_oracle_replays_the_driver(case, run, golden):
    from oracle.engine import OracleEngine

    r = golden("driver_" + case)["runs"][run]
    plan = r["plan"]
    eng = OracleEngine(plan, threads=4)
    for _ in range(r["n"] // plan["stride"]):
        eng.chunk()
    eng.close()
    assert eng.n == r["n"]
    _check(eng.results, r, 1e-10, f"{case}[{run}] oracle")


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("case,run", CASES)
def test_cuda_engine_replays_the_driver(case, run, precision, golden):
    from lightsmith_b200.engine import Engine

    r = golden("driver_" + case)["runs"][run]
    plan = r["plan"]
    eng = Engine.from_plan(plan, precision=precision)
    step, used = eng.make_runner(True)
    assert used
    for _ in range(r["n"] // plan["stride"]):
        step()
    assert eng.n_host == r["n"]

    def results(k):
        e, h = eng.results(k)
        return np.asarray(e), None if h is None else np.asarray(h)

    _check(results, r, RTOL_F64 if precision == "double" else RTOL_F32, f"{case}[{run}] {precision}")
    eng.close()
