"""The drop-in path on the GPU: ``ls.solve(problem, "fdtd", "gpu")`` with this package registered through
lightsmith's ``lightsmith.backends`` entry point (backends/base.py:96-103), run end to end on the CUDA engine.

Each problem is posed to lightsmith itself (``lightsmith`` from the reference install, ``baseline/_ref``): the
entry point hands the solve to ``B200FDTD``, lightsmith's own driver builds the plan and calls
``lightsmith_b200.engine.Engine`` where it would build its array-API engine, lightsmith's own run loop
(setup.py:722-773) drives the CUDA engine's ``make_runner``/``energy``/``release``, and lightsmith's own
post-processing reads the engine's DFT monitors. The results are compared with lightsmith's own CPU solve of
the same problem (``tests/golden/solve_results.npz``, float64): to 1e-9 when the GPU solve runs in float64,
and, in float32, to the tolerances lightsmith's own GPU-against-CPU tests use (tests/test_fdtd.py:125-132:
rtol 1e-4 on cross sections; tests/test_fdtd_periodic.py:127-132: atol 5e-5 on R and T).

Failure paths through the same chain: a run whose fields diverge raises lightsmith's ``FloatingPointError``
(setup.py:749-756; the case of tests/test_fdtd.py:89-99), as does a NaN written into a field from the host; a
progress callback raising ``progress.Cancelled`` stops the solve, and the next solve runs.
"""

import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from refsrc import add_to_path  # noqa: E402

if not add_to_path():
    pytest.skip("lightsmith (the reference install, baseline/_ref) not available", allow_module_level=True)

import lightsmith as ls  # noqa: E402
from problems import SOLVE_PROBLEMS, flatten_result, with_options  # noqa: E402

from lightsmith_b200 import plan as P  # noqa: E402

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def expected():
    return P.load(os.path.join(GOLDEN, "solve_results.npz"))


class _Counting:
    """Wraps the plugin's engine factory (what lightsmith's drivers call in place of their ``Engine``): counts the
    CUDA engines built in a solve and lets a test adjust each one."""

    def __init__(self, B, mp, adjust=None):
        self.n = 0
        real = B._b200_engine

        def make(device, **kw):
            self.n += 1
            eng = real(device, **kw)
            assert isinstance(eng, B._engine.Engine)
            return adjust(eng) if adjust else eng
        mp.setattr(B, "_b200_engine", make)


def _rel(got, want):
    scale = max(float(np.abs(want).max()), 1e-300)
    return float(np.abs(got - want).max() / scale)


# float32 tolerances: lightsmith's own GPU-against-CPU bounds for the same kind of result
def _f32_check(name, key, got, want):
    exact = ("wavelengths_nm", "angles_deg", "equivalent_radius_nm", "wavelength_nm", "offset_nm", "axis1_nm",
             "axis2_nm", "theta_deg", "phi_deg")
    if key.split("/")[-1] in exact or key.endswith("/order"):
        np.testing.assert_allclose(got, want, rtol=1e-12, err_msg=key)
    elif key.startswith(("near_field", "far_field")):
        # fields on a plane and dC_sca/dOmega at a few angles: relative to the largest value of the array (a
        # pointwise bound would fail at the near-zeros of a field pattern)
        assert _rel(got, want) < 1e-3, (key, _rel(got, want))
    elif name.startswith(("sphere", "dielectric")):
        np.testing.assert_allclose(got, want, rtol=1e-4, err_msg=key)  # tests/test_fdtd.py:131-132
    elif name.startswith("periodic"):
        np.testing.assert_allclose(got, want, rtol=0, atol=5e-5, err_msg=key)  # tests/test_fdtd_periodic.py:131
    elif name == "emission":
        np.testing.assert_allclose(got, want, rtol=1e-4, err_msg=key)
    else:  # S-parameters of the device problems
        np.testing.assert_allclose(got, want, rtol=0, atol=2e-4, err_msg=key)


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("name", sorted(SOLVE_PROBLEMS))
def test_solve_on_the_gpu_matches_lightsmiths_cpu_solve(plugin, expected, name, precision):
    problem = with_options(SOLVE_PROBLEMS[name](), precision=precision)
    with pytest.MonkeyPatch.context() as mp:
        count = _Counting(plugin, mp)
        res = ls.solve(problem, "fdtd", "gpu")
    assert count.n >= 1, "no CUDA engine was built"
    assert res.provenance["precision"] == precision
    if "framework" in res.provenance:
        assert res.provenance["framework"] == "torch"
    want = expected[name]
    if want["steps"] >= 0:
        assert int(res.provenance["steps"]) == want["steps"]
    got = flatten_result(res)
    assert sorted(got) == sorted(want["result"])
    for key, ref in want["result"].items():
        g = got[key]
        assert g.shape == ref.shape, key
        if precision == "double":
            # S-parameters come from forward/backward splits of modal overlaps, which amplify the accumulators'
            # agreement (about 1e-10 on these runs) tenfold; every other result is read off the accumulators
            tol = 1e-8 if name.startswith("device") else 1e-9
            assert _rel(g, ref) < tol, (key, _rel(g, ref))
        else:
            _f32_check(name, key, g, ref)


def _diverging_problem():
    """lightsmith's divergence case (tests/test_fdtd.py:89-99): a lossy constant index at under 3 cells per
    wavelength, stepped at the plain Courant limit."""
    return ls.Simulation(particles=[ls.Particle(shape=ls.Sphere(radius_nm=191), material=ls.ConstantIndex(
        n_real=1.2, n_imag=0.2))], medium_index=1.0, wavelengths=[500.0, 600.0, 700.0],
        options={"fdtd": {"spacing_nm": 191.0, "pml_cells": 4, "run_time_fs": 200.0}})


def test_diverging_run_raises_floating_point_error(plugin):
    from lightsmith.backends._fdtd import scattering

    with pytest.MonkeyPatch.context() as mp:
        mp.setattr(scattering, "time_step", lambda dx, courant, media, grid=None: courant * dx / np.sqrt(3))
        count = _Counting(plugin, mp)
        with pytest.raises(FloatingPointError, match="diverged.*finer mesh.*courant"):
            ls.solve(_diverging_problem(), "fdtd", "gpu")
    assert count.n == 1


def test_nan_written_from_the_host_raises_floating_point_error(plugin):
    """A NaN placed in E from the host after the third chunk: lightsmith's run loop reads a non-finite energy
    at the next chunk and raises."""
    chunks = {"n": 0}

    def poison(eng):
        run0 = eng.make_runner

        def make_runner(use_graphs):
            run, used = run0(use_graphs)

            def run_poisoned():
                run()
                chunks["n"] += 1
                if chunks["n"] == 3:
                    import torch

                    torch.cuda.synchronize()
                    eng.E_flat[eng.E_flat.numel() // 2] = float("nan")
            return run_poisoned, used
        eng.make_runner = make_runner
        return eng

    with pytest.MonkeyPatch.context() as mp:
        _Counting(plugin, mp, adjust=poison)
        with pytest.raises(FloatingPointError, match="non-finite"):
            ls.solve(with_options(SOLVE_PROBLEMS["sphere_staircase"](), precision="single"), "fdtd", "gpu")
    assert chunks["n"] >= 3


def test_cancelled_progress_stops_the_solve_and_the_next_solve_runs(plugin, expected):
    from lightsmith import progress

    seen = []

    def cb(event):  # lightsmith's callback receives one dict (progress.py:29-34)
        if event["stage"] == "fdtd_steps":
            seen.append(event.get("steps"))
            if len(seen) == 2:
                raise progress.Cancelled("stop")

    problem = with_options(SOLVE_PROBLEMS["sphere_staircase"](), precision="double")
    with pytest.raises(progress.Cancelled):
        ls.solve(problem, "fdtd", "gpu", progress=cb)
    assert len(seen) == 2
    res = ls.solve(problem, "fdtd", "gpu")
    want = expected["sphere_staircase"]["result"]
    assert _rel(np.asarray(res.c_ext_nm2), want["c_ext_nm2"]) < 1e-9


@pytest.mark.parametrize("precision", ["double", "single"])
def test_periodic_oblique_runs_are_batched_and_match_runs_one_by_one(plugin, expected, precision):
    """With a fixed run time, the periodic driver's oblique runs (one per wavelength here) advance together in
    one persistent kernel; R, T and the orders equal those of the same solve with the runs made one after
    another on the CUDA engine, and lightsmith's own CPU solve."""
    B = plugin
    problem = with_options(SOLVE_PROBLEMS["periodic_oblique"](), precision=precision)
    res_b = ls.solve(problem, "fdtd", "gpu")
    assert res_b.provenance.get("batched_oblique_runs") == 2
    assert all(r.get("batched") for r in res_b.provenance["runs"])
    with pytest.MonkeyPatch.context() as mp:
        mp.setattr(B.B200FDTD, "batch_oblique", False)
        res_s = ls.solve(problem, "fdtd", "gpu")
    assert "batched_oblique_runs" not in res_s.provenance
    got, seq, want = flatten_result(res_b), flatten_result(res_s), expected["periodic_oblique"]["result"]
    assert sorted(got) == sorted(seq) == sorted(want)
    for key in want:
        assert _rel(got[key], seq[key]) < (1e-12 if precision == "double" else 1e-5), key
        if precision == "double":
            assert _rel(got[key], want[key]) < 1e-9, key
        else:
            _f32_check("periodic_oblique", key, got[key], want[key])
