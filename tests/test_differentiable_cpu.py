"""The differentiable FDTD solve on the host: the port-amplitude rows against lightsmith's own
``ModeTable.amplitudes``, the protocol lightsmith's inverse design checks, and the permittivity mapping of
``DeviceSolver``. The lightsmith parts run where its sources are available and skip elsewhere."""

import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from refsrc import add_to_path  # noqa: E402

HAVE_LS = add_to_path()
needs_ls = pytest.mark.skipif(not HAVE_LS, reason="lightsmith sources not available")


def _problem():
    from device_problems import diff_device_problem

    return diff_device_problem()


@pytest.fixture(scope="module")
def runs():
    if not HAVE_LS:
        pytest.skip("lightsmith sources not available")
    from lightsmith_b200.backend import device_runs

    return device_runs(_problem(), keep_tables=True)


@needs_ls
def test_port_rows_restate_the_mode_amplitudes(runs):
    """Each row's linear functional gives ModeTable.amplitudes (ports.py:265-280) on random accumulators."""
    rng = np.random.default_rng(5)
    nw = len(runs["omega"])
    mons = runs["plans"][0]["monitors"]
    ne = [len(m["e_idx"]) for m in mons]
    nh = [len(m["h_idx1"]) for m in mons]
    E = [rng.normal(size=(nw, n)) + 1j * rng.normal(size=(nw, n)) for n in ne]
    H = [rng.normal(size=(nw, n)) + 1j * rng.normal(size=(nw, n)) for n in nh]
    Ecat, Hcat = np.concatenate(E, 1), np.concatenate(H, 1)
    r = 0
    for fi, tab in enumerate(runs["tables"]):
        for mm in range(tab.frame.num_modes):
            row = runs["rows"][r]
            a_ref, c_ref = tab.amplitudes(runs["omega"], E[fi], H[fi], mm)
            e0, h0 = row["e_off"], row["h_off"]
            Ef, Hf = Ecat[:, e0:e0 + ne[fi]], Hcat[:, h0:h0 + nh[fi]]
            a = (row["in_e"] * Ef).sum(1) + (row["in_h"] * Hf).sum(1)
            c = (row["out_e"] * Ef).sum(1) + (row["out_h"] * Hf).sum(1)
            np.testing.assert_allclose(a, a_ref, rtol=1e-12, atol=1e-12 * np.abs(a_ref).max())
            np.testing.assert_allclose(c, c_ref, rtol=1e-12, atol=1e-12 * np.abs(c_ref).max())
            r += 1
    assert r == len(runs["labels"]) == 2


@needs_ls
def test_runs_follow_the_device_driver(runs):
    from lightsmith.backends._fdtd import device as D
    from lightsmith.backends.fdtd import NativeFDTD

    prob = _problem()
    p = D.plan(prob, NativeFDTD._options(prob), False)
    assert tuple(runs["shape"]) == tuple(p["grid"].shape)
    assert runs["n_steps"] == p["max_steps"]
    assert runs["mesh"] == "subpixel"
    for pl in runs["plans"]:
        assert len(pl["monitors"]) == 2 and type(pl["sources"][0]).__name__ == "ModeSource"
        assert pl["stride"] == p["stride"]


@needs_ls
def test_backend_serves_lightsmiths_inverse_protocol(runs):
    from lightsmith.device import Device
    from lightsmith.inverse.topopt import check_backend

    from lightsmith_b200.backend import B200FDTD
    from lightsmith_b200.differentiable import DeviceSolver

    check_backend(B200FDTD)
    solver = DeviceSolver({k: v for k, v in runs.items() if k != "tables"})
    g = B200FDTD.design_grid(None, solver=solver)
    assert g.shape == tuple(runs["shape"]) and len(g.x) == g.shape[0] and len(g.z) == g.shape[2]
    assert np.allclose(np.diff(g.x), g.dl)
    base = B200FDTD.base_permittivity(None, solver=solver)
    assert base.shape == (len(runs["wavelengths_nm"]),) + g.shape and np.iscomplexobj(base)
    assert base.real.min() > 2.0 and base.real.max() < 12.2  # silica 1.44^2 .. silicon 3.48^2
    with pytest.raises(ValueError, match="CUDA"):
        B200FDTD.differentiable_solve(_problem(), None, Device("numpy", "cpu"), solver=solver)


def test_permittivity_mapping_on_the_box():
    """Nodes equal to the base keep the per-component 1/eps; changed nodes take 1/eps on all three; changes
    outside the interior box are rejected."""
    from lightsmith_b200.differentiable import DeviceSolver, interior_box

    shape = (12, 10, 14)
    rng = np.random.default_rng(1)
    inv = rng.uniform(0.1, 1.0, size=(3,) + shape)
    desc = {"shape": shape, "inv_eps": inv, "pml_cells": ((3, 3), (0, 0), (2, 4)), "labels": ["a"],
            "n_steps": 10, "omega": [1.0], "plans": [], "rows": []}
    s = DeviceSolver(desc)
    assert s.box == interior_box(shape, desc["pml_cells"]) == ((4, 7), (1, 9), (3, 8))
    eps = s.base_nodes.copy()
    assert np.array_equal(s.inv_eps_box(eps), inv[:, 4:7, 1:9, 3:8])
    eps[5, 2, 4] = 4.0
    got = s.inv_eps_box(eps)
    assert np.allclose(got[:, 1, 1, 1], 0.25)
    got[:, 1, 1, 1] = inv[:, 5, 2, 4]
    assert np.array_equal(got, inv[:, 4:7, 1:9, 3:8])
    eps[3, 2, 4] = 4.0  # in the x CPML slab
    with pytest.raises(ValueError, match="interior box"):
        s.inv_eps_box(eps)


@needs_ls
def test_two_d_device_design_grid_is_its_stepped_plane():
    """A 2D device: the periodic invariant axis has three nodes; the design grid is (x, y), without ``z``, as
    lightsmith's region_map tells 2D from 3D (inverse/parametrization.py:159)."""
    from device_problems import diff_device_problem

    from lightsmith_b200.backend import B200FDTD, device_runs
    from lightsmith_b200.differentiable import DeviceSolver

    desc = device_runs(diff_device_problem(2))
    assert desc["two_d"] and desc["shape"][2] == 3 and desc["plans"][0]["periodic"] == (False, False, True)
    solver = DeviceSolver(desc)
    g = B200FDTD.design_grid(None, solver=solver)
    assert not hasattr(g, "z") and g.shape == tuple(desc["shape"][:2]) == solver.design_shape
    base = B200FDTD.base_permittivity(None, solver=solver)
    assert base.shape == (2,) + g.shape
    np.testing.assert_array_equal(solver.nodes(base[0].real), solver.base_nodes)
    assert solver.box[2] == (1, 2)


@needs_ls
def test_step_count_without_a_run_time_follows_lightsmiths_run_loop():
    """Without run_time_fs the step count is the one lightsmith's run loop reaches on the base structure's
    first run (here on lightsmith's own CPU engine): the steps its own solve of the problem reports."""
    import lightsmith as ls
    from device_problems import diff_device_problem
    from lightsmith.backends._fdtd.engine import Engine as RefEngine
    from lightsmith.device import Device

    from lightsmith_b200.backend import device_runs

    p = diff_device_problem(2)
    fdtd = {k: v for k, v in p.options["fdtd"].items() if k != "run_time_fs"}
    fdtd.update(max_time_fs=600.0, decay_by=1e-2)  # decays at 6200 steps, before the 10720-step cap
    p = p.model_copy(update={"options": {"fdtd": fdtd}})
    with pytest.raises(ValueError, match="run_time_fs"):
        device_runs(p)
    desc = device_runs(p, Device("numpy", "cpu"), engine=RefEngine)
    res = ls.solve(p, "fdtd", "cpu")
    assert desc["n_steps"] == res.provenance["runs"][0]["steps"] < 10720


@needs_ls
def test_lightsmiths_optimiser_takes_the_backend(monkeypatch):
    """lightsmith's TopologyOptimizer (inverse/topopt.py:96-130) set up on the FDTD backend: it prepares the
    runs, maps a design region onto the design grid and composes the permittivity; the solve itself needs a
    CUDA device (raised here, on the host)."""
    from device_problems import diff_device_problem
    from lightsmith import inverse
    from lightsmith.backends import base as ls_base
    from lightsmith.inverse.topopt import TopologyOptimizer

    from lightsmith_b200.backend import B200FDTD

    monkeypatch.setattr(ls_base, "_REGISTRY", {**ls_base._REGISTRY, "lightsmith-fdtd": B200FDTD})
    monkeypatch.setattr(ls_base, "_PLUGINS_LOADED", True)
    import lightsmith as ls

    dev = diff_device_problem(3)
    spec = inverse.OptimizationProblem(
        device=dev, backend="lightsmith-fdtd",
        design_regions=[inverse.DesignRegion(center_nm=(0, 0, 0), size_nm=(400, 600, 220),
                                             material_low=ls.ConstantIndex(n_real=1.44),
                                             material_high=ls.ConstantIndex(n_real=3.48))],
        objective=[inverse.SParameterTerm(out_port="o2", in_port="o1")])
    opt = TopologyOptimizer(spec, device="cpu")
    assert opt.grid.shape == tuple(opt.ctx["solver"].design_shape) and opt.sources == ["o1"]
    (reg,) = opt.regions
    expect = tuple(int(np.sum(np.abs(c) <= h + 1e-9)) for c, h in ((opt.grid.x, 200), (opt.grid.y, 300)))
    assert reg.shape == expect and reg.mode == "extruded" and expect[0] >= 10  # nodes of a 400 x 600 nm box
    import torch

    eps, proj, _ = opt.permittivity(torch.as_tensor(opt.initial_x()), 1.0)
    assert tuple(eps.shape) == (2,) + opt.grid.shape
    assert float(eps.real.max()) < 12.2 and float(eps.real.min()) > 2.0
    with pytest.raises(ValueError, match="CUDA"):
        opt.solve(eps)
