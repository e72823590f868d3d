"""The GPU voxeliser (``lightsmith_b200.voxel``, ``csrc/voxel.cu``) against lightsmith's own ``voxelise``
(backends/_fdtd/setup.py:110-289) on the calls lightsmith's drivers make: each scene is posed to lightsmith
(its CPU solve), the driver's call of ``voxelise`` is answered by both and the solve stopped there. inv_eps,
the dispersive groups (indices, media, fractions, weights), the statistics and the conformal off-diagonal
terms must be identical, bit for bit."""

import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from refsrc import add_to_path  # noqa: E402

if not add_to_path():
    pytest.skip("lightsmith (the reference install, baseline/_ref) not available", allow_module_level=True)

import lightsmith as ls  # noqa: E402
from lightsmith.backends._fdtd import emission as E_drv  # noqa: E402
from lightsmith.backends._fdtd import scattering as S_drv  # noqa: E402
from problems import DRUDE_LORENTZ, c0_problem, dielectric_sphere_problem, emission_problem, sphere_problem  # noqa: E402
from problems import with_options  # noqa: E402

from lightsmith_b200 import voxel  # noqa: E402

pytestmark = pytest.mark.gpu


class _Stop(Exception):
    pass


def _both(prob):
    """(lightsmith's voxelise result, the GPU one or None where it does not serve the call, the mesh mode) for
    the driver's first call of voxelise on ``prob``."""
    got = {}
    drv = E_drv if isinstance(prob, ls.problems.EmissionProblem) else S_drv
    slot_attr = "particle_slot_fn" if drv is E_drv else "_slot_fn"
    saved = getattr(drv, slot_attr), drv.voxelise

    def slots(*a):
        sim, slot_of = a[0], a[1]
        sub = None
        if drv is S_drv and sim.substrate is not None:
            sub = (sim.substrate.interface_z_nm, a[2] - 1)
        return voxel.ShapeSlots(saved[0](*a), sim.particles, slot_of, sub)

    def both(slot_fn, media, shape, origin, dx, roi_lo, roi_hi, *, mode="subpixel", samples=8, base=None,
             background=(), grid=None, **kw):
        host = saved[1](slot_fn, media, shape, origin, dx, roi_lo, roi_hi, mode=mode, samples=samples,
                        base=None if base is None else (base[0].copy(), list(base[1])), background=background,
                        grid=grid, **kw)
        gpu = None
        if voxel.supports(slot_fn, media, mode, samples, grid):
            gpu = voxel.voxelise_gpu(slot_fn, media, shape, origin, dx, roi_lo, roi_hi, mode=mode, samples=samples,
                                     base=base, background=background, device="cuda:0")
        got.update(host=host, gpu=gpu, mode=mode)
        raise _Stop

    setattr(drv, slot_attr, slots)
    drv.voxelise = both
    try:
        ls.solve(prob, method="fdtd", device="cpu")
    except _Stop:
        pass
    finally:
        setattr(drv, slot_attr, saved[0])
        drv.voxelise = saved[1]
    return got["host"], got["gpu"], got["mode"]


def _assert_same(host, gpu):
    inv_h, groups_h, stats_h, od_h = host
    inv_g, groups_g, stats_g, od_g = gpu
    assert inv_g.shape == inv_h.shape and np.array_equal(inv_g, inv_h)
    assert stats_g == stats_h
    assert len(groups_g) == len(groups_h)
    for gh, gg in zip(groups_h, groups_g):
        assert np.array_equal(gg.idx, gh.idx)
        assert [m is n for m, n in zip(gg.media, gh.media)] == [True] * len(gh.media) and len(gg.media) == len(gh.media)
        assert np.array_equal(gg.frac, gh.frac)
        assert (gg.w is None) == (gh.w is None) and (gh.w is None or np.array_equal(gg.w, gh.w))
    assert (od_g is None) == (od_h is None)
    if od_h is not None:
        assert np.array_equal(od_g.idx3, od_h.idx3) and np.array_equal(od_g.comp, od_h.comp)
        assert np.array_equal(od_g.coef, od_h.coef)


def _mixed_scene(mode: str, dispersive: bool = True, substrate: bool = False):
    """Four overlapping particles of every shape the voxeliser serves (the first listed wins overlaps): a
    layered sphere with two shells, a spheroid, a cylinder and a sphere, in n = 1.33, 4 nm cells."""
    metal = ls.DrudeLorentz(**DRUDE_LORENTZ) if dispersive else ls.ConstantIndex(n_real=1.9)
    parts = [
        ls.Particle(shape=ls.LayeredSphere(core_radius_nm=10.0, shells=[
            ls.Shell(thickness_nm=4.0, material=ls.ConstantIndex(n_real=2.2)),
            ls.Shell(thickness_nm=5.0, material=metal)]), material=ls.ConstantIndex(n_real=1.5),
            position_nm=(-9.0, 3.0, 1.0)),
        ls.Particle(shape=ls.Spheroid(semi_axis_xy_nm=9.0, semi_axis_z_nm=15.0), material=ls.ConstantIndex(n_real=2.6),
                    position_nm=(14.0, -6.0, 2.0)),
        ls.Particle(shape=ls.Cylinder(radius_nm=7.0, length_nm=26.0), material=metal, position_nm=(2.0, 15.0, -5.0)),
        ls.Particle(shape=ls.Sphere(radius_nm=8.0), material=ls.ConstantIndex(n_real=3.1), position_nm=(3.0, 3.0, 12.0)),
    ]
    kw = {}
    if substrate:
        kw["substrate"] = ls.Substrate(material=ls.ConstantIndex(n_real=1.45), interface_z_nm=-14.0)
    return ls.Simulation(particles=parts, medium_index=1.33, wavelengths={"start_nm": 500.0, "stop_nm": 700.0, "num": 3},
                         options={"fdtd": dict(spacing_nm=4.0, pml_cells=8, symmetry="off", mesh_refinement=mode,
                                               padding_nm=8.0, pml_gap_nm=8.0, run_time_fs=1.0)}, **kw)


SCENES = {
    "sphere_staircase": lambda: sphere_problem("staircase"),
    "sphere_subpixel": lambda: sphere_problem("subpixel"),
    "sphere_volume_average": lambda: sphere_problem("volume_average"),
    "sphere_symmetric": lambda: sphere_problem("staircase", "auto"),
    "dielectric_conformal": dielectric_sphere_problem,
    "c0_full_size": c0_problem,
    "mixed_subpixel": lambda: _mixed_scene("subpixel"),
    "mixed_staircase": lambda: _mixed_scene("staircase"),
    "mixed_volume_average": lambda: _mixed_scene("volume_average"),
    "mixed_conformal_dielectric": lambda: _mixed_scene("conformal", dispersive=False),
    "mixed_subpixel_substrate": lambda: _mixed_scene("subpixel", substrate=True),
    "emission": emission_problem,
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_gpu_voxelise_equals_lightsmiths(name):
    host, gpu, mode = _both(SCENES[name]())
    assert gpu is not None, f"the GPU voxeliser does not serve {name} ({mode})"
    _assert_same(host, gpu)
    if mode != "staircase":
        assert host[2]["interface_cells"] > 0  # the scene has interface cells to supersample


def test_conformal_next_to_a_dispersive_medium_stays_on_the_host():
    host, gpu, mode = _both(sphere_problem("conformal"))
    assert mode == "conformal" and gpu is None and host[2]["tensor_vertices"] > 0


def test_a_solve_through_the_plugin_meshes_on_the_gpu(plugin, monkeypatch):
    """``ls.solve(sim, "fdtd", "gpu")`` with the plugin: the scattering driver's voxelise runs on the GPU (the
    result's provenance says so), and every number of the result equals that of the same solve meshed on the
    host by lightsmith."""
    from problems import flatten_result

    prob = with_options(sphere_problem("subpixel"), precision="double")
    res = ls.solve(prob, method="fdtd", device="gpu")
    assert res.provenance.get("voxelise_on_gpu") == "subpixel"
    monkeypatch.setattr(plugin.B200FDTD, "gpu_voxelise", False)
    ref = ls.solve(prob, method="fdtd", device="gpu")
    assert "voxelise_on_gpu" not in ref.provenance
    got, want = flatten_result(res), flatten_result(ref)
    assert sorted(got) == sorted(want)
    for k in want:
        assert np.array_equal(got[k], want[k]), k
