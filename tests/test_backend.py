"""The lightsmith plugin (``lightsmith_b200.backend.B200FDTD``) on the host: registration through the entry
point, what it rejects, and that a solve on a CUDA device hands lightsmith's own driver plan to the CUDA
engine. These run where the lightsmith sources are available and skip elsewhere (the GPU host has none)."""

import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from refsrc import add_to_path  # noqa: E402

if not add_to_path():
    pytest.skip("lightsmith sources not available", allow_module_level=True)

import lightsmith as ls  # noqa: E402
from lightsmith.backends import base as ls_base  # noqa: E402
from lightsmith.device import Device  # noqa: E402

from lightsmith_b200 import backend as B  # noqa: E402
from lightsmith_b200 import plan as P  # noqa: E402

CUDA0 = Device("torch", "cuda:0")


def sphere(mesh="staircase", **extra):
    """The dispersive-sphere problem of the ``solve_sphere_*`` fixtures."""
    mat = ls.DrudeLorentz(eps_inf=5.9, wp_ev=9.0, gamma_ev=0.07,
                          poles=[{"delta_eps": 1.3, "omega0_ev": 2.6, "gamma_ev": 0.6},
                                 {"delta_eps": 1.5, "omega0_ev": 3.7, "gamma_ev": 1.0}])
    fdtd = dict(spacing_nm=4.0, pml_cells=8, symmetry="off", mesh_refinement=mesh, padding_nm=8.0,
                pml_gap_nm=8.0, dft_stride=10, run_time_fs=399.5 * 2.2863 / 299.792458)
    fdtd.update(extra)
    return ls.Simulation(particles=[ls.Particle(shape=ls.Sphere(radius_nm=16.0), material=mat)], medium_index=1.33,
                         wavelengths={"start_nm": 400.0, "stop_nm": 800.0, "num": 9}, options={"fdtd": fdtd})


def test_class_mirrors_the_builtin_backend():
    from lightsmith.backends.fdtd import NativeFDTD

    assert issubclass(B.B200FDTD, NativeFDTD)
    assert (B.B200FDTD.name, B.B200FDTD.method, B.B200FDTD.gpu) == ("lightsmith-fdtd", "fdtd", True)
    assert B.B200FDTD.problem_kinds == NativeFDTD.problem_kinds
    assert B.B200FDTD.options_model is NativeFDTD.options_model


def test_entry_point_replaces_the_builtin_backend(tmp_path, monkeypatch):
    """An installed distribution declaring the entry point (as pyproject.toml does) takes the FDTD slot."""
    dist = tmp_path / "lightsmith_b200-0.1.0.dist-info"
    dist.mkdir()
    (dist / "METADATA").write_text("Metadata-Version: 2.1\nName: lightsmith-b200\nVersion: 0.1.0\n")
    (dist / "entry_points.txt").write_text(
        "[lightsmith.backends]\nlightsmith-fdtd-b200 = lightsmith_b200.backend:B200FDTD\n")
    monkeypatch.syspath_prepend(str(tmp_path))
    monkeypatch.setattr(ls_base, "_REGISTRY", dict(ls_base._REGISTRY))
    monkeypatch.setattr(ls_base, "_PLUGINS_LOADED", False)
    assert ls_base.get_backend("fdtd", kind="scattering") is B.B200FDTD
    assert ls_base.get_backend("lightsmith-fdtd") is B.B200FDTD


@pytest.mark.parametrize("extra, why", [
    (dict(grid="auto"), "graded"),
])
def test_supports_rejects_options_without_a_cuda_path(extra, why):
    ok, msg = B.B200FDTD.supports(sphere(**extra))
    assert not ok and why in msg


def test_supports_rejects_resonances_output():
    sim = sphere().model_copy(update={"outputs": sphere().outputs.model_copy(update={"resonances": {}})})
    ok, msg = B.B200FDTD.supports(sim)
    if sim.outputs.resonances is None:  # the model normalised the empty request away
        pytest.skip("resonances output could not be requested this way")
    assert not ok and "resonances" in msg


def test_supports_accepts_the_sphere_problem():
    for mesh in ("staircase", "subpixel", "volume_average", "conformal"):
        assert B.B200FDTD.supports(sphere(mesh)) == (True, "")


class _Recorded(Exception):
    pass


def test_solve_hands_lightsmiths_plan_to_the_cuda_engine(monkeypatch, golden):
    """On a CUDA device the scattering driver builds the B200 engine with the very plan the fixture recorded
    from lightsmith's CPU solve (precision aside: 'auto' is single on a GPU)."""
    seen = {}

    class Recorder:
        def __init__(self, device, **kw):
            seen["device"] = device
            seen["plan"] = P.make_plan(**kw)
            raise _Recorded

    monkeypatch.setattr(B._engine, "Engine", Recorder)
    saved = [m.Engine for m in B._DRIVERS]
    with pytest.raises(_Recorded):
        B.B200FDTD.solve(sphere(), CUDA0)
    assert [m.Engine for m in B._DRIVERS] == saved  # the drivers' own engine is back
    assert seen["device"] is CUDA0
    got, want = P.dumps(seen["plan"]), P.dumps(golden("solve_sphere_staircase")["plan"])
    assert seen["plan"]["single"] is True
    skel = lambda a: bytes(a["__skeleton__"]).decode().replace('"single": true', '"single": false')  # noqa: E731
    assert skel(got) == skel(want)
    assert sorted(got) == sorted(want)
    for k in want:
        if k != "__skeleton__":
            np.testing.assert_array_equal(got[k], want[k], err_msg=k)


def test_mirror_planes_reach_the_cuda_engine(monkeypatch):
    """symmetry='auto' gives this sphere mirror planes: the driver hands the CUDA engine a plan that keeps them
    (a half or quarter grid stepped with PEC/PMC planes at node 1)."""
    seen = {}

    class Recorder:
        def __init__(self, device, **kw):
            seen["plan"] = P.make_plan(**kw)
            raise _Recorded

    monkeypatch.setattr(B._engine, "Engine", Recorder)
    with pytest.raises(_Recorded):
        B.B200FDTD.solve(sphere(symmetry="auto"), CUDA0)
    mirror = seen["plan"].get("mirror", (0, 0, 0))
    assert any(mirror) and all(m in (-1, 0, 1) for m in mirror)


def test_solve_on_cuda_without_a_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="CUDA"):
        B.B200FDTD.solve(sphere(), CUDA0)


def dielectric_sphere(mesh="conformal"):
    """A non-dispersive sphere (n = 2) in n = 1.33: conformal interfaces take off-diagonal 1/eps terms."""
    fdtd = dict(spacing_nm=4.0, pml_cells=8, symmetry="off", mesh_refinement=mesh, padding_nm=8.0,
                pml_gap_nm=8.0, dft_stride=10, run_time_fs=399.5 * 2.2863 / 299.792458)
    return ls.Simulation(particles=[ls.Particle(shape=ls.Sphere(radius_nm=16.0), material=ls.ConstantIndex(n_real=2.0))],
                         medium_index=1.33, wavelengths={"start_nm": 400.0, "stop_nm": 800.0, "num": 9},
                         options={"fdtd": fdtd})


def test_conformal_dielectric_reaches_the_cuda_engine_with_its_offdiagonal_terms(monkeypatch):
    """mesh_refinement='conformal' on a dielectric: supported, and the driver's OffDiagonal rows arrive as the
    plan's gather tables."""
    assert B.B200FDTD.supports(dielectric_sphere()) == (True, "")
    seen = {}

    class Recorder:
        def __init__(self, device, **kw):
            seen["plan"] = P.make_plan(**kw)
            raise _Recorded

    monkeypatch.setattr(B._engine, "Engine", Recorder)
    with pytest.raises(_Recorded):
        B.B200FDTD.solve(dielectric_sphere(), CUDA0)
    od = seen["plan"]["offdiag"]
    assert len(od["e"]) > 0 and od["h"].shape == od["w"].shape and od["h"].shape[1] >= 1


def _compare_plans(got, want, path=""):
    """Plans equal array for array, the off-diagonal tables as operators (their layout is this package's own)."""
    if isinstance(want, dict):
        assert isinstance(got, dict) and sorted(got) == sorted(want), path
        if path.endswith("offdiag") and "w" in want:
            from test_oracle_golden import sparse_operator

            ka, va = sparse_operator(got["e"], got["h"], got["w"])
            kb, vb = sparse_operator(want["e"], want["h"], want["w"])
            keys = np.union1d(ka, kb)
            da, db = np.zeros(len(keys), complex), np.zeros(len(keys), complex)
            da[np.searchsorted(keys, ka)], db[np.searchsorted(keys, kb)] = va, vb
            np.testing.assert_allclose(da, db, rtol=0, atol=1e-14 * np.abs(vb).max(), err_msg=path)
            return
        for k in want:
            _compare_plans(got[k], want[k], f"{path}/{k}")
    elif isinstance(want, (list, tuple)):
        assert len(got) == len(want), path
        for i, (g, w) in enumerate(zip(got, want)):
            _compare_plans(g, w, f"{path}/{i}")
    elif isinstance(want, np.ndarray):
        np.testing.assert_array_equal(np.asarray(got), want, err_msg=path)
    elif hasattr(want, "__dict__"):
        _compare_plans(got.__dict__, want.__dict__, path)
    elif path.endswith("/single"):
        assert got is True, path  # 'auto' precision is single on a GPU, the fixture's CPU solve double
    else:
        assert got == want, path


@pytest.mark.parametrize("name", ["sphere_staircase", "sphere_subpixel", "sphere_conformal", "sphere_symmetric",
                                  "sphere_defaults", "dielectric_conformal"])
def test_driver_plan_on_cuda_equals_lightsmiths(monkeypatch, golden, name):
    """The plan the scattering driver hands the CUDA engine (groups, vertex-tensor tables, off-diagonal terms,
    mirror planes, TF/SF tables, monitors) equals the one recorded from lightsmith's own CPU solve of the same
    problem; the conformal off-diagonal terms as the same operator as lightsmith's tables."""
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from problems import SOLVE_PROBLEMS

    seen = {}

    class Recorder:
        def __init__(self, device, **kw):
            seen["plan"] = P.make_plan(**kw)
            raise _Recorded

    monkeypatch.setattr(B._engine, "Engine", Recorder)
    with pytest.raises(_Recorded):
        B.B200FDTD.solve(SOLVE_PROBLEMS[name](), CUDA0)
    got = P.loads(P.dumps(seen["plan"]))  # through the fixture format, as the recorded plan went
    _compare_plans(got, golden("solve_" + name)["plan"])
