"""lightsmith's FDTD backend with its time loop on a B200 (sm_100a).

lightsmith finds backends through the ``lightsmith.backends`` entry-point group and keys its registry by
``Backend.name`` (backends/base.py:91-103). ``B200FDTD`` carries the built-in FDTD backend's own name,
``"lightsmith-fdtd"`` (backends/fdtd.py:48-56), so once this package is installed ``ls.solve(sim, "fdtd",
"gpu")`` reaches it with no change to lightsmith.

It is lightsmith's ``NativeFDTD`` with one part swapped: on a CUDA device, the problem drivers
(backends/_fdtd/scattering.py:416, emission.py:179, periodic.py:409,444, device.py:540) construct
``lightsmith_b200.engine.Engine`` where they would construct lightsmith's array-API ``Engine``. Options,
``supports``, ``estimate``, the drivers' set-up (voxelisation, sources, monitors, time step), the run loop
(setup.py:722-773) and the post-processing (cross sections, orders, S-parameters) are lightsmith's own.

On a CPU device the class is ``NativeFDTD`` unchanged: this package adds no CPU path. On a CUDA device there is
no fallback: a problem that needs a feature with no CUDA path here (graded grids, time monitors, substrates,
Gaussian beams) is rejected by ``supports`` or raises
``ValueError`` when its engine is built, and a missing or unloadable ``liblsfdtd.so`` raises from the engine.
"""

from __future__ import annotations

import threading

import numpy as np
from contextlib import contextmanager

from lightsmith.backends._fdtd import device as _device_driver
from lightsmith.backends._fdtd import emission as _emission_driver
from lightsmith.backends._fdtd import periodic as _periodic_driver
from lightsmith.backends._fdtd import scattering as _scattering_driver
from lightsmith.backends.fdtd import NativeFDTD
from lightsmith.problems import DeviceProblem, EmissionProblem, LayerStackProblem, PeriodicProblem
from lightsmith.spec import Simulation

from . import engine as _engine
from . import voxel as _voxel

__all__ = ["B200FDTD"]

# the modules whose `Engine` name the solve rebinds (each imports it with `from .engine import ... Engine`)
_DRIVERS = (_scattering_driver, _emission_driver, _periodic_driver, _device_driver)
_SWAP_LOCK = threading.RLock()


def _b200_engine(device, **kw):
    """lightsmith's ``Engine(device, **kw)`` call, answered by the CUDA engine."""
    try:
        return _engine.Engine(device, **kw)
    except NotImplementedError as e:  # a feature with no CUDA path: lightsmith's error for unsupported problems
        raise ValueError(f"{B200FDTD.name} (B200): {e}") from e


@contextmanager
def _engine_swapped():
    """Rebind the drivers' ``Engine`` to the CUDA engine for the duration of one solve."""
    with _SWAP_LOCK:
        saved = [m.Engine for m in _DRIVERS]
        try:
            for m in _DRIVERS:
                m.Engine = _b200_engine
            yield
        finally:
            for m, e in zip(_DRIVERS, saved):
                m.Engine = e


@contextmanager
def _nothing():
    yield


@contextmanager
def _voxeliser_swapped(device, used: list):
    """For the duration of one solve, the particle meshing of the scattering and emission drivers
    (``voxelise`` of their particle slot functions, setup.py:110-289) by the GPU voxeliser
    (``lightsmith_b200.voxel``) where it serves the scene; every call it serves is appended to ``used``."""
    S, E = _scattering_driver, _emission_driver
    saved = (S._slot_fn, S.voxelise, E.particle_slot_fn, E.voxelise)
    dev = _engine._device_name(device)

    def scattering_slots(sim, slot_of, n_media):
        sub = None if sim.substrate is None else (sim.substrate.interface_z_nm, n_media - 1)
        return _voxel.ShapeSlots(saved[0](sim, slot_of, n_media), sim.particles, slot_of, sub)

    def emission_slots(prob, slot_of):
        return _voxel.ShapeSlots(saved[2](prob, slot_of), prob.particles, slot_of)

    import torch

    on_gpu = torch.cuda.is_available()  # (the drivers' set-up runs without a GPU in the host-only tests)

    def dispatch(host_voxelise):
        def voxelise(slot_fn, media, shape, origin, dx, roi_lo, roi_hi, *, mode="subpixel", samples=8, base=None,
                     background=(), grid=None, **kw):
            if on_gpu and _voxel.supports(slot_fn, media, mode, samples, grid):
                used.append(mode)
                return _voxel.voxelise_gpu(slot_fn, media, shape, origin, dx, roi_lo, roi_hi, mode=mode,
                                           samples=samples, base=base, background=background, device=dev)
            return host_voxelise(slot_fn, media, shape, origin, dx, roi_lo, roi_hi, mode=mode, samples=samples,
                                 base=base, background=background, grid=grid, **kw)
        return voxelise

    with _SWAP_LOCK:
        try:
            S._slot_fn, S.voxelise = scattering_slots, dispatch(saved[1])
            E.particle_slot_fn, E.voxelise = emission_slots, dispatch(saved[3])
            yield
        finally:
            S._slot_fn, S.voxelise, E.particle_slot_fn, E.voxelise = saved


def _static_rejection(sim, opts) -> str:
    """Features known from the problem and its options alone that have no CUDA path here ('' if none)."""
    if isinstance(sim, (Simulation, DeviceProblem)) and _scattering_driver.graded(opts):
        return "does not support graded grids (grid='auto', mesh_override) on the GPU"
    if isinstance(sim, Simulation):
        if sim.outputs.resonances is not None:
            return "does not support the resonances output (time monitors) on the GPU"
        if sim.substrate is not None:
            return "does not support substrates on the GPU"
        if sim.illumination.kind == "gaussian_beam":
            return "does not support gaussian_beam illumination on the GPU"
    return ""


def _port_rows(tables, omega, e_counts, h_counts) -> list[dict]:
    """The port amplitudes of every port mode as linear functionals of its monitor's DFT accumulators.

    ``ModeTable.amplitudes`` (ports.py:265-280) forms p1 = <E, h> and p2 = <e, H> (unconjugated overlaps with
    the weights wa, wb), X = (p1 / u2 + p2) / (2 c N), Y = (u2 p1 - p2) / (2 c N) with u2 = exp(i beta s / 2),
    c = cos(beta s / 2), N = <e, h>, and moves them to the reference plane (exp(+-i beta ds)). Every step is
    linear in (E, H), so each amplitude is sum(kE E) + sum(kH H); the rows hold kE and kH, (n_w, points), for
    the incoming and the outgoing amplitude, and the offsets of the monitor's points in the concatenation of
    all port monitors."""
    e_off = np.concatenate([[0], np.cumsum(e_counts)])
    h_off = np.concatenate([[0], np.cumsum(h_counts)])
    rows = []
    for fi, tab in enumerate(tables):
        fr = tab.frame
        e, h, beta = tab.at(omega)
        for mm in range(fr.num_modes):
            em, hm, b = e[:, mm], h[:, mm], beta[:, mm]
            N = tab.overlap(em, hm)
            kE = np.stack([tab.wa * hm[:, 1], -tab.wb * hm[:, 0]], axis=1)  # p1 = sum kE E
            kH = np.stack([-tab.wb * em[:, 1], tab.wa * em[:, 0]], axis=1)  # p2 = sum kH H
            u2 = np.exp(0.5j * b * tab.spacing)
            c = np.cos(0.5 * b * tab.spacing)
            ds = fr.s_ref - fr.s_m
            x = (np.exp(1j * b * ds) / (2 * c * N))[:, None, None, None]
            y = (np.exp(-1j * b * ds) / (2 * c * N))[:, None, None, None]
            fwd = (kE * x / u2[:, None, None, None], kH * x)
            bwd = (kE * y * u2[:, None, None, None], -kH * y)
            inc, out = (fwd, bwd) if fr.delta > 0 else (bwd, fwd)
            nw = len(omega)
            rows.append({"e_off": int(e_off[fi]), "h_off": int(h_off[fi]),
                         "in_e": inc[0].reshape(nw, -1), "in_h": inc[1].reshape(nw, -1),
                         "out_e": out[0].reshape(nw, -1), "out_h": out[1].reshape(nw, -1)})
    return rows


def _decay_steps(problem, opts, p, src, kw, device, engine) -> int:
    """The step count lightsmith's run loop picks for the first port mode's run of the base structure
    (device.py:547-550 calling setup.py:722-773: until the monitors' energy has decayed, or the time cap), run
    on ``engine`` (the CUDA engine by default, on ``device``)."""
    import math

    from lightsmith.backends._fdtd import device as D
    from lightsmith.backends._fdtd.setup import run_until_decayed
    from lightsmith.problems import wavelength_array

    if engine is None:
        if device is None or not device.is_gpu:
            raise ValueError("the differentiable FDTD solve runs a fixed step count: set options['fdtd']"
                             "['run_time_fs'], pass n_steps, or give a CUDA device to find it by a decay run")
        engine = _engine.Engine
    wl = wavelength_array(problem.wavelengths)
    w1, dt, stride = p["band"][0], p["dt"], p["stride"]
    n_max = D._n_max(problem, wl)
    transit = 1.5 * n_max * float(np.sum(problem.domain_size_nm))
    eng = engine(device, **kw)
    steps, _, _ = run_until_decayed(eng, opts, max_steps=p["max_steps"], min_steps=int((src.t_off + transit) / dt),
                                    window=math.ceil(2 * np.pi * n_max / (w1 * stride * dt)), warnings=[])
    return int(steps)


def device_runs(problem, device=None, n_steps: int | None = None, keep_tables: bool = False,
                engine=None) -> dict:
    """The runs lightsmith's device driver makes for ``problem`` (backends/_fdtd/device.py:475-561), as the
    plain description ``lightsmith_b200.differentiable.DeviceSolver`` solves: one plan per port mode (its mode
    source and one DFT monitor per port), the driver's 1/eps, the port-amplitude rows, the design grid's node
    coordinates and the step count.

    The set-up is lightsmith's own (plan, voxelisation, mode tables, pulse band, CPML), with two choices the
    adjoint needs: the mesh is subpixel or staircase as the options ask (conformal asks for subpixel: the
    adjoint has no off-diagonal terms or vertex tensor; subpixel interface cells of a dispersive medium are mixed
    D-form groups, which it serves); the step count is fixed: the options' ``run_time_fs`` (the driver's ``max_steps``),
    ``n_steps``, or else the count lightsmith's run loop reaches on the base structure's first run (on
    ``engine``: the CUDA engine on ``device`` by default). ``keep_tables`` adds lightsmith's mode tables (not
    plain data) under ``"tables"``."""
    from lightsmith.backends._fdtd import device as D
    from lightsmith.backends._fdtd.engine import DFTMonitor, PMLSpec
    from lightsmith.backends._fdtd.ports import ModeSource, ModeTable
    from lightsmith.backends._fdtd.setup import voxelise
    from lightsmith.problems import wavelength_array

    from . import plan as P

    if not isinstance(problem, DeviceProblem):
        raise ValueError("the differentiable FDTD solve takes device problems")
    ok, why = D.supports(problem)
    if not ok:
        raise ValueError(why)
    problem = D._resolved(problem)
    opts = B200FDTD._options(problem)
    if D.graded(opts):
        raise NotImplementedError("graded grids have no CUDA path in lightsmith-b200")
    single = D.uses_single(opts, device) if device is not None else opts.precision == "single"
    p = D.plan(problem, opts, single)
    grid, frames, dt, stride = p["grid"], p["frames"], p["dt"], p["stride"]
    media = p["media"]
    wl = wavelength_array(problem.wavelengths)
    omega = 2 * np.pi / wl
    _, slots = D._media(problem, wl, [])
    w1, w2, wc, sigma, wa, wb = p["band"]
    dx = grid.engine_spacing()
    two_d = bool(grid.two_d)
    slot_fn = D._slot_fn(problem, slots, problem.domain_center_nm[2] if two_d else None)
    asked = opts.mesh_refinement or ("subpixel" if opts.subpixel else "staircase")
    mode = "staircase" if asked == "staircase" else "subpixel"
    inv_eps, groups, _, _ = voxelise(slot_fn, media, grid.shape, grid.origin, dx, np.array([1, 1, 1]),
                                     np.array(grid.shape) - 1, mode=mode, samples=opts.subpixel_samples,
                                     periodic=grid.periodic, grid=grid.graded)
    pol = {"te": "x", "tm": "y"}[opts.polarization or "te"] if two_d else None
    tables = [ModeTable(f, f.ds, dt, wa, wb, D._eps_fn(f, inv_eps, groups, dt), polarization=pol) for f in frames]
    n_bg = float(np.sqrt(max(media[0].eps_inf, 1.0)))
    cells = tuple((0, 0) if per else (grid.n_pml, grid.n_pml) for per in grid.periodic)
    pml = PMLSpec(cells=cells, kappa_max=opts.pml_kappa, alpha_max=0.05 * 2 * np.pi * n_bg / float(wl.max()),
                  eps_ref=media[0].eps_inf)
    if n_steps is None and opts.run_time_fs:
        n_steps = p["max_steps"]
    labels = [lab for f in frames for lab in f.labels()]
    plans, decided = [], None
    for f, tab in zip(frames, tables):
        for m in range(f.num_modes):
            src = ModeSource(tab, m, inv_eps=inv_eps, dt=dt, omega_c=wc, sigma=sigma,
                             n_steps=p["max_steps"] + 4 * stride)
            mons = [DFTMonitor(omega, g.e_nodes(g.k_m), g.h_nodes(g.k_m), g.h_nodes(g.k_m), energy=True)
                    for g in frames]
            kw = dict(shape=grid.shape, dx=dx, dt=dt, single=single, inv_eps=inv_eps, groups=groups, pml=pml,
                      sources=[src], monitors=mons, dft_stride=stride, periodic=grid.periodic,
                      widths=grid.engine_widths())
            if n_steps is None and decided is None:
                decided = _decay_steps(problem, opts, p, src, kw, device, engine)
            pl = P.make_plan(**kw)
            pl.pop("inv_eps")
            plans.append(pl)
    n_steps = int(n_steps if n_steps is not None else decided) // stride * stride
    e_counts = [len(m["e_idx"]) for m in plans[0]["monitors"]]
    h_counts = [len(m["h_idx1"]) for m in plans[0]["monitors"]]
    coords = [np.array([grid.coord(a, i) for i in range(grid.shape[a])], float) for a in range(3)]
    out = {"shape": tuple(int(v) for v in grid.shape), "inv_eps": np.asarray(inv_eps, float), "plans": plans,
           "labels": labels, "rows": _port_rows(tables, omega, e_counts, h_counts), "omega": omega,
           "wavelengths_nm": wl, "n_steps": n_steps, "pml_cells": cells, "coords": coords, "dl": float(grid.dx),
           "mesh": mode, "two_d": two_d, "polarization": (opts.polarization or "te") if two_d else None}
    if keep_tables:
        out["tables"] = tables
    return out


_GRID_DESCS: dict[str, dict] = {}  # the last few problems' run descriptions, for design_grid/base_permittivity


def _grid_desc(problem, desc=None) -> dict:
    """A run description of ``problem`` for its grid and base permittivity (the step count does not matter
    there): ``desc`` when given (and kept), else one made earlier for the same problem, else a new one.
    lightsmith's optimiser asks for the grid and the base permittivity without the prepared context
    (inverse/topopt.py:113-116), so this saves it the driver's set-up twice over."""
    key = problem.model_dump_json()
    if desc is None:
        desc = _GRID_DESCS.get(key)
        if desc is None:
            desc = device_runs(problem, n_steps=0)
    _GRID_DESCS.pop(key, None)
    _GRID_DESCS[key] = desc
    while len(_GRID_DESCS) > 4:
        _GRID_DESCS.pop(next(iter(_GRID_DESCS)))
    return desc


class _Deferred(Exception):
    """Raised in place of lightsmith's run loop while the runs of a batch are collected."""


class _BatchedRun:
    """One oblique run of a periodic solve: lightsmith's own set-up of it (``_run_oblique``, periodic.py:426-459)
    built its CUDA engine; the batch advances it; the driver's post-processing then reads it."""

    def __init__(self, key, eng, max_steps):
        self.key, self.eng, self.max_steps = key, eng, int(max_steps)


def _oblique_key(pol, kpar, wavelength):
    return (str(pol), round(float(kpar[0]), 15), round(float(kpar[1]), 15), round(float(wavelength), 12))


@contextmanager
def _patched(module, **attrs):
    saved = {k: getattr(module, k) for k in attrs}
    try:
        for k, v in attrs.items():
            setattr(module, k, v)
        yield
    finally:
        for k, v in saved.items():
            setattr(module, k, v)


def _solve_periodic_batched(cls, sim, device, steps_per_launch: int = 512):
    """A periodic solve whose oblique runs (one per angle, wavelength and polarisation; lightsmith runs them one
    after another, periodic.py:503-518) advance together in one persistent kernel (``BlochBatch``).

    Pass 1 runs lightsmith's driver with each oblique run recorded instead of made (and the normal-incidence
    runs skipped); each recorded run is then set up by lightsmith's own ``_run_oblique`` up to its run loop,
    which is where its CUDA engine is taken; the batch advances every engine to the run's fixed step count
    (``run_time_fs``); pass 2 runs the driver again, and each oblique run's set-up gets its advanced engine back
    (its new monitors bound to that engine's accumulators) and a run loop that only reports the steps, so the
    driver's own post-processing (orders, R and T) reads the batched results. Returns None where the runs cannot
    be batched (no fixed step count, fewer than two oblique runs, or a feature the batch does not serve: then
    the caller solves as usual)."""
    import math

    import torch

    from .batch import BlochBatch

    P = _periodic_driver
    opts = cls._options(sim)
    if not opts.run_time_fs or not isinstance(sim, PeriodicProblem):
        return None, "no fixed run time (run_time_fs): each run stops when its own fields have decayed"
    from lightsmith.problems import wavelength_array

    if sum(abs(a) > 1e-12 for a in P._angles(sim)) * len(wavelength_array(sim.wavelengths)) < 2:
        return None, "fewer than two oblique runs"  # a normal-incidence run is one broadband run
    calls = []
    placeholder = {"steps": 0, "decay_level": 0.0}  # what the driver's provenance reads of each run

    def record(c, pol, kpar, wavelength):
        calls.append((c, pol, kpar, wavelength))
        nx, ny = c.cell.n_cells
        return np.zeros((1, nx, ny)), np.zeros((1, nx, ny)), dict(placeholder)

    def skip_normal(c, pol, p, omega):
        nx, ny = c.cell.n_cells
        z = np.zeros((len(omega), nx, ny))
        return z, z.copy(), (None, None), dict(placeholder)

    with _patched(P, _run_oblique=record, _run_normal=skip_normal):
        NativeFDTD.solve.__func__(cls, sim, device)
    if len(calls) < 2:
        return None, "fewer than two oblique runs"

    runs, taken = [], {}

    def take(eng, opts_, *, max_steps, **_):
        taken["eng"], taken["max_steps"] = eng, max_steps
        raise _Deferred

    original = P._run_oblique
    with _patched(P, run_until_decayed=take):
        for c, pol, kpar, wavelength in calls:
            try:
                original(c, pol, kpar, wavelength)
            except _Deferred:
                pass
            runs.append(_BatchedRun(_oblique_key(pol, kpar, wavelength), taken.pop("eng"), taken.pop("max_steps")))
    try:
        batch = BlochBatch([r.eng for r in runs], [r.max_steps for r in runs])
    except Exception as e:  # noqa: BLE001 (a run the batch does not serve: the caller solves run by run)
        return None, str(e)
    try:
        batch.run_to_end(steps_per_launch)
        bad = batch.diverged()
    finally:
        batch.close()
    if bad:  # lightsmith's run loop raises the same error for a run it steps itself (setup.py:749-756)
        r = runs[bad[0]]
        raise FloatingPointError(
            f"FDTD diverged after {int(r.eng.n.item())} steps (non-finite fields in the batched oblique run "
            f"{r.key}); the results would be meaningless. Use a finer mesh (smaller spacing_nm or larger "
            "cells_per_wavelength), lower courant, or give lossy/dispersive materials as Drude/DrudeLorentz")
    by_key = {r.key: r for r in runs}
    current = {}

    def engine_back(device_, **kw):
        r = current["run"]
        for obj, m in zip(kw["monitors"], r.eng.monitors):
            obj.acc_e, obj.acc_h = m["acc_e"], m["acc_h"]
        return r.eng

    def loop_done(eng, opts_, *, max_steps, **_):
        return int(eng.n_host), float("nan"), True

    def replay(c, pol, kpar, wavelength):
        current["run"] = by_key[_oblique_key(pol, kpar, wavelength)]
        with _patched(P, Engine=engine_back, run_until_decayed=loop_done):
            r, t, prov = original(c, pol, kpar, wavelength)
        return r, t, {**prov, "batched": True}

    with _engine_swapped(), _patched(P, _run_oblique=replay):
        res = NativeFDTD.solve.__func__(cls, sim, device)
    for r in runs:
        r.eng.close()
    res.provenance["batched_oblique_runs"] = len(runs)
    res.provenance["batch_steps_per_launch"] = int(steps_per_launch)
    return res, ""


class B200FDTD(NativeFDTD):
    """``NativeFDTD`` (backends/fdtd.py:47) whose engine is the B200 one on CUDA devices, and which serves
    lightsmith's differentiable-backend protocol (inverse/__init__.py:14-43) for device problems on CUDA
    devices (``lightsmith_b200.differentiable``)."""

    name = "lightsmith-fdtd"
    method = "fdtd"
    gpu = True
    differentiable = True
    citation = NativeFDTD.citation + "; time loop: lightsmith-b200 (sm_100a CUDA kernels)"
    # a periodic solve with a fixed run time advances its oblique runs together in one persistent kernel
    batch_oblique = True
    # the scattering and emission drivers' particle meshing runs on the GPU where the scene allows it
    gpu_voxelise = True

    # --- the differentiable-backend protocol -----------------------------------------------------------------
    @classmethod
    def prepare(cls, problem) -> dict:
        """The runs' description and their solver, reused across optimisation iterations."""
        import torch
        from lightsmith.device import resolve_device

        from .differentiable import DeviceSolver

        dev = resolve_device("gpu") if torch.cuda.is_available() else None
        desc = device_runs(problem, dev)
        _grid_desc(problem, desc)
        return {"solver": DeviceSolver(desc)}

    @classmethod
    def design_grid(cls, problem, solver=None):
        """The FDTD grid's nodes (``x``, ``y``, ``z`` in nm, ``dl``, ``shape``); node (i, j, k) carries the
        permittivity of its three E components. A 2D device's grid is (x, y): its stepped plane."""
        from .differentiable import DesignGrid, DesignGrid2D

        d = solver.desc if solver is not None else _grid_desc(problem)
        x, y, z = d["coords"]
        if d.get("two_d"):
            return DesignGrid2D(x=x, y=y, dl=d["dl"], shape=tuple(d["shape"][:2]))
        return DesignGrid(x=x, y=y, z=z, dl=d["dl"], shape=tuple(d["shape"]))

    @classmethod
    def base_permittivity(cls, problem, solver=None) -> np.ndarray:
        """(n_wl, Nx, Ny, Nz), or (n_wl, Nx, Ny) for a 2D device, complex: per node, 1 over the mean of its three
        E components' 1/eps."""
        d = solver.desc if solver is not None else _grid_desc(problem)
        nodes = 1.0 / np.asarray(d["inv_eps"], float).mean(axis=0)
        if d.get("two_d"):
            nodes = nodes[:, :, 1]
        return np.broadcast_to(nodes, (len(d["wavelengths_nm"]),) + nodes.shape).astype(complex)

    @classmethod
    def differentiable_solve(cls, problem, eps_grid_override=None, device="gpu", sources=None,
                             with_fields: bool = True, solver=None):
        """S-parameters as torch tensors connected to ``eps_grid_override`` ((n_wl, Nx, Ny[, Nz]) or (Nx, Ny[, Nz]),
        real and equal across wavelengths), by the CUDA engine and the discrete adjoint. ``with_fields``: the
        DFT field per unit incident mode amplitude, (n_wl, n_src, 3, Nx, Ny, Nz) of E, or (n_wl, n_src, Nx, Ny)
        of H_z (TE) or E_z (TM) for a 2D device, as lightsmith's field objectives read it."""
        import torch
        from lightsmith.backends.fdfd import DifferentiableSolution
        from lightsmith.device import resolve_device

        from .differentiable import DeviceSolver, s_parameters

        dev = resolve_device(device) if isinstance(device, str) else device
        if not dev.is_gpu or dev.framework != "torch":
            raise ValueError(f"{cls.name} (B200): the differentiable solve runs on PyTorch CUDA devices")
        if solver is None:
            solver = DeviceSolver(device_runs(problem, dev))
        if eps_grid_override is None:
            eps = torch.as_tensor(solver.base_design, dtype=torch.float64)
        else:
            e = torch.as_tensor(eps_grid_override)
            if e.dim() == len(solver.design_shape):
                e = e[None]
            if torch.is_complex(e):
                if torch.any(e.imag.detach() != 0):
                    raise ValueError("FDTD steps a real permittivity: the override must have no imaginary part")
                e = e.real
            e = e.to(torch.float64)
            ref = e[0].detach()
            if torch.any((e.detach() - ref).abs() > 1e-12 * ref.abs()):
                raise ValueError("FDTD steps a frequency-independent permittivity: the override must be equal "
                                 "across wavelengths")
            eps = e.mean(0)
        labels = solver.labels if sources is None else list(sources)
        S, F = s_parameters(eps, solver, labels, fields=True) if with_fields else (s_parameters(eps, solver, labels),
                                                                                  None)
        return DifferentiableSolution(s=S, fields=F, outputs=list(solver.labels), inputs=labels,
                                      wavelengths_nm=np.asarray(solver.desc["wavelengths_nm"]),
                                      grid=cls.design_grid(problem, solver))

    @classmethod
    def supports(cls, sim):
        ok, why = NativeFDTD.supports(sim)
        if not ok:
            return ok, why
        if isinstance(sim, (Simulation, DeviceProblem, EmissionProblem, PeriodicProblem, LayerStackProblem)):
            try:
                opts = cls._options(sim)
            except ValueError as e:
                return False, str(e)
            why = _static_rejection(sim, opts)
            if why:
                return False, why
        return True, ""

    @classmethod
    def solve(cls, sim, device):
        if not device.is_gpu:
            return NativeFDTD.solve.__func__(cls, sim, device)
        if device.framework != "torch":
            raise ValueError(f"{cls.name} (B200) runs on PyTorch CUDA devices, not {device.framework!r}")
        used: list = []
        with _engine_swapped(), (_voxeliser_swapped(device, used) if cls.gpu_voxelise else _nothing()):
            why = ""
            if isinstance(sim, PeriodicProblem) and cls.batch_oblique:
                res, why = _solve_periodic_batched(cls, sim, device)
                if res is not None:
                    return res
            res = NativeFDTD.solve.__func__(cls, sim, device)
            if why:
                res.provenance["oblique_runs_one_by_one"] = why
            if used:
                res.provenance["voxelise_on_gpu"] = used[-1]
            return res
