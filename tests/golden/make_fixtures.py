"""Generate the golden fixtures in this directory by running lightsmith's own FDTD (v0.3.0, CPU, float64).

Run here (where the lightsmith sources are available), not on the GPU host:

    python tests/golden/make_fixtures.py [/path/to/lightsmith/src]

Each ``engine_*.npz`` holds the plan of one small seeded ``Engine`` run (built from the same objects the
reference engine was given, before it bound them) and the reference's fields, DFT accumulators and monitor
energy after a number of chunks. ``solve_*.npz`` holds one ``ls.solve(sim, "fdtd", "cpu")`` run: the plan
the reference's scattering driver built, its post-processing inputs and its cross sections.

``array_api_compat`` is not installed here; ``shim/`` supplies the few names the reference uses.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [HERE, REPO]
from refsrc import REF_SRC, add_to_path  # noqa: E402

if not add_to_path(sys.argv[1] if len(sys.argv) > 1 else REF_SRC):
    sys.exit("lightsmith sources not found (pass their src/ directory or set LIGHTSMITH_SRC)")

import lightsmith as ls  # noqa: E402
from lightsmith.backends._fdtd import engine as ref_engine  # noqa: E402
from lightsmith.backends._fdtd import scattering as ref_scattering  # noqa: E402
from lightsmith.backends._fdtd import device as ref_device  # noqa: E402
from lightsmith.backends._fdtd import emission as ref_emission  # noqa: E402
from lightsmith.backends._fdtd import periodic as ref_periodic  # noqa: E402
from lightsmith.backends._fdtd import symmetry as ref_symmetry  # noqa: E402
from lightsmith.backends._fdtd.emission import PointDipole  # noqa: E402
from lightsmith.backends._fdtd.layered import ObliqueLayeredPlaneWave  # noqa: E402
from lightsmith.backends._fdtd.media import Medium, Pole  # noqa: E402
from lightsmith.backends._fdtd.ports import ModeSource  # noqa: E402
from device_problems import device_problem, diff_device_problem  # noqa: E402
from problems import (SOLVE_PROBLEMS, c0_problem, dielectric_sphere_problem, emission_problem,  # noqa: E402
                      flatten_result, periodic_problem, sphere_problem)
from lightsmith.backends._fdtd.setup import flux_points, voxelise  # noqa: E402
from lightsmith.backends._fdtd.tfsf import BlochPlaneSource, TFSFPlaneWave  # noqa: E402
from lightsmith.device import Device  # noqa: E402

from lightsmith_b200 import plan as P  # noqa: E402

CPU = Device("numpy", "cpu")
HBARC = 197.3269804
# the dispersive metal of the 128^3 sphere workload: eps_inf 5.9, Drude 9.0 eV / 0.07 eV, Lorentz poles
# (1.3 @ 2.6 eV, 0.6 eV) and (1.5 @ 3.7 eV, 1.0 eV)
METAL = Medium(5.9, (Pole((9.0 / HBARC) ** 2, 0.0, 0.07 / HBARC),
                     Pole(1.3 * (2.6 / HBARC) ** 2, 2.6 / HBARC, 0.6 / HBARC),
                     Pole(1.5 * (3.7 / HBARC) ** 2, 3.7 / HBARC, 1.0 / HBARC)), "metal")


def advance_pulse(src, n_steps: int, lead: int = 12):
    """Start a source's pulse `lead` steps before its waveform first reaches 1e-3 of its peak, so that a short
    fixture run sees the whole pulse: the same waveform, advanced in time (tables: all start times moved
    together, which keeps the incident field consistent)."""
    if hasattr(src, "tables"):
        env = np.abs(src.tables).reshape(-1, src.tables.shape[-1]).max(axis=0)
        first = int(np.nonzero(env > 1e-3 * env.max())[0][0]) * src.m
        i0_min = min(int(np.min(s[4])) for s in src.slabs)
        shift = max(0, first - i0_min - lead)
        src.slabs = [(k, c, r, b, i0 + shift, u0, a, sh) for k, c, r, b, i0, u0, a, sh in src.slabs]
        src.inc = (src.inc[0], src.inc[1] + shift, src.inc[2])
        return
    w = np.asarray(src.wave)
    first = int(np.nonzero(np.abs(w) > 1e-3 * np.abs(w).max())[0][0])
    shift = max(0, first - lead)
    src.wave = np.concatenate([w[shift:], np.zeros(shift)])[:n_steps + 8]


def run_engine_case(name: str, kw: dict, n_chunks: int, snap: int = 1):
    for src in kw["sources"]:
        if not isinstance(src, ModeSource):
            advance_pulse(src, n_chunks * kw["dft_stride"])
    plan = P.make_plan(**kw)  # before Engine() binds the sources (the table source drops its tables then)
    eng = ref_engine.Engine(CPU, **kw)
    snaps = {}
    for i in range(n_chunks):
        eng.chunk()
        if i + 1 == snap:
            snaps["E_snap"], snaps["H_snap"] = eng.E.copy(), eng.H.copy()
    out = {"E": np.asarray(eng.E), "H": np.asarray(eng.H), "n": int(eng.n[0]), "energy": np.asarray(eng.energy),
           "n_chunks": n_chunks, "snap": snap, **snaps,
           "acc_e": [np.asarray(m.acc_e) for m in kw["monitors"]],
           "acc_h": [np.zeros(0) if m.acc_h is None else np.asarray(m.acc_h) for m in kw["monitors"]]}
    if getattr(eng, "od", None) is not None:  # the reference's off-diagonal gather tables, and the rows
        out["od_e"], out["od_h"], out["od_w"] = (np.asarray(x) for x in eng.od)
        od = kw["offdiag"]
        out["od_rows"] = {"idx3": np.asarray(od.idx3), "comp": np.asarray(od.comp), "coef": np.asarray(od.coef)}
    for src in kw["sources"]:
        if hasattr(src, "col"):
            out["col_E"], out["col_H"] = np.asarray(src.col.E), np.asarray(src.col.H)
        if isinstance(src, TFSFPlaneWave):
            out["line_E"], out["line_H"] = np.asarray(src.E_flat), np.asarray(src.H_flat)
    P.save(os.path.join(HERE, f"engine_{name}.npz"), {"plan": plan, "out": out})
    print(name, plan["shape"], "steps", out["n"], "max|E|", float(np.abs(out["E"]).max()))


def plane_monitor(shape, k, omega, energy):
    """E_x, E_y on node plane k with the H pair straddling it (the periodic driver's plane layout)."""
    i, j = np.meshgrid(np.arange(1, shape[0] - 1), np.arange(1, shape[1] - 1), indexing="ij")
    i, j = i.ravel(), j.ravel()
    e = np.concatenate([P.flat_index(0, i, j, k, shape), P.flat_index(1, i, j, k, shape)])
    h1 = np.concatenate([P.flat_index(1, i, j, k - 1, shape), P.flat_index(0, i, j, k - 1, shape)])
    h2 = np.concatenate([P.flat_index(1, i, j, k, shape), P.flat_index(0, i, j, k, shape)])
    return ref_engine.DFTMonitor(omega, e, h1, h2, energy=energy)


def case_yee_cpml_dipole():
    rng = np.random.default_rng(1)
    shape, dx = (18, 16, 20), 5.0
    dt = 0.99 * dx / np.sqrt(3)
    ie = 1.0 / rng.uniform(1.0, 12.25, size=(3,) + shape)
    pml = ref_engine.PMLSpec(cells=((4, 3), (3, 4), (4, 4)), alpha_max=0.02, eps_ref=1.7)
    om = 2 * np.pi / np.array([300.0, 400.0, 550.0])
    dip = PointDipole(shape=shape, origin=np.zeros(3), dx=dx, dt=dt, pos=(41.3, 38.2, 52.7), pdir=(0.3, 0.5, 0.8),
                      inv_eps=ie, omega_c=om.mean(), omega_half=0.5 * np.ptp(om), max_steps=20000)
    mons = [plane_monitor(shape, 10, om, 1), plane_monitor(shape, 6, om, 2)]
    kw = dict(shape=shape, dx=dx, dt=dt, single=False, inv_eps=ie, groups=[], pml=pml, sources=[dip],
              monitors=mons, dft_stride=3)
    run_engine_case("yee_cpml_dipole", kw, 12, snap=1)


def case_kappa_noncubic():
    rng = np.random.default_rng(2)
    shape, sp = (14, 17, 15), (4.0, 5.0, 6.0)
    dt = 0.95 / np.sqrt(sum(1 / d ** 2 for d in sp))
    ie = np.broadcast_to(1.0 / rng.uniform(1.0, 6.0, size=shape), (3,) + shape).copy()
    pml = ref_engine.PMLSpec(cells=((3, 4), (4, 3), (3, 3)), kappa_max=3.0, alpha_max=0.03, eps_ref=1.2,
                             eps_ref_high=2.25)
    om = 2 * np.pi / np.array([350.0, 500.0])
    dip = PointDipole(shape=shape, origin=np.zeros(3), dx=4.0, dt=dt, pos=(28.0, 30.0, 31.0), pdir=(0.0, 0.0, 1.0),
                      inv_eps=ie, omega_c=om.mean(), omega_half=0.5 * np.ptp(om), max_steps=20000)
    dip_idx = dip.idx  # the dipole is spread on a 4 nm lattice: only its node list and weights matter here
    mons = [plane_monitor(shape, 7, om, 1)]
    kw = dict(shape=shape, dx=sp, dt=dt, single=False, inv_eps=ie, groups=[], pml=pml, sources=[dip],
              monitors=mons, dft_stride=4)
    assert len(dip_idx)
    run_engine_case("kappa_noncubic", kw, 8, snap=2)


def case_mirror():
    """Mirror planes at node 1 (engine.py:47-60): symmetric (PMC) along x and z, antisymmetric (PEC) along y;
    CPML on the high sides only."""
    rng = np.random.default_rng(8)
    shape, dx = (14, 15, 16), 5.0
    dt = 0.99 * dx / np.sqrt(3)
    ie = 1.0 / rng.uniform(1.0, 6.0, size=(3,) + shape)
    pml = ref_engine.PMLSpec(cells=((0, 3), (0, 3), (0, 3)), alpha_max=0.02, eps_ref=1.5)
    om = 2 * np.pi / np.array([300.0, 450.0])
    dip = PointDipole(shape=shape, origin=np.zeros(3), dx=dx, dt=dt, pos=(22.3, 31.7, 41.2), pdir=(0.6, 0.3, 0.7),
                      inv_eps=ie, omega_c=om.mean(), omega_half=0.5 * np.ptp(om), max_steps=20000)
    mons = [plane_monitor(shape, 9, om, 1)]
    kw = dict(shape=shape, dx=dx, dt=dt, single=False, inv_eps=ie, groups=[], pml=pml, sources=[dip],
              monitors=mons, dft_stride=3, mirror=(1, -1, 1))
    run_engine_case("mirror", kw, 10, snap=2)


def _offdiag_rows(rng, shape, n):
    """n random conformal rows: E_comp at interior nodes, small random (1/eps)_cd with column comp zero."""
    idx3 = np.stack([rng.integers(2, s - 3, n) for s in shape], axis=1)
    comp = rng.integers(0, 3, n)
    coef = rng.uniform(-0.06, 0.06, (n, 3))
    coef[np.arange(n), comp] = 0.0
    return ref_engine.OffDiagonal(idx3, comp, coef)


def case_offdiag():
    """Conformal off-diagonal 1/eps terms (engine.py:421-518, 653-655) on random rows, with a pure Drude-Lorentz
    group overlapping some of them (their couplings are dropped) and CPML on every face."""
    rng = np.random.default_rng(9)
    shape, dx = (16, 15, 14), 5.0
    dt = 0.99 * dx / np.sqrt(3)
    ie = 1.0 / rng.uniform(1.0, 6.0, size=(3,) + shape)
    pml = ref_engine.PMLSpec(cells=((3, 3), (3, 3), (3, 3)), alpha_max=0.02, eps_ref=1.5)
    om = 2 * np.pi / np.array([300.0, 450.0])
    dip = PointDipole(shape=shape, origin=np.zeros(3), dx=dx, dt=dt, pos=(31.3, 33.7, 26.2), pdir=(0.4, 0.8, 0.3),
                      inv_eps=ie, omega_c=om.mean(), omega_half=0.5 * np.ptp(om), max_steps=20000)
    cells = int(np.prod(shape))
    node = np.ravel_multi_index(np.meshgrid(np.arange(9, 11), np.arange(5, 7), np.arange(6, 8), indexing="ij"),
                                shape).ravel()
    idx = np.concatenate([c * cells + node for c in range(3)])
    ie.reshape(3, -1)[:, node] = 1.0
    grp = ref_engine.DispersiveGroup(idx=idx, media=[METAL], frac=np.ones((1, len(idx))), w=None)
    mons = [plane_monitor(shape, 8, om, 1)]
    kw = dict(shape=shape, dx=dx, dt=dt, single=False, inv_eps=ie, groups=[grp], pml=pml, sources=[dip],
              monitors=mons, dft_stride=3, offdiag=_offdiag_rows(rng, shape, 240))
    run_engine_case("offdiag", kw, 10, snap=2)


def case_offdiag_mirror():
    """Off-diagonal terms with mirror planes (symmetric along x, antisymmetric along y): the rows' images and
    the folded sources (engine.py:475-483, 540-553)."""
    rng = np.random.default_rng(10)
    shape, dx = (14, 15, 16), 5.0
    dt = 0.99 * dx / np.sqrt(3)
    ie = 1.0 / rng.uniform(1.0, 6.0, size=(3,) + shape)
    pml = ref_engine.PMLSpec(cells=((0, 3), (0, 3), (3, 3)), alpha_max=0.02, eps_ref=1.5)
    om = 2 * np.pi / np.array([300.0, 450.0])
    dip = PointDipole(shape=shape, origin=np.zeros(3), dx=dx, dt=dt, pos=(22.3, 31.7, 41.2), pdir=(0.6, 0.3, 0.7),
                      inv_eps=ie, omega_c=om.mean(), omega_half=0.5 * np.ptp(om), max_steps=20000)
    od = _offdiag_rows(rng, shape, 200)
    od.idx3[:40, 0] = 1  # rows on the symmetric plane
    od.idx3[40:70, 1] = 1  # and on the antisymmetric one
    mons = [plane_monitor(shape, 9, om, 1)]
    kw = dict(shape=shape, dx=dx, dt=dt, single=False, inv_eps=ie, groups=[], pml=pml, sources=[dip],
              monitors=mons, dft_stride=3, mirror=(1, -1, 0), offdiag=od)
    run_engine_case("offdiag_mirror", kw, 10, snap=2)


def sphere_slot_fn(center, radius, slot=1):
    c = np.asarray(center, float)

    def fn(pts):
        return np.where(np.sum((pts - c) ** 2, axis=-1) <= radius ** 2, slot, 0).astype(int)
    return fn


def case_ade_groups():
    shape, dx = (22, 22, 22), 2.0
    host = Medium(1.33 ** 2, (), "medium")
    media = [host, METAL]
    ctr = np.array([21.0, 21.3, 20.7])
    inv_eps, groups, stats, od = voxelise(sphere_slot_fn(ctr, 9.0), media, shape, np.zeros(3), dx,
                                          np.array([2, 2, 2]), np.array([20, 20, 20]), mode="subpixel")
    assert od is None and any(g.w is not None for g in groups) and any(g.w is None for g in groups)
    dt = 0.99 * dx / np.sqrt(3)
    pml = ref_engine.PMLSpec(cells=((4, 4),) * 3, alpha_max=0.01, eps_ref=host.eps_inf)
    om = 2 * np.pi / np.array([450.0, 550.0, 700.0])
    dip = PointDipole(shape=shape, origin=np.zeros(3), dx=dx, dt=dt, pos=(21.0, 30.5, 22.0), pdir=(1.0, 0.0, 0.0),
                      inv_eps=inv_eps, omega_c=om.mean(), omega_half=0.5 * np.ptp(om), max_steps=20000)
    lo, hi = np.array([5, 5, 5]), np.array([16, 16, 16])
    sca = flux_points(lo, hi, shape, dx)
    mons = [ref_engine.DFTMonitor(om, sca[0], sca[1], sca[2], energy=1), plane_monitor(shape, 11, om, 2)]
    kw = dict(shape=shape, dx=dx, dt=dt, single=False, inv_eps=inv_eps, groups=groups, pml=pml, sources=[dip],
              monitors=mons, dft_stride=5)
    run_engine_case("ade_groups", kw, 16, snap=2)


def case_tfsf_table():
    shape, dx = (27, 25, 29), 3.0
    host = Medium(1.33 ** 2, (), "medium")
    glass = Medium(2.25, (), "glass")
    media = [host, METAL, glass]
    ctr = np.array([13, 12, 14]) * dx

    def slot(pts):
        r1 = np.sum((pts - ctr - np.array([-4.0, 0.0, 0.0])) ** 2, axis=-1) <= 7.0 ** 2
        r2 = np.sum((pts - ctr - np.array([6.0, 1.0, 2.0])) ** 2, axis=-1) <= 5.0 ** 2
        return np.where(r1, 1, np.where(r2, 2, 0)).astype(int)
    inv_eps, groups, stats, od = voxelise(slot, media, shape, np.zeros(3), dx, np.array([5, 5, 5]),
                                          np.array([22, 20, 24]), mode="staircase")
    dt = 0.99 * dx / np.sqrt(3)
    wl = np.linspace(420.0, 780.0, 5)
    om = 2 * np.pi / wl
    omega_c, omega_half = 0.5 * (om.min() + om.max()), max(0.5 * np.ptp(om), 0.15 * om.mean())
    lo, hi = np.array([6, 6, 6]), np.array([20, 18, 22])
    khat = np.array([0.3, -0.4, 1.0])
    khat /= np.linalg.norm(khat)
    ehat = np.cross(khat, [0.0, 1.0, 0.0])
    ehat /= np.linalg.norm(ehat)
    src = ObliqueLayeredPlaneWave(shape=shape, origin=np.zeros(3), spacing=dx, dt=dt, lo=lo, hi=hi, khat=khat,
                                  ehat=ehat, inv_eps=inv_eps, host=host, omega_c=omega_c, omega_half=omega_half,
                                  max_steps=400, omega_min=om.min())
    pml = ref_engine.PMLSpec(cells=((4, 4),) * 3, alpha_max=0.02, eps_ref=host.eps_inf)
    sca = flux_points(lo - 2, hi + 2, shape, dx)
    tot = flux_points(lo + 2, hi - 2, shape, dx)
    mons = [ref_engine.DFTMonitor(om, sca[0], sca[1], sca[2], energy=True),
            ref_engine.DFTMonitor(om, tot[0], tot[1], tot[2], energy=2),
            ref_engine.DFTMonitor(om, np.arange(3), source=src.view)]
    kw = dict(shape=shape, dx=dx, dt=dt, single=False, inv_eps=inv_eps, groups=groups, pml=pml, sources=[src],
              monitors=mons, dft_stride=7)
    run_engine_case("tfsf_table", kw, 20, snap=3)


def case_line_periodic():
    shape, dx = (8, 7, 40), 10.0
    sp = (12.0, 11.0, 10.0)
    rng = np.random.default_rng(4)
    ie = np.full((3,) + shape, 1.0)
    ie[:, :, :, 20:26] = 1.0 / rng.uniform(2.0, 6.0, size=(3, shape[0], shape[1], 6))
    dt = 0.95 / np.sqrt(sum(1 / d ** 2 for d in sp))
    om = 2 * np.pi / np.array([500.0, 650.0, 800.0])
    big = 10 ** 9
    src = TFSFPlaneWave(shape=shape, origin=np.array([-12.0, -11.0, -100.0]), dx=sp, dt=dt,
                        r0=np.array([0.0, 0.0, 50.0]), lo=np.array([-big, -big, 14]), hi=np.array([big, big, big]),
                        khat=np.array([0.0, 0.0, 1.0]), ehat=np.array([0.6, 0.8, 0.0]), eps_b=1.0,
                        omega_c=om.mean(), omega_half=0.5 * np.ptp(om), max_steps=20000, periodic=(True, True, False))
    pml = ref_engine.PMLSpec(cells=((0, 0), (0, 0), (8, 8)), alpha_max=0.01, eps_ref=1.0, eps_ref_high=2.0)
    e, h1, h2 = src.probe()
    mons = [plane_monitor(shape, 12, om, 1), plane_monitor(shape, 29, om, 1),
            ref_engine.DFTMonitor(om, e, h1, h2, source=src)]
    kw = dict(shape=shape, dx=sp, dt=dt, single=False, inv_eps=ie, groups=[], pml=pml, sources=[src],
              monitors=mons, dft_stride=4, periodic=(True, True, False))
    run_engine_case("line_periodic", kw, 20, snap=2)


def case_bloch_column():
    shape = (9, 8, 44)
    sp = (30.0, 32.0, 10.0)
    rng = np.random.default_rng(5)
    ie = np.full((3,) + shape, 1.0)
    xx = np.arange(shape[0])[:, None]
    yy = np.arange(shape[1])[None, :]
    pillar = ((xx - 4) ** 2 + (yy - 4) ** 2 <= 4)
    for z in range(22, 30):
        ie[:, :, :, z] = np.where(pillar, 1 / 5.76, 1.0)
    ie[:, :, :, 30:] = 1 / 2.1025
    ie *= rng.uniform(0.98, 1.0, size=ie.shape)
    dt = 0.95 / np.sqrt(sum(1 / d ** 2 for d in sp))
    lam = 600.0
    omega = 2 * np.pi / lam
    kpar = (omega * np.sin(0.5) * np.cos(0.3), omega * np.sin(0.5) * np.sin(0.3))
    pml = ref_engine.PMLSpec(cells=((0, 0), (0, 0), (8, 8)), alpha_max=0.01, eps_ref=1.0, eps_ref_high=2.1)
    from dataclasses import replace
    src = BlochPlaneSource(shape=shape, spacing=sp, dt=dt, k_src=14, k_launch=13, kpar=kpar, pol="p", eps_b=1.0,
                           pml=replace(pml, eps_ref_high=None), omega_c=omega, omega_half=0.1 * omega, max_steps=20000)
    om = np.array([omega])
    e, h1, h2 = src.probe(16)
    mons = [plane_monitor(shape, 11, om, 1), plane_monitor(shape, 34, om, 1),
            ref_engine.DFTMonitor(om, e, h1, h2, source=src)]
    kw = dict(shape=shape, dx=sp, dt=dt, single=False, inv_eps=ie, groups=[], pml=pml, sources=[src],
              monitors=mons, dft_stride=3, periodic=(True, True, False), bloch=(kpar[0], kpar[1], 0.0))
    run_engine_case("bloch_column", kw, 25, snap=2)


def case_mode_source():
    rng = np.random.default_rng(6)
    shape, dx = (16, 14, 18), 20.0
    ie = 1.0 / rng.uniform(2.0, 12.0, size=(3,) + shape)
    dt = 0.95 * dx / np.sqrt(3)
    pml = ref_engine.PMLSpec(cells=((3, 3),) * 3, alpha_max=0.01, eps_ref=2.07)
    # a port plane at x = 5: H targets on the half plane outside it, E targets on the plane (ports.py:346-360)
    jj, kk = np.meshgrid(np.arange(3, 11), np.arange(4, 14), indexing="ij")
    jj, kk = jj.ravel(), kk.ravel()
    nw = jj.size
    src = ModeSource.__new__(ModeSource)
    src.h_idx = np.concatenate([P.flat_index(2, 4, jj, kk, shape), P.flat_index(1, 4, jj, kk, shape)])
    src.e_idx = np.concatenate([P.flat_index(1, 5, jj, kk, shape), P.flat_index(2, 5, jj, kk, shape)])
    r_e, r_h, L = 3, 2, 200
    src.mH = rng.normal(size=(2 * nw, r_e)) * 0.05
    src.mE = rng.normal(size=(2 * nw, r_h)) * 0.05
    t = np.arange(L) * dt
    env = np.exp(-((t - 60 * dt) / (18 * dt)) ** 2)
    src.tab_E = env[:, None] * np.sin(0.2 * np.arange(L)[:, None] + rng.uniform(0, 3, r_e)[None, :])
    src.tab_H = env[:, None] * np.cos(0.2 * np.arange(L)[:, None] + rng.uniform(0, 3, r_h)[None, :])
    om = np.array([2 * np.pi / 1550.0, 2 * np.pi / 1300.0])
    i, k = np.meshgrid(np.arange(1, 15), np.arange(1, 17), indexing="ij")
    e = P.flat_index(1, i.ravel(), 11, k.ravel(), shape)
    h1 = P.flat_index(2, i.ravel(), 10, k.ravel(), shape)
    h2 = P.flat_index(2, i.ravel(), 11, k.ravel(), shape)
    mons = [ref_engine.DFTMonitor(om, e, h1, h2, energy=1)]
    kw = dict(shape=shape, dx=dx, dt=dt, single=False, inv_eps=ie, groups=[], pml=pml, sources=[src],
              monitors=mons, dft_stride=2)
    run_engine_case("mode_source", kw, 30, snap=5)


# --- a whole ls.solve of the dispersive-sphere scattering problem ---------------------------------------


def solve_case(name: str, sim):
    rec = {}
    Base = ref_scattering.Engine
    fp_orig = ref_scattering.flux_points

    class Recording(Base):
        def __init__(self, device, **kw):
            rec["plan"] = P.make_plan(**kw)
            rec["kw"] = kw
            super().__init__(device, **kw)
            rec["eng"] = self

    boxes = []

    def flux_points_rec(*a, **k):
        out = fp_orig(*a, **k)
        boxes.append(out)
        return out
    ref_scattering.Engine = Recording
    ref_scattering.flux_points = flux_points_rec
    try:
        res = ls.solve(sim, "fdtd", "cpu")
    finally:
        ref_scattering.Engine = Base
        ref_scattering.flux_points = fp_orig
    kw, eng = rec["kw"], rec["eng"]
    src = kw["sources"][0]
    omega = 2 * np.pi / sim.wavelength_array()
    sca, tot = boxes
    n_sym = float(ref_symmetry.factor(kw.get("mirror", (0, 0, 0))))
    post = {"omega": omega, "n_sym": n_sym, "n_inc": float(src.n_inc), "sca_coeff": sca[3], "tot_coeff": tot[3],
            "unit": src.incident_reference(omega), "bg_e": src.background(omega, tot[0], "E"),
            "bg_h": 0.5 * (src.background(omega, tot[1], "H") + src.background(omega, tot[2], "H")),
            "steps": int(res.provenance["steps"])}
    out = {"c_ext": np.asarray(res.c_ext_nm2), "c_sca": np.asarray(res.c_sca_nm2), "c_abs": np.asarray(res.c_abs_nm2),
           "acc_e": [np.asarray(m.acc_e) for m in kw["monitors"]],
           "acc_h": [np.zeros(0) if m.acc_h is None else np.asarray(m.acc_h) for m in kw["monitors"]],
           "energy": np.asarray(eng.energy), "n": int(eng.n[0])}
    P.save(os.path.join(HERE, f"solve_{name}.npz"), {"plan": rec["plan"], "post": post, "out": out})
    print(name, rec["plan"]["shape"], "steps", post["steps"], "C_ext", out["c_ext"])


def c0_case():
    """The full-size sphere: the plan and post-processing inputs lightsmith's scattering driver builds, then
    lightsmith's own engine run on the host for exactly 4000 steps twice, in float64 and in float32 (its GPU
    precision; here through PyTorch on the CPU), and the cross sections at all 81 wavelengths from each run's
    accumulators by oracle/post.py (which reproduces lightsmith's post-processing to 1e-13 on the other solve
    fixtures). The background's flux through the total-field box is kept per wavelength (``bg_flux``, the
    unit-amplitude flux; the post-processing scales it by the measured incident amplitude), which keeps the
    fixture small. ``ls.solve`` itself is not used for the run: its run loop stops this one at step 3100 with
    its divergence test (setup.py:749-756), whose reference is the monitor energy of the run's first half,
    before the pulse has reached the scattered-field box; the energy per chunk is kept in the fixture."""
    import torch
    from lightsmith.device import resolve_device

    from oracle.post import cross_sections, flux

    sim = c0_problem()

    class Stop(Exception):
        pass

    def setup():
        rec, boxes = {}, []

        def capture(device, **kw):
            rec["kw"] = kw
            raise Stop()

        def flux_points_rec(*a, **k):
            out = fp_orig(*a, **k)
            boxes.append(out)
            return out
        fp_orig, Base = ref_scattering.flux_points, ref_scattering.Engine
        ref_scattering.Engine, ref_scattering.flux_points = capture, flux_points_rec
        try:
            ls.solve(sim, "fdtd", "cpu")
        except Stop:
            pass
        finally:
            ref_scattering.Engine, ref_scattering.flux_points = Base, fp_orig
        return rec["kw"], boxes

    torch.set_num_threads(os.cpu_count() or 1)
    steps = 4000
    runs = {}
    for prec in ("double", "single"):
        kw, boxes = setup()
        if prec == "double":
            plan = P.make_plan(**kw)
        kw = {**kw, "single": prec == "single"}
        eng = ref_scattering.Engine(resolve_device("torch-cpu"), **kw)
        energy = []
        for _ in range(steps // plan["stride"]):
            eng.chunk()
            energy.append(Device.to_numpy(eng.energy).astype(float).copy())
        runs[prec] = (kw, eng, boxes, np.asarray(energy))
    kw, eng, boxes, energy = runs["double"]
    src = kw["sources"][0]
    omega = 2 * np.pi / sim.wavelength_array()
    sca, tot = boxes
    bg_e = src.background(omega, tot[0], "E")
    bg_h = 0.5 * (src.background(omega, tot[1], "H") + src.background(omega, tot[2], "H"))
    post = {"omega": omega, "n_sym": 1.0, "n_inc": float(src.n_inc), "sca_coeff": sca[3], "tot_coeff": tot[3],
            "unit": src.incident_reference(omega), "bg_flux": flux(bg_e, bg_h, tot[3]), "steps": steps}
    out = {"n": int(Device.to_numpy(eng.n)[0]), "energy": energy}
    for prec, tag in (("double", "fp64"), ("single", "fp32")):
        kw_p, eng_p = runs[prec][:2]
        acc_e = [Device.to_numpy(m.acc_e).astype(complex) for m in kw_p["monitors"]]
        acc_h = [None if m.acc_h is None else Device.to_numpy(m.acc_h).astype(complex) for m in kw_p["monitors"]]
        cs = cross_sections(acc_e, acc_h, post)
        if prec == "double":
            out.update({k: cs[k] for k in ("c_ext", "c_sca", "c_abs")})
        else:
            out["lightsmith_fp32"] = {k: cs[k] for k in ("c_ext", "c_sca", "c_abs")}
    P.save(os.path.join(HERE, "solve_c0.npz"), {"plan": plan, "post": post, "out": out})
    err = {k: float(np.max(np.abs(out["lightsmith_fp32"][k] - out[k]) / np.abs(out[k]))) for k in ("c_ext", "c_sca",
                                                                                                  "c_abs")}
    print("c0", plan["shape"], "steps", steps, "lightsmith fp32 vs fp64 (max rel over 81 wavelengths)", err)


def driver_case(name: str, problem, module):
    """Every Engine a lightsmith driver builds in ``ls.solve(problem, "fdtd", "cpu")`` (a periodic solve builds
    one per incidence and polarisation): its plan, step count, final DFT accumulators and energy."""
    runs = []
    Base = module.Engine

    class Recording(Base):
        def __init__(self, device, **kw):
            plan = P.make_plan(**kw)  # before the engine binds the sources
            super().__init__(device, **kw)
            runs.append((plan, kw, self))

    module.Engine = Recording
    try:
        ls.solve(problem, "fdtd", "cpu")
    finally:
        module.Engine = Base
    out = []
    for plan, kw, eng in runs:
        out.append({"plan": plan, "n": int(eng.n[0]), "energy": np.asarray(eng.energy),
                    "acc_e": [np.asarray(m.acc_e) for m in kw["monitors"]],
                    "acc_h": [np.zeros(0) if m.acc_h is None else np.asarray(m.acc_h) for m in kw["monitors"]]})
    P.save(os.path.join(HERE, f"driver_{name}.npz"), {"runs": out})
    print(name, [(r["plan"]["shape"], r["n"], r["plan"]["complex"]) for r in out])






def diff_device_case(dimension: int):
    """``backend.device_runs`` of the width step and lightsmith's own S of the same problem."""
    from lightsmith_b200.backend import device_runs
    prob = diff_device_problem(dimension)
    desc = device_runs(prob)
    res = ls.solve(prob, "fdtd", "cpu")
    assert list(res.ports) == desc["labels"]
    S = np.asarray(res.s_real) + 1j * np.asarray(res.s_imag)
    name = f"diff_device_{dimension}d"
    P.save(os.path.join(HERE, name + ".npz"), {"desc": desc, "s": S})
    print(name, desc["shape"], desc["n_steps"], desc["mesh"], np.abs(S[:, 1, 0]))





def results_case():
    """lightsmith's own ``ls.solve(problem, "fdtd", "cpu")`` (float64) result for every problem of
    ``problems.SOLVE_PROBLEMS``: the numeric content of each result (``flatten_result``), for the tests that
    pose the same problems to ``ls.solve(problem, "fdtd", "gpu")`` through the plugin."""
    out = {}
    for name, make in SOLVE_PROBLEMS.items():
        res = ls.solve(make(), "fdtd", "cpu")
        out[name] = {"result": flatten_result(res), "steps": int(res.provenance.get("steps", -1))}
        print(name, type(res).__name__, out[name]["steps"], sorted(out[name]["result"]))
    P.save(os.path.join(HERE, "solve_results.npz"), out)


CASES = {"yee_cpml_dipole": case_yee_cpml_dipole, "kappa_noncubic": case_kappa_noncubic,
         "ade_groups": case_ade_groups, "tfsf_table": case_tfsf_table, "line_periodic": case_line_periodic,
         "bloch_column": case_bloch_column, "mode_source": case_mode_source, "mirror": case_mirror,
         "offdiag": case_offdiag, "offdiag_mirror": case_offdiag_mirror,
         "solve_sphere_staircase": lambda: solve_case("sphere_staircase", sphere_problem("staircase")),
         "solve_sphere_subpixel": lambda: solve_case("sphere_subpixel", sphere_problem("subpixel")),
         "solve_sphere_symmetric": lambda: solve_case("sphere_symmetric", sphere_problem("staircase", "auto")),
         "solve_dielectric_conformal": lambda: solve_case("dielectric_conformal", dielectric_sphere_problem()),
         "solve_sphere_conformal": lambda: solve_case("sphere_conformal", sphere_problem("conformal")),
         "solve_sphere_defaults": lambda: solve_case("sphere_defaults", sphere_problem("conformal", "auto")),
         "driver_periodic_normal": lambda: driver_case("periodic_normal", periodic_problem(0.0, 0.0, "s"),
                                                       ref_periodic),
         "driver_periodic_oblique": lambda: driver_case("periodic_oblique", periodic_problem(30.0, 10.0, "p"),
                                                        ref_periodic),
         "driver_emission": lambda: driver_case("emission", emission_problem(), ref_emission),
         "driver_device_2d": lambda: driver_case("device_2d", device_problem(2), ref_device),
         "driver_device_3d": lambda: driver_case("device_3d", device_problem(3), ref_device),
         "solve_c0": c0_case,
         "diff_device_3d": lambda: diff_device_case(3),
         "diff_device_2d": lambda: diff_device_case(2),
         "solve_results": results_case}

if __name__ == "__main__":
    which = sys.argv[2:] or list(CASES)
    for c in which:
        CASES[c]()
