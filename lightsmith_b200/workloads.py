"""Synthetic workloads with the shapes of lightsmith's FDTD benchmark cases.

``throughput_plan``: the plain FDTD throughput case, a cubic grid of i.i.d. permittivity uniform in
[1, 12.25] drawn from a seed, CPML on every face, a Gaussian point-current pulse at the centre and a running
DFT at 16 frequencies on the centre z plane. lightsmith itself does not fix the cell size, band or DFT
stride of that case; they are fixed here: dx = 20 nm, dt = 0.99 dx / sqrt(3), band 1000-2000 nm, and the
stride lightsmith's drivers pick for that band (``scattering.py:257-261``: the largest step count whose
sampling does not alias the pulse onto the band).
"""

from __future__ import annotations

import math

import numpy as np

from .plan import DFTMonitor, DipoleSource, PMLSpec, flat_index, make_plan


def point_dipole(shape, origin, dx: float, dt: float, pos, pdir, inv_eps_at, omega_c: float, omega_half: float,
                 max_steps: int) -> DipoleSource:
    """A point current J = j(t) p_hat at ``pos`` spread trilinearly over the eight E_c nodes around it, with j
    the exact step difference of a Gaussian-modulated sine (``emission.py:97-128``): E_c -= dt (1/eps) w j.
    ``inv_eps_at(flat)`` gives 1/eps at flat E indices."""
    idx, w = [], []
    pos, origin = np.asarray(pos, float), np.asarray(origin, float)
    for c in range(3):
        if abs(pdir[c]) < 1e-12:
            continue
        off = np.zeros(3)
        off[c] = 0.5
        f = (pos - origin) / dx - off
        i0 = np.floor(f).astype(int)
        t = f - i0
        for corner in range(8):
            bits = np.array([(corner >> a) & 1 for a in range(3)])
            wt = float(np.prod(np.where(bits, t, 1 - t)))
            if wt > 1e-12:
                idx.append(int(flat_index(c, *(i0 + bits), shape)))
                w.append(wt * pdir[c])
    idx, w = np.asarray(idx, np.int64), np.asarray(w, float)
    coef = dt * inv_eps_at(idx) * w
    tau = 2.0 / omega_half
    t0 = 5.0 * tau
    t = np.arange(max_steps + 3) * dt
    g = np.exp(-(((t - t0) / tau) ** 2)) * np.sin(omega_c * (t - t0))
    return DipoleSource(idx=idx, coef=coef, wave=np.diff(g) / (omega_c * dt))


def plane_monitor(shape, k: int, omega, energy: int = 1) -> DFTMonitor:
    """E_x, E_y on node plane k over the interior nodes, each with the two H samples straddling the plane
    (the layout of lightsmith's periodic R/T planes, ``periodic.py:335-344``)."""
    i, j = np.meshgrid(np.arange(1, shape[0] - 1), np.arange(1, shape[1] - 1), indexing="ij")
    i, j = i.ravel(), j.ravel()
    e = np.concatenate([flat_index(0, i, j, k, shape), flat_index(1, i, j, k, shape)])
    h1 = np.concatenate([flat_index(1, i, j, k - 1, shape), flat_index(0, i, j, k - 1, shape)])
    h2 = np.concatenate([flat_index(1, i, j, k, shape), flat_index(0, i, j, k, shape)])
    return DFTMonitor(np.asarray(omega, float), e, h1, h2, energy=energy)


def throughput_band(dx: float = 20.0, lam=(1000.0, 2000.0), n_freq: int = 16):
    dt = 0.99 * dx / math.sqrt(3)
    wl = np.linspace(lam[0], lam[1], n_freq)
    om = 2 * np.pi / wl
    omega_c = 0.5 * (om.min() + om.max())
    omega_half = max(0.5 * (om.max() - om.min()), 0.15 * omega_c)
    stride = max(1, int(2 * np.pi / (omega_c + 4 * omega_half + om.max()) / dt))
    return dt, om, omega_c, omega_half, stride


def throughput_plan(n: int | tuple = 640, pml: int = 16, dx: float = 20.0, n_freq: int = 16, max_steps: int = 2000,
                    seed: int = 0, inv_eps=None, single: bool = True, stride: int | None = None) -> dict:
    """Plan of the throughput case on an n^3 grid (or shape n). ``inv_eps``: (N0, N1, N2) isotropic 1/eps as a
    NumPy array, or None to draw it here from ``seed`` (float64, ``np.random.default_rng(seed)``); the caller
    may also pass a device tensor (the CUDA engine accepts one)."""
    shape = (n, n, n) if np.isscalar(n) else tuple(int(v) for v in n)
    dt, om, omega_c, omega_half, st = throughput_band(dx, n_freq=n_freq)
    if inv_eps is None:
        inv_eps = 1.0 / np.random.default_rng(seed).uniform(1.0, 12.25, size=shape)
    ctr = (np.asarray(shape) // 2) * dx + 0.37 * dx  # off-node, so the current spreads over 8 nodes per component

    def at(flat):
        rest = np.asarray(flat) % (shape[0] * shape[1] * shape[2])
        ijk = np.unravel_index(rest, shape)
        if hasattr(inv_eps, "detach"):
            import torch

            v = inv_eps[tuple(torch.as_tensor(a, device=inv_eps.device) for a in ijk)]
            return v.detach().double().cpu().numpy()
        return np.asarray(inv_eps)[ijk]
    dip = point_dipole(shape, np.zeros(3), dx, dt, ctr, (0.0, 0.0, 1.0), at, omega_c, omega_half, max_steps)
    mon = plane_monitor(shape, shape[2] // 2, om, energy=1)
    spec = PMLSpec(cells=((pml, pml),) * 3, alpha_max=0.05 * 2 * np.pi / 2000.0 if pml else 0.0, eps_ref=1.0)
    if hasattr(inv_eps, "detach"):
        # make_plan takes host arrays: a device tensor for 1/eps is put in place afterwards
        plan = _plan_on_device(shape, dx, dt, single, spec, dip, mon, stride or st)
        plan["inv_eps"] = inv_eps
        return plan
    return make_plan(shape=shape, dx=dx, dt=dt, single=single, inv_eps=inv_eps, groups=[], pml=spec, sources=[dip],
                     monitors=[mon], dft_stride=stride or st)


def _plan_on_device(shape, dx, dt, single, spec, dip, mon, stride):
    plan = make_plan(shape=(3, 3, 3), dx=dx, dt=dt, single=single, inv_eps=np.ones((3, 3, 3)), groups=[],
                     pml=PMLSpec(cells=((0, 0),) * 3), sources=[dip], monitors=[mon], dft_stride=stride)
    plan["shape"] = tuple(shape)
    plan["pml"] = {"cells": tuple(tuple(int(v) for v in c) for c in spec.cells), "m": float(spec.m),
                   "kappa_max": float(spec.kappa_max), "alpha_max": float(spec.alpha_max),
                   "eps_ref": float(spec.eps_ref), "eps_ref_high": None}
    return plan


def cells_in_cpml(plan) -> int:
    """Per step, the number of (cell, axis) pairs inside a CPML slab (each carries 4 psi values)."""
    shape = plan["shape"]
    tot = 0
    for d, (lo, hi) in enumerate(plan["pml"]["cells"]):
        thick = (lo + 1 if lo else 0) + (hi + 1 if hi else 0)
        tot += thick * int(np.prod([shape[a] for a in range(3) if a != d]))
    return tot
