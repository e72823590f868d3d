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

from .plan import (ColumnSource, DFTMonitor, DipoleSource, DispersiveGroup, Medium, PMLSpec, Pole, flat_index,
                   make_plan)


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


# --- the batched oblique sweep of a periodic metasurface cell ---------------------------------------------


def metasurface_run(period: float, theta_deg: float, phi_deg: float, wavelength: float, pol: str, *,
                    dz: float = 10.0, nz: int = 200, pml: int = 12, single: bool = True, steps: int = 3000,
                    n_pillar: float = 2.4, n_sub: float = 1.45, height: float = 600.0) -> dict:
    """Plan of one fixed-k_par oblique run of a periodic cell (the structure of lightsmith's
    ``periodic._run_oblique``, ``periodic.py:426-459``): a cylinder of index ``n_pillar``, radius 0.3 x period
    and ``height`` on a substrate of index ``n_sub``, air above, square period ``period``.

    Cells: ceil(period / 10 nm) per period (spacing period / n, as ``periodic.py:172``), ``dz`` along z, ``nz``
    nodes (fixed here; lightsmith derives it from gaps), CPML of ``pml`` cells at both ends. Along z: the
    reflection plane, the TF/SF plane (k_src, fed by the Bloch column, ``tfsf.py:214-296``), the incident probe,
    the pillar, the substrate and the transmission plane. The permittivity is sampled at the nodes (staircase,
    isotropic). The pulse is lightsmith's oblique-run pulse: a Gaussian of half-width 0.15 omega around the
    wavelength (the upper clip of ``periodic._oblique_half_width``)."""
    n = int(math.ceil(period / 10.0))
    d = period / n
    shape = (n + 2, n + 2, nz)
    spacing = (d, d, dz)
    dt = 0.99 / math.sqrt(2 / d ** 2 + 1 / dz ** 2)
    k_r, k_src = pml + 4, pml + 10
    k_launch, k_probe = k_src - 1, k_src + 3
    z_top = k_src + 8
    z_sub = z_top + int(round(height / dz))
    k_t = nz - pml - 4
    if not (z_sub < k_t):
        raise ValueError("the cell is too short for the pillar")
    # nodes: x, y periodic over the real cells (ghosts repeat them), z as laid out above
    xi = (np.arange(shape[0]) - 1) % n
    xc = (xi + 0.5) * d - 0.5 * period
    r2 = xc[:, None] ** 2 + xc[None, :] ** 2
    pillar = r2 <= (0.3 * period) ** 2
    eps = np.ones(shape)
    eps[:, :, z_sub:] = n_sub ** 2
    eps[:, :, z_top:z_sub][pillar] = n_pillar ** 2
    omega = 2 * np.pi / wavelength
    half = 0.15 * omega
    th, ph = math.radians(theta_deg), math.radians(phi_deg)
    kx, ky = omega * math.sin(th) * math.cos(ph), omega * math.sin(th) * math.sin(ph)
    stride = max(1, int(2 * np.pi / (2 * omega + 4 * half) / dt))
    pml_main = PMLSpec(cells=((0, 0), (0, 0), (pml, pml)), alpha_max=0.01, eps_ref=1.0, eps_ref_high=n_sub ** 2)
    pml_col = PMLSpec(cells=((0, 0), (0, 0), (pml, pml)), alpha_max=0.01, eps_ref=1.0, eps_ref_high=None)
    col = make_plan(shape=(3, 3, nz), dx=spacing, dt=dt, single=single, inv_eps=np.ones((3, 3, 3, nz)), groups=[],
                    pml=pml_col, sources=[], monitors=[], dft_stride=1, periodic=(True, True, False),
                    bloch=(kx, ky, 0.0))
    # the sheet along s = (-Ky, Kx) or p = (Kx, Ky), K the grid wavenumbers (tfsf.py:229-238)
    K = np.array([2 * math.sin(kx * d / 2) / d, 2 * math.sin(ky * d / 2) / d])
    u = K / np.linalg.norm(K) if np.linalg.norm(K) > 1e-12 else np.array([math.cos(ph), math.sin(ph)])
    a = np.array([-u[1], u[0]]) if pol == "s" else u
    amp = (complex(a[0] * np.exp(0.5j * kx * d)), complex(a[1] * np.exp(0.5j * ky * d)))
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    phase = np.exp(1j * (kx * i * d + ky * j * d))
    tau = 2.0 / half
    t0 = 3.5 * tau
    t = (np.arange(steps + 2) + 1) * dt
    wave = np.exp(-(((t - t0) / tau) ** 2)) * np.sin(omega * (t - t0))
    src = ColumnSource(column=col, k_src=k_src, k_launch=k_launch, phase=phase, amp=amp, wave=wave,
                       cE=dt / dz, cH=dt / dz)
    cs = (3, 3, nz)
    probe = DFTMonitor(np.array([omega]), np.array([flat_index(0, 1, 1, k_probe, cs), flat_index(1, 1, 1, k_probe, cs)]),
                       np.array([flat_index(1, 1, 1, k_probe - 1, cs), flat_index(0, 1, 1, k_probe - 1, cs)]),
                       np.array([flat_index(1, 1, 1, k_probe, cs), flat_index(0, 1, 1, k_probe, cs)]), source=src)
    mons = [plane_monitor(shape, k_r, [omega], energy=1), plane_monitor(shape, k_t, [omega], energy=1), probe]
    return make_plan(shape=shape, dx=spacing, dt=dt, single=single, inv_eps=1.0 / eps, groups=[], pml=pml_main,
                     sources=[src], monitors=mons, dft_stride=stride, periodic=(True, True, False),
                     bloch=(kx, ky, 0.0))


def metasurface_sweep(n_runs: int = 96, seed: int = 0, **kw) -> list[dict]:
    """``n_runs`` oblique runs drawn from ``seed``: period U(300, 600) nm, polar angle U(0, 60) deg, azimuth
    U(0, 90) deg, wavelength U(450, 750) nm, s or p polarisation."""
    rng = np.random.default_rng(seed)
    runs = []
    for _ in range(n_runs):
        period = float(rng.uniform(300, 600))
        theta, phi = float(rng.uniform(0, 60)), float(rng.uniform(0, 90))
        wl = float(rng.uniform(450, 750))
        pol = "s" if rng.integers(2) == 0 else "p"
        runs.append(metasurface_run(period, theta, phi, wl, pol, **kw))
    return runs


# --- the adjoint workload: a slab waveguide device with a design region ---------------------------------


def slab_te0(n_core: float, n_clad: float, thickness: float, wavelength: float):
    """(beta, profile(z)) of the fundamental TE mode of a symmetric slab: E_y = cos(kappa z) in the core
    (|z| <= t/2), cos(kappa t/2) exp(-gamma (|z| - t/2)) outside, from kappa tan(kappa t/2) = gamma (bisection
    on kappa in (0, pi/t))."""
    k0 = 2 * np.pi / wavelength
    V = k0 * math.sqrt(n_core ** 2 - n_clad ** 2)
    lo, hi = 1e-12, min(math.pi / thickness, V) * (1 - 1e-12)

    def f(kap):
        return kap * math.tan(kap * thickness / 2) - math.sqrt(max(V * V - kap * kap, 0.0))
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if f(lo) * f(mid) <= 0:
            hi = mid
        else:
            lo = mid
    kap = 0.5 * (lo + hi)
    gam = math.sqrt(V * V - kap * kap)
    beta = math.sqrt((n_core * k0) ** 2 - kap ** 2)

    def profile(z):
        z = np.abs(np.asarray(z, float))
        inside = z <= thickness / 2
        return np.where(inside, np.cos(kap * z), math.cos(kap * thickness / 2) * np.exp(-gam * (z - thickness / 2)))
    return beta, profile


def design_field(shape2, corr_cells: float, seed: int, beta: float = 8.0, eta: float = 0.5) -> np.ndarray:
    """rho in [0, 1] over a 2D design region: white noise from ``seed`` filtered by a Gaussian of correlation
    length ``corr_cells`` (FFT), normalised, then the tanh projection with steepness beta about eta."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape2)
    kx = np.fft.fftfreq(shape2[0])[:, None]
    ky = np.fft.fftfreq(shape2[1])[None, :]
    g = np.real(np.fft.ifft2(np.fft.fft2(w) * np.exp(-2 * (np.pi * corr_cells) ** 2 * (kx ** 2 + ky ** 2))))
    g = (g - g.mean()) / (g.std() + 1e-30)
    x = 1 / (1 + np.exp(-g))  # into (0, 1) about 0.5
    num = np.tanh(beta * eta) + np.tanh(beta * (x - eta))
    return num / (np.tanh(beta * eta) + np.tanh(beta * (1 - eta)))


def slab_device_plan(shape=(200, 200, 120), dx: float = 20.0, pml: int = 12, design=(100, 100),
                     thickness: float = 220.0, n_core: float = 3.48, n_clad: float = 1.44,
                     wavelength: float = 1550.0, n_steps: int = 8000, stride: int = 10, seed: int = 0,
                     single: bool = True):
    """The inverse-design workload: a ``thickness`` slab of index n_core in n_clad filling the grid along x and
    y (the input and output waveguides), a ``design`` (cells) region of it in the middle whose permittivity is
    eps = n_clad^2 + rho (n_core^2 - n_clad^2) for a seeded Gaussian random field rho (correlation 100 nm, tanh
    projection beta = 8), the slab's TE0 mode launched by an E_y current sheet on a plane before the design
    region (a Gaussian pulse at ``wavelength``) and the objective's monitor, E_y on a plane after it.

    Returns (plan, box, wE, info): the design box (node ranges), the overlap weights of the monitor's points
    (the mode profile times the cell area) and the pieces that map rho to 1/eps."""
    n0, n1, n2 = shape
    dt = 0.99 * dx / math.sqrt(3)
    zc = n2 // 2
    z = (np.arange(n2) - zc) * dx
    core = np.abs(z) <= thickness / 2
    eps = np.full(shape, n_clad ** 2)
    eps[:, :, core] = n_core ** 2
    x0 = (n0 - design[0]) // 2
    y0 = (n1 - design[1]) // 2
    box = ((x0, x0 + design[0]), (y0, y0 + design[1]), (int(np.nonzero(core)[0][0]), int(np.nonzero(core)[0][-1]) + 1))
    rho = design_field(design, 100.0 / dx, seed)
    eps[box[0][0]:box[0][1], box[1][0]:box[1][1], box[2][0]:box[2][1]] = (
        n_clad ** 2 + rho[:, :, None] * (n_core ** 2 - n_clad ** 2))
    inv_eps = 1.0 / eps
    beta, prof = slab_te0(n_core, n_clad, thickness, wavelength)
    # E_y nodes of the source and monitor planes: y over the non-CPML range, z within the mode's extent
    ys = np.arange(pml + 2, n1 - pml - 2)
    zs = np.arange(n2)[np.abs(z) <= thickness / 2 + 3 * wavelength / (2 * np.pi * math.sqrt(n_core ** 2 - n_clad ** 2))]
    zs = zs[(zs > pml + 1) & (zs < n2 - pml - 2)]
    Y, Z = np.meshgrid(ys, zs, indexing="ij")
    amp = prof((Z.ravel() - zc) * dx)
    x_src, x_out = pml + 6, n0 - pml - 7
    src_idx = flat_index(1, np.full(Y.size, x_src), Y.ravel(), Z.ravel(), shape).astype(np.int64)
    omega = 2 * np.pi / wavelength
    half = 0.1 * omega
    tau = 2.0 / half
    t0 = 3.5 * tau
    t = np.arange(n_steps + 3) * dt
    gpulse = np.exp(-(((t - t0) / tau) ** 2)) * np.sin(omega * (t - t0))
    flat_inv = inv_eps.reshape(-1)
    coef = dt * flat_inv[src_idx % (n0 * n1 * n2)] * amp
    src = DipoleSource(idx=src_idx, coef=coef, wave=np.diff(gpulse) / (omega * dt))
    mon_idx = flat_index(1, np.full(Y.size, x_out), Y.ravel(), Z.ravel(), shape).astype(np.int64)
    mon = DFTMonitor(np.array([omega]), mon_idx, None, None, energy=0)
    spec = PMLSpec(cells=((pml, pml),) * 3, alpha_max=0.05 * omega, eps_ref=n_clad ** 2)
    plan = make_plan(shape=shape, dx=dx, dt=dt, single=single, inv_eps=inv_eps, groups=[], pml=spec, sources=[src],
                     monitors=[mon], dft_stride=stride)
    wE = amp * dx * dx
    info = {"rho": rho, "eps_clad": n_clad ** 2, "eps_core": n_core ** 2, "n_steps": n_steps}
    return plan, box, wE, info


# --- dispersive clusters (forward + adjoint over many instances) ------------------------------------------

EV_NM = 197.3269804  # hbar c in eV nm: photon energies to angular frequencies in rad/nm (c = 1)


def drude_lorentz(eps_inf: float, wp_ev: float, gamma_ev: float, lorentz) -> Medium:
    """A Drude pole and Lorentz poles (d_eps, omega0 eV, width eV) in engine units, as lightsmith's media
    converts them (``media.py:68-75``): Drude sigma = wp^2, omega0 = 0; Lorentz sigma = d_eps omega0^2."""
    poles = [Pole((wp_ev / EV_NM) ** 2, 0.0, gamma_ev / EV_NM)]
    poles += [Pole(de * (w0 / EV_NM) ** 2, w0 / EV_NM, g / EV_NM) for de, w0, g in lorentz]
    return Medium(eps_inf, tuple(poles))


# silver of the cluster workload: eps_inf 3.7, wp 9.2 eV, gamma 0.02 eV, and the two Lorentz poles of the
# sphere benchmark (1.3 at 2.6 eV, width 0.6 eV; 1.5 at 3.7 eV, width 1.0 eV)
SILVER = drude_lorentz(3.7, 9.2, 0.02, [(1.3, 2.6, 0.6), (1.5, 3.7, 1.0)])


def box_flux_monitor(shape, lo, hi, omega):
    """The six faces of the node box [lo, hi] as one monitor: per face normal to axis a at index k, the two
    tangential E components on the face's nodes, each with the H component it pairs with averaged over planes
    k - 1 and k along a (plane_monitor's layout per face). Returns (monitor, s): the power out of the box is
    0.5 Re sum_p s_p acc_e[f, p] conj(acc_h[f, p]) (s: +-1 by pairing and outward normal)."""
    e, h1, h2, sg = [], [], [], []
    for a in range(3):
        b, c = (a + 1) % 3, (a + 2) % 3
        rng_b = np.arange(lo[b], hi[b] + 1)
        rng_c = np.arange(lo[c], hi[c] + 1)
        B, Cc = (v.ravel() for v in np.meshgrid(rng_b, rng_c, indexing="ij"))
        for side, k in ((-1, lo[a]), (1, hi[a])):
            def at(comp, kk):
                x = [None] * 3
                x[a], x[b], x[c] = np.full(B.size, kk), B, Cc
                return flat_index(comp, x[0], x[1], x[2], shape)
            # flux_a = E_b H_c* - E_c H_b*
            e += [at(b, k), at(c, k)]
            h1 += [at(c, k - 1), at(b, k - 1)]
            h2 += [at(c, k), at(b, k)]
            sg += [np.full(B.size, float(side)), np.full(B.size, -float(side))]
    mon = DFTMonitor(np.asarray(omega, float), np.concatenate(e).astype(np.int64),
                     np.concatenate(h1).astype(np.int64), np.concatenate(h2).astype(np.int64), energy=0)
    return mon, np.concatenate(sg)


def cluster_spheres(rng, dx: float):
    """3-12 spheres (radii U(10, 40) nm) at random non-overlapping positions (at least 2 dx apart), drawn from
    ``rng``: a list of (centre (3,), radius) in nm around the origin."""
    n_sph = int(rng.integers(3, 13))
    radii = rng.uniform(10.0, 40.0, n_sph)
    side = 2.2 * float(np.sum(radii ** 3)) ** (1 / 3) + 2 * radii.max()
    centres = []
    for _ in range(200):
        centres = []
        for r in radii:
            for _try in range(2000):
                c = rng.uniform(-side / 2 + r, side / 2 - r, 3)
                if all(np.linalg.norm(c - c2) >= r + r2 + 2 * dx for c2, r2 in centres):
                    centres.append((c, r))
                    break
            else:
                break
        if len(centres) == n_sph:
            break
        side *= 1.1
    return centres


def cluster_instance(seed: int, dx: float = 2.0, n_bg: float = 1.33, n_freq: int = 24, lam=(350.0, 700.0),
                     n_steps: int = 2000, shell_nm: float = 60.0, pml: int = 12, single: bool = True,
                     stride: int = 16, n_min: int = 96, n_max: int = 256):
    """One instance of the dispersive-cluster workload: 3-12 silver spheres (radii U(10, 40) nm) at random
    non-overlapping positions in a background of index n_bg on a cubic grid of dx, sized to the cluster
    (n_min^3 .. n_max^3 cells); node-centred staircase spheres (every E component of a node whose centre lies
    in a sphere belongs to one pure D-form group, with 1/eps = 1 there); a point dipole just outside the
    60 nm shell around the spheres; the power out of a closed box around the shell at n_freq wavelengths in
    lam as the objective. Returns (plan, info) with info: box (the shell's bounding box of nodes, the
    gradient's design box), shell (a bool mask over that box: background nodes within shell_nm of a sphere),
    objective (J of the accumulators), the spheres and the step count."""
    rng = np.random.default_rng(seed)
    centres = cluster_spheres(rng, dx)
    lo_nm = np.min([c - r for c, r in centres], axis=0) - shell_nm
    hi_nm = np.max([c + r for c, r in centres], axis=0) + shell_nm
    margin = 14  # cells: dipole and flux box outside the shell, then the CPML
    n = int(np.clip(math.ceil(float(np.max(hi_nm - lo_nm)) / dx) + 2 * (margin + pml + 2), n_min, n_max))
    n = min(n_max, -(-n // 4) * 4)  # rows of a multiple of 16 bytes: the fused pass's tensor copies apply
    shape = (n, n, n)
    mid = 0.5 * (lo_nm + hi_nm)
    origin = mid - (n // 2) * dx  # node i sits at origin + i dx
    pos = origin[:, None] + dx * np.arange(n)[None, :]
    X, Y, Z = np.meshgrid(pos[0], pos[1], pos[2], indexing="ij")
    inside = np.zeros(shape, bool)
    dist = np.full(shape, np.inf)
    for c, r in centres:
        d = np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) - r
        inside |= d < 0
        dist = np.minimum(dist, d)
    inv_eps = np.full(shape, 1.0 / n_bg ** 2)
    inv_eps[inside] = 1.0
    cells = n ** 3
    node = np.flatnonzero(inside.reshape(-1))
    idx = np.concatenate([cc * cells + node for cc in range(3)]).astype(np.int64)
    group = DispersiveGroup(idx=idx, media=[SILVER], frac=np.ones((1, len(idx))), w=None)
    blo = np.maximum(np.floor((lo_nm - origin) / dx).astype(int), pml + 3)
    bhi = np.minimum(np.ceil((hi_nm - origin) / dx).astype(int) + 1, n - pml - 3)
    box = tuple((int(a), int(b)) for a, b in zip(blo, bhi))
    bsl = tuple(slice(a, b) for a, b in box)
    shell = (~inside[bsl]) & (dist[bsl] <= shell_nm)
    dt = 0.99 * dx / math.sqrt(3)
    wl = np.linspace(lam[0], lam[1], n_freq)
    om = 2 * np.pi / wl  # vacuum wavelengths (c = 1)
    omega_c = 0.5 * (om.min() + om.max())
    dip_node = np.array([bhi[0] + 3, (blo[1] + bhi[1]) // 2, (blo[2] + bhi[2]) // 2])
    pdir = rng.normal(size=3)
    pdir /= np.linalg.norm(pdir)

    def at(flat):
        rest = np.asarray(flat) % cells
        return inv_eps.reshape(-1)[rest]

    dip = point_dipole(shape, np.zeros(3), dx, dt, (dip_node + 0.3) * dx, tuple(pdir), at, omega_c, 0.6 * omega_c,
                       n_steps + 8)
    flo = [int(v) - 6 for v in blo]
    fhi = [int(v) + 6 for v in bhi]
    mon, sgn = box_flux_monitor(shape, flo, fhi, om)
    spec = PMLSpec(cells=((pml, pml),) * 3, alpha_max=0.05 * omega_c, eps_ref=n_bg ** 2)
    plan = make_plan(shape=shape, dx=dx, dt=dt, single=single, inv_eps=inv_eps, groups=[group], pml=spec,
                     sources=[dip], monitors=[mon], dft_stride=stride)

    def objective(acc_e, acc_h, sgn=sgn):
        import torch

        s = torch.as_tensor(sgn, dtype=torch.float64, device=acc_e.device)
        return 0.5 * (acc_e * acc_h.conj() * s).real.sum()

    info = {"box": box, "shell": shell, "objective": objective, "sign": sgn, "spheres": centres,
            "n_steps": int(n_steps), "n_bg": n_bg, "wavelengths": wl, "cells": cells}
    return plan, info


SILVER_DRUDE_LORENTZ = dict(eps_inf=3.7, wp_ev=9.2, gamma_ev=0.02,
                            poles=[{"delta_eps": 1.3, "omega0_ev": 2.6, "gamma_ev": 0.6},
                                   {"delta_eps": 1.5, "omega0_ev": 3.7, "gamma_ev": 1.0}])


def cluster_scattering(seed: int, dx: float = 2.0, n_bg: float = 1.33, n_freq: int = 24, lam=(350.0, 700.0),
                       n_steps: int = 2000, shell_nm: float = 60.0, pml: int = 12, stride: int = 16,
                       precision: str = "single"):
    """One instance of the dispersive-cluster workload posed to lightsmith: the spheres of ``cluster_spheres``
    (silver: the sphere benchmark's Drude + two Lorentz form with eps_inf 3.7, wp 9.2 eV, gamma 0.02 eV) as a
    lightsmith ``Simulation`` in a background of index n_bg (dx cells, CPML pml, staircase meshing, n_freq
    wavelengths in lam, the TF/SF box shell_nm + 4 dx beyond the spheres' bounding box), set up by lightsmith's
    own scattering driver (``scattering.scattering_setup``: its table-fed TF/SF plane wave and flux boxes) for
    n_steps steps. Returns (plan, info): info has box (the design box: the node ranges of the shell, background
    nodes within shell_nm of a sphere), shell (a bool mask over it), objective (sum_f C_sca(f) of the
    scattered-field box, ``scattering.cross_section_objective``) with ``ref`` (its reference-view input,
    ``ref["acc_ref"]`` to be set to the run's third monitor's accumulators, and ``ref["spectrum"]``), post,
    spheres, n_steps, n_bg, cells."""
    import lightsmith as ls

    from .scattering import cross_section_objective, scattering_setup

    rng = np.random.default_rng(seed)
    centres = cluster_spheres(rng, dx)
    metal = ls.DrudeLorentz(**SILVER_DRUDE_LORENTZ)
    dt = 0.99 * dx / math.sqrt(3)
    sim = ls.Simulation(
        particles=[ls.Particle(shape=ls.Sphere(radius_nm=float(r)), material=metal,
                               position_nm=tuple(float(v) for v in c)) for c, r in centres],
        medium_index=n_bg, wavelengths={"start_nm": float(lam[0]), "stop_nm": float(lam[1]), "num": int(n_freq)},
        options={"fdtd": dict(spacing_nm=dx, pml_cells=pml, courant=0.99, symmetry="off",
                              mesh_refinement="staircase", padding_nm=shell_nm + 4 * dx, dft_stride=stride,
                              run_time_fs=(n_steps - 0.5) * dt / 299.792458, precision=precision)})
    plan, post, lay = scattering_setup(sim)
    shape = tuple(int(v) for v in plan["shape"])
    pos = [np.asarray(lay.origin, dtype=float)[a] + dx * np.arange(shape[a]) for a in range(3)]
    lo = np.min([c - r for c, r in centres], axis=0) - shell_nm
    hi = np.max([c + r for c, r in centres], axis=0) + shell_nm
    blo = [int(np.searchsorted(pos[a], lo[a])) for a in range(3)]
    bhi = [int(np.searchsorted(pos[a], hi[a], side="right")) for a in range(3)]
    box = tuple((a, b) for a, b in zip(blo, bhi))
    X, Y, Z = np.meshgrid(*[pos[a][blo[a]:bhi[a]] for a in range(3)], indexing="ij")
    dist = np.full(X.shape, np.inf)
    for c, r in centres:
        dist = np.minimum(dist, np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) - r)
    inv = np.asarray(plan["inv_eps"])
    inv = inv.reshape((-1,) + shape)
    bsl = (slice(None),) + tuple(slice(a, b) for a, b in box)
    background = np.all(np.abs(inv[bsl] - 1.0 / n_bg ** 2) < 1e-12 / n_bg ** 2, axis=0)
    shell = background & (dist > 0) & (dist <= shell_nm)
    ref: dict = {}
    info = {"box": box, "shell": shell, "objective": cross_section_objective(post, ref), "ref": ref, "post": post,
            "spheres": centres, "n_steps": int(n_steps), "n_bg": n_bg, "cells": int(np.prod(shape))}
    return plan, info

