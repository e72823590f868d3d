"""Small seeded runs for the adjoint tests: a random-permittivity grid with CPML on every face, a point
dipole near the low-x face, a DFT plane monitor, and a design box between them (outside the CPML slabs and
away from the source nodes)."""

import math

import numpy as np

from lightsmith_b200.plan import PMLSpec, make_plan
from lightsmith_b200.workloads import plane_monitor, point_dipole

SHAPE = (22, 18, 16)
BOX = ((10, 15), (6, 12), (5, 9))
DX = 20.0


def small_case(seed: int = 4, n_chunks: int = 4, pml_cells: int = 4):
    """(plan, n_steps, weights of the monitor's E and H points)."""
    dt = 0.99 * DX / math.sqrt(3)
    rng = np.random.default_rng(seed)
    inv_eps = 1.0 / rng.uniform(1.0, 4.0, size=SHAPE)
    omega = 2 * np.pi / 300.0
    stride = 7
    n_steps = n_chunks * stride

    def at(flat):
        rest = np.asarray(flat) % int(np.prod(SHAPE))
        return inv_eps[np.unravel_index(rest, SHAPE)]

    dip = point_dipole(SHAPE, np.zeros(3), DX, dt, np.array([6.37, 9.37, 8.37]) * DX, (0.3, 1.0, 0.2), at,
                       omega, 0.4 * omega, n_steps + 400)
    w = dip.wave
    first = int(np.nonzero(np.abs(w) > 1e-3 * np.abs(w).max())[0][0])
    dip.wave = np.concatenate([w[first:], np.zeros(first)])
    mon = plane_monitor(SHAPE, 12, [omega], energy=1)
    pml = PMLSpec(cells=((pml_cells, pml_cells),) * 3, alpha_max=0.02, eps_ref=1.5)
    plan = make_plan(shape=SHAPE, dx=DX, dt=dt, single=False, inv_eps=inv_eps, groups=[], pml=pml, sources=[dip],
                     monitors=[mon], dft_stride=stride)
    m = len(mon.e_idx)
    wE = rng.normal(size=m) + 1j * rng.normal(size=m)
    wH = 0.3 * (rng.normal(size=m) + 1j * rng.normal(size=m))
    return plan, n_steps, wE, wH


PERIODIC_BOX = ((1, 21), (1, 17), (5, 8))


def periodic_case(seed: int = 11, n_chunks: int = 5, pml_cells: int = 4):
    """small_case's grid periodic along x and y (ghost planes 0 and n - 1, real fields) with CPML along z, a
    dipole at z = 9.4 and the monitor on z-plane 12; the design box spans every stepped x and y node (next to
    both ghost planes of each periodic axis) at z = 5..7. Returns (plan, n_steps, wE, wH)."""
    dt = 0.99 * DX / math.sqrt(3)
    rng = np.random.default_rng(seed)
    inv_eps = 1.0 / rng.uniform(1.0, 4.0, size=SHAPE)
    omega = 2 * np.pi / 300.0
    stride = 7
    n_steps = n_chunks * stride

    def at(flat):
        rest = np.asarray(flat) % int(np.prod(SHAPE))
        return inv_eps[np.unravel_index(rest, SHAPE)]

    dip = point_dipole(SHAPE, np.zeros(3), DX, dt, np.array([3.37, 15.37, 9.37]) * DX, (0.3, 1.0, 0.6), at,
                       omega, 0.4 * omega, n_steps + 400)
    w = dip.wave
    first = int(np.nonzero(np.abs(w) > 1e-3 * np.abs(w).max())[0][0])
    dip.wave = np.concatenate([w[first:], np.zeros(first)])
    mon = plane_monitor(SHAPE, 12, [omega], energy=1)
    pml = PMLSpec(cells=((0, 0), (0, 0), (pml_cells, pml_cells)), alpha_max=0.02, eps_ref=1.5)
    plan = make_plan(shape=SHAPE, dx=DX, dt=dt, single=False, inv_eps=inv_eps, groups=[], pml=pml, sources=[dip],
                     monitors=[mon], dft_stride=stride, periodic=(True, True, False))
    m = len(mon.e_idx)
    wE = rng.normal(size=m) + 1j * rng.normal(size=m)
    wH = 0.3 * (rng.normal(size=m) + 1j * rng.normal(size=m))
    return plan, n_steps, wE, wH


def flux_objective(acc_e, acc_h):
    """The monitor plane's flux summed over its frequencies: 0.5 Re sum_p s_p acc_e[f, p] conj(acc_h[f, p]),
    s_p = +1 for the E_x / H_y half of the points and -1 for the E_y / H_x half (plane_monitor's layout)."""
    m = acc_e.shape[1] // 2
    s = acc_e.new_ones(acc_e.shape[1]).real
    s[m:] = -1
    return 0.5 * (acc_e * acc_h.conj() * s).real.sum()


def dispersive_case(seed: int = 7, n_chunks: int = 4, pml_cells: int = 4):
    """small_case's grid and dipole with a 2 x 4 x 4-node block of a Drude-Lorentz metal between the dipole and
    the design box (a pure D-form group over the three E components of those nodes, which have 1/eps = 1 as
    lightsmith's D-form nodes do), a three-frequency monitor on z-plane 12 and its flux spectrum as the
    objective. Returns (plan, n_steps, objective)."""
    from lightsmith_b200.plan import DispersiveGroup, Medium, Pole

    dt = 0.99 * DX / math.sqrt(3)
    rng = np.random.default_rng(seed)
    inv_eps = 1.0 / rng.uniform(1.0, 4.0, size=SHAPE)
    block = (slice(8, 10), slice(5, 9), slice(4, 8))
    inv_eps[block] = 1.0
    omega = 2 * np.pi / 300.0
    stride = 7
    n_steps = n_chunks * stride
    ii, jj, kk = (a.ravel() for a in np.meshgrid(*(np.arange(s.start, s.stop) for s in block), indexing="ij"))
    cells = int(np.prod(SHAPE))
    node = np.ravel_multi_index((ii, jj, kk), SHAPE)
    idx = np.concatenate([c * cells + node for c in range(3)])
    metal = Medium(3.7, (Pole(0.002, 0.0, 0.002), Pole(0.0005, 0.02, 0.004)))
    group = DispersiveGroup(idx=idx, media=[metal], frac=np.ones((1, len(idx))), w=None)

    def at(flat):
        rest = np.asarray(flat) % cells
        return inv_eps[np.unravel_index(rest, SHAPE)]

    dip = point_dipole(SHAPE, np.zeros(3), DX, dt, np.array([6.37, 9.37, 8.37]) * DX, (0.3, 1.0, 0.2), at,
                       omega, 0.4 * omega, n_steps + 400)
    w = dip.wave
    first = int(np.nonzero(np.abs(w) > 1e-3 * np.abs(w).max())[0][0])
    dip.wave = np.concatenate([w[first:], np.zeros(first)])
    mon = plane_monitor(SHAPE, 12, [0.8 * omega, omega, 1.2 * omega], energy=1)
    pml = PMLSpec(cells=((pml_cells, pml_cells),) * 3, alpha_max=0.02, eps_ref=1.5)
    plan = make_plan(shape=SHAPE, dx=DX, dt=dt, single=False, inv_eps=inv_eps, groups=[group], pml=pml,
                     sources=[dip], monitors=[mon], dft_stride=stride)
    return plan, n_steps, flux_objective


def mixed_case(seed: int = 9, n_chunks: int = 4, pml_cells: int = 4):
    """dispersive_case's grid, dipole, monitor and flux objective with its block of interface cells instead: a
    mixed D-form group (lightsmith's subpixel interface cells) of the Drude-Lorentz metal and a dielectric of
    index 1.8, each node's metal fraction drawn from U(0.2, 0.8) and its harmonic weight w from U(0, 1) (a few
    nodes at exactly 0 and 1), so that both paths run. Returns (plan, n_steps, objective)."""
    from lightsmith_b200.plan import DispersiveGroup, Medium, Pole

    dt = 0.99 * DX / math.sqrt(3)
    rng = np.random.default_rng(seed)
    inv_eps = 1.0 / rng.uniform(1.0, 4.0, size=SHAPE)
    block = (slice(8, 10), slice(5, 9), slice(4, 8))
    inv_eps[block] = 1.0
    omega = 2 * np.pi / 300.0
    stride = 7
    n_steps = n_chunks * stride
    ii, jj, kk = (a.ravel() for a in np.meshgrid(*(np.arange(s.start, s.stop) for s in block), indexing="ij"))
    cells = int(np.prod(SHAPE))
    node = np.ravel_multi_index((ii, jj, kk), SHAPE)
    idx = np.concatenate([c * cells + node for c in range(3)])
    metal = Medium(3.7, (Pole(0.002, 0.0, 0.002), Pole(0.0005, 0.02, 0.004)))
    glass = Medium(1.8 ** 2, ())
    fm = rng.uniform(0.2, 0.8, len(idx))
    w = rng.uniform(0.0, 1.0, len(idx))
    w[:3], w[3:6] = 0.0, 1.0
    group = DispersiveGroup(idx=idx, media=[metal, glass], frac=np.stack([fm, 1.0 - fm]), w=w)

    def at(flat):
        rest = np.asarray(flat) % cells
        return inv_eps[np.unravel_index(rest, SHAPE)]

    dip = point_dipole(SHAPE, np.zeros(3), DX, dt, np.array([6.37, 9.37, 8.37]) * DX, (0.3, 1.0, 0.2), at,
                       omega, 0.4 * omega, n_steps + 400)
    wv = dip.wave
    first = int(np.nonzero(np.abs(wv) > 1e-3 * np.abs(wv).max())[0][0])
    dip.wave = np.concatenate([wv[first:], np.zeros(first)])
    mon = plane_monitor(SHAPE, 12, [0.8 * omega, omega, 1.2 * omega], energy=1)
    pml = PMLSpec(cells=((pml_cells, pml_cells),) * 3, alpha_max=0.02, eps_ref=1.5)
    plan = make_plan(shape=SHAPE, dx=DX, dt=dt, single=False, inv_eps=inv_eps, groups=[group], pml=pml,
                     sources=[dip], monitors=[mon], dft_stride=stride)
    return plan, n_steps, flux_objective

