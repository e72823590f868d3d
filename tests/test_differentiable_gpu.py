"""The differentiable FDTD solve on the B200: S-parameters against lightsmith's own solve of the same device
problem, and gradients against finite differences.

``diff_device_3d.npz`` holds ``backend.device_runs`` of a silicon wire width step (500 -> 700 nm, 220 nm thick,
in silica; 73 x 83 x 73 cells at 40 nm, subpixel mesh, two ports, 279 steps) and the S matrix
``ls.solve(problem, "fdtd", "cpu")`` gave for it in float64; ``diff_device_2d.npz`` the same for the 2D width
step (TE, 123 x 139 x 3 cells at 25 nm with the invariant z axis periodic, 1640 steps).
"""

import numpy as np
import pytest

RTOL_F64 = 1e-9  # float64 on the GPU: the same arithmetic, a different summation order
RTOL_F32 = 2e-4  # float32 on the GPU against lightsmith's float64 CPU run


@pytest.fixture(scope="module", params=[3, 2], ids=["3d", "2d"])
def fixture(golden, request):
    return golden(f"diff_device_{request.param}d")


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b)))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["double", "single"])
def test_s_parameters_match_lightsmith(fixture, precision):
    import torch

    from lightsmith_b200.differentiable import DeviceSolver, s_parameters

    solver = DeviceSolver(fixture["desc"], precision=precision)
    S = s_parameters(torch.as_tensor(solver.base_design), solver).detach().cpu().numpy()
    solver.close()
    assert S.shape == fixture["s"].shape
    err = _rel(S, fixture["s"])
    assert err <= (RTOL_F64 if precision == "double" else RTOL_F32), err


def _design_block(solver):
    """A 6 x 6 (x 4) node block at the step, set to eps = 6 (between silica and silicon)."""
    eps = solver.base_design.copy()
    c = [n // 2 for n in solver.design_shape]
    half = (3, 3, 2)
    sl = tuple(slice(ci - h, ci + h) for ci, h in zip(c, half))
    eps[sl] = 6.0
    return eps, sl, c


@pytest.mark.gpu
def test_gradient_matches_finite_differences(fixture):
    """L = |S21|^2 at the first wavelength + |S12|^2 at the second: both columns' adjoints; the autograd
    gradient at nodes of the design block against central differences (h = 1e-3, float64)."""
    import torch

    from lightsmith_b200.differentiable import DeviceSolver, s_parameters

    solver = DeviceSolver(fixture["desc"], precision="double")
    eps0, sl, c = _design_block(solver)

    def loss(e):
        S = s_parameters(e, solver)
        return S[0, 1, 0].abs() ** 2 + S[1, 0, 1].abs() ** 2

    e = torch.as_tensor(eps0).requires_grad_(True)
    L = loss(e)
    L.backward()
    g = e.grad.numpy()
    assert g.shape == solver.design_shape
    outside = np.ones(solver.design_shape, bool)
    outside[solver.box_sl[:len(c)]] = False
    assert np.all(g[outside] == 0) and np.abs(g[sl]).max() > 0
    lo, hi = [s.start for s in sl], [s.stop for s in sl]
    nodes = [(lo[0], lo[1], lo[-1]), (c[0], c[1], c[-1]), (hi[0] - 1, c[1], hi[-1] - 1), (c[0] + 1, lo[1], c[-1] - 1)]
    nodes = [n[:len(c)] for n in nodes]
    h = 1e-3
    with torch.no_grad():
        for n in nodes:
            ep, em = eps0.copy(), eps0.copy()
            ep[n] += h
            em[n] -= h
            fd = (float(loss(torch.as_tensor(ep))) - float(loss(torch.as_tensor(em)))) / (2 * h)
            assert abs(g[n] - fd) <= 1e-5 * abs(fd) + 1e-9 * np.abs(g).max(), (n, g[n], fd)
    solver.close()


@pytest.mark.gpu
def test_gradient_flows_through_a_density(fixture):
    """A design density rho in [0, 1] mapped to eps = 2.07 + rho (12.1 - 2.07) inside the block, as lightsmith's
    compose_eps does (inverse/parametrization.py:187-204): d L / d rho by autograd against one directional
    finite difference."""
    import torch

    from lightsmith_b200.differentiable import DeviceSolver, s_parameters

    solver = DeviceSolver(fixture["desc"], precision="double")
    eps0, sl, _ = _design_block(solver)
    base = torch.as_tensor(eps0)
    shape = tuple(s.stop - s.start for s in sl)
    rng = np.random.default_rng(0)
    rho0 = torch.as_tensor(rng.uniform(0.3, 0.7, size=shape))
    lo, hi = 1.444 ** 2, 3.476 ** 2

    def loss(rho):
        e = base.clone()
        e[sl] = lo + rho * (hi - lo)
        S = s_parameters(e, solver, sources=["o1"])
        return (S[:, 1, 0].abs() ** 2).sum()

    rho = rho0.clone().requires_grad_(True)
    loss(rho).backward()
    d = torch.as_tensor(rng.normal(size=shape))
    t = 1e-4
    with torch.no_grad():
        fd = (float(loss(rho0 + t * d)) - float(loss(rho0 - t * d))) / (2 * t)
    ad = float((rho.grad * d).sum())
    assert abs(ad - fd) <= 1e-5 * abs(fd), (ad, fd)
    solver.close()


@pytest.mark.gpu
def test_field_outputs_and_their_gradient(fixture):
    """The field outputs (a whole-grid DFT monitor added to each run): S unchanged by it, and the gradient of a
    mean |field|^2 over a small box (lightsmith's field-intensity term, inverse/objectives.py:53-68) against
    central differences."""
    import torch

    from lightsmith_b200.differentiable import DeviceSolver, s_parameters

    solver = DeviceSolver(fixture["desc"], precision="double")
    eps0, sl, c = _design_block(solver)
    e = torch.as_tensor(eps0)
    S_plain = s_parameters(e, solver, sources=["o1"]).detach()
    S, F = s_parameters(e, solver, sources=["o1"], fields=True)
    assert torch.equal(S.detach(), S_plain)
    assert F.shape == (2, 1) + tuple(solver.field_shape())
    # a box a few nodes past the block towards port o2
    fb = tuple(slice(ci + 6, ci + 9) for ci in c)

    def loss(x):
        _, f = s_parameters(x, solver, sources=["o1"], fields=True)
        f = f[:, 0]
        if f.dim() == 5:  # 3D: |E|^2 summed over the components
            return (f[(slice(None), slice(None)) + fb].abs() ** 2).sum(1).mean()
        return (f[(slice(None),) + fb].abs() ** 2).mean()

    x = e.clone().requires_grad_(True)
    loss(x).backward()
    g = x.grad.numpy()
    h = 1e-3
    with torch.no_grad():
        for n in [tuple(ci for ci in c), tuple(s.start for s in sl)]:
            ep, em = eps0.copy(), eps0.copy()
            ep[n] += h
            em[n] -= h
            fd = (float(loss(torch.as_tensor(ep))) - float(loss(torch.as_tensor(em)))) / (2 * h)
            assert abs(g[n] - fd) <= 1e-5 * abs(fd) + 1e-9 * np.abs(g).max(), (n, g[n], fd)
    solver.close()


@pytest.mark.gpu
def test_gradient_steps_raise_the_transmission(fixture):
    """Three projected gradient steps on a design density (the step of lightsmith's optimisers, in miniature):
    the transmission sum_w |S21|^2 rises at each."""
    import torch

    from lightsmith_b200.differentiable import DeviceSolver, s_parameters

    solver = DeviceSolver(fixture["desc"], precision="single")
    eps0, sl, _ = _design_block(solver)
    base = torch.as_tensor(eps0)
    lo, hi = 1.444 ** 2, 3.476 ** 2
    rho = torch.full(tuple(s.stop - s.start for s in sl), 0.5, dtype=torch.float64)

    def transmission(r):
        e = base.clone()
        e[sl] = lo + r * (hi - lo)
        return (s_parameters(e, solver, sources=["o1"])[:, 1, 0].abs() ** 2).sum()

    values = []
    for _ in range(3):
        r = rho.clone().requires_grad_(True)
        T = transmission(r)
        T.backward()
        values.append(float(T.detach()))
        rho = (rho + 0.05 * r.grad / r.grad.abs().max()).clamp(0, 1)
    with torch.no_grad():
        values.append(float(transmission(rho)))
    solver.close()
    assert all(b > a for a, b in zip(values, values[1:])), values
