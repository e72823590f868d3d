"""The discrete adjoint on the GPU (lightsmith_b200.adjoint): its objective against the oracle's, its gradient
against torch autograd through the plain-PyTorch restatement (oracle/autograd.py) and against central finite
differences of the CUDA forward, with checkpoints every K steps for several K."""

import numpy as np
import pytest
import torch

from adjoint_cases import BOX, small_case

pytestmark = pytest.mark.gpu


def _autograd(plan, n_steps, wE, wH):
    from oracle.autograd import objective

    base = torch.as_tensor(np.asarray(plan["inv_eps"])[tuple(slice(a, b) for a, b in BOX)])
    x = base.clone().requires_grad_(True)
    J = objective(plan, x, BOX, 0, 0, wE, wH, n_steps)
    (g,) = torch.autograd.grad(J, x)
    return float(J.detach()), g.numpy(), base


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_adjoint_gradient_matches_autograd_in_double():
    from lightsmith_b200.adjoint import AdjointRun

    plan, n_steps, wE, wH = small_case()
    J_ref, g_ref, base = _autograd(plan, n_steps, wE, wH)
    run = AdjointRun(plan, BOX, wE=wE, wH=wH, checkpoint=2 * plan["stride"], precision="double")
    run.set_inv_eps_box(base)
    J, _ = run.forward(n_steps)
    g = run.backward().cpu().numpy()
    run.close()
    assert abs(J - J_ref) / J_ref < 1e-11
    assert np.abs(g_ref).max() > 0
    assert _rel(g, g_ref) < 1e-9


def test_checkpoint_interval_does_not_change_the_gradient():
    from lightsmith_b200.adjoint import AdjointRun

    plan, n_steps, wE, wH = small_case()
    grads = []
    for K in (plan["stride"], 3 * plan["stride"], n_steps):
        run = AdjointRun(plan, BOX, wE=wE, wH=wH, checkpoint=K, precision="double")
        run.forward(n_steps)
        grads.append(run.backward().cpu().numpy())
        run.close()
    assert np.array_equal(grads[0], grads[1]) and np.array_equal(grads[0], grads[2])


def test_autograd_function_and_single_precision():
    """fdtd_objective as a torch.autograd.Function (float32 engine) against the float64 autograd reference."""
    from lightsmith_b200.adjoint import AdjointRun, fdtd_objective

    plan, n_steps, wE, wH = small_case()
    J_ref, g_ref, base = _autograd(plan, n_steps, wE, wH)
    run = AdjointRun(plan, BOX, wE=wE, wH=wH, checkpoint=2 * plan["stride"], precision="single")
    x = base.clone().to("cuda").requires_grad_(True)
    J = fdtd_objective(x, run, n_steps)
    J.backward()
    run.close()
    assert abs(float(J.detach()) - J_ref) / J_ref < 1e-4
    assert _rel(x.grad.cpu().numpy(), g_ref) < 1e-3


def test_adjoint_gradient_matches_central_differences():
    from lightsmith_b200.adjoint import AdjointRun

    plan, n_steps, wE, wH = small_case()
    run = AdjointRun(plan, BOX, wE=wE, wH=wH, checkpoint=2 * plan["stride"], precision="double")
    base = torch.as_tensor(np.asarray(plan["inv_eps"])[tuple(slice(a, b) for a, b in BOX)])
    run.set_inv_eps_box(base)
    run.forward(n_steps)
    g = run.backward().cpu().numpy()
    h = 1e-6
    for flat in np.argsort(-np.abs(g).reshape(-1))[:4]:
        idx = tuple(int(v) for v in np.unravel_index(flat, g.shape))
        vals = []
        for sgn in (1, -1):
            x = base.clone()
            x[idx] += sgn * h
            run.set_inv_eps_box(x)
            vals.append(run.forward(n_steps)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-5 * abs(fd), (idx, fd, g[idx])
    run.close()


def test_periodic_axes_gradient_matches_central_differences():
    """Periodic x and y: the ghost planes' copies and their transposes; nodes next to both ghost planes of
    each axis and at a corner of the box, against central differences of the CUDA forward (float64)."""
    from adjoint_cases import PERIODIC_BOX, periodic_case

    from lightsmith_b200.adjoint import AdjointRun

    plan, n_steps, wE, wH = periodic_case()
    run = AdjointRun(plan, PERIODIC_BOX, wE=wE, wH=wH, checkpoint=2 * plan["stride"], precision="double")
    base = torch.as_tensor(np.asarray(plan["inv_eps"])[tuple(slice(a, b) for a, b in PERIODIC_BOX)])
    run.set_inv_eps_box(base)
    run.forward(n_steps)
    g = run.backward().cpu().numpy()
    nx, ny, nz = g.shape
    picks = [(0, 5, 1), (nx - 1, 5, 1), (4, 0, 2), (4, ny - 1, 2), (0, 0, 0), (nx - 1, ny - 1, nz - 1)]
    picks += [tuple(int(v) for v in np.unravel_index(f, g.shape)) for f in np.argsort(-np.abs(g).reshape(-1))[:2]]
    h = 1e-6
    for idx in picks:
        vals = []
        for sgn in (1, -1):
            x = base.clone()
            x[idx] += sgn * h
            run.set_inv_eps_box(x)
            vals.append(run.forward(n_steps)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-5 * abs(fd) + 1e-7 * np.abs(g).max(), (idx, fd, g[idx])
    run.close()


@pytest.mark.slow
def test_slab_device_gradient_in_rho_matches_finite_differences_on_32_cells():
    """The inverse-design workload at reduced size (float64): dJ/drho of the extruded design density by the
    adjoint against central differences on 32 random design cells."""
    from lightsmith_b200.adjoint import AdjointRun
    from lightsmith_b200.workloads import slab_device_plan

    plan, box, wE, info = slab_device_plan(shape=(64, 64, 48), pml=8, design=(24, 24), n_steps=1200, stride=10,
                                           single=False)
    run = AdjointRun(plan, box, wE=wE, checkpoint=200, precision="double")
    nz = box[2][1] - box[2][0]
    a, b = info["eps_clad"], info["eps_core"]

    def J_of(rho):
        eps = a + rho[:, :, None] * (b - a)
        run.set_inv_eps_box(torch.as_tensor(np.broadcast_to(1.0 / eps, rho.shape + (nz,)).copy()))
        return run.forward(info["n_steps"])[0]

    rho = info["rho"]
    J0 = J_of(rho)
    g_inv = run.backward().cpu().numpy()
    eps = a + rho[:, :, None] * (b - a)
    g = (g_inv * (-(b - a) / eps ** 2)).sum(axis=2)
    assert J0 > 0 and np.abs(g).max() > 0
    rng = np.random.default_rng(1)
    cells = rng.choice(rho.size, 32, replace=False)
    h = 1e-5
    errs = []
    for c in cells:
        i, j = np.unravel_index(c, rho.shape)
        rp, rm = rho.copy(), rho.copy()
        rp[i, j] += h
        rm[i, j] -= h
        fd = (J_of(rp) - J_of(rm)) / (2 * h)
        errs.append(abs(fd - g[i, j]) / max(np.abs(g).max(), 1e-300))
    run.close()
    assert max(errs) < 1e-5, max(errs)


@pytest.mark.slow
def test_full_size_slab_device_gradient_in_rho_matches_finite_differences_on_32_cells():
    """The inverse-design workload at its full size (200 x 200 x 120 cells of 20 nm, CPML 12, 100 x 100 x 11
    design nodes, 8000 steps, checkpoints every 256 steps), float64: dJ/drho by the adjoint against central
    differences of the CUDA forward on 32 random design cells, each within 1e-3 of its difference (the
    agreement the gradient is required to reach) and all within 1e-6 of the largest entry."""
    from lightsmith_b200.adjoint import AdjointRun
    from lightsmith_b200.workloads import slab_device_plan

    plan, box, wE, info = slab_device_plan(n_steps=8000, single=False)
    assert plan["shape"] == (200, 200, 120)
    run = AdjointRun(plan, box, wE=wE, checkpoint=256, precision="double")
    nz = box[2][1] - box[2][0]
    a, b = info["eps_clad"], info["eps_core"]

    def set_rho(rho):
        eps = a + rho[:, :, None] * (b - a)
        run.set_inv_eps_box(torch.as_tensor(np.broadcast_to(1.0 / eps, rho.shape + (nz,)).copy()))

    rho = info["rho"]
    set_rho(rho)
    J0 = run.forward(info["n_steps"])[0]
    g_inv = run.backward().cpu().numpy()
    eps = a + rho[:, :, None] * (b - a)
    g = (g_inv * (-(b - a) / eps ** 2)).sum(axis=2)
    assert J0 > 0 and np.abs(g).max() > 0
    rng = np.random.default_rng(3)
    cells = rng.choice(rho.size, 32, replace=False)
    h = 1e-5
    worst_rel, worst_abs = 0.0, 0.0
    for c in cells:
        i, j = np.unravel_index(c, rho.shape)
        vals = []
        for sgn in (1, -1):
            r = rho.copy()
            r[i, j] += sgn * h
            set_rho(r)
            vals.append(run.forward(info["n_steps"], keep=False)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[i, j]) <= 1e-3 * abs(fd) + 1e-6 * np.abs(g).max(), (i, j, fd, g[i, j])
        worst_rel = max(worst_rel, abs(fd - g[i, j]) / max(abs(fd), 1e-300))
        worst_abs = max(worst_abs, abs(fd - g[i, j]) / np.abs(g).max())
    run.close()
    print(f"full-size slab device: worst relative error {worst_rel:.2e}, worst against max|g| {worst_abs:.2e}")


def test_dispersive_group_and_flux_objective():
    """A Drude-Lorentz block (pure D-form group) between the dipole and the design box, and the monitor's
    three-frequency flux as the objective: the float64 gradient against torch autograd through the
    restatement, against central differences of the CUDA forward, and the same for two checkpoint intervals."""
    from adjoint_cases import dispersive_case
    from lightsmith_b200.adjoint import AdjointRun
    from oracle.autograd import objective

    plan, n_steps, J_of = dispersive_case()
    base = torch.as_tensor(np.asarray(plan["inv_eps"])[tuple(slice(a, b) for a, b in BOX)])
    x = base.clone().requires_grad_(True)
    J_ref = objective(plan, x, BOX, 0, 0, None, None, n_steps, J=J_of)
    (g_ref,) = torch.autograd.grad(J_ref, x)
    J_ref = float(J_ref.detach())
    grads = []
    for K in (plan["stride"], n_steps):
        run = AdjointRun(plan, BOX, objective=J_of, checkpoint=K, precision="double")
        run.set_inv_eps_box(base)
        J, _ = run.forward(n_steps)
        grads.append(run.backward().cpu().numpy())
        assert abs(J - J_ref) / abs(J_ref) < 1e-11
        if K == n_steps:
            g = grads[-1]
            h = 1e-6
            for flat in np.argsort(-np.abs(g).reshape(-1))[:3]:
                idx = tuple(int(v) for v in np.unravel_index(flat, g.shape))
                vals = []
                for sgn in (1, -1):
                    xp = base.clone()
                    xp[idx] += sgn * h
                    run.set_inv_eps_box(xp)
                    vals.append(run.forward(n_steps)[0])
                fd = (vals[0] - vals[1]) / (2 * h)
                assert abs(fd - g[idx]) <= 1e-5 * abs(fd), (idx, fd, g[idx])
        run.close()
    assert np.abs(g_ref.numpy()).max() > 0
    assert _rel(grads[0], g_ref.numpy()) < 1e-9
    assert np.array_equal(grads[0], grads[1])


def test_cluster_instance_gradient_matches_finite_differences():
    """A reduced instance of the dispersive-cluster workload (silver spheres as one pure D-form group, 4 nm
    grid, 12 nm shell, 800 steps), float64: dJ/d(1/eps) of the closed-box power on the shell's largest
    entries against central differences of the CUDA forward."""
    from lightsmith_b200.adjoint import AdjointRun
    from lightsmith_b200.workloads import cluster_instance

    plan, info = cluster_instance(1, dx=4.0, shell_nm=12.0, n_steps=800, n_min=40, n_max=128, single=False)
    box = info["box"]
    run = AdjointRun(plan, box, objective=info["objective"], checkpoint=128, precision="double")
    base = torch.as_tensor(np.asarray(plan["inv_eps"])[tuple(slice(a, b) for a, b in box)]).clone()
    run.set_inv_eps_box(base)
    J0, _ = run.forward(info["n_steps"])
    g = run.backward().cpu().numpy()
    assert J0 != 0 and np.abs(g[info["shell"]]).max() > 0
    gs = np.where(info["shell"], np.abs(g), 0)
    h = 1e-6
    for flat in np.argsort(-gs.reshape(-1))[:4]:
        idx = tuple(int(v) for v in np.unravel_index(flat, g.shape))
        vals = []
        for sgn in (1, -1):
            x = base.clone()
            x[idx] += sgn * h
            run.set_inv_eps_box(x)
            vals.append(run.forward(info["n_steps"], keep=False)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-5 * abs(fd), (idx, fd, g[idx])
    run.close()


def test_cluster_scattering_gradient_matches_finite_differences():
    """The cluster workload as lightsmith poses it (its own set-up: the table-fed TF/SF plane wave, the flux
    boxes and the incident reference view of its scattering driver), reduced: 4 nm grid, 12 nm shell, 640
    steps, float64. J = sum_f C_sca(f) of the scattered-field box; dJ/d(1/eps) on the shell's largest entries
    (the three E components of a node together) against central differences of the CUDA forward."""
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from refsrc import add_to_path

    if not add_to_path():
        pytest.skip("lightsmith (the reference install, baseline/_ref) not available")
    from lightsmith_b200.adjoint import AdjointRun
    from lightsmith_b200.workloads import cluster_scattering

    n_steps = 640
    plan, info = cluster_scattering(1, dx=4.0, shell_nm=12.0, n_steps=n_steps, precision="double")
    box, shape = info["box"], tuple(int(v) for v in plan["shape"])
    run = AdjointRun(plan, box, objective=info["objective"], checkpoint=128, precision="double")
    info["ref"]["acc_ref"] = run.eng.monitors[2]["acc_e"]
    inv = np.asarray(plan["inv_eps"]).reshape((-1,) + shape)
    base = torch.as_tensor(inv[(slice(None),) + tuple(slice(a, b) for a, b in box)]).clone()
    if base.shape[0] == 1:
        base = base[0]
    run.set_inv_eps_box(base)
    J0, _ = run.forward(n_steps)
    g = run.backward().cpu().numpy()
    shell = info["shell"]
    assert J0 > 0 and np.abs(g[shell]).max() > 0
    assert np.all(np.isfinite(info["ref"]["spectrum"])) and info["ref"]["spectrum"].shape == (24,)
    gs = np.where(shell, np.abs(g), 0)
    h = 1e-6
    for flat in np.argsort(-gs.reshape(-1))[:4]:
        idx = tuple(int(v) for v in np.unravel_index(flat, g.shape))
        vals = []
        for sgn in (1, -1):
            x = base.clone()
            if x.dim() == 4:
                x[(slice(None),) + idx] += sgn * h
            else:
                x[idx] += sgn * h
            run.set_inv_eps_box(x)
            vals.append(run.forward(n_steps, keep=False)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-5 * abs(fd), (idx, fd, g[idx])
    run.close()


def _fd_check(run, base, g, n_steps, flats, h=1e-6, tol=1e-5):
    """Central differences of the CUDA forward at the box nodes ``flats`` (the three E components of a node
    together when ``base`` holds one value per component) against the adjoint's gradient ``g``."""
    for flat in flats:
        idx = tuple(int(v) for v in np.unravel_index(int(flat), g.shape))
        vals = []
        for sgn in (1, -1):
            x = base.clone()
            if x.dim() == 4:
                x[(slice(None),) + idx] += sgn * h
            else:
                x[idx] += sgn * h
            run.set_inv_eps_box(x)
            vals.append(run.forward(n_steps, keep=False)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[idx]) <= tol * abs(fd), (idx, fd, g[idx])
    run.set_inv_eps_box(base)


def _default_pose(material, r=14.0):
    """A sphere of ``material`` (radius r nm, in water) posed to lightsmith with its default options (mirror
    planes, conformal meshing), 4 nm cells, float64: (plan, post, box, r), the box the nodes within r + 6 nm of
    the centre that every E component steps."""
    import lightsmith as ls

    from lightsmith_b200.scattering import scattering_setup

    sim = ls.Simulation(particles=[ls.Particle(shape=ls.Sphere(radius_nm=r), material=material,
                                               position_nm=(0.0, 0.0, 0.0))],
                        medium_index=1.33, wavelengths={"start_nm": 450.0, "stop_nm": 650.0, "num": 4},
                        options={"fdtd": dict(spacing_nm=4.0, pml_cells=8, padding_nm=16.0, pml_gap_nm=8.0,
                                              run_time_fs=6.0, precision="double")})
    plan, post, lay = scattering_setup(sim)
    assert tuple(plan["mirror"]) == (-1, 1, 0)
    shape = tuple(int(v) for v in plan["shape"])
    pos = [np.asarray(lay.origin, float)[a] + 4.0 * np.arange(shape[a]) for a in range(3)]
    lo_node = [2, 1, 0]  # the first node every E component steps: 2 next to the antisymmetric plane
    box = tuple((max(lo_node[a], int(np.searchsorted(pos[a], -r - 6.0))),
                 int(np.searchsorted(pos[a], r + 6.0, side="right"))) for a in range(3))
    return plan, post, box, r


def _lightsmith():
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from refsrc import add_to_path

    if not add_to_path():
        pytest.skip("lightsmith (the reference install, baseline/_ref) not available")
    import lightsmith as ls

    return ls


def test_default_pose_of_a_metal_sphere_gradient_matches_finite_differences():
    """A Drude-Lorentz sphere posed to lightsmith with its defaults: mirror planes and conformal meshing, which
    next to a dispersive medium is the vertex-tensor mesh (its nodes' E from tensor slots with their own pole
    states and plain slots), beside the metal's D-form groups; float64, J = sum_f C_sca(f). The gradient over a
    box around the sphere, which holds tensor nodes, against central differences of the CUDA forward at its
    largest entries overall and on tensor nodes, and bitwise the same for two checkpoint intervals."""
    ls = _lightsmith()
    from problems import DRUDE_LORENTZ

    from lightsmith_b200.adjoint import AdjointRun
    from lightsmith_b200.scattering import cross_section_objective

    plan, post, box, r = _default_pose(ls.DrudeLorentz(**DRUDE_LORENTZ))
    tm = plan["tensor"]
    assert tm is not None and int(tm["n_nodes"]) > 0 and len(tm["t_pos"]) > 0 and len(tm["p_pos"]) > 0
    shape = tuple(int(v) for v in plan["shape"])
    node = np.asarray(tm["idx"]) % int(np.prod(shape))
    ijk = np.stack(np.unravel_index(node, shape), axis=1)
    inside = np.all((ijk >= [a for a, _ in box]) & (ijk < [b for _, b in box]), axis=1)
    assert inside.any()
    on_tensor = np.zeros(tuple(b - a for a, b in box), bool)
    on_tensor[tuple((ijk[inside] - [a for a, _ in box]).T)] = True
    stride = int(plan["stride"])
    n_steps = 10 * stride
    inv = np.asarray(plan["inv_eps"]).reshape((-1,) + shape)
    base = torch.as_tensor(inv[(slice(None),) + tuple(slice(a, b) for a, b in box)]).clone()
    if base.shape[0] == 1:
        base = base[0]
    grads = []
    for K in (stride, 5 * stride):
        ref: dict = {}
        run = AdjointRun(plan, box, objective=cross_section_objective(post, ref), checkpoint=K, precision="double")
        ref["acc_ref"] = run.eng.monitors[2]["acc_e"]
        run.set_inv_eps_box(base)
        J0, _ = run.forward(n_steps)
        g = run.backward().cpu().numpy()
        grads.append(g)
        if K == stride:
            assert J0 > 0 and np.all(np.isfinite(g)) and np.abs(g).max() > 0
            flats = list(np.argsort(-np.abs(g).reshape(-1))[:2])
            flats += list(np.argsort(-np.where(on_tensor, np.abs(g), -1).reshape(-1))[:3])
            _fd_check(run, base, g, n_steps, flats)
        run.close()
    assert np.array_equal(grads[0], grads[1])


def test_default_pose_of_a_metal_sphere_float32_gradient_against_float64():
    """The metal sphere's default pose (mirror planes, vertex-tensor mesh, D-form groups) on the float32
    kernels: C_sca within 1e-4 and the gradient within 1e-3 of the largest float64 entry (the agreement the
    adjoint is held to), both runs from the same plan."""
    ls = _lightsmith()
    from problems import DRUDE_LORENTZ

    from lightsmith_b200.adjoint import AdjointRun
    from lightsmith_b200.scattering import cross_section_objective

    plan, post, box, r = _default_pose(ls.DrudeLorentz(**DRUDE_LORENTZ))
    shape = tuple(int(v) for v in plan["shape"])
    stride = int(plan["stride"])
    n_steps = 10 * stride
    inv = np.asarray(plan["inv_eps"]).reshape((-1,) + shape)
    base = torch.as_tensor(inv[(slice(None),) + tuple(slice(a, b) for a, b in box)]).clone()
    if base.shape[0] == 1:
        base = base[0]
    out = {}
    for prec in ("double", "single"):
        ref: dict = {}
        run = AdjointRun(plan, box, objective=cross_section_objective(post, ref), checkpoint=2 * stride,
                         precision=prec)
        ref["acc_ref"] = run.eng.monitors[2]["acc_e"]
        run.set_inv_eps_box(base)
        J, _ = run.forward(n_steps)
        out[prec] = (J, run.backward().cpu().numpy())
        run.close()
    (J64, g64), (J32, g32) = out["double"], out["single"]
    assert abs(J32 - J64) <= 1e-4 * abs(J64)
    assert np.abs(g32 - g64).max() <= 1e-3 * np.abs(g64).max()


def test_default_scattering_pose_gradient_matches_finite_differences(monkeypatch):
    """A dielectric sphere posed to lightsmith with its defaults: mirror planes through the centre (symmetry
    "auto": an antisymmetric plane normal to x and a symmetric one normal to y for the x-polarised plane wave)
    and conformal meshing (the off-diagonal terms of its tensor smoothing), float64. J = sum_f C_sca(f) of the
    scattered-field box; dJ/d(1/eps) over a box around the sphere, its interface cells with off-diagonal rows
    among its nodes, against central differences of the CUDA forward at its largest entries and at the largest
    on the planes next to each mirror plane. Without the transposed off-diagonal rows the C-ABI refuses."""
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from refsrc import add_to_path

    if not add_to_path():
        pytest.skip("lightsmith (the reference install, baseline/_ref) not available")
    import lightsmith as ls

    from lightsmith_b200 import adjoint as A
    from lightsmith_b200.scattering import cross_section_objective

    plan, post, box, r = _default_pose(ls.ConstantIndex(n_real=2.0))
    assert len(plan["offdiag"]["e"]) > 0
    shape = tuple(int(v) for v in plan["shape"])
    rest = np.asarray(plan["offdiag"]["e"]) % int(np.prod(shape))
    ijk = np.stack(np.unravel_index(rest, shape), axis=1)
    assert np.any(np.all((ijk >= [a for a, _ in box]) & (ijk < [b for _, b in box]), axis=1))
    stride = int(plan["stride"])
    n_steps = 10 * stride
    ref: dict = {}
    J_of = cross_section_objective(post, ref)
    with monkeypatch.context() as m:  # no transposed rows: refused
        m.setattr(A, "transposed_offdiag", lambda od: tuple(np.zeros(k, dt) for k, dt in
                                                             ((0, np.int64), (1, np.int64), (0, np.int64),
                                                              (0, np.float64))))
        with pytest.raises(RuntimeError, match="off-diagonal"):
            A.AdjointRun(plan, box, objective=J_of, checkpoint=2 * stride, precision="double")
    run = A.AdjointRun(plan, box, objective=J_of, checkpoint=2 * stride, precision="double")
    ref["acc_ref"] = run.eng.monitors[2]["acc_e"]
    inv = np.asarray(plan["inv_eps"]).reshape((-1,) + shape)
    base = torch.as_tensor(inv[(slice(None),) + tuple(slice(a, b) for a, b in box)]).clone()
    run.set_inv_eps_box(base)
    J0, _ = run.forward(n_steps)
    g = run.backward().cpu().numpy()
    assert J0 > 0 and np.all(np.isfinite(g)) and np.abs(g).max() > 0
    flats = list(np.argsort(-np.abs(g).reshape(-1))[:3])
    for a in (0, 1):  # the largest entry on the box's face next to each mirror plane
        face = np.zeros(g.shape, bool)
        face[(slice(None),) * a + (0,)] = True
        flats.append(int(np.argmax(np.where(face, np.abs(g), -1).reshape(-1))))
    _fd_check(run, base, g, n_steps, flats)
    run.close()


def test_mixed_dispersive_group_gradient():
    """A mixed D-form group (lightsmith's subpixel interface cells of a Drude-Lorentz metal and a dielectric,
    both paths running) between the dipole and the design box, the flux spectrum as the objective: the float64
    gradient against torch autograd through the restatement, against central differences of the CUDA forward,
    and bitwise across two checkpoint intervals."""
    from adjoint_cases import mixed_case
    from lightsmith_b200.adjoint import AdjointRun
    from oracle.autograd import objective

    plan, n_steps, J_of = mixed_case()
    base = torch.as_tensor(np.asarray(plan["inv_eps"])[tuple(slice(a, b) for a, b in BOX)])
    x = base.clone().requires_grad_(True)
    J_ref = objective(plan, x, BOX, 0, 0, None, None, n_steps, J=J_of)
    (g_ref,) = torch.autograd.grad(J_ref, x)
    J_ref = float(J_ref.detach())
    grads = []
    for K in (plan["stride"], n_steps):
        run = AdjointRun(plan, BOX, objective=J_of, checkpoint=K, precision="double")
        run.set_inv_eps_box(base)
        J, _ = run.forward(n_steps)
        grads.append(run.backward().cpu().numpy())
        assert abs(J - J_ref) / abs(J_ref) < 1e-11
        if K == n_steps:
            g = grads[-1]
            h = 1e-6
            for flat in np.argsort(-np.abs(g).reshape(-1))[:3]:
                idx = tuple(int(v) for v in np.unravel_index(flat, g.shape))
                vals = []
                for sgn in (1, -1):
                    xp = base.clone()
                    xp[idx] += sgn * h
                    run.set_inv_eps_box(xp)
                    vals.append(run.forward(n_steps)[0])
                fd = (vals[0] - vals[1]) / (2 * h)
                assert abs(fd - g[idx]) <= 1e-5 * abs(fd), (idx, fd, g[idx])
        run.close()
    assert np.abs(g_ref.numpy()).max() > 0
    assert _rel(grads[0], g_ref.numpy()) < 1e-9
    assert np.array_equal(grads[0], grads[1])
