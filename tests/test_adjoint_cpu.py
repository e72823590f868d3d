"""The plain-PyTorch restatement used to check the adjoint (oracle/autograd.py) against the NumPy oracle:
the same objective from the same run, and gradients that agree with central finite differences of itself."""

import numpy as np
import torch

from adjoint_cases import BOX, small_case


def _oracle_J(plan, n_steps, wE, wH):
    from oracle.engine import OracleEngine

    eng = OracleEngine(plan)
    for _ in range(n_steps // plan["stride"]):
        eng.chunk()
    m = eng.monitors[0]
    A = (wE * m["acc_e"][0]).sum() + (wH * m["acc_h"][0]).sum()
    return abs(A) ** 2


def test_autograd_restatement_matches_oracle():
    from oracle.autograd import objective

    plan, n_steps, wE, wH = small_case()
    box_vals = torch.as_tensor(np.asarray(plan["inv_eps"])[tuple(slice(a, b) for a, b in BOX)])
    J = float(objective(plan, box_vals, BOX, 0, 0, wE, wH, n_steps))
    J0 = _oracle_J(plan, n_steps, wE, wH)
    assert J0 > 0
    assert abs(J - J0) / J0 < 1e-12


def test_autograd_gradient_matches_finite_differences():
    from oracle.autograd import objective

    plan, n_steps, wE, wH = small_case(n_chunks=2)
    base = torch.as_tensor(np.asarray(plan["inv_eps"])[tuple(slice(a, b) for a, b in BOX)]).clone()
    x = base.clone().requires_grad_(True)
    J = objective(plan, x, BOX, 0, 0, wE, wH, n_steps)
    (g,) = torch.autograd.grad(J, x)
    assert float(g.abs().max()) > 0
    h = 1e-6
    for flat in torch.argsort(g.abs().reshape(-1), descending=True)[:3].tolist():  # the largest entries
        idx = tuple(int(v) for v in np.unravel_index(flat, g.shape))
        xp, xm = base.clone(), base.clone()
        xp[idx] += h
        xm[idx] -= h
        fd = (float(objective(plan, xp, BOX, 0, 0, wE, wH, n_steps)) -
              float(objective(plan, xm, BOX, 0, 0, wE, wH, n_steps))) / (2 * h)
        assert abs(fd - float(g[idx])) <= 1e-5 * abs(fd), (idx, fd, float(g[idx]))


def test_autograd_restatement_with_a_dispersive_group_matches_oracle():
    """The restatement's pure D-form group and multi-frequency flux objective against the oracle's run."""
    from adjoint_cases import dispersive_case
    from oracle.autograd import objective
    from oracle.engine import OracleEngine

    plan, n_steps, J_of = dispersive_case()
    box_vals = torch.as_tensor(np.asarray(plan["inv_eps"])[tuple(slice(a, b) for a, b in BOX)])
    J = float(objective(plan, box_vals, BOX, 0, 0, None, None, n_steps, J=J_of))
    eng = OracleEngine(plan)
    for _ in range(n_steps // plan["stride"]):
        eng.chunk()
    m = eng.monitors[0]
    J0 = float(J_of(torch.as_tensor(m["acc_e"]), torch.as_tensor(m["acc_h"])))
    assert abs(J0) > 0
    assert abs(J - J0) / abs(J0) < 1e-12


def test_autograd_restatement_with_a_mixed_group_matches_oracle():
    """The restatement's mixed D-form group (harmonic and arithmetic paths, lightsmith's subpixel interface
    cells) against the oracle's run of the same plan."""
    from adjoint_cases import mixed_case
    from oracle.autograd import objective
    from oracle.engine import OracleEngine

    plan, n_steps, J_of = mixed_case()
    box_vals = torch.as_tensor(np.asarray(plan["inv_eps"])[tuple(slice(a, b) for a, b in BOX)])
    J = float(objective(plan, box_vals, BOX, 0, 0, None, None, n_steps, J=J_of))
    eng = OracleEngine(plan)
    for _ in range(n_steps // plan["stride"]):
        eng.chunk()
    m = eng.monitors[0]
    J0 = float(J_of(torch.as_tensor(m["acc_e"]), torch.as_tensor(m["acc_h"])))
    assert abs(J0) > 0
    assert abs(J - J0) / abs(J0) < 1e-12

