"""The plain-PyTorch restatement used to check the adjoint (oracle/autograd.py) against the NumPy oracle:
the same objective from the same run, and gradients that agree with central finite differences of itself."""

import numpy as np
import pytest
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



def test_transposed_offdiag_rows_are_the_gather_transposed():
    """``transposed_offdiag`` against the forward gather it transposes, on a random table shaped as the plan's
    (distinct targets, padded rows with zero weights, H nodes shared between rows): <Ebar, W H> = <W^T Ebar, H>
    to rounding, distinct ascending rows, and no zero weight kept."""
    from lightsmith_b200.adjoint import transposed_offdiag

    rng = np.random.default_rng(7)
    n_flat, n_rows, width = 600, 80, 6
    e = rng.choice(n_flat, n_rows, replace=False)
    h = np.stack([rng.choice(n_flat // 4, width, replace=False) for _ in range(n_rows)])
    w = rng.normal(size=(n_rows, width))
    w[rng.random(size=w.shape) < 0.3] = 0.0
    H, Eb = rng.normal(size=n_flat), rng.normal(size=n_flat)
    WH = np.zeros(n_flat)
    WH[e] = (w * H[h]).sum(axis=1)
    rows, ptr, ee, ww = transposed_offdiag({"e": e, "h": h, "w": w})
    assert np.all(np.diff(rows) > 0) and ptr[0] == 0 and ptr[-1] == len(ee) == np.count_nonzero(w)
    assert np.all(ww != 0)
    WtE = np.zeros(n_flat)
    for r, q in enumerate(rows):
        WtE[q] = sum(ww[j] * Eb[ee[j]] for j in range(ptr[r], ptr[r + 1]))
    assert abs(Eb @ WH - WtE @ H) <= 1e-12 * np.abs(Eb).sum() * np.abs(WH).max()


def test_tensor_adjoint_maps_list_every_entry_once_under_its_node():
    """``tensor_adjoint_maps`` on a random table shaped as a vertex-tensor mesh's: every (vertex, axis, side)
    entry, tensor slot and plain slot appears once, under the node whose D it reads, in ascending order; every
    tensor slot once under its vertex; the scratch length is 6 n_vert + 2 n_tslots + n_pslots."""
    from lightsmith_b200.adjoint import tensor_adjoint_maps

    rng = np.random.default_rng(3)
    n_nodes, n_vert, n_t, n_p = 40, 9, 25, 12
    vn = rng.integers(0, n_nodes, 6 * n_vert)
    t_v = rng.integers(0, n_vert, n_t)
    t_vc = 3 * t_v + rng.integers(0, 3, n_t)
    t_g = rng.integers(0, 6 * n_vert, n_t)
    p_node = rng.integers(0, n_nodes, n_p)
    tm = {"n_nodes": n_nodes, "normal": np.zeros(3 * n_vert), "vn": vn, "t_v": t_v, "t_vc": t_vc, "t_g": t_g,
          "p_node": p_node}
    vs_ptr, vs_idx, nd_ptr, nd_src, n_work = tensor_adjoint_maps(tm)
    assert n_work == 6 * n_vert + 2 * n_t + n_p
    node_of = np.concatenate([vn, vn[t_g], p_node])
    assert sorted(nd_src.tolist()) == list(range(len(node_of)))
    for i in range(n_nodes):
        src = nd_src[nd_ptr[i]:nd_ptr[i + 1]]
        assert np.all(node_of[src] == i) and np.all(np.diff(src) > 0)
    assert sorted(vs_idx.tolist()) == list(range(n_t))
    for v in range(n_vert):
        sl = vs_idx[vs_ptr[v]:vs_ptr[v + 1]]
        assert np.all(t_v[sl] == v) and np.all(np.diff(sl) > 0)
    tm["t_vc"] = t_vc + 3  # a slot on another vertex's component: refused
    with pytest.raises(ValueError):
        tensor_adjoint_maps(tm)


def test_injection_map_groups_points_by_target_in_order():
    """``injection_map``: each distinct target once, ascending, with the points that sample it in ascending
    order; every point listed as often as it appears."""
    from lightsmith_b200.adjoint import injection_map

    targets = np.array([7, 3, 7, 9, 3, 7, 1])
    points = np.array([0, 1, 2, 3, 4, 5, 6])
    tgt, ptr, src = injection_map(targets, points)
    assert tgt.tolist() == [1, 3, 7, 9] and ptr.tolist() == [0, 1, 3, 6, 7]
    assert src.tolist() == [6, 1, 4, 0, 2, 5, 3]
    nh = 4  # H points: both samples of a point may share a target
    h1, h2 = np.array([5, 6, 5, 8]), np.array([6, 6, 9, 5])
    tgt, ptr, src = injection_map(np.concatenate([h1, h2]), np.concatenate([np.arange(nh), np.arange(nh)]))
    assert tgt.tolist() == [5, 6, 8, 9] and src[ptr[1]:ptr[2]].tolist() == [0, 1, 1]
