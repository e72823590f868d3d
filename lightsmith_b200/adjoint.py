"""Gradients of an FDTD objective by the discrete adjoint, behind ``torch.autograd``.

lightsmith's FDTD has no gradient (its inverse design runs through other solvers). This module adds one for
the FDTD path: for a run with real fields (periodic axes allowed, without a Bloch phase; mirror planes, as
lightsmith's scattering driver picks them by default) with dispersive groups, pure (staircase) or mixed
(subpixel interface cells), the conformal off-diagonal terms of its default dielectric meshing and the
vertex-tensor mesh of its default meshing next to a dispersive medium (a slab waveguide device, a metal
nanoparticle cluster, a 2D device with its periodic invariant axis, a dielectric or metal particle in a
mirrored run), a real objective J of one DFT monitor's accumulators (or several monitors'),
and its gradient with respect to 1/eps over a design box of non-dispersive nodes. J is either
|sum_p wE_p acc_e[f, p] + sum_q wH_q acc_h[f, q]|^2 at one frequency f, or any torch function of the
accumulators (a flux spectrum, say): its adjoint source G = 2 dJ/d(acc) comes from torch autograd on J.

``AdjointRun.forward`` runs the engine (the CUDA kernels: the fused pass where the run allows it, as a plain
solve would) for ``n_steps`` steps, sampling the monitors as lightsmith's chunks do, and keeps the state (E, H,
CPML psi of the current buffer parity) every ``checkpoint`` steps.
``AdjointRun.backward`` walks the segments in reverse: it restores a checkpoint, recomputes the segment's steps
while recording H of the box at every step (``lsfdtd_adjoint_record``), then applies the transposed steps
(``lsfdtd_adjoint_step``, ``csrc/adjoint.cuh``) from the segment's end to its start, accumulating
dJ/dcbE over the box. Sources only add field-independent terms, so they have no adjoint; the ones allowed
here (point dipoles, port modes, table-fed TF/SF) keep no state of their own, and their nodes must lie
outside the box (their coefficients are fixed, not functions of the design). A dispersive group's step (D, E
of the previous step and the poles' P; for a mixed group also each medium's harmonic-path E and the
arithmetic path's E) is linear too: its transpose (``k_adj_ade``) runs before the E update's, and its state
is part of each checkpoint. The off-diagonal terms (E += W H after the E update) are transposed by a gather
over the rows of W^T (``transposed_offdiag``); the gradient holds W fixed (it is the derivative with respect to
the diagonal 1/eps of the box, W's entries being separate coefficients). The vertex-tensor mesh's step runs
last in a forward step and is linear with fixed coefficients; its transpose (``k_adj_tm_*``) runs first in a
reverse step, on an adjoint state laid out as its forward state, with gathers over the inverse maps of
``tensor_adjoint_maps``; its forward state is part of each checkpoint.

``FDTDObjective.apply(inv_eps_box, run)`` is the ``torch.autograd.Function``: forward returns J, backward
dJ/d(1/eps) of the box (isotropic: the three E components of a node share its 1/eps, so the gradient is
cdx times the sum of the three components' dJ/dcbE).
"""

from __future__ import annotations

import ctypes as C
import functools

import numpy as np

from . import _abi
from .engine import Engine
from .plan import DipoleSource, ModeSource, TableSource


def _torch():
    import torch

    return torch


def transposed_offdiag(od: dict):
    """The conformal off-diagonal gather tables (``plan["offdiag"]``: row t adds sum_k w[t, k] H[h[t, k]] to
    E[e[t]]) transposed for the adjoint: (rows, ptr, e, w) with row r adding sum_{j in [ptr[r], ptr[r + 1])}
    w[j] Ebar[e[j]] to Hbar[rows[r]]. The rows are the distinct H nodes read with a nonzero weight, ascending;
    each row's entries run in ascending E index."""
    e = np.asarray(od["e"], np.int64)
    h = np.asarray(od["h"], np.int64)
    w = np.asarray(od["w"])
    ee, hh, ww = np.repeat(e, h.shape[1]), h.reshape(-1), w.reshape(-1)
    keep = ww != 0
    ee, hh, ww = ee[keep], hh[keep], ww[keep]
    order = np.lexsort((ee, hh))
    ee, hh, ww = ee[order], hh[order], ww[order]
    rows, start = np.unique(hh, return_index=True)
    return rows, np.append(start, len(hh)).astype(np.int64), ee, ww


def injection_map(targets, points):
    """(tgt, ptr, src): the distinct target nodes ``targets`` holds, ascending, and for target r the points
    src[ptr[r]:ptr[r + 1]] (from ``points``, in the same order as ``targets``) that sample it, ascending."""
    t, p = np.asarray(targets, np.int64), np.asarray(points, np.int64)
    order = np.lexsort((p, t))
    t, p = t[order], p[order]
    tgt, start = np.unique(t, return_index=True)
    return tgt.astype(np.int64), np.append(start, len(t)).astype(np.int64), p


def tensor_adjoint_maps(tm: dict):
    """The inverse maps of a vertex-tensor mesh (``plan["tensor"]``) for its transposed step: (vs_ptr, vs_idx)
    the tensor slots of each vertex, ascending; (nd_ptr, nd_src) for each node the entries that read its D,
    ascending among the 6 n_vert (vertex, axis, side) entries (node ``vn[e]``), the n_tslots tensor slots (node
    ``vn[t_g[t]]``) and the n_pslots plain slots (node ``p_node[p]``), in that order; and the scratch length,
    6 n_vert + 2 n_tslots + n_pslots."""
    def ints(key):
        a = tm.get(key)
        return np.zeros(0, np.int64) if a is None else np.asarray(a, np.int64)
    n_nodes, n_vert = int(tm["n_nodes"]), len(np.asarray(tm["normal"])) // 3
    vn, t_v, t_vc, t_g, p_node = ints("vn"), ints("t_v"), ints("t_vc"), ints("t_g"), ints("p_node")
    if len(vn) != 6 * n_vert or np.any(t_vc // 3 != t_v):
        raise ValueError("vertex-tensor tables: each slot's component must be one of its vertex's")
    vs_idx = np.argsort(t_v, kind="stable").astype(np.int64)
    vs_ptr = np.concatenate([[0], np.cumsum(np.bincount(t_v, minlength=n_vert))]).astype(np.int64)
    node_of = np.concatenate([vn, vn[t_g], p_node])
    nd_src = np.argsort(node_of, kind="stable").astype(np.int64)
    nd_ptr = np.concatenate([[0], np.cumsum(np.bincount(node_of, minlength=n_nodes))]).astype(np.int64)
    return vs_ptr, vs_idx, nd_ptr, nd_src, 6 * n_vert + 2 * len(t_v) + len(p_node)


class AdjointRun:
    """One run's forward and adjoint passes. ``box``: ((x0, x1), (y0, y1), (z0, z1)) node ranges of the design
    box; ``monitor``: the objective's monitor, or a list of monitors with the same frequencies, whose points
    the objective sees concatenated (in list order; the H points of those that record H); ``objective``: J(acc_e, acc_h) -> real torch scalar, with
    acc_e (n_freq, n_e) and acc_h (n_freq, n_h) or None the monitors' accumulators as complex128 tensors; or,
    when it is None, J = |A|^2 at frequency ``freq`` with ``wE``/``wH`` the complex weights of the E and H
    points (None: zero); ``checkpoint``: steps between saved states (a multiple of dft_stride).
    ``sources_in_box``: allow source nodes inside the box, whose injection then stays as the plan built it
    (the gradient there is that of the field update alone)."""

    def __init__(self, plan: dict, box, monitor=0, freq: int = 0, wE=None, wH=None, checkpoint: int = 256,
                 precision: str | None = None, device="cuda:0", objective=None, sources_in_box: bool = False):
        torch = _torch()
        if plan["complex"]:
            raise ValueError("the adjoint serves real fields (no Bloch phase)")
        for s in plan["sources"]:
            if not isinstance(s, (DipoleSource, ModeSource, TableSource)):
                raise ValueError(f"{type(s).__name__} keeps state of its own; the adjoint does not restore it")
        self.plan = plan
        self.eng = Engine.from_plan(plan, device=device, precision=precision)
        eng = self.eng
        self.dev = eng.dev
        self.stride = eng.stride
        self.K = max(self.stride, int(checkpoint) // self.stride * self.stride)
        self.box = tuple((int(a), int(b)) for a, b in box)
        self.box_sl = tuple(slice(a, b) for a, b in self.box)
        bshape = tuple(b - a for a, b in self.box)
        self.monitors = [int(monitor)] if np.ndim(monitor) == 0 else [int(k) for k in monitor]
        mons = [plan["monitors"][k] for k in self.monitors]
        self.monitor, self.freq = self.monitors[0], freq
        self.omegas = np.asarray(mons[0]["omega"], float)
        if any(not np.array_equal(np.asarray(m["omega"], float), self.omegas) for m in mons):
            raise ValueError("the objective's monitors must share their frequencies")
        nf = len(self.omegas)
        cd = torch.complex128
        h_mons = [m for m in mons if m["h_idx1"] is not None]
        self.has_h = bool(h_mons)  # the H points: those of the monitors that record H, in list order

        def cat(key, ms):
            return np.concatenate([np.asarray(m[key], np.int64) for m in ms])
        mon = {"e_idx": cat("e_idx", mons)}
        if self.has_h:
            mon["h_idx1"], mon["h_idx2"] = cat("h_idx1", h_mons), cat("h_idx2", h_mons)
        if objective is None:
            wE_t = torch.as_tensor(np.zeros(len(mon["e_idx"])) if wE is None else np.asarray(wE), dtype=cd,
                                   device=self.dev)
            wH_t = None
            if self.has_h:
                wH_t = torch.as_tensor(np.zeros(len(mon["h_idx1"])) if wH is None else np.asarray(wH), dtype=cd,
                                       device=self.dev)

            def objective(acc_e, acc_h, f=freq, wE_t=wE_t, wH_t=wH_t):
                A = (wE_t * acc_e[f]).sum()
                if wH_t is not None:
                    A = A + (wH_t * acc_h[f]).sum()
                return (A * A.conj()).real

        self.objective = objective
        for s in plan["sources"]:
            nodes = s.idx if isinstance(s, DipoleSource) else (np.concatenate([s.h_idx, s.e_idx]) if isinstance(
                s, ModeSource) else np.concatenate([s.E.node, s.H.node]))
            rest = np.asarray(nodes) % int(np.prod(eng.shape))
            ijk = np.stack(np.unravel_index(rest, eng.shape), axis=1)
            inside = np.all((ijk >= [a for a, _ in self.box]) & (ijk < [b for _, b in self.box]), axis=1)
            if inside.any() and not sources_in_box:
                raise ValueError("a source node lies in the design box")
        rdt = eng.rdt
        self.group_bar = [torch.zeros_like(g["state"]) for g in eng.groups]
        self.Eb = torch.zeros_like(eng.E)
        self.Hb = torch.zeros_like(eng.H)
        self.psi_bar = [[{}, {}], [{}, {}]]  # [buffer][E, H]: {(c, d, side): tensor}
        d = _abi.AdjointDesc()
        d.Eb, d.Hb = self.Eb.data_ptr(), self.Hb.data_ptr()
        for (kind, comp, ax, side), t in eng.psi.items():
            f = 0 if kind == "E" else 1
            for b in range(2):
                z = torch.zeros_like(t)
                self.psi_bar[b][f][(comp, ax, side)] = z
                d.psi_bar[(((b * 2 + f) * 3 + ax) * 3 + comp) * 2 + side] = z.data_ptr()
        d.box_lo[:] = [a for a, _ in self.box]
        d.box_hi[:] = [b for _, b in self.box]
        self.hist = torch.zeros((self.K, 3) + tuple(n + 1 for n in bshape), dtype=rdt, device=self.dev)
        d.hist, d.hist_slots = self.hist.data_ptr(), self.K
        self.grad = torch.zeros((3,) + bshape, dtype=torch.float64, device=self.dev)
        d.grad = self.grad.data_ptr()
        i64 = torch.int64
        self.e_idx = torch.as_tensor(mon["e_idx"], dtype=i64, device=self.dev)
        self.ge = torch.zeros((nf, len(mon["e_idx"]), 2), dtype=torch.float64, device=self.dev)
        d.e_idx, d.ge, d.n_e = self.e_idx.data_ptr(), self.ge.data_ptr(), len(mon["e_idx"])
        if self.has_h:
            self.h1 = torch.as_tensor(mon["h_idx1"], dtype=i64, device=self.dev)
            self.h2 = torch.as_tensor(mon["h_idx2"], dtype=i64, device=self.dev)
            self.gh = torch.zeros((nf, len(mon["h_idx1"]), 2), dtype=torch.float64, device=self.dev)
            d.h_idx1, d.h_idx2, d.gh, d.n_h = self.h1.data_ptr(), self.h2.data_ptr(), self.gh.data_ptr(), len(
                mon["h_idx1"])
        # the adjoint source gathered per target node in a fixed order (flux boxes share nodes between points)
        e_t, e_p, e_s = injection_map(mon["e_idx"], np.arange(len(mon["e_idx"])))
        self._inj = [torch.as_tensor(a, dtype=i64, device=self.dev) for a in (e_t, e_p, e_s)]
        d.inj_e_tgt, d.inj_e_ptr, d.inj_e_src = (t.data_ptr() for t in self._inj)
        d.inj_n_e = len(e_t)
        if self.has_h:
            nh = len(mon["h_idx1"])
            h_t, h_p, h_s = injection_map(np.concatenate([mon["h_idx1"], mon["h_idx2"]]),
                                          np.concatenate([np.arange(nh), np.arange(nh)]))
            self._inj += [torch.as_tensor(a, dtype=i64, device=self.dev) for a in (h_t, h_p, h_s)]
            d.inj_h_tgt, d.inj_h_ptr, d.inj_h_src = (t.data_ptr() for t in self._inj[3:])
            d.inj_n_h = len(h_t)
        self._inj.append(torch.zeros(max(len(mon["e_idx"]) + (len(mon["h_idx1"]) if self.has_h else 0), 1),
                                     dtype=torch.float64, device=self.dev))
        d.inj_work = self._inj[-1].data_ptr()
        om = (C.c_double * nf)(*self.omegas.tolist())
        d.omega = C.cast(om, C.c_void_p)
        d.n_freq = nf
        if len(self.group_bar) > 8:
            raise ValueError("the adjoint serves at most 8 dispersive groups")
        d.n_groups = len(self.group_bar)
        for gi, t in enumerate(self.group_bar):
            d.group_bar[gi] = t.data_ptr()
        od = plan.get("offdiag")
        if od is not None and len(od["e"]):  # the conformal off-diagonal terms, transposed
            rows, ptr, e, w = transposed_offdiag(od)
            self._od = [torch.as_tensor(rows, device=self.dev), torch.as_tensor(ptr, device=self.dev),
                        torch.as_tensor(e, device=self.dev), torch.as_tensor(w, dtype=eng.fdt, device=self.dev)]
            d.od_h, d.od_ptr, d.od_e, d.od_w = (t.data_ptr() for t in self._od)
            d.od_rows = len(rows)
        self._tm_bar = []
        tm = plan.get("tensor")
        if tm is not None and int(tm["n_nodes"]) > 0:  # the vertex-tensor mesh: adjoint state, scratch and maps
            vs_ptr, vs_idx, nd_ptr, nd_src, n_work = tensor_adjoint_maps(tm)
            self._tm_bar = [torch.zeros_like(eng.tensor["state"])]
            self._tm = [torch.zeros(max(n_work, 1), dtype=eng.fdt, device=self.dev)] + [
                torch.as_tensor(a, device=self.dev) for a in (vs_ptr, vs_idx, nd_ptr, nd_src)]
            d.tm_bar = self._tm_bar[0].data_ptr()
            d.tm_work, d.tm_vs_ptr, d.tm_vs_idx, d.tm_nd_ptr, d.tm_nd_src = (t.data_ptr() for t in self._tm)
        self._desc = d
        h = C.c_void_p()
        _abi.check(_abi.lib().lsfdtd_adjoint_create(eng._h, C.byref(d), C.byref(h)), "lsfdtd_adjoint_create")
        self._h = h
        self.acc = None
        self.n_steps = 0
        self._ckpt = []

    # --- state ----------------------------------------------------------------------------------------------
    def _state(self):
        return self.eng.state()

    def _save(self):
        return [t.clone() for t in self._state()]

    def _restore(self, saved, n: int):
        eng = self.eng
        for dst, src in zip(self._state(), saved):
            dst.copy_(src)
        eng.n.fill_(n)
        _abi.check(_abi.lib().lsfdtd_engine_set_steps(eng._h, int(n)), "lsfdtd_engine_set_steps")
        _torch().cuda.synchronize(self.dev)  # the engine's stream starts from the restored state

    def _reset(self):
        for t in self.eng.all_state():
            t.zero_()
        for m in self.eng.monitors:
            m["acc_e"].zero_()
            if m["acc_h"] is not None:
                m["acc_h"].zero_()
        self._restore(self._save(), 0)

    def set_inv_eps_box(self, inv_eps_box) -> None:
        """1/eps over the box, one value per node (x, y, z) or one per E component (3, x, y, z); the E curl
        coefficient of each component there becomes cdx / eps."""
        eng = self.eng
        torch = _torch()
        v = torch.as_tensor(inv_eps_box, device=self.dev, dtype=torch.float64) * eng.cdx
        shared = eng.cbE[0] is eng.cbE[1] and eng.cbE[1] is eng.cbE[2]
        if v.dim() == 3:
            v = v.expand(3, *v.shape)
        elif shared and not (torch.equal(v[0], v[1]) and torch.equal(v[0], v[2])):
            raise ValueError("this engine shares one 1/eps array between the E components; give one value per node")
        for c in range(1 if shared else 3):
            cb = eng.cbE[c]
            cb[self.box_sl] = v[c].to(cb.dtype)
        torch.cuda.synchronize(self.dev)

    # --- passes -----------------------------------------------------------------------------------------------
    def forward(self, n_steps: int, keep: bool = True):
        """Runs n_steps steps from rest (a multiple of dft_stride); returns (J, A). ``keep=False`` saves no
        checkpoints (J alone, e.g. for a line search); ``backward`` then needs another forward first."""
        torch = _torch()
        eng = self.eng
        if n_steps % self.stride:
            raise ValueError("n_steps must be a multiple of dft_stride")
        self._reset()
        self._ckpt = [self._save()]
        done = 0
        while done < n_steps:  # chunks (dft_stride steps and a sample) replayed as CUDA graphs
            seg = min(self.K, n_steps - done)
            eng.chunk(seg // self.stride, use_graph=True)
            done += seg
            if done < n_steps and keep:
                self._ckpt.append(self._save())
        self.n_steps = n_steps if keep else 0
        ms = [eng.monitors[k] for k in self.monitors]
        torch.cuda.synchronize(self.dev)
        acc_e = torch.cat([m["acc_e"].to(torch.complex128) for m in ms], dim=1)
        acc_h = (torch.cat([m["acc_h"].to(torch.complex128) for m in ms if m["acc_h"] is not None], dim=1)
                 if self.has_h else None)
        self.acc = (acc_e, acc_h)
        with torch.no_grad():
            J = self.objective(acc_e, acc_h)
        return float(J), (acc_e, acc_h)

    def backward(self, per_component: bool = False):
        """dJ/d(1/eps) over the box after forward(), as float64: (x, y, z) for a 1/eps shared by the node's
        three E components, or per component (3, x, y, z)."""
        if not self.n_steps:
            raise RuntimeError("backward needs a forward run that kept its checkpoints")
        torch = _torch()
        eng = self.eng
        L = _abi.lib()
        # the adjoint source: G = 2 dJ/d(acc) = conj of the gradient torch gives for a complex tensor
        acc_e = self.acc[0].detach().clone().requires_grad_(True)
        acc_h = self.acc[1].detach().clone().requires_grad_(True) if self.has_h else None
        with torch.enable_grad():
            J = self.objective(acc_e, acc_h)
            grads = torch.autograd.grad(J, [acc_e] + ([acc_h] if acc_h is not None else []), allow_unused=True)
        g_e = grads[0] if grads[0] is not None else torch.zeros_like(acc_e)
        self.ge.copy_(torch.view_as_real(g_e.conj().resolve_conj()))
        if self.has_h:
            g_h = grads[1] if grads[1] is not None else torch.zeros_like(acc_h)
            self.gh.copy_(torch.view_as_real(g_h.conj().resolve_conj()))
        self.Eb.zero_()
        self.Hb.zero_()
        for t in self.group_bar + self._tm_bar:
            t.zero_()
        for b in range(2):
            for f in range(2):
                for t in self.psi_bar[b][f].values():
                    t.zero_()
        self.grad.zero_()
        torch.cuda.synchronize(self.dev)
        h, he = self._h, eng._h
        st = eng.stream.cuda_stream  # every launch below on the engine's stream, in order
        for k in reversed(range(len(self._ckpt))):
            n0 = k * self.K
            n1 = min(n0 + self.K, self.n_steps)
            self._restore(self._ckpt[k], n0)
            for i in range(n1 - n0):
                _abi.check(L.lsfdtd_engine_step(he, 1, st), "lsfdtd_engine_step")
                _abi.check(L.lsfdtd_adjoint_record(h, i, st), "lsfdtd_adjoint_record")
            for i in reversed(range(n1 - n0)):
                _abi.check(L.lsfdtd_adjoint_step(h, n0 + i, i, st), "lsfdtd_adjoint_step")
            torch.cuda.synchronize(self.dev)
        return self.grad * eng.cdx if per_component else self.grad.sum(0) * eng.cdx

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _abi.lib().lsfdtd_adjoint_destroy(h)
            self._h = C.c_void_p()
        self.eng.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 (interpreter shutdown)
            pass


@functools.cache
def _function():
    torch = _torch()

    class FDTDObjective(torch.autograd.Function):
        """J(1/eps of the design box) of an ``AdjointRun``, differentiable by the discrete adjoint."""

        @staticmethod
        def forward(ctx, inv_eps_box, run: AdjointRun, n_steps: int):
            run.set_inv_eps_box(inv_eps_box.detach())
            J, _ = run.forward(n_steps)
            ctx.run = run
            return torch.tensor(J, dtype=torch.float64, device=inv_eps_box.device)

        @staticmethod
        def backward(ctx, gJ):
            g = ctx.run.backward().to(gJ.device)
            return gJ * g, None, None

    return FDTDObjective


def fdtd_objective(inv_eps_box, run: AdjointRun, n_steps: int):
    """J as a differentiable function of 1/eps over the design box."""
    return _function().apply(inv_eps_box, run, n_steps)
