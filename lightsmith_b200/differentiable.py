"""S-parameters of a device problem as a torch function of its permittivity grid, with exact gradients by the
discrete adjoint: the solve behind lightsmith's differentiable-backend protocol (inverse/__init__.py:14-43) on
the FDTD path.

lightsmith's inverse design asks a backend for ``design_grid``, ``base_permittivity`` and
``differentiable_solve`` (the FDFD backend is its one implementation, backends/fdfd.py:134-160); lightsmith's
FDTD sets ``differentiable = False``. Here the device driver's runs (backends/_fdtd/device.py:475-561: one run
per port mode, a mode source and one DFT monitor per port) are handed over as a plain description that
``lightsmith_b200.backend.device_runs`` builds with lightsmith's own set-up (voxelisation, mode tables, time
step); this module needs no lightsmith, so the GPU tests replay a recorded description.

The permittivity grid is the FDTD grid's nodes: node (i, j, k) carries one real permittivity for its three E
components (E_x at i + 1/2, E_y at j + 1/2, E_z at k + 1/2); a 2D device's grid is its one stepped z plane
(node k = 1 between the two ghost planes of the periodic invariant axis). Where the grid given equals the
base (the driver's own voxelisation, 1/eps averaged over the three components), a node keeps the driver's
per-component values; elsewhere its three components take 1/eps of the grid. FDTD steps a real,
frequency-independent permittivity: an override must be real and equal across wavelengths.

Each S column is one ``AdjointRun`` (``lightsmith_b200.adjoint``) over all port monitors: the forward runs the
CUDA engine for the description's fixed step count, keeping checkpoints; S[:, out, src] = c_out / a_src from the
port amplitudes (ports.py:265-280, device.py:553-561), which are linear functionals of the monitors' DFT
accumulators. The backward gives each run the adjoint source of Re sum conj(dL/dS) S (the same first-order
change as L) and returns dL/deps = -(1/eps^2) sum_c dL/d(1/eps_c) over the interior box (the nodes outside
every CPML slab); an override that differs from the base outside that box is rejected. The gradient is exact
for the fixed step count, with the ports' sources and mode tables built from the base permittivity (the
protocol requires that the ports do not depend on the override).
"""

from __future__ import annotations

import functools
from dataclasses import dataclass

import numpy as np

from .adjoint import AdjointRun


def _torch():
    import torch

    return torch


@dataclass
class DesignGrid:
    """The grid of ``design_grid`` of a 3D device: node coordinates (nm) along each axis, cell size, shape."""

    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    dl: float
    shape: tuple


@dataclass
class DesignGrid2D:
    """The grid of ``design_grid`` of a 2D device (lightsmith's inverse design tells 2D from 3D by ``z``)."""

    x: np.ndarray
    y: np.ndarray
    dl: float
    shape: tuple


def interior_box(shape, pml_cells):
    """Node ranges outside every E CPML slab (plan.cpml_terms: the low slab ends at node lo + 1, the high one
    starts at n - 2 - hi) and off the grid's outer nodes."""
    box = []
    for n, (lo, hi) in zip(shape, pml_cells):
        a = lo + 1 if lo else 1
        b = n - 2 - hi if hi else n - 1
        if b <= a:
            raise ValueError("the grid has no nodes outside its CPML slabs")
        box.append((int(a), int(b)))
    return tuple(box)


class DeviceSolver:
    """The runs of one device description (``backend.device_runs``), kept across evaluations: one
    ``AdjointRun`` per excited port mode, created on first use."""

    def __init__(self, desc: dict, device="cuda:0", precision: str | None = None, checkpoint: int = 256):
        self.desc = desc
        self.device, self.precision, self.checkpoint = device, precision, int(checkpoint)
        self.shape = tuple(int(v) for v in desc["shape"])
        self.two_d = bool(desc.get("two_d", False))
        self.design_shape = self.shape[:2] if self.two_d else self.shape
        self.inv_eps = np.asarray(desc["inv_eps"], float).reshape((3,) + self.shape)
        self.base_nodes = 1.0 / self.inv_eps.mean(axis=0)
        self.base_design = self.base_nodes[:, :, 1] if self.two_d else self.base_nodes
        self.box = interior_box(self.shape, desc["pml_cells"])
        self.box_sl = tuple(slice(a, b) for a, b in self.box)
        self.labels = list(desc["labels"])
        self.n_steps = int(desc["n_steps"])
        self.omega = np.asarray(desc["omega"], float)
        self._runs: dict[tuple, AdjointRun] = {}  # (label, with the field monitor)
        self._gen: dict[tuple, int] = {}
        self._amp = None

    # --- the port amplitudes -------------------------------------------------------------------------------
    def _coefficients(self, dev):
        """Per output row: (offset of its monitor's E points, of its H points, in_E, in_H, out_E, out_H) as
        complex128 tensors (n_w, points)."""
        if self._amp is None:
            torch = _torch()
            rows = []
            for r in self.desc["rows"]:
                t = [torch.as_tensor(np.asarray(r[k]), dtype=torch.complex128, device=dev)
                     for k in ("in_e", "in_h", "out_e", "out_h")]
                rows.append((int(r["e_off"]), int(r["h_off"]), *t))
            self._amp = rows
        return self._amp

    def amplitudes(self, acc_e, acc_h):
        """(incoming, outgoing) amplitudes of every port mode, (n_w, n_out) each, from the concatenated
        accumulators of the port monitors."""
        torch = _torch()
        a_in, a_out = [], []
        for e0, h0, ie, ih, oe, oh in self._coefficients(acc_e.device):
            E = acc_e[:, e0:e0 + ie.shape[1]]
            H = acc_h[:, h0:h0 + ih.shape[1]]
            a_in.append((ie * E).sum(1) + (ih * H).sum(1))
            a_out.append((oe * E).sum(1) + (oh * H).sum(1))
        return torch.stack(a_in, 1), torch.stack(a_out, 1)

    def s_column(self, label, acc_e, acc_h):
        a_in, a_out = self.amplitudes(acc_e, acc_h)
        row = self.labels.index(label)
        return a_out / a_in[:, row:row + 1]

    # --- the field outputs ---------------------------------------------------------------------------------
    def field_monitor(self) -> dict:
        """A DFT monitor of the field lightsmith's field objectives read (inverse/objectives.py:53-68): E_x,
        E_y, E_z at every node of a 3D grid; H_z (TE) or E_z (TM) at every node of a 2D device's plane k = 1
        (a TE monitor also records that plane's E_z, which is not read)."""
        n0, n1, n2 = self.shape
        cells = n0 * n1 * n2
        if not self.two_d:
            e = np.arange(3 * cells, dtype=np.int64)
            h = None
        else:
            i, j = np.meshgrid(np.arange(n0), np.arange(n1), indexing="ij")
            plane = 2 * cells + (i.ravel() * n1 + j.ravel()) * n2 + 1
            e = plane.astype(np.int64)
            h = e.copy() if self.desc.get("polarization", "te") == "te" else None
        return {"omega": self.omega, "e_idx": e, "h_idx1": h, "h_idx2": None if h is None else h.copy(),
                "energy": 0, "space": ("grid", -1)}

    def field_shape(self):
        return (3,) + self.shape if not self.two_d else self.design_shape

    def field_column(self, label, acc_e, acc_h):
        """(n_w, *field_shape) of the run of ``label`` per unit incident amplitude of its port mode."""
        a_in, _ = self.amplitudes(acc_e, acc_h)
        row = self.labels.index(label)
        ne = sum(len(m["e_idx"]) for m in self.desc["plans"][0]["monitors"])
        nh = sum(len(m["h_idx1"]) for m in self.desc["plans"][0]["monitors"] if m["h_idx1"] is not None)
        tm = self.desc.get("polarization", "te") == "tm"
        f = acc_e[:, ne:] if (not self.two_d or tm) else acc_h[:, nh:]
        f = f.reshape((f.shape[0],) + tuple(self.field_shape()))
        return f / a_in[:, row].reshape((-1,) + (1,) * (f.dim() - 1))

    # --- runs ----------------------------------------------------------------------------------------------
    def run(self, label: str, fields: bool = False) -> AdjointRun:
        key = (label, bool(fields))
        if key not in self._runs:
            k = self.labels.index(label)
            plan = dict(self.desc["plans"][k])
            plan["inv_eps"] = self.inv_eps
            if fields:
                plan["monitors"] = list(plan["monitors"]) + [self.field_monitor()]
            mons = list(range(len(plan["monitors"])))
            self._runs[key] = AdjointRun(plan, self.box, monitor=mons, checkpoint=self.checkpoint,
                                         precision=self.precision, device=self.device,
                                         objective=lambda e, h: e.real.sum() * 0, sources_in_box=True)
            self._gen[key] = 0
        return self._runs[key]

    def nodes(self, eps_design: np.ndarray) -> np.ndarray:
        """The node permittivity of the whole grid for a design-grid one (a 2D device's plane k = 1)."""
        eps_design = np.asarray(eps_design, float)
        if eps_design.shape != self.design_shape:
            raise ValueError(f"the permittivity grid must have the design grid's shape {self.design_shape}")
        if not self.two_d:
            return eps_design
        out = self.base_nodes.copy()
        out[:, :, 1] = eps_design
        return out

    def inv_eps_box(self, eps_design: np.ndarray) -> np.ndarray:
        """(3, box) 1/eps of each E component over the box for a design-grid permittivity."""
        eps_nodes = self.nodes(eps_design)
        changed = ~np.isclose(eps_nodes, self.base_nodes, rtol=1e-12, atol=0)
        inside = np.zeros(self.shape, bool)
        inside[self.box_sl] = True
        if np.any(changed & ~inside):
            raise ValueError("the permittivity grid differs from the problem's outside the interior box "
                             f"{self.box} (CPML slabs and outer nodes keep the problem's permittivity)")
        if np.any(eps_nodes[changed] <= 0):
            raise ValueError("the permittivity must be positive")
        inv = self.inv_eps[(slice(None),) + self.box_sl].copy()
        ch = changed[self.box_sl]
        inv[:, ch] = 1.0 / eps_nodes[self.box_sl][ch]
        return inv

    def forward(self, label: str, eps_nodes: np.ndarray, fields: bool = False):
        """Runs one column's forward pass; returns its accumulators (acc_e, acc_h), complex128 on the GPU."""
        run = self.run(label, fields)
        run.set_inv_eps_box(self.inv_eps_box(eps_nodes))
        _, acc = run.forward(self.n_steps)
        self._gen[(label, bool(fields))] += 1
        return acc

    def close(self):
        for r in self._runs.values():
            r.close()
        self._runs.clear()


@functools.cache
def _function():
    torch = _torch()

    class DeviceSParameters(torch.autograd.Function):
        """(S (n_w, n_out, n_src), fields (n_w, n_src, *field_shape) or an empty tensor) of a
        ``DeviceSolver`` as functions of the design-grid permittivity."""

        @staticmethod
        def forward(ctx, eps_nodes, solver: DeviceSolver, sources, fields: bool):
            eps_np = eps_nodes.detach().cpu().numpy().astype(float)
            cols, fcols, gens = [], [], []
            for lab in sources:
                acc_e, acc_h = solver.forward(lab, eps_np, fields)
                cols.append(solver.s_column(lab, acc_e, acc_h))
                if fields:
                    fcols.append(solver.field_column(lab, acc_e, acc_h))
                gens.append(solver._gen[(lab, fields)])
            ctx.solver, ctx.sources, ctx.gens, ctx.fields = solver, list(sources), gens, fields
            ctx.eps_np = eps_np
            ctx.save_for_backward(eps_nodes)
            S = torch.stack(cols, 2).to(eps_nodes.device)
            F = torch.stack(fcols, 1).to(eps_nodes.device) if fields else S.new_zeros(0)
            if not fields:
                ctx.mark_non_differentiable(F)
            return S, F

        @staticmethod
        def backward(ctx, gS, gF):
            (eps_nodes,) = ctx.saved_tensors
            solver = ctx.solver
            box_sl = solver.box_sl
            eps_box = torch.as_tensor(solver.nodes(ctx.eps_np)[box_sl], dtype=torch.float64)
            total = torch.zeros(solver.shape, dtype=torch.float64)
            use_f = ctx.fields and gF is not None and gF.numel() > 0
            for j, lab in enumerate(ctx.sources):
                g = gS[:, :, j].detach().to(torch.complex128) if gS is not None else None
                gf = gF[:, j].detach().to(torch.complex128) if use_f else None
                if not ((g is not None and torch.any(g != 0)) or (gf is not None and torch.any(gf != 0))):
                    continue
                key = (lab, ctx.fields)
                run = solver.run(lab, ctx.fields)
                if solver._gen[key] != ctx.gens[j]:  # a later forward replaced this one's checkpoints
                    solver.forward(lab, ctx.eps_np, ctx.fields)
                gd = None if g is None else g.to(run.dev)
                gfd = None if gf is None else gf.to(run.dev)

                def objective(acc_e, acc_h, lab=lab, gd=gd, gfd=gfd):
                    J = acc_e.real.sum() * 0
                    if gd is not None:
                        J = J + (gd.conj() * solver.s_column(lab, acc_e, acc_h)).sum().real
                    if gfd is not None:
                        J = J + (gfd.conj() * solver.field_column(lab, acc_e, acc_h)).sum().real
                    return J

                run.objective = objective
                gc = run.backward(per_component=True).sum(0).cpu()
                total[box_sl] += -gc / eps_box ** 2
            if solver.two_d:
                total = total[:, :, 1]
            return total.to(device=eps_nodes.device, dtype=eps_nodes.dtype), None, None, None

    return DeviceSParameters


def s_parameters(eps_nodes, solver: DeviceSolver, sources=None, fields: bool = False):
    """S (n_w, n_out, n_src) complex128, differentiable in ``eps_nodes`` (real, the design grid's shape:
    ``solver.design_shape``); with ``fields``, (S, F): F (n_w, n_src, *solver.field_shape()) the DFT field per
    unit incident amplitude of each source's port mode, differentiable too."""
    sources = list(solver.labels if sources is None else sources)
    for s in sources:
        if s not in solver.labels:
            raise ValueError(f"unknown port mode {s!r}; the ports are {solver.labels}")
    S, F = _function().apply(eps_nodes, solver, sources, bool(fields))
    return (S, F) if fields else S
