"""The B200 FDTD engine: lightsmith's ``Engine`` interface over the CUDA kernels of ``liblsfdtd.so``.

``Engine(device, shape=..., dx=..., ...)`` takes the keyword arguments of lightsmith's
``backends/_fdtd/engine.py:Engine`` (``engine.py:231-241``) and the objects its drivers pass (``PMLSpec``,
``DispersiveGroup``, ``DFTMonitor``, the source objects), so the drivers in ``scattering.py``,
``periodic.py``, ``emission.py`` and ``device.py`` run unchanged on it. ``Engine.from_plan(plan)`` builds the
same engine from a plain plan (``lightsmith_b200.plan``) without lightsmith installed.

Device memory is held as PyTorch tensors (fields, coefficients, CPML psi slabs, dispersive state, source
tables, DFT accumulators); the kernels run on a dedicated CUDA stream through the C ABI, one chunk
(``dft_stride`` steps plus one DFT sample) at a time, optionally replayed as a CUDA graph. There is no CPU
path: without a CUDA device or without the built library this module raises.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .plan import (ColumnSource, DipoleSource, LineSource, ModeSource, TableSource, cpml_profiles, make_plan,
                   pole_coefficients)


def _torch():
    import torch

    return torch


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def _csr(node: np.ndarray):
    """Entries grouped by target node, each node's entries in their original order: (nodes, offsets, order)."""
    node = np.asarray(node, np.int64)
    order = np.argsort(node, kind="stable")
    nodes, counts = np.unique(node[order], return_counts=True)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    return nodes, offsets, order


class Engine:
    """lightsmith's FDTD engine on a B200 (sm_100a): same constructor, ``chunk``/``step``/``make_runner``/
    ``release``, ``E``/``H``/``energy``/``stride`` attributes, and DFT monitors filled in place."""

    def __init__(self, device=None, *, shape, dx, dt, single, inv_eps, groups, pml, sources, monitors, dft_stride,
                 periodic=(False, False, False), bloch=(0.0, 0.0, 0.0), offdiag=None, time_monitors=(),
                 mirror=(0, 0, 0), widths=None):
        plan = make_plan(shape=shape, dx=dx, dt=dt, single=single, inv_eps=inv_eps, groups=groups, pml=pml,
                         sources=sources, monitors=monitors, dft_stride=dft_stride, periodic=periodic, bloch=bloch,
                         offdiag=offdiag, time_monitors=time_monitors, mirror=mirror, widths=widths)
        self._build(plan, _device_name(device), monitor_objs=list(monitors))

    @classmethod
    def from_plan(cls, plan: dict, device="cuda:0", precision: str | None = None, monitor_objs=None,
                  fused: bool | None = None) -> "Engine":
        """An engine for a plain plan; ``precision`` ("single"/"double") overrides the plan's; ``fused=False``
        keeps the in-place H and E kernels where the single pass would apply."""
        self = cls.__new__(cls)
        if precision is not None:
            plan = {**plan, "single": precision == "single"}
        self._build(plan, _device_name(device), monitor_objs=monitor_objs, fused=fused)
        return self

    # --- construction ---------------------------------------------------------------------------------------
    def _build(self, plan: dict, device: str, monitor_objs=None, fused: bool | None = None):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("lightsmith-b200 runs on a CUDA GPU (B200, sm_100a); no CUDA device is visible")
        L = _abi.lib()
        self.plan = plan
        self.dev = torch.device(device)
        self.shape = tuple(int(n) for n in plan["shape"])
        self.spacing = tuple(plan["spacing"])
        self.dt = float(plan["dt"])
        self.single = bool(plan["single"])
        self.complex = bool(plan["complex"])
        self.periodic = tuple(plan["periodic"])
        self.stride = int(plan["stride"])
        self.rdt = torch.float32 if self.single else torch.float64
        self.cdt = torch.complex64 if self.single else torch.complex128
        self.fdt = self.cdt if self.complex else self.rdt
        self._keep = []  # every tensor the kernels point at
        self._subs = []  # column engines
        n0, n1, n2 = self.shape
        self.cells = n0 * n1 * n2
        uniform = len(set(self.spacing)) == 1
        cdx = self.dt / self.spacing[0] if uniform else self.dt

        with torch.cuda.device(self.dev):
            self.stream = torch.cuda.Stream(device=self.dev)
            self._E = [torch.zeros((3,) + self.shape, dtype=self.fdt, device=self.dev)]
            self._H = [torch.zeros((3,) + self.shape, dtype=self.fdt, device=self.dev)]
            # the fused single-pass step alternates between two field buffers; it serves runs without periodic
            # axes whose sources only correct E (point dipoles)
            self.mirror = tuple(int(m) for m in plan.get("mirror", (0, 0, 0)))
            # (table-fed TF/SF sources too: the lean pass adds their H corrections as it steps)
            self.double_buffered = (fused is not False and not any(self.periodic) and not self.complex and
                                    not any(self.mirror) and
                                    all(isinstance(s, (DipoleSource, TableSource)) for s in plan["sources"]) and
                                    sum(isinstance(s, TableSource) for s in plan["sources"]) <= 1)
            if self.double_buffered:
                self._E.append(torch.zeros_like(self._E[0]))
                self._H.append(torch.zeros_like(self._H[0]))
            self.n = torch.zeros(1, dtype=torch.int64, device=self.dev)
            self.energy = torch.zeros(2, dtype=torch.float64, device=self.dev)
            inv_eps = plan["inv_eps"]
            self.cdx = cdx
            # cbE = (dt/dx or dt) / eps per component; one shared array when eps is isotropic (engine.py:299)
            if hasattr(inv_eps, "detach"):  # a device tensor, isotropic (N0, N1, N2)
                iso = True
                t = (inv_eps.to(device=self.dev, dtype=torch.float64) * cdx).to(self.rdt).contiguous()
                self._keep.append(t)
                cb = [t] * 3
            elif inv_eps.ndim == 3:
                iso = True
                cb = [self._dev(cdx * inv_eps, self.rdt)] * 3
            else:
                iso = bool(np.array_equal(inv_eps[0], inv_eps[1]) and np.array_equal(inv_eps[0], inv_eps[2]))
                cb = ([self._dev(cdx * inv_eps[0], self.rdt)] * 3 if iso else
                      [self._dev(cdx * inv_eps[c], self.rdt) for c in range(3)])
            self.isotropic = iso
            self.cbE = cb
            g = _abi.GridDesc()
            g.shape[:] = list(self.shape)
            g.precision = _abi.F32 if self.single else _abi.F64
            g.is_complex = int(self.complex)
            g.periodic[:] = [int(p) for p in self.periodic]
            g.mirror[:] = list(self.mirror)
            g.spacing[:] = list(self.spacing)
            g.dt = self.dt
            g.bloch[:] = list(plan["bloch"])
            g.dft_stride = self.stride
            g.E, g.H = _ptr(self._E[0]), _ptr(self._H[0])
            if self.double_buffered:
                g.E_alt, g.H_alt = _ptr(self._E[1]), _ptr(self._H[1])
            g.cbE[:] = [_ptr(t) for t in cb]
            g.step, g.energy = _ptr(self.n), _ptr(self.energy)
            h = C.c_void_p()
            _abi.check(L.lsfdtd_engine_create(C.byref(g), C.byref(h)), "lsfdtd_engine_create")
            self._h = h
            self._build_pml(plan, L)
            self.groups = [self._build_group(gr, L) for gr in plan["groups"]]
            if plan.get("tensor") is not None:  # conformal interfaces of dispersive media (engine.py:838-923)
                self._build_tensor(plan["tensor"], L)
            od = plan.get("offdiag")
            if od is not None and len(od["e"]):  # conformal off-diagonal terms (engine.py:421-518, 653-655)
                torch = _torch()
                o = _abi.OffdiagDesc()
                ee = self._dev(np.asarray(od["e"], np.int64), torch.int64)
                hh = self._dev(np.ascontiguousarray(od["h"], np.int64), torch.int64)
                ww = self._dev(np.ascontiguousarray(od["w"]), self.fdt)
                o.e, o.h, o.w = _ptr(ee), _ptr(hh), _ptr(ww)
                o.n, o.width = len(od["e"]), int(np.asarray(od["h"]).shape[1])
                _abi.check(L.lsfdtd_engine_add_offdiag(self._h, C.byref(o)), "lsfdtd_engine_add_offdiag")
            self._src_state = [self._build_source(s, L) for s in plan["sources"]]
            self.monitors = []
            objs = monitor_objs if monitor_objs is not None else [None] * len(plan["monitors"])
            for m, obj in zip(plan["monitors"], objs):
                self.monitors.append(self._build_monitor(m, obj, L))
            nbytes = C.c_size_t()
            _abi.check(L.lsfdtd_engine_scratch_bytes(self._h, C.byref(nbytes)), "lsfdtd_engine_scratch_bytes")
            self.scratch = torch.zeros(max(int(nbytes.value), 8), dtype=torch.uint8, device=self.dev)
            _abi.check(L.lsfdtd_engine_set_scratch(self._h, _ptr(self.scratch), int(nbytes.value)),
                       "lsfdtd_engine_set_scratch")
        self._graph_used = False

    def _dev(self, a, dtype):
        t = _torch().as_tensor(np.ascontiguousarray(a)).to(device=self.dev, dtype=dtype).contiguous()
        self._keep.append(t)
        return t

    def _zeros(self, shape, dtype):
        t = _torch().zeros(tuple(int(s) for s in shape), dtype=dtype, device=self.dev)
        self._keep.append(t)
        return t

    def _build_pml(self, plan, L):
        spec = _Spec(plan["pml"])
        pad = int(plan.get("pad_z") or 0)  # rows padded along z (plan.pad_rows): the profiles of the original grid
        orig = (self.shape[0], self.shape[1], self.shape[2] - pad)
        prof = cpml_profiles(spec, orig, self.spacing, self.dt)
        if pad and 2 in prof:  # the high z slab widened over the frozen planes, where psi stays zero
            lo_n, hi_n, pr = prof[2]
            one, zero = np.ones(pad), np.zeros(pad)
            prof[2] = (lo_n, hi_n + pad if hi_n else 0,
                       {k: (np.concatenate([b, zero]), np.concatenate([c, zero]), np.concatenate([kap, one]))
                        for k, (b, c, kap) in pr.items()})
        shp = (C.c_int32 * 3)(*self.shape)
        per = (C.c_int32 * 3)(*[int(p) for p in self.periodic])
        self.psi = {}
        self.psi_alt = {}  # the H slabs that go with the second field buffers of the fused pass
        for d, (lo_n, hi_n, pr) in prof.items():
            if self.periodic[d]:
                raise ValueError("a periodic axis cannot have a PML")
            p = _abi.PmlDesc()
            p.axis, p.cells_lo, p.cells_hi = d, lo_n, hi_n
            for f, kind in enumerate(("E", "H")):
                b, c, kap = pr[kind]
                p.b[f] = _ptr(self._dev(b, self.rdt))
                p.c[f] = _ptr(self._dev(c, self.rdt))
                p.k[f] = _ptr(self._dev(1 / kap - 1, self.rdt)) if np.any(kap > 1) else None
                for comp in range(3):
                    for side in range(2):
                        st, ln = C.c_int32(), C.c_int32()
                        _abi.check(L.lsfdtd_cpml_slab(shp, per, d, lo_n, hi_n, f, comp, side, C.byref(st),
                                                      C.byref(ln)), "lsfdtd_cpml_slab")
                        if ln.value > 0:
                            dims = list(self.shape)
                            dims[d] = ln.value
                            t = self._zeros(dims, self.fdt)
                            self.psi[(kind, comp, d, side)] = t
                            p.psi[f][comp][side] = _ptr(t)
                            if kind == "H" and self.double_buffered:
                                alt = self._zeros(dims, self.fdt)
                                self.psi_alt[(kind, comp, d, side)] = alt
                                p.psi_alt[comp][side] = _ptr(alt)
            _abi.check(L.lsfdtd_engine_set_pml(self._h, C.byref(p)), "lsfdtd_engine_set_pml")

    def _build_group(self, gr, L):
        media = gr["media"]
        idx = np.asarray(gr["idx"], np.int64)
        n = len(idx)
        g = _abi.GroupDesc()
        g.n = n
        g.idx = _ptr(self._dev(idx, _torch().int64))
        if gr["w"] is None:
            (m,) = media
            disp = [m]
            g.mixed, g.has_h, g.has_a = 0, 0, 0
            g.inv_eps_inf[0] = 1.0 / m["eps_inf"]
        else:
            f = np.asarray(gr["frac"], float)
            dis = [s for s, m in enumerate(media) if m["poles"]]
            disp = [media[s] for s in dis]
            if not dis:
                raise ValueError("a mixed dispersive group without a dispersive medium")
            w = np.asarray(gr["w"], float)
            h0 = sum(f[s] / m["eps_inf"] for s, m in enumerate(media) if not m["poles"]) + 0 * f[0]
            inv_a = 1.0 / sum(f[s] * m["eps_inf"] for s, m in enumerate(media))
            g.mixed = 1
            g.has_h, g.has_a = int(np.any(w > 0)), int(np.any(w < 1))
            g.h0 = _ptr(self._dev(h0, self.rdt))
            g.inv_a = _ptr(self._dev(inv_a, self.rdt))
            g.w = _ptr(self._dev(w, self.rdt))
            g.frac = _ptr(self._dev(f[dis], self.rdt))
            for s, m in enumerate(disp):
                g.inv_eps_inf[s] = 1.0 / m["eps_inf"]
        if len(disp) > _abi.MAX_MEDIA:
            raise ValueError(f"at most {_abi.MAX_MEDIA} dispersive media per group")
        g.n_media = len(disp)
        npoles = []
        for s, m in enumerate(disp):
            if len(m["poles"]) > _abi.MAX_POLES:
                raise ValueError(f"at most {_abi.MAX_POLES} poles per medium")
            npoles.append(len(m["poles"]))
            g.n_poles[s] = len(m["poles"])
            for k, pole in enumerate(m["poles"]):
                c1, c2, c3 = pole_coefficients(_Pole(*pole), self.dt)
                g.c1[s][k], g.c2[s][k], g.c3[s][k] = c1, c2, c3
        arr = (C.c_int32 * _abi.MAX_MEDIA)(*(npoles + [0] * (_abi.MAX_MEDIA - len(npoles))))
        slen = int(L.lsfdtd_group_state_len(g.mixed, g.n_media, arr))
        state = self._zeros((slen, max(n, 1)), self.fdt)
        g.state = _ptr(state)
        _abi.check(L.lsfdtd_engine_add_group(self._h, C.byref(g)), "lsfdtd_engine_add_group")
        return {"idx": idx, "state": state, "mixed": bool(g.mixed)}

    def _build_tensor(self, t, L):
        """The vertex-tensor mesh's tables (plan.py:tensor_plan) on the device and its zeroed state."""
        torch = _torch()
        i64 = torch.int64
        d = _abi.TensorDesc()
        keep = {}

        def arr(name, dtype):
            a = t[name]
            if a is None or not len(a):
                return None
            keep[name] = self._dev(np.asarray(a), dtype)
            return _ptr(keep[name])

        d.idx, d.n_nodes = arr("idx", i64), int(t["n_nodes"])
        d.vn, d.scale, d.normal = arr("vn", i64), arr("scale", self.fdt), arr("normal", self.rdt)
        d.n_vert = len(np.asarray(t["normal"])) // 3
        for k in ("t_pos", "t_v", "t_vc", "t_g"):
            setattr(d, k, arr(k, i64))
        d.t_nc, d.t_conj = arr("t_nc", self.rdt), arr("t_conj", self.fdt)
        d.frac = arr("frac", self.rdt)
        d.n_tslots = len(t["t_pos"])
        d.p_pos, d.p_node, d.p_medium = arr("p_pos", i64), arr("p_node", i64), arr("p_medium", i64)
        d.n_pslots = len(t["p_pos"])
        media = t["media"]
        if len(media) > _abi.MAX_MEDIA:
            raise ValueError(f"at most {_abi.MAX_MEDIA} media in a vertex-tensor mesh")
        d.n_media = len(media)
        npoles = []
        for s, m in enumerate(media):
            if len(m["poles"]) > _abi.MAX_POLES:
                raise ValueError(f"at most {_abi.MAX_POLES} poles per medium")
            npoles.append(len(m["poles"]))
            d.n_poles[s] = len(m["poles"])
            d.eps_inf[s] = float(m["eps_inf"])
            for k, pole in enumerate(m["poles"]):
                d.c1[s][k], d.c2[s][k], d.c3[s][k] = pole_coefficients(_Pole(*pole), self.dt)
        arr_np = (C.c_int32 * _abi.MAX_MEDIA)(*(npoles + [0] * (_abi.MAX_MEDIA - len(npoles))))
        n = int(L.lsfdtd_tensor_state_len(d.n_nodes, d.n_vert, d.n_tslots, d.n_pslots, d.n_media, arr_np))
        if n < 0:
            raise ValueError("vertex-tensor mesh sizes out of range")
        state = self._zeros((max(n, 1),), self.fdt)
        d.state = _ptr(state)
        _abi.check(L.lsfdtd_engine_add_tensor(self._h, C.byref(d)), "lsfdtd_engine_add_tensor")
        self.tensor = {"state": state, **keep}

    def _points(self, pts, fields):
        """CSR device arrays of a TablePoints/LinePoints (fields: its per-entry arrays and their dtypes)."""
        torch = _torch()
        nodes, offsets, order = _csr(pts.node)
        out = {"nodes": self._dev(nodes, torch.int64), "offsets": self._dev(offsets, torch.int64),
               "n_nodes": len(nodes), "n_entries": len(order), "order": order}
        for name, dt in fields:
            out[name] = self._dev(np.asarray(getattr(pts, name))[order], dt)
        return out

    def _build_source(self, s, L):
        torch = _torch()
        i64 = torch.int64
        if isinstance(s, TableSource):
            d = _abi.TableSourceDesc()
            T = self._dev(s.tables, self.rdt)
            Ti = self._dev(s.inc_table, self.rdt)
            d.table, d.table_len = _ptr(T), T.numel()
            d.inc_table, d.inc_len = _ptr(Ti), Ti.numel()
            d.m, d.cmax = int(s.m), int(s.cmax)
            for k, pts in enumerate((s.E, s.H)):
                if pts is None:
                    continue
                if np.max(pts.base) + s.cmax + 5 >= T.numel() or np.min(pts.base) < 0 or np.min(pts.i0) < 0:
                    raise ValueError("table source reads outside its tables")
                q = self._points(pts, [("base", i64), ("i0", i64), ("u0", self.rdt), ("coef", self.rdt)])
                if k == 1:
                    q_h = q
                d.pts[k].n_nodes, d.pts[k].nodes, d.pts[k].offsets = q["n_nodes"], _ptr(q["nodes"]), _ptr(q["offsets"])
                d.pts[k].n_entries = q["n_entries"]
                d.base[k], d.i0[k], d.u0[k], d.coef[k] = (_ptr(q[x]) for x in ("base", "i0", "u0", "coef"))
            base, i0, u0 = s.inc
            if np.max(base) + s.cmax + 5 >= Ti.numel():
                raise ValueError("incident view reads outside its table")
            d.inc_base, d.inc_i0 = _ptr(self._dev(base, i64)), _ptr(self._dev(i0, i64))
            d.inc_u0 = _ptr(self._dev(u0, self.rdt))
            view = self._zeros((3,), self.rdt)
            d.view = _ptr(view)
            _abi.check(L.lsfdtd_engine_add_table_source(self._h, C.byref(d)), "lsfdtd_engine_add_table_source")
            if self.double_buffered and s.H is not None:
                self._table_boxes(s.H, q_h, L)
            return {"kind": "table", "view": view}
        if isinstance(s, DipoleSource):
            idx = np.asarray(s.idx, np.int64)
            if len(np.unique(idx)) != len(idx):
                raise ValueError("a point dipole's nodes must be distinct")
            d = _abi.DipoleDesc()
            d.n = len(idx)
            d.idx = _ptr(self._dev(idx, i64))
            d.coef = _ptr(self._dev(s.coef, self.rdt))
            wave = self._dev(s.wave, self.rdt)
            d.wave, d.wave_len = _ptr(wave), wave.numel()
            _abi.check(L.lsfdtd_engine_add_dipole(self._h, C.byref(d)), "lsfdtd_engine_add_dipole")
            return {"kind": "dipole"}
        if isinstance(s, LineSource):
            d = _abi.LineSourceDesc()
            d.M, d.m_src = int(s.M), int(s.m_src)
            for name in ("ca", "cb", "da", "db"):
                setattr(d, name, _ptr(self._dev(getattr(s, name), self.rdt)))
            wave = self._dev(s.wave, self.rdt)
            d.wave, d.wave_len = _ptr(wave), wave.numel()
            E_line, H_line = self._zeros((s.M,), self.rdt), self._zeros((s.M,), self.rdt)
            d.E_line, d.H_line = _ptr(E_line), _ptr(H_line)
            for k, pts in enumerate((s.E, s.H)):
                if pts is None:
                    continue
                if np.min(pts.i0) < 0 or np.max(pts.i0) + 1 >= s.M:
                    raise ValueError("1D-fed source reads outside its line")
                q = self._points(pts, [("i0", i64), ("w", self.rdt), ("coef", self.rdt)])
                d.pts[k].n_nodes, d.pts[k].nodes, d.pts[k].offsets = q["n_nodes"], _ptr(q["nodes"]), _ptr(q["offsets"])
                d.pts[k].n_entries = q["n_entries"]
                d.i0[k], d.w[k], d.coef[k] = _ptr(q["i0"]), _ptr(q["w"]), _ptr(q["coef"])
            _abi.check(L.lsfdtd_engine_add_line_source(self._h, C.byref(d)), "lsfdtd_engine_add_line_source")
            return {"kind": "line", "E": E_line, "H": H_line}
        if isinstance(s, ColumnSource):
            col = Engine.from_plan(s.column, device=str(self.dev), precision="single" if self.single else "double")
            if not col.complex or not self.complex:
                raise ValueError("a Bloch column source needs complex fields on both grids")
            self._subs.append(col)
            d = _abi.ColumnSourceDesc()
            d.column = col._h
            d.k_src, d.k_launch = int(s.k_src), int(s.k_launch)
            ph = np.asarray(s.phase, complex)
            if ph.shape != (self.shape[0] - 2, self.shape[1] - 2):
                raise ValueError("column phase must cover the real cells of the plane")
            d.phase = _ptr(self._dev(ph, self.cdt))
            d.amp[0][0], d.amp[0][1] = s.amp[0].real, s.amp[0].imag
            d.amp[1][0], d.amp[1][1] = s.amp[1].real, s.amp[1].imag
            wave = self._dev(s.wave, self.rdt)
            d.wave, d.wave_len = _ptr(wave), wave.numel()
            d.cE, d.cH = float(s.cE), float(s.cH)
            _abi.check(L.lsfdtd_engine_add_column_source(self._h, C.byref(d)), "lsfdtd_engine_add_column_source")
            return {"kind": "column", "col": col}
        if isinstance(s, ModeSource):
            d = _abi.ModeSourceDesc()
            mH, mE = np.atleast_2d(s.mH), np.atleast_2d(s.mE)
            tE, tH = np.atleast_2d(s.tab_E), np.atleast_2d(s.tab_H)
            d.n_h, d.r_e = mH.shape
            d.n_e, d.r_h = mE.shape
            if tE.shape[1] != d.r_e or tH.shape[1] != d.r_h:
                raise ValueError("mode source tables do not match its basis")
            for idx in (s.h_idx, s.e_idx):
                if len(np.unique(idx)) != len(idx):
                    raise ValueError("a mode source's target nodes must be distinct")
            d.h_idx, d.e_idx = _ptr(self._dev(s.h_idx, i64)), _ptr(self._dev(s.e_idx, i64))
            d.mH, d.mE = _ptr(self._dev(mH, self.rdt)), _ptr(self._dev(mE, self.rdt))
            d.tab_E, d.tab_H = _ptr(self._dev(tE, self.rdt)), _ptr(self._dev(tH, self.rdt))
            d.len_E, d.len_H = tE.shape[0], tH.shape[0]
            _abi.check(L.lsfdtd_engine_add_mode_source(self._h, C.byref(d)), "lsfdtd_engine_add_mode_source")
            return {"kind": "mode"}
        raise NotImplementedError(f"no CUDA path for the source {type(s).__name__}")

    def _table_boxes(self, pts, q, L):
        """Give the fused pass the H corrections of the (only) table-fed source as slab boxes (plan.slab_boxes),
        with the position of each slab-order entry among the source's CSR entries and a value array. Sources
        whose points do not form at most 24 boxes keep the in-place kernels."""
        from .plan import slab_boxes

        torch = _torch()
        try:
            boxes = slab_boxes(pts.node, self.shape)
        except ValueError:
            return
        if not 1 <= len(boxes) <= 24:
            return
        rows = np.array([[bc, *lo, *hi, off] for bc, lo, hi, off in boxes], dtype=np.int32)
        perm = np.empty(len(q["order"]), np.int64)
        perm[q["order"]] = np.arange(len(q["order"]))  # slab-order entry e sits at CSR position perm[e]
        perm_d = self._dev(perm, torch.int64)
        vals = self._zeros((len(perm),), self.rdt)
        _abi.check(L.lsfdtd_engine_set_table_boxes(self._h, 0, len(boxes), rows.ctypes.data_as(C.c_void_p),
                                                   _ptr(perm_d), len(perm), _ptr(vals)),
                   "lsfdtd_engine_set_table_boxes")
        self._keep.append(rows)

    def _build_monitor(self, m, obj, L):
        torch = _torch()
        kind, i = m["space"]
        if kind == "grid":
            space, E_src, H_src = 0, self._E[0], self._H[0]
        elif kind == "view":
            v = self._src_state[i]["view"]
            space, E_src, H_src = 1, v, v
        elif kind == "line":
            st = self._src_state[i]
            space, E_src, H_src = 1, st["E"], st["H"]
        elif kind == "column":
            col = self._src_state[i]["col"]
            space, E_src, H_src = 2, col.E, col.H
        else:
            raise ValueError(kind)
        omega = np.asarray(m["omega"], float)
        nf = len(omega)
        acc_e = torch.zeros((nf, len(m["e_idx"])), dtype=torch.complex128, device=self.dev)
        acc_h = None
        d = _abi.MonitorDesc()
        d.n_freq = nf
        d.omega = _ptr(self._dev(omega, torch.float64))
        d.n_e, d.e_idx = len(m["e_idx"]), _ptr(self._dev(m["e_idx"], torch.int64))
        if m["h_idx1"] is not None:
            acc_h = torch.zeros((nf, len(m["h_idx1"])), dtype=torch.complex128, device=self.dev)
            d.n_h = len(m["h_idx1"])
            d.h_idx1 = _ptr(self._dev(m["h_idx1"], torch.int64))
            d.h_idx2 = _ptr(self._dev(m["h_idx2"], torch.int64))
            d.acc_h = _ptr(acc_h)
        d.acc_e = _ptr(acc_e)
        d.energy, d.space = int(m["energy"]), space
        d.E_src, d.H_src = _ptr(E_src), _ptr(H_src)
        n_src_e = E_src.numel()
        for name in ("e_idx", "h_idx1", "h_idx2"):
            a = m[name]
            if a is not None and len(a) and (np.min(a) < 0 or np.max(a) >= n_src_e):
                raise ValueError(f"monitor {name} out of range")
        _abi.check(L.lsfdtd_engine_add_monitor(self._h, C.byref(d)), "lsfdtd_engine_add_monitor")
        if obj is not None:
            obj.acc_e, obj.acc_h = acc_e, acc_h
        return {"acc_e": acc_e, "acc_h": acc_h}

    # --- running ---------------------------------------------------------------------------------------------
    def _prime(self):
        """The engine's stream waits for the caller's: whatever the caller did to the engine's arrays on its own
        stream (writes, or reads such as a checkpoint's copy) comes before the engine's next kernels."""
        torch = _torch()
        self.stream.wait_stream(torch.cuda.current_stream(self.dev))

    def _finish(self):
        _torch().cuda.current_stream(self.dev).wait_stream(self.stream)

    def step(self, n: int = 1):
        """n time steps without a DFT sample (Engine.step, engine.py:665-678)."""
        self._prime()
        _abi.check(_abi.lib().lsfdtd_engine_step(self._h, int(n), self.stream.cuda_stream), "lsfdtd_engine_step")
        self._finish()

    def sample(self):
        self._prime()
        _abi.check(_abi.lib().lsfdtd_engine_sample(self._h, self.stream.cuda_stream), "lsfdtd_engine_sample")
        self._finish()

    def chunk(self, n_chunks: int = 1, use_graph: bool = False):
        """dft_stride steps then one DFT sample, n_chunks times (Engine.chunk, engine.py:680-683)."""
        self._prime()
        _abi.check(_abi.lib().lsfdtd_engine_chunk(self._h, int(n_chunks), int(bool(use_graph)),
                                                  self.stream.cuda_stream), "lsfdtd_engine_chunk")
        self._graph_used |= bool(use_graph)
        self._finish()

    def chunk_timed(self, n_chunks: int = 1) -> tuple[float, int]:
        """Eager chunks with CUDA events around every bulk Yee-update kernel on the engine's stream:
        (summed kernel milliseconds, number of those launches). Synchronises."""
        self._prime()
        ms, n = C.c_double(), C.c_int64()
        _abi.check(_abi.lib().lsfdtd_engine_chunk_timed(self._h, int(n_chunks), self.stream.cuda_stream,
                                                        C.byref(ms), C.byref(n)), "lsfdtd_engine_chunk_timed")
        self._finish()
        return float(ms.value), int(n.value)

    def load_inv_eps(self, inv_eps) -> None:
        """Replace an isotropic 1/eps (N0, N1, N2) in place, e.g. from pinned host memory (asynchronous on the
        engine's stream): the curl coefficients become cdx / eps."""
        if not self.isotropic:
            raise ValueError("load_inv_eps needs an engine built with isotropic permittivity")
        torch = _torch()
        with torch.cuda.stream(self.stream):
            self.cbE[0].copy_(inv_eps, non_blocking=True)
            self.cbE[0].mul_(self.cdx)

    def make_runner(self, use_graphs: bool):
        """(run one chunk, used graphs) as Engine.make_runner (engine.py:685-709): the chunk is captured once as
        a CUDA graph and replayed."""
        def run():
            self.chunk(1, use_graph=use_graphs)
            self.check_status()  # the driver synchronises once per chunk anyway to read the energy
        return run, bool(use_graphs)

    def release(self):
        """Nothing to drop between chunks; the captured graph lives until the engine is closed."""
        _torch().cuda.synchronize(self.dev)

    @property
    def E(self):
        """The current E (3, N0, N1, N2): one of two buffers on the fused path."""
        return self._E[int(_abi.lib().lsfdtd_engine_buffer(self._h))]

    @property
    def H(self):
        return self._H[int(_abi.lib().lsfdtd_engine_buffer(self._h))]

    def state(self) -> list:
        """The fields, CPML psi and dispersive state of the current step, in a fixed order (E, H, psi in
        ``self.psi``'s order, the groups' state, the vertex-tensor mesh's state): on the fused path, the buffers
        of the current parity."""
        b = int(_abi.lib().lsfdtd_engine_buffer(self._h))
        return [self._E[b], self._H[b]] + [self.psi_alt[k] if b and k in self.psi_alt else t
                                           for k, t in self.psi.items()] + [g["state"] for g in self.groups] + \
            self._tensor_state()

    def _tensor_state(self) -> list:
        t = getattr(self, "tensor", None)
        return [] if t is None else [t["state"]]

    def all_state(self) -> list:
        """Every state buffer of both parities (for clearing the state)."""
        return (self._E + self._H + list(self.psi.values()) + list(self.psi_alt.values()) +
                [g["state"] for g in self.groups] + self._tensor_state())

    @property
    def E_flat(self):
        return self.E.view(-1)

    @property
    def H_flat(self):
        return self.H.view(-1)

    @property
    def fused(self) -> bool:
        """Whether a step is the fused single pass (decided once the engine is described)."""
        return bool(_abi.lib().lsfdtd_engine_fused(self._h))

    @property
    def uses_tma(self) -> bool:
        """Whether the fused pass copies its planes with the Tensor Memory Accelerator."""
        return bool(_abi.lib().lsfdtd_engine_uses_tma(self._h))

    def set_copy_engine(self, use_tma: bool) -> None:
        """TMA (default) or cp.async copies for the fused pass; before the first step."""
        _abi.check(_abi.lib().lsfdtd_engine_set_copy_engine(self._h, int(bool(use_tma))),
                   "lsfdtd_engine_set_copy_engine")

    def check_status(self) -> None:
        """Raise if a kernel gave up waiting for its own copies (synchronises the engine's stream)."""
        st = C.c_int32()
        _abi.check(_abi.lib().lsfdtd_engine_status(self._h, self.stream.cuda_stream, C.byref(st)),
                   "lsfdtd_engine_status")

    def clear_status(self) -> None:
        """Clear the status word a timed-out copy wait set (on the engine's stream)."""
        _abi.check(_abi.lib().lsfdtd_engine_clear_status(self._h, self.stream.cuda_stream),
                   "lsfdtd_engine_clear_status")

    def set_wait_budget(self, cycles: int) -> None:
        """Clock cycles the fused pass waits for one plane's copies before it gives up (default about 2 s when
        ``cycles`` is 0; negative: a test of the timeout path, every wait on a barrier nothing completes for
        -cycles cycles); before the first graph capture."""
        _abi.check(_abi.lib().lsfdtd_engine_set_wait_budget(self._h, int(cycles)), "lsfdtd_engine_set_wait_budget")

    def set_clean_split(self, on: bool) -> None:
        """Variant 4: step the grid's clean interior (no CPML, no walls) with its own kernel beside the lean
        kernel on the rest (on, the default), or every tile with the lean kernel; the same values either way.
        Before the first graph capture."""
        _abi.check(_abi.lib().lsfdtd_engine_set_clean_split(self._h, 1 if on else 0), "lsfdtd_engine_set_clean_split")

    def set_tuning(self, variant: int, tile_y: int, planes: int, stages: int = 4) -> None:
        """Kernel choice and launch shape (before the first graph capture): variant 0 the in-place H and E
        kernels, 2 their four-node vector form, 1 the fused pass (CTA tile rows 8 or 16, x planes per tile,
        copy ring 4/6/8), 3 the fused pass split into an interior box and CPML/wall shell kernels, 4 the fused
        pass with lean CPML terms (the default, with tile rows 8, planes per grid and ring 4; runs the fused pass
        does not serve take the in-place kernels). ``planes=0`` chooses per grid: 48, or fewer on grids too
        small for about three waves of CTAs."""
        _abi.check(_abi.lib().lsfdtd_engine_set_tuning(self._h, int(variant), int(tile_y), int(planes),
                                                       int(stages)), "lsfdtd_engine_set_tuning")

    @property
    def n_host(self) -> int:
        return int(_abi.lib().lsfdtd_engine_steps(self._h))

    def launches_per_chunk(self) -> int:
        return int(_abi.lib().lsfdtd_engine_launches_per_chunk(self._h))

    def results(self, k: int):
        m = self.monitors[k]
        return (m["acc_e"].cpu().numpy(), None if m["acc_h"] is None else m["acc_h"].cpu().numpy())

    def source_arrays(self, i: int):
        """Device arrays a source keeps (the 1D line's E/H, the column engine, the incident view)."""
        return self._src_state[i]

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _torch().cuda.synchronize(self.dev)
            _abi.lib().lsfdtd_engine_destroy(h)
            self._h = C.c_void_p()
        for s in getattr(self, "_subs", []):
            s.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 (interpreter shutdown)
            pass


class _Spec:
    def __init__(self, d):
        self.__dict__.update(d)


class _Pole:
    def __init__(self, sigma, omega0, gamma):
        self.sigma, self.omega0, self.gamma = sigma, omega0, gamma


def _device_name(device) -> str:
    if device is None:
        return "cuda:0"
    name = getattr(device, "name", device)
    name = str(name)
    if not name.startswith("cuda"):
        raise RuntimeError(f"lightsmith-b200 runs on a CUDA device, not {name!r}")
    return name
