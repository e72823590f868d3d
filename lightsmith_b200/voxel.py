"""Material on the Yee E grid from lightsmith's particle shapes, on the GPU.

lightsmith's scattering and emission drivers mesh their particles on the host (``voxelise``,
backends/_fdtd/setup.py:110-289): the medium slot at every point of a half-cell lattice over the particles'
region, a test of every node's cell for an interface, and 8^3 samples of each interface cell. Here the
per-point work runs in CUDA (``csrc/voxel.cu``: ``lsfdtd_vox_lattice``, ``_classify``, ``_supersample``) and
this module assembles what ``voxelise`` returns from it: ``inv_eps`` (3, *shape), the dispersive groups, the
statistics and the conformal off-diagonal terms, in the same order and with the same values (the kernels
evaluate every coordinate and formula as numpy does on the host).

It serves uniform grids (no graded grid) with sphere, spheroid, cylinder and layered-sphere particles (at
most ``MAX_REGIONS`` regions each, ``MAX_MEDIA`` media) in every mesh mode except conformal meshing next to a
dispersive medium (whose vertex tensor stays on the host); ``supports`` says which.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi

MAX_REGIONS = _abi.VOX_MAX_REGIONS
MAX_MEDIA = _abi.VOX_MAX_MEDIA
KINDS = {"sphere": 0, "spheroid": 1, "cylinder": 2, "layered_sphere": 3}
MODES = {"staircase": 0, "volume_average": 1, "subpixel": 2, "conformal": 3}


class ShapeSlots:
    """lightsmith's slot function (``pts -> medium slot``) with the scene it was made from: the particles (in
    list order, the first winning overlaps), each particle's region -> slot list, and the substrate (interface
    height and slot) or None. Calling it calls lightsmith's own function."""

    def __init__(self, fn, particles, slot_of, substrate=None):
        self.fn, self.particles, self.slot_of, self.substrate = fn, list(particles), [list(s) for s in slot_of], substrate

    def __call__(self, pts):
        return self.fn(pts)


def _particle(p, slots) -> _abi.VoxParticle | None:
    shp = p.shape
    kind = KINDS.get(getattr(shp, "kind", None))
    if kind is None:
        return None
    v = _abi.VoxParticle()
    v.kind = kind
    v.pos[:] = [float(x) for x in p.position_nm]
    if kind == 0:
        v.a, radii = float(shp.radius_nm), [float(shp.radius_nm)]
    elif kind == 1:
        v.a, v.b, radii = float(shp.semi_axis_xy_nm), float(shp.semi_axis_z_nm), [0.0]
    elif kind == 2:
        v.a, v.b, radii = float(shp.radius_nm), float(shp.length_nm), [0.0]
    else:
        radii = [float(r) for r in shp.radii_nm]
        v.a = radii[-1]
    n_reg = len(radii)
    if n_reg > MAX_REGIONS or len(slots) < (n_reg if kind == 3 else 1):
        return None
    v.n_regions = n_reg if kind == 3 else 1
    for r in range(v.n_regions):
        v.radii[r] = radii[r] if kind == 3 else 0.0
        v.slot[r] = int(slots[r])
    return v


def supports(slot_fn, media, mode: str, samples: int, grid) -> bool:
    """Whether ``voxelise_gpu`` serves this call of ``voxelise``."""
    if not isinstance(slot_fn, ShapeSlots) or grid is not None or mode not in MODES:
        return False
    if not 1 <= len(media) <= MAX_MEDIA or not 1 <= int(samples) <= 64:
        return False
    if mode == "conformal" and any(m.dispersive for m in media):
        return False  # the vertex tensor of conformal meshing next to a dispersive medium stays on the host
    return all(_particle(p, s) is not None for p, s in zip(slot_fn.particles, slot_fn.slot_of))


def voxelise_gpu(slot_fn: ShapeSlots, media, shape, origin, dx, roi_lo, roi_hi, *, mode: str = "subpixel",
                 samples: int = 8, base=None, background=(), device="cuda:0"):
    """``voxelise``'s result (inv_eps, groups, stats, offdiag) for a scene ``supports`` accepts, with the
    per-point work on ``device``."""
    import torch

    from lightsmith.backends._fdtd.engine import DispersiveGroup, OffDiagonal

    L = _abi.lib()
    dev = torch.device(device)
    stream = torch.cuda.current_stream(dev)
    shape = tuple(int(n) for n in shape)
    lo, hi = [int(v) for v in roi_lo], [int(v) for v in roi_hi]
    dxv = np.broadcast_to(np.asarray(dx, dtype=float), (3,))
    S = len(media)
    eps_inf = np.array([m.eps_inf for m in media], dtype=float)
    disp = np.array([bool(m.dispersive) for m in media])
    bg = np.zeros(S, dtype=bool)
    bg[list(background)] = True
    inv_eps = np.full((3,) + shape, 1.0 / eps_inf[0]) if base is None else base[0].copy()
    flat_inv = inv_eps.reshape(-1)
    stats = {"interface_cells": 0, "dispersive_cells": 0, "mesh_refinement": mode, "offdiagonal_cells": 0,
             "tensor_vertices": 0}
    n_roi = [h - l for l, h in zip(lo, hi)]
    if min(n_roi) <= 0:
        return inv_eps, (list(base[1]) if base is not None else []), stats, None

    parts = [_particle(p, s) for p, s in zip(slot_fn.particles, slot_fn.slot_of)]
    raw = (_abi.VoxParticle * max(1, len(parts)))(*parts)
    d_parts = torch.frombuffer(bytearray(bytes(raw)), dtype=torch.uint8).to(dev)
    scene = _abi.VoxScene()
    scene.n_particles = len(parts)
    scene.particles = d_parts.data_ptr()
    if slot_fn.substrate is not None:
        scene.has_substrate, scene.z_int, scene.sub_slot = 1, float(slot_fn.substrate[0]), int(slot_fn.substrate[1])
    scene.origin[:] = [float(v) for v in origin]
    scene.dx[:] = [float(v) for v in dxv]
    scene.shape[:] = list(shape)
    scene.roi_lo[:] = lo
    scene.roi_hi[:] = hi
    med = _abi.VoxMedia()
    med.n, med.samples, med.mode = S, int(samples), MODES[mode]
    med.eps_inf[:S] = list(eps_inf)
    med.dispersive[:S] = [int(v) for v in disp]
    med.background[:S] = [int(v) for v in bg]

    lat = torch.empty(int(np.prod([2 * n + 2 for n in n_roi])), dtype=torch.int16, device=dev)
    _abi.check(L.lsfdtd_vox_lattice(C.byref(scene), C.c_void_p(lat.data_ptr()), C.c_void_p(stream.cuda_stream)),
               "lsfdtd_vox_lattice")
    cls = torch.empty(int(np.prod(n_roi)), dtype=torch.int16, device=dev)
    ii, jj, kk = (a.reshape(-1) for a in np.meshgrid(*[np.arange(l, h) for l, h in zip(lo, hi)], indexing="ij"))
    subpixel = mode != "staircase"
    claimed, pure = [], {s: [] for s in range(S) if disp[s]}
    mix_idx, mix_f, mix_w = [], [], []
    od_idx3, od_comp, od_coef = [], [], []
    for c in range(3):
        _abi.check(L.lsfdtd_vox_classify(C.byref(scene), C.c_void_p(lat.data_ptr()), c, int(subpixel),
                                         C.c_void_p(cls.data_ptr()), C.c_void_p(stream.cuda_stream)),
                   "lsfdtd_vox_classify")
        kind = cls.cpu().numpy()
        flat = ((c * shape[0] + ii) * shape[1] + jj) * shape[2] + kk
        # cells of one medium: 1/eps_inf, or 1 (D form) for a dispersive medium; the background set keeps base
        for s in range(1, S):
            if bg[s]:
                continue
            sel = kind == s
            if not sel.any():
                continue
            claimed.append(flat[sel])
            if disp[s]:
                pure[s].append(flat[sel])
                flat_inv[flat[sel]] = 1.0
            else:
                flat_inv[flat[sel]] = 1.0 / eps_inf[s]
        mi = np.flatnonzero(kind == -1)
        if not len(mi):
            continue
        r = _supersample(L, scene, med, c, mi, S, dev, stream)
        keep = r["part"].astype(bool) if bg.any() else np.ones(len(mi), dtype=bool)
        mi = mi[keep]
        if not len(mi):
            continue
        r = {k: (v[:, keep] if k == "frac" else v[keep]) for k, v in r.items()}
        f_idx = flat[mi]
        claimed.append(f_idx)
        stats["interface_cells"] += len(mi)
        hd = r["has_disp"].astype(bool)
        nd = ~hd
        if nd.any():
            flat_inv[f_idx[nd]] = r["inv"][nd]
            if mode == "conformal":
                coef = r["od"][nd]
                big = np.any(np.abs(coef) > 1e-9, axis=1)
                od_idx3.append(np.stack([ii[mi][nd][big], jj[mi][nd][big], kk[mi][nd][big]], axis=1))
                od_comp.append(np.full(int(big.sum()), c))
                od_coef.append(coef[big])
        if hd.any():
            mix_idx.append(f_idx[hd])
            mix_f.append(r["frac"][:, hd])
            mix_w.append(r["w"][hd])
            flat_inv[f_idx[hd]] = 1.0

    groups = []
    if base is not None:
        taken = np.concatenate(claimed) if claimed else np.zeros(0, dtype=np.int64)
        for g in base[1]:
            left = ~np.isin(g.idx, taken)
            if left.any():
                groups.append(DispersiveGroup(g.idx[left], g.media, g.frac[:, left], None if g.w is None else g.w[left]))
    for s, lst in pure.items():
        if lst:
            idx = np.concatenate(lst)
            groups.append(DispersiveGroup(idx, [media[s]], np.ones((1, len(idx))), None))
    if mix_idx:
        f = np.concatenate(mix_f, axis=1)
        used = [s for s in range(S) if np.any(f[s] > 0)]
        groups.append(DispersiveGroup(np.concatenate(mix_idx), [media[s] for s in used], f[used], np.concatenate(mix_w)))
    offdiag = OffDiagonal(np.concatenate(od_idx3), np.concatenate(od_comp), np.concatenate(od_coef)) if od_comp else None
    stats["dispersive_cells"] = int(sum(len(g.idx) for g in groups))
    stats["offdiagonal_cells"] = 0 if offdiag is None else len(offdiag.comp)
    stats["interface_cells"] = int(stats["interface_cells"])
    return inv_eps, groups, stats, offdiag


def _supersample(L, scene, med, c: int, mi: np.ndarray, S: int, dev, stream) -> dict:
    import torch

    n = len(mi)
    cells = torch.as_tensor(mi.astype(np.int64), device=dev)
    out = {"frac": torch.empty(S * n, dtype=torch.float64, device=dev),
           "nhat": torch.empty(3 * n, dtype=torch.float64, device=dev),
           "w": torch.empty(n, dtype=torch.float64, device=dev),
           "part": torch.empty(n, dtype=torch.int8, device=dev),
           "has_disp": torch.empty(n, dtype=torch.int8, device=dev),
           "inv": torch.empty(n, dtype=torch.float64, device=dev),
           "od": torch.empty(3 * n, dtype=torch.float64, device=dev)}
    vc = _abi.VoxCells(*[out[k].data_ptr() for k in ("frac", "nhat", "w", "part", "has_disp", "inv", "od")])
    _abi.check(L.lsfdtd_vox_supersample(C.byref(scene), C.byref(med), c, C.c_void_p(cells.data_ptr()), n, vc,
                                        C.c_void_p(stream.cuda_stream)), "lsfdtd_vox_supersample")
    h = {k: v.cpu().numpy() for k, v in out.items()}
    h["frac"] = h["frac"].reshape(S, n)
    h["nhat"] = h["nhat"].reshape(n, 3)
    h["od"] = h["od"].reshape(n, 3)
    return h
