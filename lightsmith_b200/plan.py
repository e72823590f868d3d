"""Plain-array descriptions of one FDTD run (the "plan"), shared by the CUDA engine and the CPU oracle.

A plan holds only NumPy arrays and Python scalars, so it can be built from lightsmith's own engine inputs
(duck-typed: ``PMLSpec``, ``DispersiveGroup``, ``DFTMonitor`` and the source objects of
``lightsmith/backends/_fdtd``), from this module's dataclasses of the same names, or loaded from an ``.npz``
fixture, with no lightsmith installation.

Layouts follow lightsmith's engine (``backends/_fdtd/engine.py:16-18``): fields stacked as F[3, N0, N1, N2]
(C order, N2 fastest), flat index ``((c * N0 + i) * N1 + j) * N2 + k`` (``engine.py:103-105``). E_c sits at
node + e_c/2 and H_c at node + (1 - e_c)/2 in cell units.
"""

from __future__ import annotations

import io
import json
from dataclasses import dataclass, field, replace

import numpy as np

# --- material / boundary / monitor descriptions (same fields as lightsmith's engine dataclasses) ---------


@dataclass(frozen=True)
class Pole:
    """One ADE pole P'' + gamma P' + omega0^2 P = sigma E (``media.py:25-29``)."""

    sigma: float
    omega0: float
    gamma: float


@dataclass(frozen=True)
class Medium:
    """eps_inf plus poles (``media.py:32-40``)."""

    eps_inf: float
    poles: tuple = ()
    label: str = ""

    @property
    def dispersive(self) -> bool:
        return bool(self.poles)


@dataclass
class PMLSpec:
    """CPML thickness per axis and its grading (``engine.py:184-191``)."""

    cells: tuple
    m: float = 3.0
    kappa_max: float = 1.0
    alpha_max: float = 0.0
    eps_ref: float = 1.0
    eps_ref_high: float | None = None


@dataclass
class DispersiveGroup:
    """E nodes integrated in D-form (``engine.py:129-137``): flat E indices, media, fractions (S, n) and the
    harmonic-path weight w (None for pure cells)."""

    idx: np.ndarray
    media: list
    frac: np.ndarray
    w: np.ndarray | None


@dataclass
class DFTMonitor:
    """Running DFT of E at e_idx and of the mean of H at h_idx1/h_idx2 (``engine.py:194-210``).

    ``source`` selects whose arrays are sampled: None for the grid, else a source object (its own E/H, e.g.
    the 1D feed line or the Bloch column) or a source's incident-reference view."""

    omega: np.ndarray
    e_idx: np.ndarray
    h_idx1: np.ndarray | None = None
    h_idx2: np.ndarray | None = None
    energy: int = 0
    source: object | None = None
    acc_e: object = field(default=None, repr=False)
    acc_h: object = field(default=None, repr=False)

    def results(self):
        def host(a):
            if a is None:
                return None
            if hasattr(a, "detach"):
                a = a.detach().cpu().numpy()
            return np.asarray(a).astype(complex)
        return host(self.acc_e), host(self.acc_h)


# --- region helpers ----------------------------------------------------------------------------------


def _parity(kind: str, c: int, a: int, m: int) -> int:
    """Sign a field component takes under reflection in a mirror plane normal to axis a (m = +1 symmetric, -1
    antisymmetric in E): an E component parallel to the plane keeps the plane's sign m, the normal one takes the
    opposite; H, a pseudovector, takes the opposite of E's."""
    e = m if c != a else -m
    return e if kind == "E" else -e


def _on_node_planes(kind: str, c: int, a: int) -> bool:
    """Whether component c of E or H sits on the node planes along axis a (Yee staggering: E_c is half a cell
    off along c, H_c half a cell off along both other axes)."""
    return (c != a) if kind == "E" else (c == a)


def _first_stepped(kind: str, c: int, a: int, m: int) -> int:
    """First stepped index along a mirror axis (the plane at node 1, a ghost plane at 0): a component that is odd
    under the reflection and sits on the plane vanishes there and is stepped from index 2; every other one is
    stepped from index 1."""
    return 2 if _parity(kind, c, a, m) < 0 and _on_node_planes(kind, c, a) else 1


def e_range(c: int, a: int, n: int, periodic: bool, mirror: int = 0) -> tuple[int, int]:
    """Stepped index range [lo, hi) of E_c along axis a (``engine.py:47-60``): tangential E stays 0 on the
    outer (PEC) planes; periodic axes step the real cells 1..n-2 between two ghost planes; on a mirror axis
    (mirror = +1 or -1, the plane at node 1, a ghost plane at 0) the range starts at 1 or 2."""
    if mirror:
        return _first_stepped("E", c, a, mirror), n - 1
    if periodic or a != c:
        return 1, n - 1
    return 0, n - 1


def h_range(c: int, a: int, n: int, periodic: bool, mirror: int = 0) -> tuple[int, int]:
    """Stepped index range of H_c along axis a (``engine.py:63-66``)."""
    if mirror:
        return _first_stepped("H", c, a, mirror), (n if a == c else n - 1)
    if periodic:
        return 1, n - 1
    return (0, n) if a == c else (0, n - 1)


def flat_index(c, i, j, k, shape):
    n0, n1, n2 = shape
    return ((np.asarray(c) * n0 + np.asarray(i)) * n1 + np.asarray(j)) * n2 + np.asarray(k)


def pole_coefficients(pole, dt: float) -> tuple[float, float, float]:
    """Central-difference ADE coefficients (c1, c2, c3) of P^{n+1} = c1 P^n + c2 P^{n-1} + c3 E^n
    (``engine.py:108-111``)."""
    half = pole.gamma * dt / 2
    den = 1 + half
    return (2 - pole.omega0 ** 2 * dt ** 2) / den, -(1 - half) / den, pole.sigma * dt ** 2 / den


# --- CPML terms --------------------------------------------------------------------------------------


def _depth_fraction(x, n_cells: int):
    """How far into an n-cell layer a position lies, as a fraction clipped to [0, 1] (x: cells inward from the
    layer's inner face); zero everywhere when the side has no layer."""
    return np.clip(x / n_cells, 0, 1) if n_cells else np.zeros_like(x)


def _grading(rho, sigma_max, pml, dt):
    """CPML coefficients at depth fraction rho in [0, 1] (the grading of ``engine.py:361-371``: polynomial sigma
    and kappa of order m, alpha falling linearly to zero at the outer face and zero outside the layer), as
    (b, c, kappa) with b = exp(-(sigma/kappa + alpha) dt) and c = sigma (b - 1) / (sigma kappa + kappa^2
    alpha), c = 0 where sigma = 0."""
    poly = rho ** pml.m
    sigma = sigma_max * poly
    kappa = 1 + (pml.kappa_max - 1) * poly
    alpha = pml.alpha_max * (1 - rho) * (rho > 0)
    b = np.exp(-(sigma / kappa + alpha) * dt)
    c = np.zeros_like(rho)
    live = sigma > 0
    c[live] = sigma[live] * (b[live] - 1) / (sigma[live] * kappa[live] + kappa[live] ** 2 * alpha[live])
    return b, c, kappa


def cpml_profiles(pml, shape, spacing, dt):
    """Per axis d with a CPML: (lo_n, hi_n, {"E": (b, c, kappa), "H": (b, c, kappa)}), 1D profiles over the
    axis' node positions (E) and half-integer positions (H). A position's depth fraction is taken in whichever
    layer it lies deeper in; sigma_max = 0.8 (m + 1) / (sqrt(eps_ref) dx), with the high side's own eps_ref
    where one is given."""
    out = {}
    for d in range(3):
        lo_n, hi_n = (int(v) for v in pml.cells[d])
        if not (lo_n or hi_n):
            continue
        n, dx = shape[d], spacing[d]
        smax_lo, smax_hi = (0.8 * (pml.m + 1) / (np.sqrt(eps) * dx)
                            for eps in (pml.eps_ref, pml.eps_ref_high or pml.eps_ref))
        nodes = np.arange(n, dtype=float)
        prof = {}
        for kind, u in (("E", nodes), ("H", nodes + 0.5)):
            into_lo = _depth_fraction(lo_n - u, lo_n)
            into_hi = _depth_fraction(u - (n - 1 - hi_n), hi_n)
            sigma_max = np.where(into_lo >= into_hi, smax_lo, smax_hi)
            prof[kind] = _grading(np.maximum(into_lo, into_hi), sigma_max, pml, dt)
        out[d] = (lo_n, hi_n, prof)
    return out


def cpml_terms(pml, shape, periodic, mirror=(0, 0, 0)):
    """The CPML correction terms in lightsmith's order (``engine.py:373-418``): per axis d, per field (E then
    H), per component c != d, per side (low, high) a slab of c's stepped region restricted along d.

    Returns dicts {field, c, d, src, sgn, lo, hi, region}: ``src`` is the differentiated component, ``sgn`` the
    curl sign of the term, ``region`` the slab as three (start, stop) pairs."""
    terms = []
    for d in range(3):
        lo_n, hi_n = (int(v) for v in pml.cells[d])
        if not (lo_n or hi_n):
            continue
        if periodic[d]:
            raise ValueError("a periodic axis cannot have a PML")
        N = shape[d]
        for fld in ("E", "H"):
            for c in range(3):
                if c == d:
                    continue
                d1, d2 = (c + 1) % 3, (c + 2) % 3
                src, sgn = (d2, 1.0) if d == d1 else (d1, -1.0)
                if fld == "H":
                    sgn = -sgn
                rng = e_range if fld == "E" else h_range
                R = [rng(c, a, shape[a], periodic[a], mirror[a]) for a in range(3)]
                start, stop = R[d]
                sides = []
                if lo_n:
                    sides.append((start, min(stop, lo_n + 1)))
                if hi_n:
                    sides.append((max(start, N - 2 - hi_n), stop))
                for a, b in sides:
                    if b <= a:
                        continue
                    reg = list(R)
                    reg[d] = (a, b)
                    terms.append({"field": fld, "c": c, "d": d, "src": src, "sgn": sgn, "region": tuple(reg)})
    return terms


# --- sources -----------------------------------------------------------------------------------------


@dataclass
class TablePoints:
    """Correction points of a table-fed TF/SF box for one kind ("E": E nodes fed by H_inc, "H": the
    reverse), in application order: target flat node, first table index of its quintic stencil, integer
    and fractional fine time at n = 0, and the coefficient."""

    node: np.ndarray
    base: np.ndarray
    i0: np.ndarray
    u0: np.ndarray
    coef: np.ndarray


@dataclass
class TableSource:
    """TF/SF plane wave fed from time tables of the exact discrete background (``layered.py:254-482``)."""

    tables: np.ndarray  # flat (rows * L,)
    inc_table: np.ndarray  # flat (3 * L,)
    m: int
    cmax: int
    E: TablePoints | None
    H: TablePoints | None
    inc: tuple  # (base[3], i0[3], u0[3]) of the incident-reference view
    view: object = None  # the object DFTMonitor(source=...) names for the incident view


@dataclass
class DipoleSource:
    """Point current spread over the E nodes around it (``emission.py:97-142``): E[idx] -= coef * wave[n]."""

    idx: np.ndarray
    coef: np.ndarray
    wave: np.ndarray


@dataclass
class LinePoints:
    """1D-feed corrections of one kind: target flat node, 1D index i0, interpolation weight w (0 when the
    slab has none), coefficient; in application order (``tfsf.py:184-193``)."""

    node: np.ndarray
    i0: np.ndarray
    w: np.ndarray
    coef: np.ndarray


@dataclass
class LineSource:
    """TF/SF fed by a 1D auxiliary Yee line with graded absorbers (``tfsf.py:108-211``)."""

    M: int
    m_src: int
    ca: np.ndarray
    cb: np.ndarray
    da: np.ndarray
    db: np.ndarray
    wave: np.ndarray
    E: LinePoints | None
    H: LinePoints | None
    owner: object = None  # the object DFTMonitor(source=...) names for the line's own arrays


@dataclass
class ColumnSource:
    """One-sided TF/SF plane of a Bloch-periodic cell fed by a 3 x 3 x nz column engine with the same Bloch
    phases (``tfsf.py:214-296``)."""

    column: dict  # the column's own plan
    k_src: int
    k_launch: int
    phase: np.ndarray  # (nx, ny) complex
    amp: tuple  # two complex sheet amplitudes (E_x, E_y)
    wave: np.ndarray
    cE: float
    cH: float
    owner: object = None


@dataclass
class ModeSource:
    """Rank-r mode source on a port plane (``ports.py:294-378``): H[h] += mH @ tE[n], E[e] += mE @ tH[n]."""

    h_idx: np.ndarray
    mH: np.ndarray
    tab_E: np.ndarray
    e_idx: np.ndarray
    mE: np.ndarray
    tab_H: np.ndarray


def _points_by_slab(slabs, shape, kind, make):
    n_cells = int(np.prod(shape))
    grid = np.arange(n_cells).reshape(shape)
    rows = []
    for s in slabs:
        if s[0] != kind:
            continue
        rows.append(make(s, grid, n_cells))
    if not rows:
        return None
    return rows


def slab_boxes(node, shape) -> list[tuple]:
    """The boxes a list of flat field nodes enumerates: [(component, lo (3,), hi (3,), offset)], each box's
    nodes in row-major order starting at its offset, the boxes one after another (a table-fed source's
    correction points come slab by slab this way, ``layered.py:190-228``). Each box is grown as far as the
    list continues its pattern: along z, then rows along y, then planes along x. Raises ValueError if the
    boxes do not reproduce the list."""
    node = np.asarray(node, np.int64)
    n0, n1, n2 = (int(v) for v in shape)
    c, r = np.divmod(node, n0 * n1 * n2)
    i, r = np.divmod(r, n1 * n2)
    j, k = np.divmod(r, n2)
    boxes, e, total = [], 0, len(node)

    def same(s, length, di, dj, dk):
        """Entries s .. s + length: component c[e], at (i[e] + di, j[e] + dj, k[e] + dk + t)."""
        if s + length > total:
            return False
        sl = slice(s, s + length)
        return bool(np.all(c[sl] == c[e]) and np.all(i[sl] == i[e] + di) and np.all(j[sl] == j[e] + dj) and
                    np.array_equal(k[sl], k[e] + dk + np.arange(length)))

    while e < total:
        lz = 1
        while same(e + lz, 1, 0, 0, lz):
            lz += 1
        ly = 1
        while same(e + ly * lz, lz, 0, ly, 0):
            ly += 1
        lx = 1
        while all(same(e + (lx * ly + row) * lz, lz, lx, row, 0) for row in range(ly)):
            lx += 1
        lo = (int(i[e]), int(j[e]), int(k[e]))
        boxes.append((int(c[e]), lo, (lo[0] + lx, lo[1] + ly, lo[2] + lz), e))
        e += lx * ly * lz
    rebuilt = np.concatenate([
        flat_index(bc, *np.meshgrid(np.arange(lo[0], hi[0]), np.arange(lo[1], hi[1]), np.arange(lo[2], hi[2]),
                                    indexing="ij"), shape).reshape(-1) for bc, lo, hi, _ in boxes]) if boxes else node
    if not np.array_equal(rebuilt, node):
        raise ValueError("the nodes are not a sequence of row-major boxes")
    return boxes


def table_source_from(src, shape) -> TableSource:
    """TableSource from a constructed ``ObliqueLayeredPlaneWave`` (before ``bind``, which drops its tables).

    Its ``slabs`` are (kind, c, region, base, i0, u0, coef array, slab shape) (``layered.py:397-402``)."""
    out = {}
    for kind in ("E", "H"):
        def make(s, grid, n_cells):
            _, c, region, base, i0, u0, arr, shape_ = s
            nodes = c * n_cells + grid[region].reshape(-1)
            n = nodes.size
            return (nodes, np.broadcast_to(np.asarray(base), (n,)), np.broadcast_to(np.asarray(i0), (n,)),
                    np.broadcast_to(np.asarray(u0, dtype=float), (n,)),
                    np.broadcast_to(np.asarray(arr, dtype=float), shape_).reshape(-1))
        rows = _points_by_slab(src.slabs, shape, kind, make)
        out[kind] = None if rows is None else TablePoints(*(np.concatenate([r[j] for r in rows]) for j in range(5)))
    base, i0, u0 = src.inc
    return TableSource(tables=np.asarray(src.tables, dtype=float).reshape(-1),
                       inc_table=np.asarray(src.inc_table, dtype=float).reshape(-1), m=int(src.m),
                       cmax=int(src.cmax), E=out["E"], H=out["H"],
                       inc=(np.asarray(base, np.int64), np.asarray(i0, np.int64), np.asarray(u0, float)),
                       view=getattr(src, "view", None))


def line_source_from(src, shape) -> LineSource:
    """LineSource from a constructed ``TFSFPlaneWave``: slabs (kind, c, region, coef, i0, w, shape)
    (``tfsf.py:141-147``)."""
    out = {}
    for kind in ("E", "H"):
        def make(s, grid, n_cells):
            _, c, region, coef, i0, w, shape_ = s
            nodes = c * n_cells + grid[region].reshape(-1)
            n = nodes.size
            return (nodes, np.asarray(i0, np.int64).reshape(-1),
                    np.zeros(n) if w is None else np.asarray(w, float).reshape(-1), np.full(n, float(coef)))
        rows = _points_by_slab(src.slabs, shape, kind, make)
        out[kind] = None if rows is None else LinePoints(*(np.concatenate([r[j] for r in rows]) for j in range(4)))
    return LineSource(M=int(src.M), m_src=int(src.m_src), ca=np.asarray(src.ca, float), cb=np.asarray(src.cb, float),
                      da=np.asarray(src.da, float), db=np.asarray(src.db, float), wave=np.asarray(src.wave, float),
                      E=out["E"], H=out["H"], owner=src)


def column_source_from(src, single: bool) -> ColumnSource:
    """ColumnSource from a constructed ``BlochPlaneSource`` (``tfsf.py:227-246,256-269``)."""
    nz = src.shape[2]
    col = make_plan(shape=(3, 3, nz), dx=src.spacing, dt=src.dt, single=single,
                    inv_eps=np.full((3, 3, 3, nz), 1 / src.eps_b), groups=[], pml=src.pml, sources=[], monitors=[],
                    dft_stride=1, periodic=(True, True, False), bloch=(*src.kpar, 0.0))
    return ColumnSource(column=col, k_src=int(src.k_src), k_launch=int(src.k_launch),
                        phase=np.asarray(src.phase, complex).reshape(src.shape[0] - 2, src.shape[1] - 2),
                        amp=(complex(src.amp[0]), complex(src.amp[1])), wave=np.asarray(src.wave, float),
                        cE=src.dt / (src.eps_b * src.spacing[2]), cH=src.dt / src.spacing[2], owner=src)


def source_plan(src, shape, single: bool):
    """Plain description of one source object; raises for kinds without a CUDA implementation."""
    if isinstance(src, (TableSource, DipoleSource, LineSource, ColumnSource, ModeSource)):
        return src
    kind = type(src).__name__
    if kind == "ObliqueLayeredPlaneWave":
        return table_source_from(src, shape)
    if kind == "PointDipole":
        return DipoleSource(np.asarray(src.idx, np.int64), np.asarray(src.coef, float), np.asarray(src.wave, float))
    if kind == "TFSFPlaneWave":
        return line_source_from(src, shape)
    if kind == "BlochPlaneSource":
        return column_source_from(src, single)
    if kind == "ModeSource":
        return ModeSource(np.asarray(src.h_idx, np.int64), np.asarray(src.mH, float), np.asarray(src.tab_E, float),
                          np.asarray(src.e_idx, np.int64), np.asarray(src.mE, float), np.asarray(src.tab_H, float))
    raise NotImplementedError(f"lightsmith-b200 has no CUDA path for the source {kind}")


# --- the plan ----------------------------------------------------------------------------------------


def _media_plan(media):
    return [{"eps_inf": float(m.eps_inf), "poles": [(float(p.sigma), float(p.omega0), float(p.gamma)) for p in m.poles]}
            for m in media]


def _inv_eps(inv_eps, shape):
    a = np.asarray(inv_eps)
    if a.shape == tuple(shape):
        return a
    return np.asarray(a, dtype=float).reshape((3,) + tuple(shape))


# --- mirror-plane geometry ----------------------------------------------------------------------------
# A mirror plane normal to axis a lies on node plane 1; index 0 is its ghost plane. Reflection maps a node
# position j to 2 - j and the half-integer position of the normal E component (j + 1/2) to (1 - j) + 1/2; it
# multiplies E_c by the component's reflection sign (_parity) and a (1/eps) tensor entry (c, d) by s_c s_d,
# with s_x = -1 for x = a.


def _reflected_index(comp, j, a):
    """Index along axis a of the mirror image of E_comp's position j."""
    return np.where(comp == a, 1 - j, 2 - j)


def fold_to_stepped(comp, idx3, mirror):
    """E nodes (comp (n,), idx3 (n, 3)) on the ghost side of the mirror planes (index <= 0 along a mirror axis)
    replaced by their images on the stepped side: (idx3, sign), sign the product of the reflection signs taken,
    and 0 for a node whose image is an odd component lying on a plane (it vanishes there)."""
    idx3 = np.array(idx3, dtype=np.int64)
    comp = np.broadcast_to(np.asarray(comp), (len(idx3),))
    sign = np.ones(len(idx3), dtype=np.int64)
    for a, m in enumerate(mirror):
        if not m:
            continue
        refl = np.where(comp == a, -m, m)  # the reflection sign of E_comp, vectorised _parity("E", ...)
        ghost = idx3[:, a] <= 0
        idx3[:, a] = np.where(ghost, _reflected_index(comp, idx3[:, a], a), idx3[:, a])
        sign = sign * np.where(ghost, refl, 1)
        sign[(refl < 0) & (comp != a) & (idx3[:, a] == 1)] = 0
    return idx3, sign


def _with_mirror_twins(idx3, comp, coef, mirror):
    """The off-diagonal rows of the whole symmetric grid that the stepped part couples to: for each mirror axis
    in turn, every row not lying on the plane gains its reflected twin, whose tensor row is reflected too."""
    for a, m in enumerate(mirror):
        if not m:
            continue
        img = _reflected_index(comp, idx3[:, a], a)
        off = img != idx3[:, a]
        twin = idx3[off].copy()
        twin[:, a] = img[off]
        s_ax = np.where(np.arange(3) == a, -1.0, 1.0)
        idx3 = np.concatenate([idx3, twin])
        coef = np.concatenate([coef, coef[off] * (s_ax[comp[off]][:, None] * s_ax[None, :])])
        comp = np.concatenate([comp, comp[off]])
    return idx3, comp, coef


# --- conformal off-diagonal terms ---------------------------------------------------------------------


def _period_phase(shift, bloch, shape, spacing):
    """exp(i k . L n) for a position shifted by ``shift`` periods (..., 3) along the periodic axes, L the period
    (n - 2 real cells) per axis."""
    period = np.array([(n - 2) * h for n, h in zip(shape, spacing)], float)
    return np.exp(1j * (np.asarray(shift, float) * (np.asarray(bloch, float) * period)).sum(-1))


def _curl_taps(d, q, shape, spacing, dt):
    """The four H taps of dt (curl H)_d at E_d nodes q (Yee backward differences, as the E update takes them):
    (flat H index (4, n), weight (4, n))."""
    d1, d2 = (d + 1) % 3, (d + 2) % 3
    n = len(d)
    eye = np.eye(3, dtype=np.int64)
    inv = 1.0 / np.asarray(spacing, float)
    taps, wts = np.empty((4, n), np.int64), np.empty((4, n))
    for k, (cmp, back, sgn, ax) in enumerate(((d2, None, 1.0, d1), (d2, d1, -1.0, d1),
                                               (d1, None, -1.0, d2), (d1, d2, 1.0, d2))):
        at = q if back is None else q - eye[back]
        taps[k] = flat_index(cmp, at[:, 0], at[:, 1], at[:, 2], shape)
        wts[k] = dt * sgn * inv[ax]
    return taps, wts


def offdiag_tables(od, shape, spacing, dt, periodic, bloch, mirror, group_idx, complex_fields):
    """Gather tables of the conformal off-diagonal 1/eps terms of tensor subpixel smoothing (``OffDiagonal``,
    applied in ``engine.py:421-518, 653-655``; cubic or rectangular cells, no graded axes): (targets (n,),
    h (n, W), w (n, W)); row r adds sum_k w[r, k] H_flat[h[r, k]] to E_flat[targets[r]] after the E curl
    update, one row per target node.

    The tables are one merged sparse operator, built in two products. First the E-to-E coupling K: the row of
    E_c at node p couples to D_d (the time integral of curl_d H) at the four E_d nodes q on the cell edges
    around p, entered in both directions, (1/eps)_cd(p) / 8 from q to p and its conjugate from p to q, so that
    K is Hermitian (periodic axes wrap q onto the real cells with the Bloch phase of the period crossed; along
    other axes q must be an E_d node inside the grid). Mirror planes extend the rows by their reflected twins;
    targets on the ghost side are dropped and ghost-side sources act through their stepped images with their
    reflection signs. Couplings touching a dispersive node are dropped. Then K times the curl: every source
    D_d(q) is replaced by its four H taps with dt / dx along each difference's axis, and entries with the same
    (target, H node) are summed, so each H value is read once per target."""
    shape = tuple(int(n) for n in shape)
    nflat = 3 * int(np.prod(shape))
    idx3 = np.asarray(od.idx3, np.int64)
    comp = np.asarray(od.comp, np.int64)
    coef = np.asarray(od.coef, float)
    if any(mirror):
        idx3, comp, coef = _with_mirror_twins(idx3, comp, coef, mirror)
    eye = np.eye(3, dtype=np.int64)
    pairs = []  # (target comp, target idx3, source comp, source idx3, value)
    for d in range(3):
        rows = np.nonzero((comp != d) & (coef[:, d] != 0))[0]
        p, c, o = idx3[rows], comp[rows], coef[rows, d]
        for along_c in (0, 1):
            for back_d in (0, 1):
                q = p + eye[c] * along_c
                q[:, d] -= back_d
                shift = np.zeros(q.shape, np.int64)
                inside = np.ones(len(q), bool)
                for a in range(3):
                    n = shape[a]
                    if periodic[a]:  # ghost planes 0 and n-1 stand for the real planes n-2 and 1
                        shift[:, a] = (q[:, a] == n - 1).astype(np.int64) - (q[:, a] == 0)
                        q[:, a] -= shift[:, a] * (n - 2)
                    else:
                        lo, hi = e_range(d, a, n, False)
                        inside &= (q[:, a] < hi) & ((q[:, a] >= lo) | bool(mirror[a]))
                kq = o[inside] * _period_phase(shift[inside], bloch, shape, spacing)
                dd = np.full(int(inside.sum()), d)
                pairs.append((c[inside], p[inside], dd, q[inside], kq / 8))
                pairs.append((dd, q[inside], c[inside], p[inside], np.conj(kq) / 8))
    tc, ti, sc, si, v = (np.concatenate([x[k] for x in pairs]) for k in range(5))
    if any(mirror):
        tf, t_sign = fold_to_stepped(tc, ti, mirror)
        si, s_sign = fold_to_stepped(sc, si, mirror)
        keep = (np.all(tf == ti, axis=1) & (t_sign != 0) & (s_sign != 0) &
                np.all(si < np.asarray(shape) - 1, axis=1))
        tc, ti, sc, si, v = tc[keep], ti[keep], sc[keep], si[keep], v[keep] * s_sign[keep]
    t = flat_index(tc, ti[:, 0], ti[:, 1], ti[:, 2], shape)
    src = flat_index(sc, si[:, 0], si[:, 1], si[:, 2], shape)
    if len(group_idx):
        keep = ~(np.isin(t, group_idx) | np.isin(src, group_idx))
        t, sc, si, v = t[keep], sc[keep], si[keep], v[keep]
    if not len(t):
        return None
    taps, wts = _curl_taps(sc, si, shape, spacing, dt)
    key = (np.repeat(t[None], 4, 0) * nflat + taps).ravel()
    val = (wts * v[None]).ravel()
    key, inv = np.unique(key, return_inverse=True)
    merged = np.bincount(inv, val.real, len(key)) + 1j * np.bincount(inv, val.imag, len(key))
    nz = merged != 0
    key, merged = key[nz], merged[nz]
    if not len(key):
        return None
    tgt, hh = key // nflat, key % nflat
    targets, first, count = np.unique(tgt, return_index=True, return_counts=True)
    width = int(count.max())
    slot = np.arange(len(tgt)) - np.repeat(first, count)
    row = np.repeat(np.arange(len(targets)), count)
    h = np.zeros((len(targets), width), np.int64)  # padding: index 0 with weight 0
    w = np.zeros((len(targets), width), complex)
    h[row, slot], w[row, slot] = hh, merged
    return targets.astype(np.int64), h, (w if complex_fields else w.real)


def tensor_plan(tm, shape, spacing, bloch, complex_fields) -> dict:
    """The vertex-tensor ADE of conformal interfaces with dispersive media (``TensorMesh``, ``_Tensor``,
    ``engine.py:140-175, 838-923``) as flat index tables, cubic or rectangular cells (no graded axes).

    Per step: each node's D += E - E_prev; per vertex v the mean D~ of its two d-nodes for every d (their
    values times a Bloch phase and mirror parity, ``scale``) and s = n . D~; per tensor slot (a node next to
    v) sigma = s + n_c (D_p - D~_c) and out = (1/2) (b[D_p - n_c sigma] + n_c a[sigma]) (times the conjugate
    phase under a Bloch wavevector), a (``_Harmonic``) and b (``_Arithmetic``) with their own pole states and
    the vertex's medium fractions; per plain slot out = (1/2) medium[D] of its one medium; a node's E is the sum
    of its two slots."""
    n_nodes = len(tm.node_comp)
    idx = np.asarray(tm.idx, np.int64)
    ph = _period_phase(tm.shift, bloch, shape, spacing)  # per vertex, d and side: (nV, 3, 2)
    parity = np.ones(ph.shape) if tm.sign is None else np.asarray(tm.sign, float)
    scale = ph * parity if complex_fields else parity
    sv = np.asarray(tm.slot_vert)
    tk, tnode = np.nonzero((sv >= 0).T)  # slots ordered (k, node)
    tv = sv[tnode, tk]
    tc = np.asarray(tm.node_comp)[tnode]
    side = 1 - tk
    nrm = np.asarray(tm.normal, float)
    pk, pnode = np.nonzero((sv < 0).T)
    out = {"idx": idx, "n_nodes": n_nodes, "vn": np.asarray(tm.vert_nodes, np.int64).reshape(-1),
           "normal": nrm.reshape(-1), "t_pos": (tk * n_nodes + tnode).astype(np.int64), "t_v": tv.astype(np.int64),
           "t_vc": (tv * 3 + tc).astype(np.int64), "t_g": ((tv * 3 + tc) * 2 + side).astype(np.int64),
           "t_nc": nrm[tv, tc], "frac": np.asarray(tm.frac, float)[:, tv],
           "p_pos": (pk * n_nodes + pnode).astype(np.int64), "p_node": pnode.astype(np.int64),
           "p_medium": np.asarray(tm.slot_medium, np.int64)[pnode, pk], "media": _media_plan(tm.media)}
    scaled = complex_fields or tm.sign is not None
    out["scale"] = (scale.reshape(-1) if complex_fields else scale.real.reshape(-1)) if scaled else None
    out["t_conj"] = np.conj(ph[tv, tc, side]) if complex_fields else None
    return out


def make_plan(*, shape, dx, dt, single, inv_eps, groups, pml, sources, monitors, dft_stride,
              periodic=(False, False, False), bloch=(0.0, 0.0, 0.0), offdiag=None, time_monitors=(),
              mirror=(0, 0, 0), widths=None) -> dict:
    """The plan of lightsmith's ``Engine(...)`` keyword arguments (``engine.py:231-241``).

    Graded grids and the conformal off-diagonal / vertex-tensor terms have no CUDA path here and are rejected.
    Mirror planes (``mirror`` per axis: +1 symmetric, -1 antisymmetric, at node 1) are kept."""
    shape = tuple(int(n) for n in shape)
    spacing = tuple(float(v) for v in np.broadcast_to(np.asarray(dx, dtype=float), (3,)))
    if widths is not None and any(w is not None for w in widths):
        raise NotImplementedError("graded grids have no CUDA path in lightsmith-b200")
    mirror = tuple(int(np.sign(m)) for m in mirror)
    for a, m in enumerate(mirror):  # engine.py:259-261
        if m and (bool(periodic[a]) or int(pml.cells[a][0])):
            raise ValueError("a mirror plane needs a non-periodic axis without PML on its low side")
    if time_monitors:
        raise NotImplementedError("time monitors have no CUDA path in lightsmith-b200")
    periodic = tuple(bool(p) for p in periodic)
    bloch = tuple(float(k) for k in bloch)
    if any(k and not p for k, p in zip(bloch, periodic)):
        raise ValueError("a Bloch wavevector needs a periodic axis")
    grp, tensor = [], None
    for g in groups:
        if type(g).__name__ == "TensorMesh":
            if tensor is not None:
                raise NotImplementedError("more than one vertex-tensor mesh")
            tensor = g
            continue
        grp.append({"idx": np.asarray(g.idx, np.int64), "media": _media_plan(g.media),
                    "frac": np.asarray(g.frac, float), "w": None if g.w is None else np.asarray(g.w, float)})
    plan = {
        "shape": shape, "spacing": spacing, "dt": float(dt), "single": bool(single), "periodic": periodic,
        "bloch": bloch, "complex": any(bloch), "stride": int(dft_stride),
        # (3, N0, N1, N2) per component, or (N0, N1, N2) when eps is isotropic everywhere
        "inv_eps": _inv_eps(inv_eps, shape),
        "pml": {"cells": tuple(tuple(int(v) for v in c) for c in pml.cells), "m": float(pml.m),
                "kappa_max": float(pml.kappa_max), "alpha_max": float(pml.alpha_max), "eps_ref": float(pml.eps_ref),
                "eps_ref_high": None if pml.eps_ref_high is None else float(pml.eps_ref_high)},
        "groups": grp,
        "sources": [source_plan(s, shape, single) for s in sources],
    }
    if any(mirror):  # only then (plans without mirror planes keep their earlier form)
        plan["mirror"] = mirror
    if tensor is not None:
        plan["tensor"] = tensor_plan(tensor, shape, spacing, bloch, any(bloch))
    if offdiag is not None and len(getattr(offdiag, "comp", ())):
        gidx = [g["idx"] for g in grp] + ([plan["tensor"]["idx"]] if tensor is not None else [])
        gidx = np.concatenate(gidx) if gidx else np.zeros(0, np.int64)
        tab = offdiag_tables(offdiag, shape, spacing, dt, periodic, bloch, mirror, gidx, any(bloch))
        if tab is not None:
            plan["offdiag"] = {"e": tab[0], "h": tab[1], "w": tab[2]}
    mons = []
    for m in monitors:
        space = _monitor_space(m.source, sources, plan["sources"])
        mons.append({"omega": np.asarray(m.omega, float), "e_idx": np.asarray(m.e_idx, np.int64),
                     "h_idx1": None if m.h_idx1 is None else np.asarray(m.h_idx1, np.int64),
                     "h_idx2": None if m.h_idx2 is None else np.asarray(m.h_idx2, np.int64),
                     "energy": int(m.energy), "space": space})
    plan["monitors"] = mons
    return plan


# --- rows padded for the tensor-memory copies -----------------------------------------------------------
# The fused pass moves planes with tensor-memory (TMA) copies, whose row stride must be a multiple of 16 bytes;
# lightsmith's scattering layouts are odd along every axis (setup.py:640). pad_rows appends planes along z so
# that a row of nodes is a multiple of `multiple` values, and freezes them: every E component from z = n2 - 1
# on (where lightsmith steps none: e_range) gets a zero curl coefficient, so it keeps its zero start value, and
# H there, whose every difference then reads zeros, stays zero too. The high z CPML slab keeps its start (the
# engine widens it over the new planes, where its profile is b = 0, c = 0, kappa = 1, so psi stays zero), and
# every flat index of the plan is moved to the wider rows. The run's values on the original nodes are then
# the original run's.


def _remap_flat(idx, shape, n2p):
    """Flat indices (component-stacked, c * N + (x * n1 + y) * n2 + z) of a grid of `shape` on rows of n2p."""
    a = np.asarray(idx, np.int64)
    n0, n1, n2 = shape
    N = n0 * n1 * n2
    c, rest = np.divmod(a, N)
    xy, z = np.divmod(rest, n2)
    return c * (n0 * n1 * n2p) + xy * n2p + z


def pad_rows(plan: dict, multiple: int = 4) -> dict:
    """The plan on rows padded to a multiple of `multiple` nodes along z (the plan itself when its rows are
    already, or when it has complex fields, periodic axes or a z mirror plane, or already padded)."""
    n0, n1, n2 = (int(v) for v in plan["shape"])
    n2p = -(-n2 // multiple) * multiple
    if (n2p == n2 or plan["complex"] or any(plan["periodic"]) or plan.get("mirror", (0, 0, 0))[2]
            or plan.get("pad_z")):
        return plan
    shape = (n0, n1, n2)

    def rm(a):
        return None if a is None else _remap_flat(a, shape, n2p)

    out = dict(plan)
    out["shape"] = (n0, n1, n2p)
    out["pad_z"] = n2p - n2
    inv = np.asarray(plan["inv_eps"])
    pad = [(0, 0)] * (inv.ndim - 1) + [(0, n2p - n2)]
    inv = np.pad(inv, pad).astype(inv.dtype, copy=False)
    inv[..., n2 - 1:] = 0
    out["inv_eps"] = inv
    out["groups"] = [{**g, "idx": rm(g["idx"])} for g in plan["groups"]]
    srcs = []
    for src in plan["sources"]:
        if isinstance(src, DipoleSource):
            src = replace(src, idx=rm(src.idx))
        elif isinstance(src, TableSource):
            src = replace(src, E=None if src.E is None else replace(src.E, node=rm(src.E.node)),
                          H=None if src.H is None else replace(src.H, node=rm(src.H.node)))
        elif isinstance(src, LineSource):
            src = replace(src, E=None if src.E is None else replace(src.E, node=rm(src.E.node)),
                          H=None if src.H is None else replace(src.H, node=rm(src.H.node)))
        elif isinstance(src, ModeSource):
            src = replace(src, h_idx=rm(src.h_idx), e_idx=rm(src.e_idx))
        else:
            raise NotImplementedError(f"pad_rows: no row padding for the source {type(src).__name__}")
        srcs.append(src)
    out["sources"] = srcs
    if plan.get("tensor") is not None:
        out["tensor"] = {**plan["tensor"], "idx": rm(plan["tensor"]["idx"])}
    if plan.get("offdiag") is not None:
        od = plan["offdiag"]
        out["offdiag"] = {**od, "e": rm(od["e"]), "h": rm(od["h"])}
    mons = []
    for m in plan["monitors"]:
        if m["space"][0] == "grid":
            m = {**m, "e_idx": rm(m["e_idx"]), "h_idx1": rm(m["h_idx1"]), "h_idx2": rm(m["h_idx2"])}
        mons.append(m)
    out["monitors"] = mons
    return out


def _monitor_space(obj, sources, plans):
    """("grid",) or (kind, source number): which arrays a monitor samples."""
    if obj is None:
        return ("grid", -1)
    for i, (s, p) in enumerate(zip(sources, plans)):
        if isinstance(p, TableSource) and (obj is p.view or obj is getattr(s, "view", None)):
            return ("view", i)
        if isinstance(p, (LineSource, ColumnSource)) and (obj is s or obj is p.owner):
            return ("line" if isinstance(p, LineSource) else "column", i)
    raise NotImplementedError(f"a monitor samples {type(obj).__name__}, which has no CUDA path")


# --- (de)serialisation -------------------------------------------------------------------------------


def _flatten(obj, prefix, arrays):
    """JSON skeleton of obj with its arrays moved into `arrays` under path-like keys."""
    if isinstance(obj, np.ndarray):
        key = prefix or "root"
        arrays[key] = obj
        return {"__array__": key}
    if isinstance(obj, dict):
        return {k: _flatten(v, f"{prefix}/{k}", arrays) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return {"__seq__": type(obj).__name__, "items": [_flatten(v, f"{prefix}/{i}", arrays) for i, v in enumerate(obj)]}
    if isinstance(obj, complex):
        return {"__complex__": [obj.real, obj.imag]}
    for cls in (TableSource, TablePoints, DipoleSource, LineSource, LinePoints, ColumnSource, ModeSource):
        if isinstance(obj, cls):
            d = {k: v for k, v in obj.__dict__.items() if k not in ("view", "owner")}
            return {"__class__": cls.__name__, "fields": _flatten(d, prefix, arrays)}
    if isinstance(obj, (np.integer,)):
        return int(obj)
    if isinstance(obj, (np.floating,)):
        return float(obj)
    if isinstance(obj, np.bool_):
        return bool(obj)
    return obj


_CLASSES = {c.__name__: c for c in (TableSource, TablePoints, DipoleSource, LineSource, LinePoints, ColumnSource,
                                     ModeSource)}


def _unflatten(obj, arrays):
    if isinstance(obj, dict):
        if "__array__" in obj:
            return np.asarray(arrays[obj["__array__"]])
        if "__seq__" in obj:
            items = [_unflatten(v, arrays) for v in obj["items"]]
            return tuple(items) if obj["__seq__"] == "tuple" else items
        if "__complex__" in obj:
            return complex(*obj["__complex__"])
        if "__class__" in obj:
            return _CLASSES[obj["__class__"]](**_unflatten(obj["fields"], arrays))
        return {k: _unflatten(v, arrays) for k, v in obj.items()}
    return obj


def dumps(tree) -> dict:
    """A dict of arrays (for ``np.savez_compressed``) holding `tree` (plans, results, nested dicts)."""
    arrays = {}
    skel = _flatten(tree, "", arrays)
    arrays["__skeleton__"] = np.frombuffer(json.dumps(skel).encode(), dtype=np.uint8)
    return arrays


def loads(arrays) -> dict:
    skel = json.loads(bytes(np.asarray(arrays["__skeleton__"])).decode())
    return _unflatten(skel, arrays)


def save(path, tree) -> None:
    np.savez_compressed(path, **dumps(tree))


def load(path) -> dict:
    with np.load(path, allow_pickle=False) as z:
        return loads({k: z[k] for k in z.files})


def to_bytes(tree) -> bytes:
    buf = io.BytesIO()
    np.savez_compressed(buf, **dumps(tree))
    return buf.getvalue()
