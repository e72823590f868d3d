"""CPU oracle: a NumPy restatement of lightsmith's FDTD time step, used as the checker for the CUDA engine.

TEST INFRASTRUCTURE ONLY. Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this package; the product path never calls it.

It follows ``backends/_fdtd/engine.py`` of lightsmith v0.3.0 (cited per function) and consumes the same plan
(``lightsmith_b200.plan``) as the CUDA engine. It is pinned against golden vectors produced by lightsmith's
own ``Engine`` in ``tests/golden/`` (``tests/test_oracle_golden.py``).

``threads`` splits every field update into x slabs run on a thread pool (NumPy releases the GIL inside its
ufuncs); the per-cell arithmetic and its order are unchanged, so results do not depend on it.
"""

from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np

from lightsmith_b200.plan import (ColumnSource, DipoleSource, LineSource, ModeSource, TableSource, cpml_profiles,
                                  cpml_terms, e_range, h_range, pole_coefficients)

# quintic Lagrange stencil of the table reads (layered.py:164-165)
STENCIL = np.arange(-2, 4)
DENOM = [float(np.prod([xj - xk for xk in STENCIL if xk != xj])) for xj in STENCIL]


def _sl(r):
    return slice(r[0], r[1])


class OracleEngine:
    """One run of the plan on the CPU in float64 (complex128 under a Bloch phase), or float32 when
    ``dtype=np.float32`` (the reference GPU precision)."""

    def __init__(self, plan: dict, dtype=np.float64, threads: int = 1):
        self.plan = plan
        self.shape = tuple(plan["shape"])
        self.spacing = tuple(plan["spacing"])
        self.dt = plan["dt"]
        self.periodic = tuple(plan["periodic"])
        self.bloch = tuple(plan["bloch"])
        self.complex = bool(plan["complex"])
        self.rdt = np.dtype(dtype)
        self.fdt = np.dtype(np.complex128 if self.rdt == np.float64 else np.complex64) if self.complex else self.rdt
        self.stride = int(plan["stride"])
        self.uniform = len(set(self.spacing)) == 1
        self.threads = max(1, int(threads))
        self._pool = ThreadPoolExecutor(self.threads) if self.threads > 1 else None
        n0, n1, n2 = self.shape
        self.E = np.zeros((3, n0, n1, n2), self.fdt)
        self.H = np.zeros((3, n0, n1, n2), self.fdt)
        self.n = 0
        P = self.periodic
        M = self.mirror = tuple(plan.get("mirror", (0, 0, 0)))
        self.RE = [tuple(e_range(c, a, self.shape[a], P[a], M[a]) for a in range(3)) for c in range(3)]
        self.RH = [tuple(h_range(c, a, self.shape[a], P[a], M[a]) for a in range(3)) for c in range(3)]
        # symmetric (PMC) mirror planes: tangential H's ghost plane 0 is minus its image, plane 1, before every
        # E update (engine.py:290-298, 649-650)
        self._mirror_ghosts = []
        for a, m in enumerate(M):
            if m > 0:
                for t in range(3):
                    if t != a:
                        g, s = [slice(None)] * 3, [slice(None)] * 3
                        g[a], s[a] = slice(0, 1), slice(1, 2)
                        self._mirror_ghosts.append((t, tuple(g), tuple(s)))
        # uniform cubic cells fold dt/dx into the coefficients; otherwise differences are scaled by 1/d_axis and
        # the coefficients carry dt alone (engine.py:274-276, 622-627)
        cdx = self.dt / self.spacing[0] if self.uniform else self.dt
        inv_eps = plan["inv_eps"]
        if inv_eps.ndim == 3:  # isotropic: one array for every component
            inv_eps = np.broadcast_to(inv_eps, (3,) + inv_eps.shape)
        self.cbE = [np.asarray(cdx * inv_eps[c][tuple(_sl(r) for r in self.RE[c])], self.rdt) for c in range(3)]
        self.cH = cdx
        self.inv_d = tuple(1.0 / d for d in self.spacing)
        self._build_pml(inv_eps, cdx)
        self.groups = [_Group(self, g) for g in plan["groups"]]
        if plan.get("tensor") is not None:  # the vertex-tensor mesh steps after the D-form groups
            self.groups.append(_TensorMesh(self, plan["tensor"]))
        self.sources = [self._bind_source(s) for s in plan["sources"]]
        self.monitors = []
        for m in plan["monitors"]:
            nf = len(m["omega"])
            acc_e = np.zeros((nf, len(m["e_idx"])), np.complex128)
            acc_h = None if m["h_idx1"] is None else np.zeros((nf, len(m["h_idx1"])), np.complex128)
            self.monitors.append({**m, "acc_e": acc_e, "acc_h": acc_h})
        self.energy = np.zeros(2)

    # --- CPML (engine.py:344-418) ---------------------------------------------------------------------
    def _build_pml(self, inv_eps, cdx):
        prof = cpml_profiles(_Spec(self.plan["pml"]), self.shape, self.spacing, self.dt)
        self.pml = {"E": [], "H": []}
        for t in cpml_terms(_Spec(self.plan["pml"]), self.shape, self.periodic, self.mirror):
            d, fld = t["d"], t["field"]
            a, b = t["region"][d]
            bb, cc, kk = (v[a:b] for v in prof[d][2][fld])
            bshape = [1, 1, 1]
            bshape[d] = b - a
            reg = tuple(_sl(r) for r in t["region"])
            scale = cdx * inv_eps[t["c"]][reg] if fld == "E" else np.full([r[1] - r[0] for r in t["region"]], cdx)
            if not self.uniform:
                scale = scale / self.spacing[d]
            cprime = t["sgn"] * scale * cc.reshape(bshape)
            kprime = t["sgn"] * scale * (1 / kk - 1).reshape(bshape) if np.any(kk > 1) else None
            self.pml[fld].append({**t, "reg": reg, "b": np.asarray(bb.reshape(bshape), self.rdt),
                                  "cp": np.asarray(cprime, self.rdt),
                                  "kp": None if kprime is None else np.asarray(kprime, self.rdt),
                                  "psi": np.zeros(cprime.shape, self.fdt)})

    # --- sources ----------------------------------------------------------------------------------------
    def _bind_source(self, s):
        if isinstance(s, TableSource):
            return _Table(self, s)
        if isinstance(s, DipoleSource):
            return _Dipole(self, s)
        if isinstance(s, LineSource):
            return _Line(self, s)
        if isinstance(s, ColumnSource):
            return _Column(self, s)
        if isinstance(s, ModeSource):
            return _Mode(self, s)
        raise TypeError(type(s))

    # --- helpers ------------------------------------------------------------------------------------------
    def _xchunks(self, lo, hi):
        if self._pool is None or hi - lo < 2 * self.threads:
            return [(lo, hi)]
        cuts = np.linspace(lo, hi, self.threads + 1).astype(int)
        return [(int(a), int(b)) for a, b in zip(cuts[:-1], cuts[1:]) if b > a]

    def _parallel(self, fn, lo, hi):
        chunks = self._xchunks(lo, hi)
        if len(chunks) == 1:
            fn(*chunks[0])
        else:
            list(self._pool.map(lambda ab: fn(*ab), chunks))

    # --- periodic ghosts (engine.py:595-611) ---------------------------------------------------------------
    def _ghosts(self, F, low: bool):
        for a, per in enumerate(self.periodic):
            if not per:
                continue
            n = self.shape[a]
            dst, src = (0, n - 2) if low else (n - 1, 1)
            ix_d = [slice(None)] * 4
            ix_s = [slice(None)] * 4
            ix_d[a + 1], ix_s[a + 1] = slice(dst, dst + 1), slice(src, src + 1)
            k = self.bloch[a]
            if k:
                kl = k * (n - 2) * self.spacing[a] * (-1 if low else 1)
                F[tuple(ix_d)] = F[tuple(ix_s)] * complex(np.cos(kl), np.sin(kl))
            else:
                F[tuple(ix_d)] = F[tuple(ix_s)]

    # --- curl updates (engine.py:613-663) -----------------------------------------------------------------
    def _curl_part(self, F, c, R, forward: bool, coef):
        """coef * (difference of F_{d2} along d1 - difference of F_{d1} along d2) over region R (slices)."""
        d1, d2 = (c + 1) % 3, (c + 2) % 3

        def sh(R, d, s):
            R = list(R)
            R[d] = slice(R[d].start + s, R[d].stop + s)
            return tuple(R)
        if forward:
            a = F[d2][sh(R, d1, 1)] - F[d2][R]
            b = F[d1][sh(R, d2, 1)] - F[d1][R]
        else:
            a = F[d2][R] - F[d2][sh(R, d1, -1)]
            b = F[d1][R] - F[d1][sh(R, d2, -1)]
        if not self.uniform:
            a = a * self.inv_d[d1]
            b = b * self.inv_d[d2]
        return (a - b) * coef

    def _update(self, kind: str, x0: int, x1: int):
        """Bulk curl update then the CPML terms of one field over the x planes [x0, x1)."""
        E, H = self.E, self.H
        tgt, src = (H, E) if kind == "H" else (E, H)
        regions = self.RH if kind == "H" else self.RE
        for c in range(3):
            R = regions[c]
            lo, hi = max(R[0][0], x0), min(R[0][1], x1)
            if hi <= lo:
                continue
            Rs = (slice(lo, hi), _sl(R[1]), _sl(R[2]))
            if kind == "H":
                tgt[c][Rs] -= self._curl_part(src, c, Rs, True, self.cH)
            else:
                coef = self.cbE[c][lo - R[0][0]:hi - R[0][0]]
                tgt[c][Rs] += self._curl_part(src, c, Rs, False, coef)
        for t in self.pml[kind]:
            reg = t["reg"]
            lo, hi = max(reg[0].start, x0), min(reg[0].stop, x1)
            if hi <= lo:
                continue
            o0, o1 = lo - reg[0].start, hi - reg[0].start
            R = (slice(lo, hi), reg[1], reg[2])
            d, s = t["d"], t["src"]
            Rp = list(R)
            if kind == "H":
                Rp[d] = slice(R[d].start + 1, R[d].stop + 1)
                der = src[s][tuple(Rp)] - src[s][R]
            else:
                Rp[d] = slice(R[d].start - 1, R[d].stop - 1)
                der = src[s][R] - src[s][tuple(Rp)]
            # psi, c' and k' are slab-shaped; b is a profile along d only
            psi = t["psi"][o0:o1]
            b = t["b"][o0:o1] if d == 0 else t["b"]
            psi *= b
            if t["kp"] is not None:
                tgt[t["c"]][R] += t["kp"][o0:o1] * der
            psi += der * t["cp"][o0:o1]
            tgt[t["c"]][R] += psi

    def update_H(self):
        if any(self.periodic):
            self._ghosts(self.E, low=False)
        self._parallel(lambda a, b: self._update("H", a, b), 0, self.shape[0])

    def update_E(self):
        if any(self.periodic):
            self._ghosts(self.H, low=True)
        for t, g, s in self._mirror_ghosts:
            self.H[t][g] = -self.H[t][s]
        self._parallel(lambda a, b: self._update("E", a, b), 0, self.shape[0])
        od = self.plan.get("offdiag")
        if od is not None:  # conformal off-diagonal terms (engine.py:653-655; added here after the CPML terms,
            # which changes only the order of the additions)
            Ef, Hf = self.E.reshape(-1), self.H.reshape(-1)
            Ef[od["e"]] += np.sum(np.asarray(od["w"]) * Hf[od["h"]], axis=1)

    # --- step order (engine.py:665-683) -----------------------------------------------------------------
    def step(self):
        self.update_H()
        for s in self.sources:
            s.correct_H()
        for s in self.sources:
            s.advance_H()
        self.update_E()
        for s in self.sources:
            s.correct_E()
        for g in self.groups:
            g.step()
        for s in self.sources:
            s.advance_E()
        self.n += 1

    def chunk(self):
        for _ in range(self.stride):
            self.step()
        self.sample()

    # --- DFT monitors (engine.py:564-592) ---------------------------------------------------------------
    def _arrays(self, space):
        kind, i = space
        if kind == "grid":
            return self.E.reshape(-1), self.H.reshape(-1)
        s = self.sources[i]
        return s.E_flat, s.H_flat

    def sample(self):
        t_e = float(self.n) * self.dt
        t_h = t_e - 0.5 * self.dt
        energy = [None, None]
        for m in self.monitors:
            ef, hf = self._arrays(m["space"])
            se = ef[m["e_idx"]].astype(np.complex128)
            wt = m["omega"] * t_e
            m["acc_e"] += (np.cos(wt) + 1j * np.sin(wt))[:, None] * se[None, :]
            if m["acc_h"] is not None:
                sh = 0.5 * (hf[m["h_idx1"]] + hf[m["h_idx2"]])
                wt = m["omega"] * t_h
                m["acc_h"] += (np.cos(wt) + 1j * np.sin(wt))[:, None] * sh.astype(np.complex128)[None, :]
                if m["energy"]:
                    if np.iscomplexobj(sh):
                        v = float(np.sum((se * np.conj(se)).real) + np.sum((sh * np.conj(sh)).real))
                    else:
                        se_r = ef[m["e_idx"]]
                        v = float(np.sum(se_r * se_r) + np.sum(sh * sh))
                    g = int(m["energy"]) - 1
                    energy[g] = v if energy[g] is None else energy[g] + v
        for g, v in enumerate(energy):
            if v is not None:
                self.energy[g] = v

    def results(self, k: int):
        m = self.monitors[k]
        return m["acc_e"], m["acc_h"]

    def close(self):
        if self._pool is not None:
            self._pool.shutdown()


class _Spec:
    """Attribute view of the plan's CPML dict."""

    def __init__(self, d):
        self.__dict__.update(d)


# --- dispersive groups (engine.py:722-793) -------------------------------------------------------------


class _Group:
    """D-form ADE: D += E - E_prev; poles P^{n+1} = c1 P^n + c2 P^{n-1} + c3 E_drive; E = (D - sum P)/eps_inf.
    Mixed (subpixel) nodes run a harmonic path (per medium s its own E_s driving its poles) and an arithmetic
    path (all poles driven by E_a), E = w harm + (1 - w) E_a."""

    def __init__(self, eng: OracleEngine, g: dict):
        self.eng = eng
        self.idx = np.asarray(g["idx"], np.int64)
        n = len(self.idx)
        z = lambda: np.zeros(n, eng.fdt)  # noqa: E731
        self.D, self.E_prev = z(), z()
        media = g["media"]
        dt = eng.dt
        coefs = [[pole_coefficients(_P(*p), dt) for p in m["poles"]] for m in media]
        self.coef = coefs
        self.pure = g["w"] is None
        if self.pure:
            (m,) = media
            self.inv_inf = 1.0 / m["eps_inf"]
            self.P = [(z(), z()) for _ in m["poles"]]
            return
        f = np.asarray(g["frac"], float)
        disp = [s for s, m in enumerate(media) if m["poles"]]
        self.disp = disp
        self.h0 = sum(f[s] / m["eps_inf"] for s, m in enumerate(media) if not m["poles"]) + 0 * f[0]
        self.f = {s: f[s] for s in disp}
        self.inv_inf_s = {s: 1.0 / media[s]["eps_inf"] for s in disp}
        self.inv_a = 1.0 / sum(f[s] * m["eps_inf"] for s, m in enumerate(media))
        self.w = np.asarray(g["w"], float)
        self.has_h, self.has_a = bool(np.any(self.w > 0)), bool(np.any(self.w < 1))
        self.Eh = {s: z() for s in disp}
        self.Ea = z()
        self.Ph = {s: [(z(), z()) for _ in media[s]["poles"]] for s in disp}
        self.Pa = {s: [(z(), z()) for _ in media[s]["poles"]] for s in disp}
        rd = eng.rdt
        self.h0, self.inv_a, self.w = (np.asarray(v, rd) for v in (self.h0, self.inv_a, self.w))
        self.f = {s: np.asarray(v, rd) for s, v in self.f.items()}

    @staticmethod
    def _poles(pairs, coefs, drive):
        tot = None
        for (P, Pp), (c1, c2, c3) in zip(pairs, coefs):
            new = c1 * P + c2 * Pp + c3 * drive
            Pp[...] = P
            P[...] = new
            tot = P.copy() if tot is None else tot + P
        return tot

    def step(self):
        Ef = self.eng.E.reshape(-1)
        e_now = Ef[self.idx]
        self.D += e_now - self.E_prev
        if self.pure:
            tot = self._poles(self.P, self.coef[0], self.E_prev)
            e_new = (self.D - tot) * self.inv_inf
        else:
            parts = []
            if self.has_h:
                harm = self.D * self.h0
                for s in self.disp:
                    tot = self._poles(self.Ph[s], self.coef[s], self.Eh[s])
                    self.Eh[s][...] = (self.D - tot) * self.inv_inf_s[s]
                    harm = harm + self.f[s] * self.Eh[s]
                parts.append(self.w * harm)
            if self.has_a:
                acc = self.D
                for s in self.disp:
                    tot = self._poles(self.Pa[s], self.coef[s], self.Ea)
                    acc = acc - self.f[s] * tot
                self.Ea[...] = acc * self.inv_a
                parts.append((1 - self.w) * self.Ea)
            e_new = parts[0] if len(parts) == 1 else parts[0] + parts[1]
        Ef[self.idx] = e_new
        self.E_prev[...] = e_new


class _Harmonic:
    """<1/eps>[u] over slots with medium fractions F (S, n) (engine.py:796-818): y = sum_s F_s E_s with
    E_s = (u - P_s) / eps_inf_s, each dispersive medium's poles driven by its own E_s of the step before."""

    def __init__(self, eng, media, F):
        n = F.shape[1]
        self.h0 = sum(F[s] / m["eps_inf"] for s, m in enumerate(media) if not m["poles"]) + 0 * F[0]
        self.disp = [s for s, m in enumerate(media) if m["poles"] and np.any(F[s] > 0)]
        self.f = {s: F[s] for s in self.disp}
        self.inv = {s: 1.0 / media[s]["eps_inf"] for s in self.disp}
        self.coef = {s: [pole_coefficients(_P(*p), eng.dt) for p in media[s]["poles"]] for s in self.disp}
        z = lambda: np.zeros(n, eng.fdt)  # noqa: E731
        self.E = {s: z() for s in self.disp}
        self.P = {s: [(z(), z()) for _ in media[s]["poles"]] for s in self.disp}

    def __call__(self, u):
        y = u * self.h0
        for s in self.disp:
            tot = _Group._poles(self.P[s], self.coef[s], self.E[s])
            self.E[s][...] = (u - tot) * self.inv[s]
            y = y + self.f[s] * self.E[s]
        return y


class _Arithmetic:
    """(1/<eps>)[u] (engine.py:820-835): y = (u - sum_s F_s P_s) / sum_s F_s eps_inf_s, every pole driven by the
    y of the step before."""

    def __init__(self, eng, media, F):
        n = F.shape[1]
        self.disp = [s for s, m in enumerate(media) if m["poles"] and np.any(F[s] > 0)]
        self.f = {s: F[s] for s in self.disp}
        self.inv_a = 1.0 / sum(F[s] * m["eps_inf"] for s, m in enumerate(media))
        self.coef = {s: [pole_coefficients(_P(*p), eng.dt) for p in media[s]["poles"]] for s in self.disp}
        z = lambda: np.zeros(n, eng.fdt)  # noqa: E731
        self.y = z()
        self.P = {s: [(z(), z()) for _ in media[s]["poles"]] for s in self.disp}

    def __call__(self, u):
        acc = u
        for s in self.disp:
            acc = acc - self.f[s] * _Group._poles(self.P[s], self.coef[s], self.y)
        self.y[...] = acc * self.inv_a
        return self.y


class _TensorMesh:
    """The D-form update of a vertex-tensor mesh's nodes (engine.py:838-923), from the plan's index tables
    (lightsmith_b200/plan.py:tensor_plan)."""

    def __init__(self, eng, t):
        self.eng = eng
        self.idx = np.asarray(t["idx"], np.int64)
        nN = self.nN = int(t["n_nodes"])
        self.D = np.zeros(nN, eng.fdt)
        self.E_prev = np.zeros(nN, eng.fdt)
        self.out = np.zeros(2 * nN, eng.fdt)
        self.vn = np.asarray(t["vn"], np.int64)
        self.scale = None if t["scale"] is None else np.asarray(t["scale"])
        self.n = np.asarray(t["normal"], float).reshape(-1, 3)
        self.nV = len(self.n)
        self.t_pos, self.t_v, self.t_vc, self.t_g = (np.asarray(t[k], np.int64) for k in ("t_pos", "t_v", "t_vc", "t_g"))
        self.t_nc = np.asarray(t["t_nc"], float)
        self.t_conj = None if t["t_conj"] is None else np.asarray(t["t_conj"])
        media = t["media"]
        F = np.asarray(t["frac"], float)
        self.a = _Harmonic(eng, media, F)
        self.b = _Arithmetic(eng, media, F)
        self.p_pos, self.p_node = np.asarray(t["p_pos"], np.int64), np.asarray(t["p_node"], np.int64)
        onehot = np.zeros((len(media), len(self.p_node)))
        onehot[np.asarray(t["p_medium"], np.int64), np.arange(len(self.p_node))] = 1.0
        self.plain = _Harmonic(eng, media, onehot)

    def step(self):
        Ef = self.eng.E.reshape(-1)
        e_now = Ef[self.idx]
        self.D += e_now - self.E_prev
        dv = self.D[self.vn]
        if self.scale is not None:
            dv = dv * self.scale
        dv = dv.reshape(self.nV, 3, 2)
        dbar = 0.5 * (dv[..., 0] + dv[..., 1])
        s = np.sum(self.n * dbar, axis=1)
        dp = dv.reshape(-1)[self.t_g]
        nc = self.t_nc
        sigma = s[self.t_v] + nc * (dp - dbar.reshape(-1)[self.t_vc])
        contrib = 0.5 * (self.b(dp - nc * sigma) + nc * self.a(sigma))
        if self.t_conj is not None:
            contrib = contrib * self.t_conj
        self.out[self.t_pos] = contrib
        if len(self.p_node):
            self.out[self.p_pos] = 0.5 * self.plain(self.D[self.p_node])
        e_new = self.out[:self.nN] + self.out[self.nN:]
        Ef[self.idx] = e_new
        self.E_prev[...] = e_new


class _P:
    def __init__(self, sigma, omega0, gamma):
        self.sigma, self.omega0, self.gamma = sigma, omega0, gamma


# --- sources ---------------------------------------------------------------------------------------------


class _Source:
    E_flat = H_flat = None

    def correct_H(self):
        pass

    def advance_H(self):
        pass

    def correct_E(self):
        pass

    def advance_E(self):
        pass


def read_tables(T, n: int, m: int, cmax: int, base, i0, u0, rdt):
    """Quintic interpolation of tables sampled every m steps at fine time (n + i0 + u0) / m = c + u, c clamped
    to cmax (``layered.py:169-187``); u is formed in the field precision as the reference does."""
    q = n + np.asarray(i0, np.int64)
    r = q % m
    c = np.minimum((q - r) // m, cmax)
    u = (r.astype(rdt) + np.asarray(u0, rdt)) / rdt.type(m)
    d = [u - rdt.type(x) for x in STENCIL]
    idx = np.asarray(base, np.int64) + c
    out = None
    for j in range(len(STENCIL)):
        w = None
        for k in range(len(STENCIL)):
            if k != j:
                w = d[k] if w is None else w * d[k]
        term = (w / rdt.type(DENOM[j])) * T[idx + j]
        out = term if out is None else out + term
    return out


class _Table(_Source):
    """Table-fed TF/SF box (``layered.py:459-482``): per correction point target += coef * interpolated table;
    the incident-reference view holds the incident E at the end of each step."""

    def __init__(self, eng, s: TableSource):
        self.eng, self.s = eng, s
        self.T = np.asarray(s.tables, eng.rdt)
        self.Tinc = np.asarray(s.inc_table, eng.rdt)
        self.E_flat = np.zeros(3, eng.rdt)
        self.H_flat = self.E_flat

    def _apply(self, pts, F):
        if pts is None:
            return
        vals = read_tables(self.T, self.eng.n, self.s.m, self.s.cmax, pts.base, pts.i0, pts.u0, self.eng.rdt)
        vals = np.asarray(pts.coef, self.eng.rdt) * vals
        np.add.at(F.reshape(-1), pts.node, vals.astype(F.dtype))

    def correct_H(self):
        self._apply(self.s.H, self.eng.H)

    def correct_E(self):
        self._apply(self.s.E, self.eng.E)

    def advance_E(self):
        b, i0, u0 = self.s.inc
        self.E_flat[...] = read_tables(self.Tinc, self.eng.n, self.s.m, self.s.cmax, b, i0, u0, self.eng.rdt)


class _Dipole(_Source):
    """E[idx] -= coef * wave[n] after the E curl (``emission.py:139-140``)."""

    def __init__(self, eng, s: DipoleSource):
        self.eng, self.s = eng, s
        self.coef = np.asarray(s.coef, eng.rdt)
        self.wave = np.asarray(s.wave, eng.rdt)

    def correct_E(self):
        Ef = self.eng.E.reshape(-1)
        Ef[self.s.idx] -= self.coef * self.wave[self.eng.n]


class _Line(_Source):
    """1D-grid-fed TF/SF (``tfsf.py:174-211``)."""

    def __init__(self, eng, s: LineSource):
        self.eng, self.s = eng, s
        rd = eng.rdt
        self.E_flat = np.zeros(s.M, rd)
        self.H_flat = np.zeros(s.M, rd)
        self.ca, self.cb = np.asarray(s.ca[1:-1], rd), np.asarray(s.cb[1:-1], rd)
        self.da, self.db = np.asarray(s.da[:-1], rd), np.asarray(s.db[:-1], rd)
        self.wave = np.asarray(s.wave, rd)

    def _apply(self, pts, F, src):
        if pts is None:
            return
        vals = src[pts.i0]
        vals = vals + np.asarray(pts.w, self.eng.rdt) * (src[pts.i0 + 1] - vals)
        Ff = F.reshape(-1)
        # slabs are applied one after another, so a node on two slabs receives both (tfsf.py:187-193)
        np.add.at(Ff, pts.node, (np.asarray(pts.coef, self.eng.rdt) * vals).astype(F.dtype))

    def correct_H(self):
        self._apply(self.s.H, self.eng.H, self.E_flat)

    def correct_E(self):
        self._apply(self.s.E, self.eng.E, self.H_flat)

    def advance_H(self):
        E, H = self.E_flat, self.H_flat
        H[:-1] *= self.da
        H[:-1] -= self.db * (E[1:] - E[:-1])

    def advance_E(self):
        E, H = self.E_flat, self.H_flat
        E[1:-1] *= self.ca
        E[1:-1] -= self.cb * (H[1:-1] - H[:-2])
        E[self.s.m_src] += self.wave[self.eng.n]


class _Column(_Source):
    """Bloch column source (``tfsf.py:256-296``): a 3 x 3 x nz engine of its own, plane corrections with the
    transverse phase, and a current sheet at k_launch."""

    def __init__(self, eng, s: ColumnSource):
        self.eng, self.s = eng, s
        self.col = OracleEngine(s.column, dtype=eng.rdt.type)
        self.E_flat, self.H_flat = self.col.E.reshape(-1), self.col.H.reshape(-1)
        self.phase = np.asarray(s.phase, eng.fdt)[:, :, None]
        self.amp = [np.asarray(a, eng.fdt) for a in s.amp]
        self.wave = np.asarray(s.wave, eng.rdt)
        nx, ny = eng.shape[0] - 2, eng.shape[1] - 2
        self.X, self.Y = slice(1, nx + 1), slice(1, ny + 1)

    def correct_H(self):
        k, E, H = self.s.k_src, self.col.E, self.eng.H
        H[0][self.X, self.Y, k - 1:k] -= self.s.cH * (self.phase * E[1][1:2, 1:2, k:k + 1])
        H[1][self.X, self.Y, k - 1:k] += self.s.cH * (self.phase * E[0][1:2, 1:2, k:k + 1])

    def correct_E(self):
        k, Hc, E = self.s.k_src, self.col.H, self.eng.E
        E[0][self.X, self.Y, k:k + 1] += self.s.cE * (self.phase * Hc[1][1:2, 1:2, k - 1:k])
        E[1][self.X, self.Y, k:k + 1] -= self.s.cE * (self.phase * Hc[0][1:2, 1:2, k - 1:k])

    def advance_H(self):
        self.col.update_H()

    def advance_E(self):
        self.col.update_E()
        w = self.wave[self.eng.n]
        k = self.s.k_launch
        self.col.E[0][1:2, 1:2, k:k + 1] += self.amp[0] * w
        self.col.E[1][1:2, 1:2, k:k + 1] += self.amp[1] * w


class _Mode(_Source):
    """Rank-r port mode source (``ports.py:368-372``)."""

    def __init__(self, eng, s: ModeSource):
        self.eng, self.s = eng, s
        rd = eng.rdt
        self.mH, self.mE = np.asarray(s.mH, rd), np.asarray(s.mE, rd)
        self.tE, self.tH = np.asarray(s.tab_E, rd), np.asarray(s.tab_H, rd)

    def correct_H(self):
        Hf = self.eng.H.reshape(-1)
        Hf[self.s.h_idx] += np.sum(self.mH * self.tE[self.eng.n], axis=1)

    def correct_E(self):
        Ef = self.eng.E.reshape(-1)
        Ef[self.s.e_idx] += np.sum(self.mE * self.tH[self.eng.n], axis=1)
