"""A plain-PyTorch restatement of the FDTD step, differentiated by torch.autograd: TEST INFRASTRUCTURE ONLY.

The checker of ``lightsmith_b200.adjoint``: the same update equations as ``oracle/engine.py`` (lightsmith's
``engine.py:613-663`` curl updates over the stepped regions, ``engine.py:344-418`` CPML terms in their order,
``emission.py:130-140`` point-current corrections after the E update, ``engine.py:769-793`` D-form ADE groups,
pure and mixed, after the sources), for real fields, no periodic axes and point-dipole sources, written out of
place so
that autograd can differentiate a DFT objective (|sum_p wE_p acc_e[f, p] + sum_q wH_q acc_h[f, q]|^2, or any
function of the accumulators) with respect to 1/eps over a box of nodes.
"""

from __future__ import annotations

import numpy as np
import torch

from lightsmith_b200.plan import DipoleSource, cpml_profiles, cpml_terms, e_range, h_range, pole_coefficients

from .engine import _P as _Pole
from .engine import _Spec


def _put(F, region, delta):
    """F with delta added over region (out of place)."""
    Z = torch.zeros_like(F)
    Z[region] = delta
    return F + Z


def objective(plan: dict, inv_eps_box, box, monitor: int, freq: int, wE, wH, n_steps: int, J=None):
    """J (float64 tensor) after n_steps steps from rest, differentiable in inv_eps_box (the box's 1/eps). J:
    a function of the monitor's accumulators (acc_e (n_freq, n_e), acc_h or None, complex128); None: the
    |A|^2 of weights wE, wH at frequency index freq."""
    dt = torch.float64
    shape = tuple(plan["shape"])
    spacing = tuple(plan["spacing"])
    step_dt = float(plan["dt"])
    stride = int(plan["stride"])
    uniform = len(set(spacing)) == 1
    cdx = step_dt / spacing[0] if uniform else step_dt
    inv_d = [1.0 / s for s in spacing]
    per = (False, False, False)
    inv0 = np.asarray(plan["inv_eps"], float)
    if inv0.ndim != 3:
        raise ValueError("isotropic permittivity only")
    bsl = tuple(slice(a, b) for a, b in box)
    full = torch.as_tensor(inv0, dtype=dt).clone()
    full[bsl] = inv_eps_box
    RE = [tuple(e_range(c, a, shape[a], per[a]) for a in range(3)) for c in range(3)]
    RH = [tuple(h_range(c, a, shape[a], per[a]) for a in range(3)) for c in range(3)]
    sl = lambda R: tuple(slice(r[0], r[1]) for r in R)  # noqa: E731
    cb = [cdx * full[sl(RE[c])] for c in range(3)]
    cH = cdx

    # CPML terms (oracle/engine.py:_build_pml)
    spec = _Spec(plan["pml"])
    prof = cpml_profiles(spec, shape, spacing, step_dt)
    terms = {"E": [], "H": []}
    for t in cpml_terms(spec, shape, per):
        d, fld = t["d"], t["field"]
        a, b = t["region"][d]
        bb, cc, kk = (v[a:b] for v in prof[d][2][fld])
        bshape = [1, 1, 1]
        bshape[d] = b - a
        reg = sl(t["region"])
        scale = cdx * full[reg] if fld == "E" else torch.full([r[1] - r[0] for r in t["region"]], cdx, dtype=dt)
        if not uniform:
            scale = scale / spacing[d]
        cp = t["sgn"] * scale * torch.as_tensor(cc.reshape(bshape), dtype=dt)
        kp = t["sgn"] * scale * torch.as_tensor((1 / kk - 1).reshape(bshape), dtype=dt) if np.any(kk > 1) else None
        terms[fld].append({**t, "reg": reg, "b": torch.as_tensor(bb.reshape(bshape), dtype=dt), "cp": cp, "kp": kp,
                           "psi": torch.zeros(cp.shape, dtype=dt)})

    def shifted(R, d, s):
        R = list(R)
        R[d] = slice(R[d].start + s, R[d].stop + s)
        return tuple(R)

    def curl(F, c, R, forward):
        d1, d2 = (c + 1) % 3, (c + 2) % 3
        if forward:
            a = F[d2][shifted(R, d1, 1)] - F[d2][R]
            b = F[d1][shifted(R, d2, 1)] - F[d1][R]
        else:
            a = F[d2][R] - F[d2][shifted(R, d1, -1)]
            b = F[d1][R] - F[d1][shifted(R, d2, -1)]
        if not uniform:
            a, b = a * inv_d[d1], b * inv_d[d2]
        return a - b

    def pml(tgt, src, kind):
        out = list(tgt)
        for t in terms[kind]:
            R, d, s = t["reg"], t["d"], t["src"]
            if kind == "H":
                der = src[s][shifted(R, d, 1)] - src[s][R]
            else:
                der = src[s][R] - src[s][shifted(R, d, -1)]
            psi = t["psi"] * t["b"]
            delta = torch.zeros_like(der)
            if t["kp"] is not None:
                delta = delta + t["kp"] * der
            psi = psi + der * t["cp"]
            t["psi"] = psi
            out[t["c"]] = _put(out[t["c"]], R, delta + psi)
        return out

    E = [torch.zeros(shape, dtype=dt) for _ in range(3)]
    H = [torch.zeros(shape, dtype=dt) for _ in range(3)]
    dips = [s for s in plan["sources"] if isinstance(s, DipoleSource)]
    if len(dips) != len(plan["sources"]):
        raise ValueError("point dipoles only")
    mon = plan["monitors"][monitor]
    omegas = torch.as_tensor(np.asarray(mon["omega"], float))
    e_idx = torch.as_tensor(mon["e_idx"])
    h1 = None if mon["h_idx1"] is None else torch.as_tensor(mon["h_idx1"])
    h2 = None if mon["h_idx2"] is None else torch.as_tensor(mon["h_idx2"])
    acc_e = torch.zeros((len(omegas), len(e_idx)), dtype=torch.complex128)
    acc_h = None if h1 is None else torch.zeros((len(omegas), len(h1)), dtype=torch.complex128)
    cells = int(np.prod(shape))

    # dispersive groups (lightsmith's engine.py:722-793, _Group): D, E_prev and (P, P') per pole; a mixed group
    # (interface cells) also a harmonic path per dispersive medium (its E_s driving its poles, weight w) and an
    # arithmetic path (one E_a driving every medium's poles, weight 1 - w); out of place
    groups = []
    for g in plan["groups"]:
        idx = torch.as_tensor(np.asarray(g["idx"], np.int64))
        z = torch.zeros(len(idx), dtype=dt)
        coef = [[pole_coefficients(_Pole(*p), step_dt) for p in m["poles"]] for m in g["media"]]
        if g["w"] is None:
            (m,) = g["media"]
            groups.append({"idx": idx, "pure": True, "D": z, "Ep": z, "P": [(z, z) for _ in coef[0]],
                           "coef": coef[0], "inv_inf": 1.0 / m["eps_inf"]})
            continue
        f = np.asarray(g["frac"], float)
        media = g["media"]
        disp = [s for s, m in enumerate(media) if m["poles"]]
        w = np.asarray(g["w"], float)
        groups.append({"idx": idx, "pure": False, "D": z, "Ep": z, "disp": disp, "coef": coef,
                       "h0": torch.as_tensor(sum(f[s] / m["eps_inf"] for s, m in enumerate(media)
                                                 if not m["poles"]) + 0 * f[0], dtype=dt),
                       "f": {s: torch.as_tensor(f[s], dtype=dt) for s in disp},
                       "inv_inf": {s: 1.0 / media[s]["eps_inf"] for s in disp},
                       "inv_a": torch.as_tensor(1.0 / sum(f[s] * m["eps_inf"] for s, m in enumerate(media)), dtype=dt),
                       "w": torch.as_tensor(w, dtype=dt), "has_h": bool(np.any(w > 0)), "has_a": bool(np.any(w < 1)),
                       "Eh": {s: z for s in disp}, "Ea": z,
                       "Ph": {s: [(z, z) for _ in coef[s]] for s in disp},
                       "Pa": {s: [(z, z) for _ in coef[s]] for s in disp}})

    def advance(pairs, coefs, drive):
        """The poles' new (P, P') and their sum (lightsmith's _Group._advance)."""
        tot, new = None, []
        for (P, Pp), (c1, c2, c3) in zip(pairs, coefs):
            nw = c1 * P + c2 * Pp + c3 * drive
            new.append((nw, P))
            tot = nw if tot is None else tot + nw
        return new, tot
    for n in range(n_steps):
        H = [_put(H[c], sl(RH[c]), -curl(E, c, sl(RH[c]), True) * cH) for c in range(3)]
        H = pml(H, E, "H")
        E = [_put(E[c], sl(RE[c]), curl(H, c, sl(RE[c]), False) * cb[c]) for c in range(3)]
        E = pml(E, H, "E")
        for s in dips:  # E_flat[idx] -= coef * wave[n] (after the E update)
            flat = torch.cat([e.reshape(-1) for e in E])
            upd = torch.zeros_like(flat).index_add(0, torch.as_tensor(s.idx),
                                                   torch.as_tensor(s.coef * s.wave[n], dtype=dt))
            flat = flat - upd
            E = [flat[c * cells:(c + 1) * cells].reshape(shape) for c in range(3)]
        if groups:  # D += E - E_prev; P <- c1 P + c2 P' + c3 drive; E from D and P; E_prev = E
            flat = torch.cat([e.reshape(-1) for e in E])
            for g in groups:
                e_now = flat[g["idx"]]
                g["D"] = g["D"] + (e_now - g["Ep"])
                if g["pure"]:
                    g["P"], tot = advance(g["P"], g["coef"], g["Ep"])
                    e_new = (g["D"] - tot) * g["inv_inf"]
                else:
                    parts = []
                    if g["has_h"]:
                        harm = g["D"] * g["h0"]
                        for s in g["disp"]:
                            g["Ph"][s], tot = advance(g["Ph"][s], g["coef"][s], g["Eh"][s])
                            g["Eh"][s] = (g["D"] - tot) * g["inv_inf"][s]
                            harm = harm + g["f"][s] * g["Eh"][s]
                        parts.append(g["w"] * harm)
                    if g["has_a"]:
                        acc = g["D"]
                        for s in g["disp"]:
                            g["Pa"][s], tot = advance(g["Pa"][s], g["coef"][s], g["Ea"])
                            acc = acc - g["f"][s] * tot
                        g["Ea"] = acc * g["inv_a"]
                        parts.append((1 - g["w"]) * g["Ea"])
                    e_new = parts[0] if len(parts) == 1 else parts[0] + parts[1]
                g["Ep"] = e_new
                flat = flat.index_put((g["idx"],), e_new)
            E = [flat[c * cells:(c + 1) * cells].reshape(shape) for c in range(3)]
        if (n + 1) % stride == 0:
            t_e = (n + 1) * step_dt
            flat_e = torch.cat([e.reshape(-1) for e in E])
            ph_e = torch.exp(1j * omegas * t_e)[:, None]
            acc_e = acc_e + ph_e * flat_e[e_idx].to(torch.complex128)[None, :]
            if acc_h is not None:
                flat_h = torch.cat([h.reshape(-1) for h in H])
                havg = ((flat_h[h1] + flat_h[h2]) * 0.5).to(torch.complex128)
                acc_h = acc_h + torch.exp(1j * omegas * (t_e - 0.5 * step_dt))[:, None] * havg[None, :]
    if J is not None:
        return J(acc_e, acc_h)
    wE = torch.as_tensor(np.asarray(wE), dtype=torch.complex128)
    A = (wE * acc_e[freq]).sum()
    if wH is not None and acc_h is not None:
        A = A + (torch.as_tensor(np.asarray(wH), dtype=torch.complex128) * acc_h[freq]).sum()
    return (A * A.conj()).real
