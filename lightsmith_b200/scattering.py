"""lightsmith scattering problems for this package's engine and adjoint.

``scattering_setup`` returns the plan lightsmith's scattering driver builds for a ``Simulation``
(backends/_fdtd/scattering.py:301-364: the layout, the meshing, the table-fed TF/SF plane wave, and the
monitors in the driver's order: the scattered-field flux box, the total-field flux box, the incident reference
view) together with what its post-processing reads (scattering.py:428-462: the boxes' flux weights, the
incidence medium's index, the mirror factor). It runs lightsmith's own set-up on the host and stops where the
driver would build its engine, so nothing is stepped. ``cross_section_objective`` is the scattering cross
section summed over the frequencies as a torch function of the scattered-field box's accumulators: an
objective for ``lightsmith_b200.adjoint.AdjointRun``.
"""

from __future__ import annotations

import numpy as np


class _Built(Exception):
    pass


def scattering_setup(sim):
    """(plan, post, layout) for lightsmith ``Simulation`` ``sim``: ``plan`` as ``plan.make_plan`` makes it from the
    driver's ``Engine(...)`` arguments; ``post`` with ``wavelengths_nm``, ``omega``, ``n_inc``, ``n_sym``,
    ``sca_coeff`` and ``tot_coeff`` (the flux weights of the scattered- and total-field boxes, in their points'
    order); ``layout`` lightsmith's grid layout of the run (origin, TF/SF box, spacing; with mirror planes the
    part the run steps, symmetry.py:116-127)."""
    from lightsmith.backends._fdtd import scattering as S
    from lightsmith.backends._fdtd import symmetry as Y
    from lightsmith.backends._fdtd.setup import scattering_layout
    from lightsmith.backends.fdtd import NativeFDTD
    from lightsmith.device import resolve_device

    from .plan import make_plan

    got, boxes = {}, []
    saved = S.Engine, S.flux_points

    def engine(device, **kw):
        got["kw"] = kw
        got["plan"] = make_plan(**kw)
        raise _Built

    def flux_points(*a, **k):
        out = saved[1](*a, **k)
        boxes.append(out)
        return out

    opts = NativeFDTD._options(sim)
    S.Engine, S.flux_points = engine, flux_points
    try:
        S.solve(sim, opts, resolve_device("cpu"))
    except _Built:
        pass
    finally:
        S.Engine, S.flux_points = saved
    if "plan" not in got or len(boxes) < 2:
        raise ValueError("lightsmith's scattering driver did not reach its engine for this problem")
    kw = got["kw"]
    wl = np.asarray(sim.wavelength_array(), dtype=float)
    src = kw["sources"][0]
    post = {"wavelengths_nm": wl, "omega": 2 * np.pi / wl, "n_inc": float(getattr(src, "n_inc", sim.medium_index)),
            "n_sym": float(Y.factor(kw.get("mirror", (0, 0, 0)))),
            "sca_coeff": np.asarray(boxes[0][3], dtype=float), "tot_coeff": np.asarray(boxes[1][3], dtype=float)}
    lay = Y.halve(scattering_layout(sim, opts, float(opts.spacing_nm)), tuple(kw.get("mirror", (0, 0, 0))))
    return got["plan"], post, lay


def cross_section_objective(post: dict, ref: dict):
    """J(acc_e, acc_h) = sum_f C_sca(f) (nm^2): the outward flux of the scattered field through the
    scattered-field box, 0.5 Re sum_p w_p E[f, p] conj(H[f, p]) (setup.py:564), times the mirror factor, over
    the incident intensity 0.5 n_inc |E_ref[f]|^2 (scattering.py:433-435, 457-459). ``ref["acc_ref"]``: the
    run's reference-view accumulators (n_freq, 3), read when J is evaluated, after the forward steps (the
    incident wave does not depend on the design: a constant of J). ``ref["spectrum"]`` gets C_sca per
    frequency (detached)."""
    import torch

    def J(acc_e, acc_h):
        w = torch.as_tensor(post["sca_coeff"], dtype=torch.float64, device=acc_e.device)
        flux = 0.5 * ((acc_e * acc_h.conj()).real * w).sum(dim=1)
        e_ref = torch.as_tensor(ref["acc_ref"]).detach().to(device=acc_e.device, dtype=torch.complex128)
        inten = 0.5 * post["n_inc"] * (e_ref.abs() ** 2).sum(dim=1)
        c_sca = post["n_sym"] * flux / inten
        ref["spectrum"] = c_sca.detach().cpu().numpy()
        return c_sca.sum()
    return J
