"""CPU restatement of lightsmith's scattering post-processing: flux-box cross sections from DFT accumulators.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__``): the checker for whole-solve fixtures. On the product path
this step is lightsmith's own driver code, which runs unchanged on the host after the CUDA engine's run.

Follows lightsmith v0.3.0: ``flux`` (backends/_fdtd/setup.py:564-566) and the table-fed TF/SF branch of the
cross sections (backends/_fdtd/scattering.py:428-446, 457-462).
"""

from __future__ import annotations

import numpy as np


def flux(e: np.ndarray, h: np.ndarray, coeff: np.ndarray) -> np.ndarray:
    """Outward flux 0.5 Re sum_p coeff[p] E[f, p] conj(H[f, p]), one value per frequency row (setup.py:564)."""
    return 0.5 * np.real((e * np.conj(h)) @ coeff)


def cross_sections(acc_e, acc_h, post: dict) -> dict:
    """C_sca, C_abs, C_ext (nm^2) of a table-fed scattering run.

    acc_e / acc_h: the DFT accumulators of the run's monitors in the driver's order (scattered-field box,
    total-field box, incident reference view; scattering.py:344-363). ``post`` holds what the driver computes
    from its source object on the host: ``n_inc`` and ``n_sym``, the flux weights of the two boxes
    (``sca_coeff``, ``tot_coeff``), the incident reference polarisation ``unit`` (f, 3) and the unit-amplitude
    background fields on the total-field box, ``bg_e`` and the H average ``bg_h`` (scattering.py:438-441), or
    instead their flux through that box per frequency, ``bg_flux``.
    """
    e_ref = np.asarray(acc_e[2], complex)
    e0sq = np.sum(np.abs(e_ref) ** 2, axis=1)
    intensity = 0.5 * post["n_inc"] * e0sq  # scattering.py:433-435
    unit = np.asarray(post["unit"], complex)
    amp = np.sum(e_ref * np.conj(unit), axis=1) / np.sum(np.abs(unit) ** 2, axis=1)
    n_sym = post.get("n_sym", 1.0)
    if "bg_flux" in post:
        # the flux is bilinear in (E, H) and both background fields carry the same amplitude: the unit-amplitude
        # background's flux per frequency, times |amp|^2
        bg_out = n_sym * np.abs(amp) ** 2 * np.asarray(post["bg_flux"], float)
    else:
        e_bg = amp[:, None] * post["bg_e"]
        h_bg = amp[:, None] * post["bg_h"]
        bg_out = n_sym * flux(e_bg, h_bg, post["tot_coeff"])  # scattering.py:442
    c_sca = n_sym * flux(acc_e[0], acc_h[0], post["sca_coeff"]) / intensity  # scattering.py:457-459
    c_abs = -(n_sym * flux(acc_e[1], acc_h[1], post["tot_coeff"]) - bg_out) / intensity
    return {"c_sca": c_sca, "c_abs": c_abs, "c_ext": c_sca + c_abs}
