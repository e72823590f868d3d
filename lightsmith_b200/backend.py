"""lightsmith's FDTD backend with its time loop on a B200 (sm_100a).

lightsmith finds backends through the ``lightsmith.backends`` entry-point group and keys its registry by
``Backend.name`` (backends/base.py:91-103). ``B200FDTD`` carries the built-in FDTD backend's own name,
``"lightsmith-fdtd"`` (backends/fdtd.py:48-56), so once this package is installed ``ls.solve(sim, "fdtd",
"gpu")`` reaches it with no change to lightsmith.

It is lightsmith's ``NativeFDTD`` with one part swapped: on a CUDA device, the problem drivers
(backends/_fdtd/scattering.py:416, emission.py:179, periodic.py:409,444, device.py:540) construct
``lightsmith_b200.engine.Engine`` where they would construct lightsmith's array-API ``Engine``. Options,
``supports``, ``estimate``, the drivers' set-up (voxelisation, sources, monitors, time step), the run loop
(setup.py:722-773) and the post-processing (cross sections, orders, S-parameters) are lightsmith's own.

On a CPU device the class is ``NativeFDTD`` unchanged: this package adds no CPU path. On a CUDA device there is
no fallback: a problem that needs a feature with no CUDA path here (graded grids, time monitors, substrates,
Gaussian beams) is rejected by ``supports`` or raises
``ValueError`` when its engine is built, and a missing or unloadable ``liblsfdtd.so`` raises from the engine.
"""

from __future__ import annotations

import threading
from contextlib import contextmanager

from lightsmith.backends._fdtd import device as _device_driver
from lightsmith.backends._fdtd import emission as _emission_driver
from lightsmith.backends._fdtd import periodic as _periodic_driver
from lightsmith.backends._fdtd import scattering as _scattering_driver
from lightsmith.backends.fdtd import NativeFDTD
from lightsmith.problems import DeviceProblem, EmissionProblem, LayerStackProblem, PeriodicProblem
from lightsmith.spec import Simulation

from . import engine as _engine

__all__ = ["B200FDTD"]

# the modules whose `Engine` name the solve rebinds (each imports it with `from .engine import ... Engine`)
_DRIVERS = (_scattering_driver, _emission_driver, _periodic_driver, _device_driver)
_SWAP_LOCK = threading.RLock()


def _b200_engine(device, **kw):
    """lightsmith's ``Engine(device, **kw)`` call, answered by the CUDA engine."""
    try:
        return _engine.Engine(device, **kw)
    except NotImplementedError as e:  # a feature with no CUDA path: lightsmith's error for unsupported problems
        raise ValueError(f"{B200FDTD.name} (B200): {e}") from e


@contextmanager
def _engine_swapped():
    """Rebind the drivers' ``Engine`` to the CUDA engine for the duration of one solve."""
    with _SWAP_LOCK:
        saved = [m.Engine for m in _DRIVERS]
        try:
            for m in _DRIVERS:
                m.Engine = _b200_engine
            yield
        finally:
            for m, e in zip(_DRIVERS, saved):
                m.Engine = e


def _static_rejection(sim, opts) -> str:
    """Features known from the problem and its options alone that have no CUDA path here ('' if none)."""
    if isinstance(sim, (Simulation, DeviceProblem)) and _scattering_driver.graded(opts):
        return "does not support graded grids (grid='auto', mesh_override) on the GPU"
    if isinstance(sim, Simulation):
        if sim.outputs.resonances is not None:
            return "does not support the resonances output (time monitors) on the GPU"
        if sim.substrate is not None:
            return "does not support substrates on the GPU"
        if sim.illumination.kind == "gaussian_beam":
            return "does not support gaussian_beam illumination on the GPU"
    return ""


class B200FDTD(NativeFDTD):
    """``NativeFDTD`` (backends/fdtd.py:47) whose engine is the B200 one on CUDA devices."""

    name = "lightsmith-fdtd"
    method = "fdtd"
    gpu = True
    citation = NativeFDTD.citation + "; time loop: lightsmith-b200 (sm_100a CUDA kernels)"

    @classmethod
    def supports(cls, sim):
        ok, why = NativeFDTD.supports(sim)
        if not ok:
            return ok, why
        if isinstance(sim, (Simulation, DeviceProblem, EmissionProblem, PeriodicProblem, LayerStackProblem)):
            try:
                opts = cls._options(sim)
            except ValueError as e:
                return False, str(e)
            why = _static_rejection(sim, opts)
            if why:
                return False, why
        return True, ""

    @classmethod
    def solve(cls, sim, device):
        if not device.is_gpu:
            return NativeFDTD.solve.__func__(cls, sim, device)
        if device.framework != "torch":
            raise ValueError(f"{cls.name} (B200) runs on PyTorch CUDA devices, not {device.framework!r}")
        with _engine_swapped():
            return NativeFDTD.solve.__func__(cls, sim, device)
