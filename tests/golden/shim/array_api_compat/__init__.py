"""Minimal stand-in for the ``array_api_compat`` package, used only to import the reference's CPU FDTD in
this container when generating golden fixtures (the package itself is not installed here). It supplies the
few names the reference touches: ``device``, ``array_namespace`` and the ``numpy``/``torch`` namespaces."""

import numpy as _np


def device(x):
    dev = getattr(x, "device", None)
    return "cpu" if dev is None or isinstance(x, _np.ndarray) else dev


def array_namespace(*xs):
    for x in xs:
        if type(x).__module__.startswith("torch"):
            from . import torch as ns
            return ns
    from . import numpy as ns
    return ns
