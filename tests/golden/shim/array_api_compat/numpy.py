"""NumPy namespace with the array-API extras the reference uses (``astype``)."""

from numpy import *  # noqa: F401,F403
import numpy as _np


def astype(x, dtype, copy=True):
    return _np.asarray(x).astype(dtype, copy=copy)


def asarray(a, dtype=None, device=None, copy=None):  # noqa: A002
    return _np.asarray(a, dtype=dtype)


def zeros(shape, dtype=None, device=None):  # noqa: A002
    return _np.zeros(shape, dtype=dtype)
