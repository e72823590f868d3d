"""PyTorch namespace with the array-API spellings the reference uses."""

import torch as _t
from torch import *  # noqa: F401,F403

float32, float64, complex64, complex128, int64 = _t.float32, _t.float64, _t.complex64, _t.complex128, _t.int64


def astype(x, dtype, copy=True):
    return x.to(dtype)


def reshape(x, shape):
    return _t.reshape(x, shape)


def sum(x, axis=None):  # noqa: A001
    return _t.sum(x) if axis is None else _t.sum(x, dim=axis)


def asarray(a, dtype=None, device=None, copy=None):  # noqa: A002
    if isinstance(a, _t.Tensor):
        return a.to(dtype=dtype or a.dtype, device=device or a.device)
    import numpy as _np
    arr = _np.asarray(a)
    t = _t.from_numpy(arr.copy()) if arr.dtype != object else _t.tensor(arr)
    return t.to(dtype=dtype or t.dtype, device=device or "cpu")


def zeros(shape, dtype=None, device=None):  # noqa: A002
    return _t.zeros(shape, dtype=dtype, device=device)


def minimum(a, b):
    return _t.minimum(a, b if isinstance(b, _t.Tensor) else _t.as_tensor(b))
