"""Device-buffer helpers for the GPU tests (torch is used for allocation only)."""

import ctypes

import numpy as np


def to_dev(a):
    import torch
    a = np.ascontiguousarray(a)
    view = a.view(np.int64 if a.dtype.itemsize == 8 else np.int32)
    t = torch.from_numpy(view.copy()).cuda()
    torch.cuda.synchronize()
    return t


def from_dev(t, dtype):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy().view(dtype)


def empty_dev(shape, dtype):
    import torch
    t = torch.zeros(shape, dtype=torch.int64 if np.dtype(dtype).itemsize == 8 else torch.int32,
                    device="cuda")
    torch.cuda.synchronize()
    return t


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())
