"""Conversions between dense (z, y, x) arrays and the FP32 solver's padded
level layout (one ghost node per face, x offset 4, row pitch from
pb_level_geometry)."""

import ctypes

import numpy as np


def geometry(L, n):
    pitch, count = ctypes.c_int64(), ctypes.c_int64()
    assert L.pb_level_geometry(n, ctypes.byref(pitch), ctypes.byref(count)) == 0
    return pitch.value, count.value


def to_padded(L, a):
    import torch

    n = a.shape[0]
    pitch, count = geometry(L, n)
    out = np.zeros(count, np.float32)
    view = out.reshape(n + 2, n + 2, pitch)
    view[1:n + 1, 1:n + 1, 4:n + 4] = a
    return torch.from_numpy(out).cuda()


def from_padded(L, t, n):
    pitch, _ = geometry(L, n)
    v = t.cpu().numpy().reshape(n + 2, n + 2, pitch)
    return v[1:n + 1, 1:n + 1, 4:n + 4].astype(np.float64)


def ghosts_zero(L, t, n):
    pitch, _ = geometry(L, n)
    v = t.cpu().numpy().reshape(n + 2, n + 2, pitch).copy()
    v[1:n + 1, 1:n + 1, 4:n + 4] = 0
    return not v.any()
