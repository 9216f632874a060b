"""Seeded synthetic RGB-D sequences (ctypes wrapper of rgbd_synth/synth.cpp).

The sequences stand in for the recorded RGB-D sequence the reference reads
(MainTum.cc:78-96) and for its live camera (Core/Camera.cc:117-144): u16 depth
in 1/depth_scale metres plus packed RGB8, one pair per frame.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class SynthParams(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int),
        ("height", ctypes.c_int),
        ("fx", ctypes.c_float),
        ("fy", ctypes.c_float),
        ("cx", ctypes.c_float),
        ("cy", ctypes.c_float),
        ("seed", ctypes.c_uint64),
        ("depth_scale", ctypes.c_float),
        ("min_range", ctypes.c_float),
        ("max_range", ctypes.c_float),
        ("dropout", ctypes.c_float),
        ("noise", ctypes.c_int),
        ("fps", ctypes.c_float),
        ("max_speed", ctypes.c_float),
        ("max_rate_deg", ctypes.c_float),
    ]


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libfbsynth.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run `python -m rgbd_synth.build` first")
        lib = ctypes.CDLL(path)
        lib.fbs_default_params.argtypes = [ctypes.POINTER(SynthParams), ctypes.c_int,
                                           ctypes.c_int, ctypes.c_uint64]
        lib.fbs_splitmix64.restype = ctypes.c_uint64
        lib.fbs_splitmix64.argtypes = [ctypes.c_uint64]
        lib.fbs_render.argtypes = [ctypes.POINTER(SynthParams), ctypes.c_int, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.fbs_render.restype = ctypes.c_int
        lib.fbs_num_threads.restype = ctypes.c_int
        _LIB = lib
    return _LIB


def session_seed(config_id, session_id):
    """seed = splitmix64(config_id << 32 | session_id)."""
    return int(_lib().fbs_splitmix64(ctypes.c_uint64(((config_id & 0xFFFFFFFF) << 32)
                                                     | (session_id & 0xFFFFFFFF))))


def params(width, height, seed, **overrides):
    p = SynthParams()
    _lib().fbs_default_params(ctypes.byref(p), width, height, ctypes.c_uint64(seed))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def render(p, first, count, depth=True, rgb=True, poses=True):
    """Render frames [first, first+count).  Returns (depth u16 [n,H,W],
    rgb u8 [n,H,W,3], poses f64 [n,4,4] camera-to-world); skipped outputs are None."""
    n, H, W = count, p.height, p.width
    d = np.zeros((n, H, W), np.uint16) if depth else None
    c = np.zeros((n, H, W, 3), np.uint8) if rgb else None
    T = np.zeros((n, 4, 4), np.float64) if poses else None
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p) if a is not None else None
    rc = _lib().fbs_render(ctypes.byref(p), first, count, ptr(d), ptr(c), ptr(T))
    if rc != 0:
        raise ValueError("fbs_render: bad parameters")
    return d, c, T


def num_threads():
    return int(_lib().fbs_num_threads())
