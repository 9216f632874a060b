"""Configuration limits of the C ABI, checked on the host (no GPU):
fb_session_bytes is 0 for a configuration fb_session_create refuses."""
import ctypes

from fusion_b200 import _lib
from fusion_b200.system import make_config


def _bytes(cfg):
    return int(_lib.load().fb_session_bytes(ctypes.byref(cfg)))


def test_image_size_limits():
    # width <= 4096 and height <= 2048 (the packed photometric correspondence
    # holds a 12-bit column and an 11-bit row)
    assert _bytes(make_config(2048, 2047, 0.01, 4, 1 << 16, 1 << 14, 1 << 14)) > 0
    assert _bytes(make_config(4096, 1024, 0.01, 4, 1 << 16, 1 << 14, 1 << 14)) > 0
    assert _bytes(make_config(4096, 2048, 0.01, 4, 1 << 16, 1 << 14, 1 << 14)) > 0
    assert _bytes(make_config(4096, 2049, 0.01, 4, 1 << 16, 1 << 14, 1 << 14)) == 0
    assert _bytes(make_config(4097, 16, 0.01, 4, 1 << 16, 1 << 14, 1 << 14)) == 0
    assert _bytes(make_config(16, 16, 0.01, 4, 1 << 16, 1 << 14, 1 << 14)) > 0
    assert _bytes(make_config(15, 16, 0.01, 4, 1 << 16, 1 << 14, 1 << 14)) == 0


def test_map_and_form_limits():
    c = make_config(320, 240, 0.01, 4, 1 << 16, 1 << 14, 1 << 14)
    assert _bytes(c) > 0
    for field, bad in (("num_buckets", 0), ("num_blocks", 0), ("num_excess", -1), ("voxel_size", 0.0),
                       ("trunc_dist", 0.0), ("form", 2)):
        d = make_config(320, 240, 0.01, 4, 1 << 16, 1 << 14, 1 << 14)
        setattr(d, field, bad)
        assert _bytes(d) == 0, field
    d = make_config(320, 240, 0.01, 4, 1 << 16, 1 << 14, 1 << 14)
    d.iters[0] = 1001
    assert _bytes(d) == 0
