"""ORACLE / TEST INFRASTRUCTURE ONLY.

ctypes wrapper of oracle/liboracle.so, the CPU restatement of the reference's
per-frame path (see oracle.hpp).  Only tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py may import this module, and only as the checker.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
_LIB = None


class OracleConfig(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int),
        ("fx", ctypes.c_float), ("fy", ctypes.c_float), ("cx", ctypes.c_float), ("cy", ctypes.c_float),
        ("depth_scale", ctypes.c_float), ("depth_cutoff", ctypes.c_float),
        ("voxel_size", ctypes.c_float), ("trunc_dist", ctypes.c_float),
        ("depth_min", ctypes.c_float), ("depth_max", ctypes.c_float),
        ("num_buckets", ctypes.c_int), ("num_excess", ctypes.c_int), ("num_blocks", ctypes.c_int),
        ("iters", ctypes.c_int * 3),
        ("precision", ctypes.c_int),
    ]


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            import subprocess
            subprocess.check_call(["make", "-C", _HERE, "liboracle.so"])
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.fbo_map_create.restype = vp
        L.fbo_system_create.restype = vp
        L.fbo_system_map.restype = vp
        for n in ["fbo_map_destroy", "fbo_map_reset", "fbo_system_destroy"]:
            getattr(L, n).argtypes = [vp]
        L.fbo_system_map.argtypes = [vp]
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f(x):
    return ctypes.c_float(x)


def config(width, height, fx, fy, cx, cy, depth_scale=5000.0, depth_cutoff=3.0,
           voxel_size=0.006, trunc_dist=None, depth_min=0.1, depth_max=3.0,
           num_buckets=1000000, num_excess=500000, num_blocks=700000, iters=(10, 5, 3),
           precision=64):
    c = OracleConfig()
    c.width, c.height = width, height
    c.fx, c.fy, c.cx, c.cy = fx, fy, cx, cy
    c.depth_scale, c.depth_cutoff = depth_scale, depth_cutoff
    c.voxel_size = voxel_size
    # TruncateDist = VoxelSize * 8 in float (Mapping/DeviceMap.h:146)
    c.trunc_dist = trunc_dist if trunc_dist is not None else float(np.float32(voxel_size) * np.float32(8))
    c.depth_min, c.depth_max = depth_min, depth_max
    c.num_buckets, c.num_excess, c.num_blocks = num_buckets, num_excess, num_blocks
    for i in range(3):
        c.iters[i] = iters[i]
    c.precision = precision
    return c


# ---------------------------------------------------------------- stages --

def filter_depth(depth_u16, depth_scale, depth_cutoff, prec=64):
    H, W = depth_u16.shape
    raw = np.zeros((H, W), np.float32)
    filt = np.zeros((H, W), np.float32)
    lib().fbo_filter_depth(prec, W, H, _p(np.ascontiguousarray(depth_u16)), _f(depth_scale),
                           _f(depth_cutoff), _p(raw), _p(filt))
    return raw, filt


def intensity(rgb):
    H, W, _ = rgb.shape
    g = np.zeros((H, W), np.uint8)
    lib().fbo_intensity(W, H, _p(np.ascontiguousarray(rgb)), _p(g))
    return g


def pyrdown(src, prec=64):
    H, W = src.shape
    dst = np.zeros((H // 2, W // 2), src.dtype)
    fn = lib().fbo_pyrdown_f32 if src.dtype == np.float32 else lib().fbo_pyrdown_u8
    fn(prec, W, H, _p(np.ascontiguousarray(src)), _p(dst))
    return dst


def vmap(depth, fx, fy, cx, cy, depth_cutoff, prec=64):
    H, W = depth.shape
    out = np.zeros((H, W, 4), np.float32)
    lib().fbo_vmap(prec, W, H, _p(np.ascontiguousarray(depth, np.float32)), _f(fx), _f(fy), _f(cx),
                   _f(cy), _f(depth_cutoff), _p(out))
    return out


def nmap(vm, prec=64):
    H, W, _ = vm.shape
    out = np.zeros((H, W, 4), np.float32)
    lib().fbo_nmap(prec, W, H, _p(np.ascontiguousarray(vm, np.float32)), _p(out))
    return out


def derivative(gray):
    H, W = gray.shape
    dx = np.zeros((H, W), np.int16)
    dy = np.zeros((H, W), np.int16)
    lib().fbo_derivative(W, H, _p(np.ascontiguousarray(gray)), _p(dx), _p(dy))
    return dx, dy


def resize_map(vm, nm, prec=64):
    H, W, _ = vm.shape
    vd = np.zeros((H // 2, W // 2, 4), np.float32)
    nd = np.zeros((H // 2, W // 2, 4), np.float32)
    lib().fbo_resize_map(prec, W, H, _p(np.ascontiguousarray(vm, np.float32)),
                         _p(np.ascontiguousarray(nm, np.float32)), _p(vd), _p(nd))
    return vd, nd


def icp_step(vcurr, vlast, ncurr, nlast, pose_curr, pose_last, fx, fy, cx, cy, prec=64):
    H, W, _ = vcurr.shape
    s = np.zeros(29, np.float64)
    c = lambda a: _p(np.ascontiguousarray(a, np.float32))
    lib().fbo_icp_step(prec, W, H, c(vcurr), c(vlast), c(ncurr), c(nlast),
                       _p(np.ascontiguousarray(pose_curr, np.float64)),
                       _p(np.ascontiguousarray(pose_last, np.float64)), _f(fx), _f(fy), _f(cx), _f(cy), _p(s))
    return s


def rgb_step(gcurr, glast, vcurr, vlast, dx, dy, pose_curr, pose_last, fx, fy, cx, cy, prec=64):
    H, W = gcurr.shape
    s = np.zeros(29, np.float64)
    r = np.zeros(2, np.int64)
    c = lambda a: _p(np.ascontiguousarray(a, np.float32))
    lib().fbo_rgb_step(prec, W, H, _p(np.ascontiguousarray(gcurr)), _p(np.ascontiguousarray(glast)),
                       c(vcurr), c(vlast), _p(np.ascontiguousarray(dx)), _p(np.ascontiguousarray(dy)),
                       _p(np.ascontiguousarray(pose_curr, np.float64)),
                       _p(np.ascontiguousarray(pose_last, np.float64)), _f(fx), _f(fy), _f(cx), _f(cy),
                       _p(s), _p(r))
    return s, r


def unpack29(s):
    """CreateMatrix<6,7> (Tracking/Reduction.cu:6-16): symmetric A, b."""
    A = np.zeros((6, 6))
    b = np.zeros(6)
    k = 0
    for i in range(6):
        for j in range(i, 7):
            if j == 6:
                b[i] = s[k]
            else:
                A[i, j] = A[j, i] = s[k]
            k += 1
    return A, b


# ------------------------------------------------------------------- map --

class Map:
    def __init__(self, cfg, handle=None):
        self.cfg = cfg
        self.owned = handle is None
        self.h = handle if handle is not None else lib().fbo_map_create(ctypes.byref(cfg))

    def close(self):
        if self.owned and self.h:
            lib().fbo_map_destroy(ctypes.c_void_p(self.h))
        self.h = None

    def __del__(self):
        self.close()

    @property
    def n_entries(self):
        return self.cfg.num_buckets + self.cfg.num_excess

    def reset(self):
        lib().fbo_map_reset(ctypes.c_void_p(self.h))

    def fuse(self, raw, rgb, nm, pose):
        n = ctypes.c_uint32(0)
        lib().fbo_map_fuse(ctypes.c_void_p(self.h), _p(np.ascontiguousarray(raw, np.float32)),
                           _p(np.ascontiguousarray(rgb)), _p(np.ascontiguousarray(nm, np.float32)),
                           _p(np.ascontiguousarray(pose, np.float64)), ctypes.byref(n))
        return int(n.value)

    def allocate(self, raw, pose):
        n = ctypes.c_uint32(0)
        lib().fbo_map_allocate(ctypes.c_void_p(self.h), _p(np.ascontiguousarray(raw, np.float32)),
                               _p(np.ascontiguousarray(pose, np.float64)), ctypes.byref(n))
        return int(n.value)

    def raycast(self, pose, vm=None, nm=None):
        W, H = self.cfg.width, self.cfg.height
        vm = np.full((H, W, 4), np.nan, np.float32) if vm is None else vm.copy()
        nm = np.full((H, W, 4), np.nan, np.float32) if nm is None else nm.copy()
        zc, zr = (W + 7) // 8, (H + 7) // 8
        zmin = np.zeros((zr, zc), np.float32)
        zmax = np.zeros((zr, zc), np.float32)
        tiles = lib().fbo_map_raycast(ctypes.c_void_p(self.h), _p(np.ascontiguousarray(pose, np.float64)),
                                      _p(vm), _p(nm), _p(zmin), _p(zmax))
        return vm, nm, zmin, zmax, tiles

    def counters(self):
        hc, ep, nv = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_uint32()
        lib().fbo_map_counters(ctypes.c_void_p(self.h), ctypes.byref(hc), ctypes.byref(ep), ctypes.byref(nv))
        return hc.value, ep.value, nv.value

    def entries(self):
        e = np.zeros((self.n_entries, 5), np.int32)
        lib().fbo_map_entries(ctypes.c_void_p(self.h), _p(e))
        return e

    def allocated(self):
        """Occupied slots sorted by (x, y, z): (slots, entries[n,5])."""
        e = self.entries()
        occ = np.nonzero(e[:, 3] >= 0)[0]
        rows = e[occ]
        order = np.lexsort((rows[:, 2], rows[:, 1], rows[:, 0]))
        return occ[order].astype(np.int32), rows[order]

    def visible(self):
        n = self.counters()[2]
        s = np.zeros(n, np.int32)
        lib().fbo_map_visible(ctypes.c_void_p(self.h), _p(s))
        return s

    def set_entries(self, slots, entries, heap_counter, entry_ptr):
        slots = np.ascontiguousarray(slots, np.int32)
        entries = np.ascontiguousarray(entries, np.int32)
        lib().fbo_map_set_entries(ctypes.c_void_p(self.h), _p(slots), _p(entries), len(slots),
                                  int(heap_counter), int(entry_ptr))

    def set_visible(self, slots):
        slots = np.ascontiguousarray(slots, np.int32)
        lib().fbo_map_set_visible(ctypes.c_void_p(self.h), _p(slots), len(slots))

    def load_blocks(self, ptrs, sdf, weight, rgb):
        ptrs = np.ascontiguousarray(ptrs, np.int32)
        lib().fbo_map_load_blocks(ctypes.c_void_p(self.h), _p(ptrs), len(ptrs),
                                  _p(np.ascontiguousarray(sdf, np.float64)),
                                  _p(np.ascontiguousarray(weight, np.uint8)),
                                  _p(np.ascontiguousarray(rgb, np.uint8)))

    def voxels(self, ptrs):
        ptrs = np.ascontiguousarray(ptrs, np.int32)
        n = len(ptrs)
        sdf = np.zeros((n, 512), np.float64)
        w = np.zeros((n, 512), np.uint8)
        rgb = np.zeros((n, 512, 3), np.uint8)
        lib().fbo_map_voxels(ctypes.c_void_p(self.h), _p(ptrs), n, _p(sdf), _p(w), _p(rgb))
        return sdf, w, rgb

    def visibility(self, pose):
        """CheckBlockVisibility at `pose` (4x4) for the configured camera and
        depth range; returns the visible block count."""
        n = ctypes.c_uint32()
        lib().fbo_map_visibility(ctypes.c_void_p(self.h), _p(np.ascontiguousarray(pose, np.float64)),
                                 ctypes.byref(n))
        return n.value

    def mesh(self, tri, ntri, fused=1):
        """MeshScene on this map with case table (tri [256, 16] edge triples,
        ntri [256]): (vertex, normal, color), three rows per triangle."""
        tri = np.ascontiguousarray(tri, np.int8)
        ntri = np.ascontiguousarray(ntri, np.int32)
        n = ctypes.c_uint64()
        L = lib()
        L.fbo_map_mesh.argtypes = [ctypes.c_void_p] * 7 + [ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]
        L.fbo_map_mesh(ctypes.c_void_p(self.h), _p(tri), _p(ntri), fused, None, None, None, 0, ctypes.byref(n))
        V = np.zeros((3 * n.value, 3), np.float32)
        N = np.zeros((3 * n.value, 3), np.float32)
        C = np.zeros((3 * n.value, 3), np.uint8)
        L.fbo_map_mesh(ctypes.c_void_p(self.h), _p(tri), _p(ntri), fused, _p(V), _p(N), _p(C), n.value,
                       ctypes.byref(n))
        return V, N, C


class System:
    def __init__(self, cfg):
        self.cfg = cfg
        self.h = lib().fbo_system_create(ctypes.byref(cfg))
        self.map = Map(cfg, handle=lib().fbo_system_map(ctypes.c_void_p(self.h)))

    def close(self):
        if self.h:
            lib().fbo_system_destroy(ctypes.c_void_p(self.h))
        self.h = None

    def __del__(self):
        self.close()

    def grab(self, depth, rgb):
        info = np.zeros(8, np.float64)
        lib().fbo_system_grab(ctypes.c_void_p(self.h), _p(np.ascontiguousarray(depth)),
                              _p(np.ascontiguousarray(rgb)), _p(info))
        return info

    def pose(self, which=0):
        T = np.zeros((4, 4), np.float64)
        lib().fbo_system_pose(ctypes.c_void_p(self.h), which, _p(T))
        return T

    def level(self, which, lv):
        W, H = self.cfg.width >> lv, self.cfg.height >> lv
        out = dict(vmap=np.zeros((H, W, 4), np.float32), nmap=np.zeros((H, W, 4), np.float32),
                   depth=np.zeros((H, W), np.float32), image=np.zeros((H, W), np.uint8),
                   dx=np.zeros((H, W), np.int16), dy=np.zeros((H, W), np.int16))
        lib().fbo_system_level(ctypes.c_void_p(self.h), which, lv, _p(out["vmap"]), _p(out["nmap"]),
                               _p(out["depth"]), _p(out["image"]), _p(out["dx"]), _p(out["dy"]))
        return out


def track(cfg, nxt, last, last_pose, grid=None):
    """Tracker::ComputeSE3 on given inputs.  nxt / last: lists of three dicts
    (levels 0-2) with vmap, nmap, image (+ dx, dy for nxt).  Returns
    (pose, info[ok, icp_err, icp_count, rgb_err, rgb_count]).
    grid (reference precision only): the library's tracking grid per level
    (fb_track_reduction_grid); the normal equations are then summed and
    solved in the order of its kernels, for a bit-for-bit comparison."""
    keep = []

    def arr(lst, key, dtype):
        ptrs = (ctypes.c_void_p * 3)()
        for i in range(3):
            a = np.ascontiguousarray(lst[i][key], dtype)
            keep.append(a)
            ptrs[i] = a.ctypes.data
        return ptrs
    out = np.zeros((4, 4), np.float64)
    info = np.zeros(5, np.float64)
    args = [arr(nxt, "vmap", np.float32), arr(nxt, "nmap", np.float32), arr(nxt, "image", np.uint8),
            arr(nxt, "dx", np.int16), arr(nxt, "dy", np.int16), arr(last, "vmap", np.float32),
            arr(last, "nmap", np.float32), arr(last, "image", np.uint8),
            _p(np.ascontiguousarray(last_pose, np.float64)), _p(out), _p(info)]
    if grid is None:
        lib().fbo_track(ctypes.byref(cfg), *args)
    else:
        assert cfg.precision == 32, "the kernels' summation order is a reference-precision mode"
        g = (ctypes.c_int * 3)(*[int(x) for x in grid])
        if lib().fbo_track_gpu_order(ctypes.byref(cfg), g, *args) != 0:
            raise ValueError(f"bad tracking grid {list(grid)}")
    return out, info


def num_threads():
    return int(lib().fbo_num_threads())
