"""ORACLE / TEST INFRASTRUCTURE ONLY.

ctypes wrapper of oracle/_ref/libfusion_ref.so: the reference's own CUDA
kernels (compiled unmodified from the reference tree by oracle/Makefile) driven
by the restated host loop in oracle/ref_harness/harness.cu.  Needs a GPU.
Used only to generate golden vectors and for side-by-side checks; never by the
shipped library.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libfusion_ref.so")

_c_double_p = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def available():
    return os.path.exists(LIB_PATH)


class RefHarness:
    def __init__(self, cols, rows, fx, fy, cx, cy, depth_scale, depth_cutoff, iters=(10, 5, 3)):
        lib = ctypes.CDLL(LIB_PATH)
        lib.ref_create.restype = ctypes.c_void_p
        lib.ref_create.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_float] * 6 + [ctypes.c_void_p]
        for name in ["ref_destroy", "ref_swap"]:
            getattr(lib, name).argtypes = [ctypes.c_void_p]
        self.lib = lib
        self.cols, self.rows = cols, rows
        it = np.array(iters, np.int32)
        self.h = lib.ref_create(cols, rows, fx, fy, cx, cy, depth_scale, depth_cutoff, _p(it))
        if not self.h:
            raise RuntimeError("ref_create failed")

    def close(self):
        if self.h:
            self.lib.ref_destroy(ctypes.c_void_p(self.h))
            self.h = None

    def __del__(self):
        self.close()

    def _call(self, name, *args):
        fn = getattr(self.lib, name)
        return fn(ctypes.c_void_p(self.h), *args)

    def constants(self):
        out = np.zeros(12, np.float64)
        self.lib.ref_constants(_p(out))
        keys = ["voxel_size", "trunc_dist", "depth_min", "depth_max", "num_buckets",
                "num_excess", "num_blocks", "max_rendering_blocks", "step_scale",
                "sizeof_hash_entry", "sizeof_voxel", "sizeof_rendering_block"]
        return dict(zip(keys, out.tolist()))

    def grab(self, depth, rgb):
        info = np.zeros(8, np.float64)
        self._call("ref_grab", _p(np.ascontiguousarray(depth)), _p(np.ascontiguousarray(rgb)), _p(info))
        return info

    def get_pose(self, which):
        T = np.zeros((4, 4), np.float64)
        self._call("ref_get_pose", ctypes.c_int(which), _p(T))
        return T

    def set_pose(self, which, T):
        T = np.ascontiguousarray(T, np.float64)
        self._call("ref_set_pose", ctypes.c_int(which), _p(T))

    def swap(self):
        self._call("ref_swap")

    def fill_images(self, which, depth, rgb):
        self._call("ref_fill_images", ctypes.c_int(which), _p(np.ascontiguousarray(depth)),
                   _p(np.ascontiguousarray(rgb)))

    def resize_images(self, which):
        self._call("ref_resize_images", ctypes.c_int(which))

    def level(self, which, lv):
        c, r = self.cols >> lv, self.rows >> lv
        out = dict(vmap=np.zeros((r, c, 4), np.float32), nmap=np.zeros((r, c, 4), np.float32),
                   depth=np.zeros((r, c), np.float32), image=np.zeros((r, c), np.uint8),
                   dx=np.zeros((r, c), np.int16), dy=np.zeros((r, c), np.int16))
        self._call("ref_download_level", ctypes.c_int(which), ctypes.c_int(lv), _p(out["vmap"]),
                   _p(out["nmap"]), _p(out["depth"]), _p(out["image"]), _p(out["dx"]), _p(out["dy"]))
        return out

    def range(self, which):
        out = np.zeros((self.rows, self.cols), np.float32)
        self._call("ref_download_range", ctypes.c_int(which), _p(out))
        return out

    def upload_maps(self, which, lv, vmap, nmap):
        self._call("ref_upload_maps", ctypes.c_int(which), ctypes.c_int(lv),
                   _p(np.ascontiguousarray(vmap, np.float32)), _p(np.ascontiguousarray(nmap, np.float32)))

    def icp_step(self, lv):
        A = np.zeros(36, np.float64); b = np.zeros(6, np.float64); res = np.zeros(2, np.float32)
        self._call("ref_icp_step", ctypes.c_int(lv), _p(A), _p(b), _p(res))
        return A.reshape(6, 6), b, res

    def rgb_step(self, lv):
        A = np.zeros(36, np.float64); b = np.zeros(6, np.float64); res = np.zeros(2, np.float32)
        self._call("ref_rgb_step", ctypes.c_int(lv), _p(A), _p(b), _p(res))
        return A.reshape(6, 6), b, res

    def reset_map(self):
        self._call("ref_reset_map")

    def fuse(self, which):
        n = ctypes.c_uint32(0)
        self._call("ref_fuse", ctypes.c_int(which), ctypes.byref(n))
        return int(n.value)

    def raytrace(self, which, no_visible):
        self._call("ref_raytrace", ctypes.c_int(which), ctypes.c_uint32(no_visible))

    def hash_entries(self):
        n = int(self.constants()["num_buckets"] + self.constants()["num_excess"])
        e = np.zeros((n, 5), np.int32)
        cnt = np.zeros(2, np.int32)
        self._call("ref_download_hash", _p(e), _p(cnt))
        return e, cnt

    def visible(self, n):
        e = np.zeros((n, 5), np.int32)
        self._call("ref_download_visible", _p(e), ctypes.c_uint32(n))
        return e

    def blocks(self, ptrs):
        ptrs = np.ascontiguousarray(ptrs, np.int32)
        n = len(ptrs)
        sdf = np.zeros((n, 512), np.float32)
        w = np.zeros((n, 512), np.uint8)
        rgb = np.zeros((n, 512, 3), np.uint8)
        self._call("ref_download_blocks", _p(ptrs), ctypes.c_int(n), _p(sdf), _p(w), _p(rgb))
        return sdf, w, rgb

    def mesh(self):
        """Mapping::CreateModel with the reference's MeshScene and tables:
        (vertex, normal, color), three rows per triangle."""
        n = ctypes.c_uint32(0)
        fn = self.lib.ref_mesh_scene
        fn.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_uint32, ctypes.c_void_p]
        fn(ctypes.c_void_p(self.h), None, None, None, ctypes.c_uint32(0), ctypes.byref(n))
        # the count is only known after a run; run again to download
        V = np.zeros((3 * n.value, 3), np.float32)
        N = np.zeros((3 * n.value, 3), np.float32)
        C = np.zeros((3 * n.value, 3), np.uint8)
        fn(ctypes.c_void_p(self.h), _p(V), _p(N), _p(C), ctypes.c_uint32(n.value), ctypes.byref(n))
        return V, N, C

    def write_map(self, path):
        """System::WriteMapToDisk of the harness's map to `path`."""
        fn = self.lib.ref_write_map
        fn.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        if fn(ctypes.c_void_p(self.h), os.fsencode(path)) != 0:
            raise RuntimeError("ref_write_map failed")

    def read_map(self, path):
        """The map part of System::ReadMapFromDisk from `path`."""
        fn = self.lib.ref_read_map
        fn.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        if fn(ctypes.c_void_p(self.h), os.fsencode(path)) != 0:
            raise RuntimeError("ref_read_map failed")

    def mesh_time(self, iters=5):
        """Mean wall ms of the reference's MeshScene on the current map (its
        buffers allocated once) and its triangle count."""
        ms = ctypes.c_double()
        n = ctypes.c_uint32()
        fn = self.lib.ref_mesh_time
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        fn(ctypes.c_void_p(self.h), iters, ctypes.byref(ms), ctypes.byref(n))
        return ms.value, n.value

    def zrange(self):
        zmin = np.zeros((60, 80), np.float32)
        zmax = np.zeros((60, 80), np.float32)
        self._call("ref_download_zrange", _p(zmin), _p(zmax))
        return zmin, zmax


def render_image(vmap, nmap, light):
    """The reference's RenderImage on host float4 maps; uint8 [H, W, 4]."""
    lib = ctypes.CDLL(LIB_PATH)
    H, W, _ = vmap.shape
    out = np.zeros((H, W, 4), np.uint8)
    lib.ref_render_image(W, H, _p(np.ascontiguousarray(vmap, np.float32)), _p(np.ascontiguousarray(nmap, np.float32)),
                         _p(np.ascontiguousarray(light, np.float32)), _p(out))
    return out


def depth_to_image(depth):
    lib = ctypes.CDLL(LIB_PATH)
    H, W = depth.shape
    out = np.zeros((H, W, 4), np.uint8)
    lib.ref_depth_to_image(W, H, _p(np.ascontiguousarray(depth, np.float32)), _p(out))
    return out


def rgb_to_rgba(rgb):
    lib = ctypes.CDLL(LIB_PATH)
    H, W, _ = rgb.shape
    out = np.zeros((H, W, 4), np.uint8)
    lib.ref_rgb_to_rgba(W, H, _p(np.ascontiguousarray(rgb, np.uint8)), _p(out))
    return out


def mesh_tables():
    """The reference's marching-cubes tables (Mapping/Constant.h): (tri int8
    [256, 16], triangles per case int32 [256])."""
    lib = ctypes.CDLL(LIB_PATH)
    tri = np.zeros((256, 16), np.int8)
    ntri = np.zeros(256, np.int32)
    lib.ref_mesh_tables(_p(tri), _p(ntri))
    return tri, ntri


def sizeof_surf():
    return int(ctypes.CDLL(LIB_PATH).ref_sizeof_surf())
