"""Host-side mirror of the reference's per-frame interface over the C ABI.

`System` mirrors Core/System.h (System(SysDesc*), GrabImage(image, depth),
RebootSystem) for one camera; `Session` exposes the full C ABI session
(frame results, map inspection).  The stage functions at the bottom mirror the
reference's kernel free functions (Tracking/Reduction.h, Mapping/RenderScene.h)
on torch CUDA tensors, which serve only as device memory here.
"""
import ctypes
import os

import numpy as np

from . import _lib
from ._lib import Config, FrameResult, Image, MapStats, check


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


# --------------------------------------------------------------- configs --

def reference_config(width, height, fx=None, fy=None, cx=None, cy=None, depth_scale=1000.0,
                     depth_cutoff=3.0):
    """The reference's compile-time constants (Mapping/DeviceMap.h:135-151,
    Tracking/Tracking.h:98-100) for a width x height camera."""
    c = Config()
    _lib.load().fb_default_config(ctypes.byref(c), width, height)
    if fx is not None:
        c.fx = fx
    if fy is not None:
        c.fy = fy
    if cx is not None:
        c.cx = cx
    if cy is not None:
        c.cy = cy
    c.depth_scale = depth_scale
    c.depth_cutoff = depth_cutoff
    c.trunc_dist = float(np.float32(c.voxel_size) * np.float32(8))
    return c


def make_config(width, height, voxel_size, trunc_voxels, num_buckets, num_excess, num_blocks,
                iters=(10, 5, 3), depth_scale=5000.0, depth_cutoff=4.0, depth_min=0.1, depth_max=4.0,
                fx=None, fy=None, cx=None, cy=None):
    c = Config()
    _lib.load().fb_default_config(ctypes.byref(c), width, height)
    c.fx = fx if fx is not None else 525.0 * width / 640.0
    c.fy = fy if fy is not None else c.fx
    c.cx = cx if cx is not None else width / 2.0
    c.cy = cy if cy is not None else height / 2.0
    c.depth_scale, c.depth_cutoff = depth_scale, depth_cutoff
    c.voxel_size = voxel_size
    c.trunc_dist = float(np.float32(voxel_size) * np.float32(trunc_voxels))
    c.depth_min, c.depth_max = depth_min, depth_max
    c.num_buckets, c.num_excess, c.num_blocks = num_buckets, num_excess, num_blocks
    for i in range(3):
        c.iters[i] = iters[i]
    return c


def config_c1():
    """320x240, 8 mm voxels, truncation 3 voxels, 2^18 buckets (2^17 excess,
    2^17 blocks), 10/5/4 iterations (levels 0/1/2)."""
    return make_config(320, 240, 0.008, 3, 1 << 18, 1 << 17, 1 << 17, iters=(10, 5, 4))


def config_c2():
    """640x480, 5 mm voxels, truncation 4 voxels, 2^20 buckets + 2^18 excess,
    2^18 blocks, 10/5/3 iterations."""
    return make_config(640, 480, 0.005, 4, 1 << 20, 1 << 18, 1 << 18, iters=(10, 5, 3))


def config_dict(c):
    return {k: (list(getattr(c, k)) if k == "iters" else getattr(c, k)) for k, _ in Config._fields_}


# --------------------------------------------------------------- session --

class Session:
    """One camera's frames, tracker and voxel-block map on the GPU."""

    def __init__(self, cfg, stream=None):
        self.lib = _lib.load()
        self.cfg = cfg
        h = ctypes.c_void_p()
        check("fb_session_create", self.lib.fb_session_create(ctypes.byref(cfg), stream, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.fb_session_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def reset(self):
        check("fb_session_reset", self.lib.fb_session_reset(self.h))

    def snapshot(self):
        """The session's whole state as bytes (fb_snapshot)."""
        n = ctypes.c_size_t()
        check("fb_snapshot_bytes", self.lib.fb_snapshot_bytes(self.h, ctypes.byref(n)))
        buf = np.empty(n.value, np.uint8)
        w = ctypes.c_size_t()
        check("fb_snapshot", self.lib.fb_snapshot(self.h, _p(buf), buf.nbytes, ctypes.byref(w)))
        return buf[:w.value]

    def restore(self, snap):
        """Continue from a snapshot of a session with the same configuration."""
        snap = np.ascontiguousarray(snap, np.uint8)
        check("fb_restore", self.lib.fb_restore(self.h, _p(snap), snap.nbytes))

    def mesh(self, max_triangles=None, device=False):
        """MeshScene (fb_mesh_scene): the map's marching-cubes triangle soup as
        (vertex, normal, color), three rows per triangle -- float32 [3T, 3]
        metres and unit normals, uint8 [3T, 3] colours -- as numpy arrays, or
        as CUDA tensors with device=True.  At most max_triangles triangles."""
        import torch
        n = ctypes.c_uint64()
        check("fb_mesh_scene", self.lib.fb_mesh_scene(self.h, None, None, None, 0, ctypes.byref(n), None))
        cap = n.value if max_triangles is None else min(n.value, int(max_triangles))
        V = torch.empty((3 * cap, 3), dtype=torch.float32, device="cuda")
        N = torch.empty((3 * cap, 3), dtype=torch.float32, device="cuda")
        C = torch.empty((3 * cap, 3), dtype=torch.uint8, device="cuda")
        if cap:
            torch.cuda.current_stream().synchronize()
            check("fb_mesh_scene", self.lib.fb_mesh_scene(self.h, V.data_ptr(), N.data_ptr(), C.data_ptr(), cap,
                                                          ctypes.byref(n), None))
        if device:
            return V, N, C
        return V.cpu().numpy(), N.cpu().numpy(), C.cpu().numpy()

    def save_mesh(self, path):
        """System::WriteMeshToDisk: mesh the map and write it to `path` as
        ASCII PLY (fb_save_mesh).  Returns the triangle count."""
        n = ctypes.c_uint64()
        check("fb_save_mesh", self.lib.fb_save_mesh(self.h, os.fsencode(path), ctypes.byref(n)))
        return n.value

    def set_keypoints(self, on):
        """Key points on every frame, the bootstrap from the last frame's key
        points, keyframes, the key map and relocalisation (fb_session_set_keypoints)."""
        check("fb_session_set_keypoints", self.lib.fb_session_set_keypoints(self.h, 1 if on else 0))

    def keypoint_stats(self):
        st = _lib.KeypointStats()
        check("fb_session_keypoint_stats", self.lib.fb_session_keypoint_stats(self.h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.KeypointStats._fields_}

    def keypoints(self, which=0):
        """The key points of the last (0) or next (1) frame: kp [n, 4] (x, y,
        scale, angle), pts [n, 4], nrm [n, 4], desc [n, 64]."""
        n = ctypes.c_uint32()
        check("fb_download_keypoints", self.lib.fb_download_keypoints(self.h, which, None, None, None, None, 0,
                                                                      ctypes.byref(n)))
        k = n.value
        kp, pts, nrm = (np.zeros((k, 4), np.float32) for _ in range(3))
        desc = np.zeros((k, 64), np.float32)
        check("fb_download_keypoints", self.lib.fb_download_keypoints(self.h, which, _p(kp), _p(pts), _p(nrm),
                                                                      _p(desc), k, ctypes.byref(n)))
        return {"kp": kp, "pts": pts, "nrm": nrm, "desc": desc}

    def write_map_file(self, path):
        """System::WriteMapToDisk: the map in the reference's dump layout."""
        check("fb_write_map_file", self.lib.fb_write_map_file(self.h, os.fsencode(path)))

    def read_map_file(self, path):
        """System::ReadMapFromDisk: load a map in the reference's dump layout;
        the tracker restarts and mapping is disabled (set_mapping)."""
        check("fb_read_map_file", self.lib.fb_read_map_file(self.h, os.fsencode(path)))

    def set_mapping(self, on):
        """Fuse frames into the map (True) or only track against it."""
        check("fb_session_set_mapping", self.lib.fb_session_set_mapping(self.h, 1 if on else 0))

    def prepare(self, shared=False):
        """Capture every frame graph now (for frames alone, or in batch steps
        with shared=True)."""
        check("fb_session_prepare", self.lib.fb_session_prepare(self.h, 1 if shared else 0))

    def prepare_some(self, max_graphs=1, shared=False):
        """Capture at most max_graphs of the missing frame graphs; returns how
        many are still missing."""
        left = ctypes.c_int()
        check("fb_session_prepare_some", self.lib.fb_session_prepare_some(
            self.h, 1 if shared else 0, int(max_graphs), ctypes.byref(left)))
        return left.value

    def stage(self, depth, rgb):
        """Start copying a later frame (host numpy arrays, ideally pinned) to
        the device (fb_stage_frame); grab(None, None) takes it."""
        depth = np.ascontiguousarray(depth, np.uint16)
        rgb = np.ascontiguousarray(rgb, np.uint8)
        self._staged = getattr(self, "_staged", [])[-1:] + [(depth, rgb)]   # keep the host memory alive
        check("fb_stage_frame", self.lib.fb_stage_frame(self.h, _p(depth), depth.strides[0], _p(rgb),
                                                        rgb.strides[0]))

    def grab(self, depth, rgb, on_device=False):
        """One frame.  depth: u16 [H, W]; rgb: u8 [H, W, 3]; numpy arrays
        (host) or, with on_device, objects with data_ptr() (device); None and
        None: the oldest frame given to stage()."""
        r = FrameResult()
        if depth is None and rgb is None:
            code = self.lib.fb_grab_frame(self.h, None, 0, None, 0, 0, ctypes.byref(r))
        elif on_device:
            W = self.cfg.width
            code = self.lib.fb_grab_frame(self.h, depth.data_ptr(), 2 * W, rgb.data_ptr(), 3 * W, 1,
                                          ctypes.byref(r))
        else:
            depth = np.ascontiguousarray(depth, np.uint16)
            rgb = np.ascontiguousarray(rgb, np.uint8)
            code = self.lib.fb_grab_frame(self.h, _p(depth), depth.strides[0], _p(rgb), rgb.strides[0], 0,
                                          ctypes.byref(r))
        check("fb_grab_frame", code)
        return r

    @staticmethod
    def result_dict(r):
        return dict(status=r.status, tracked=r.tracked, tracker_state=r.tracker_state, fused=r.fused,
                    no_visible=r.no_visible, no_allocated=r.no_allocated, no_new=r.no_new,
                    error_flags=r.error_flags, icp_error=r.icp_error, icp_count=r.icp_count,
                    rgb_error=r.rgb_error, rgb_count=r.rgb_count,
                    pose=np.array(r.pose[:]).reshape(4, 4), frame_id=r.frame_id)

    STAGES = ["resize", "pyramid", "tracking", "allocation", "visibility", "integration", "zrange", "raycast"]

    def set_profiling(self, on=True):
        check("fb_session_set_profiling", self.lib.fb_session_set_profiling(self.h, 1 if on else 0))

    def stage_times(self):
        """{stage: (total device ms, calls)} since profiling was switched on."""
        ms = np.zeros(8, np.float64)
        calls = np.zeros(8, np.uint64)
        check("fb_session_stage_times", self.lib.fb_session_stage_times(self.h, _p(ms), _p(calls), 8))
        return {k: (float(ms[i]), int(calls[i])) for i, k in enumerate(self.STAGES)}

    def set_graphs(self, on=True):
        check("fb_session_set_graphs", self.lib.fb_session_set_graphs(self.h, 1 if on else 0))


    def launch_count(self):
        n = ctypes.c_uint64()
        check("fb_session_launch_count", self.lib.fb_session_launch_count(self.h, ctypes.byref(n)))
        return int(n.value)

    def transfer_bytes(self):
        h2d, d2h = ctypes.c_size_t(), ctypes.c_size_t()
        check("fb_frame_transfer_bytes", self.lib.fb_frame_transfer_bytes(ctypes.byref(self.cfg), ctypes.byref(h2d),
                                                                         ctypes.byref(d2h)))
        return int(h2d.value), int(d2h.value)

    def pose(self):
        T = np.zeros((4, 4))
        check("fb_get_pose", self.lib.fb_get_pose(self.h, _p(T)))
        return T

    def level(self, which, lv):
        W, H = self.cfg.width >> lv, self.cfg.height >> lv
        out = dict(vmap=np.zeros((H, W, 4), np.float32), nmap=np.zeros((H, W, 4), np.float32),
                   depth=np.zeros((H, W), np.float32), image=np.zeros((H, W), np.uint8),
                   dx=np.zeros((H, W), np.int16), dy=np.zeros((H, W), np.int16))
        check("fb_download_level", self.lib.fb_download_level(
            self.h, which, lv, _p(out["vmap"]), _p(out["nmap"]), _p(out["depth"]), _p(out["image"]),
            _p(out["dx"]), _p(out["dy"])))
        return out

    def raw(self, which):
        out = np.zeros((self.cfg.height, self.cfg.width), np.float32)
        check("fb_download_raw", self.lib.fb_download_raw(self.h, which, _p(out)))
        return out

    def stats(self):
        s = MapStats()
        check("fb_map_get_stats", self.lib.fb_map_get_stats(self.h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in MapStats._fields_}

    def entries(self):
        n = self.cfg.num_buckets + self.cfg.num_excess
        e = np.zeros((n, 5), np.int32)
        check("fb_map_download_entries", self.lib.fb_map_download_entries(self.h, _p(e)))
        return e

    def allocated(self):
        """Occupied slots sorted by (x, y, z): (slots, entries[n, 5])."""
        e = self.entries()
        occ = np.nonzero(e[:, 3] >= 0)[0]
        rows = e[occ]
        order = np.lexsort((rows[:, 2], rows[:, 1], rows[:, 0]))
        return occ[order].astype(np.int32), rows[order]

    def blocks(self, ptrs):
        ptrs = np.ascontiguousarray(ptrs, np.int32)
        n = len(ptrs)
        sdf = np.zeros((n, 512), np.float32)
        w = np.zeros((n, 512), np.uint8)
        rgb = np.zeros((n, 512, 3), np.uint8)
        check("fb_map_download_blocks", self.lib.fb_map_download_blocks(self.h, _p(ptrs), n, _p(sdf), _p(w), _p(rgb)))
        return sdf, w, rgb

    def visible(self):
        n = ctypes.c_uint32()
        check("fb_map_download_visible", self.lib.fb_map_download_visible(self.h, None, 0, ctypes.byref(n)))
        s = np.zeros(n.value, np.int32)
        if n.value:
            check("fb_map_download_visible",
                  self.lib.fb_map_download_visible(self.h, _p(s), n.value, ctypes.byref(n)))
        return s


class System:
    """Mirror of the reference's System (Core/System.h:29-80) for the dense
    path: System(desc) builds the map and tracker; GrabImage(image, depth)
    tracks, fuses and raycasts one frame and returns True (the reference's
    GrabImage always returns true, Core/System.cc:137)."""

    def __init__(self, cfg):
        self.session = Session(cfg)
        self.state = True
        self.nFrames = 0
        self.last = None

    def GrabImage(self, image, depth):
        r = self.session.grab(depth, image)
        self.last = r
        self.state = bool(r.tracked)
        if self.state:
            self.nFrames += 1
        return True

    def RebootSystem(self):
        self.session.reset()
        self.nFrames = 0

    def GetCurrentPose(self):
        return self.session.pose()


# ----------------------------------------------------- per-stage functions --
# Arguments are torch CUDA tensors (contiguous rows; pitch = row stride).

def _img(t, elem_bytes):
    rows, cols = t.shape[0], t.shape[1]
    return Image(t.data_ptr(), t.stride(0) * t.element_size(), cols, rows)


def _stream(stream):
    return None if stream is None else ctypes.c_void_p(stream.cuda_stream)


def filter_depth(depth, raw, filtered, depth_scale, depth_cutoff, stream=None):
    L = _lib.load()
    check("fb_filter_depth", L.fb_filter_depth(ctypes.byref(_img(depth, 2)), ctypes.byref(_img(raw, 4)),
                                                ctypes.byref(_img(filtered, 4)), depth_scale, depth_cutoff,
                                                _stream(stream)))


def image_to_intensity(rgb, gray, stream=None):
    check("fb_image_to_intensity", _lib.load().fb_image_to_intensity(
        ctypes.byref(_img(rgb, 3)), ctypes.byref(_img(gray, 1)), _stream(stream)))


def pyrdown_gauss(src, dst, stream=None):
    L = _lib.load()
    fn = L.fb_pyrdown_gauss_f32 if src.element_size() == 4 else L.fb_pyrdown_gauss_u8
    check("fb_pyrdown_gauss", fn(ctypes.byref(_img(src, 0)), ctypes.byref(_img(dst, 0)), _stream(stream)))


def compute_vmap(depth, vmap, fx, fy, cx, cy, depth_cutoff, stream=None):
    check("fb_compute_vmap", _lib.load().fb_compute_vmap(ctypes.byref(_img(depth, 4)), ctypes.byref(_img(vmap, 16)),
                                                        fx, fy, cx, cy, depth_cutoff, _stream(stream)))


def compute_nmap(vmap, nmap, stream=None):
    check("fb_compute_nmap", _lib.load().fb_compute_nmap(ctypes.byref(_img(vmap, 16)), ctypes.byref(_img(nmap, 16)),
                                                        _stream(stream)))


def compute_derivative_image(gray, dx, dy, stream=None):
    check("fb_compute_derivative_image", _lib.load().fb_compute_derivative_image(
        ctypes.byref(_img(gray, 1)), ctypes.byref(_img(dx, 2)), ctypes.byref(_img(dy, 2)), _stream(stream)))


def resize_map(vsrc, nsrc, vdst, ndst, stream=None):
    check("fb_resize_map", _lib.load().fb_resize_map(ctypes.byref(_img(vsrc, 16)), ctypes.byref(_img(nsrc, 16)),
                                                    ctypes.byref(_img(vdst, 16)), ctypes.byref(_img(ndst, 16)),
                                                    _stream(stream)))


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def icp_step(vcurr, vlast, ncurr, nlast, Rcurr, tcurr, Rlast, RlastInv, tlast, K, scratch, stream=None):
    """Returns (residual[2], A[6,6], b[6]) like the reference's ICPStep."""
    res = np.zeros(2, np.float32)
    A = np.zeros(36)
    b = np.zeros(6)
    args = [_f32(Rcurr), _f32(tcurr), _f32(Rlast), _f32(RlastInv), _f32(tlast), _f32(K)]
    check("fb_icp_step", _lib.load().fb_icp_step(
        ctypes.byref(_img(vcurr, 16)), ctypes.byref(_img(vlast, 16)), ctypes.byref(_img(ncurr, 16)),
        ctypes.byref(_img(nlast, 16)), *[_p(a) for a in args], scratch.data_ptr(),
        scratch.numel() * scratch.element_size(), _p(res), _p(A), _p(b), _stream(stream)))
    return res, A.reshape(6, 6), b


def rgb_step(gcurr, glast, vcurr, vlast, dx, dy, Rcurr, RcurrInv, Rlast, RlastInv, tcurr, tlast, K, scratch,
             stream=None):
    res = np.zeros(2, np.float32)
    A = np.zeros(36)
    b = np.zeros(6)
    args = [_f32(Rcurr), _f32(RcurrInv), _f32(Rlast), _f32(RlastInv), _f32(tcurr), _f32(tlast), _f32(K)]
    check("fb_rgb_step", _lib.load().fb_rgb_step(
        ctypes.byref(_img(gcurr, 1)), ctypes.byref(_img(glast, 1)), ctypes.byref(_img(vcurr, 16)),
        ctypes.byref(_img(vlast, 16)), ctypes.byref(_img(dx, 2)), ctypes.byref(_img(dy, 2)),
        *[_p(a) for a in args], scratch.data_ptr(), scratch.numel() * scratch.element_size(), _p(res), _p(A),
        _p(b), _stream(stream)))
    return res, A.reshape(6, 6), b


def rgb_step_static(gcurr, glast, vcurr, vlast, dx, dy, Rcurr, RcurrInv, Rlast, RlastInv, tcurr, tlast, K,
                    stream=None):
    """rgb_step without a scratch argument: for callers that cannot allocate
    device memory where they track (a frame loop that cannot wait for
    cudaFree, a plug-in in a host that owns all device memory).  The
    library's own fixed device buffer limits images to 640 x 480 pixels, and
    calls that overlap on the GPU share that buffer.  Synchronous."""
    res = np.zeros(2, np.float32)
    A = np.zeros(36)
    b = np.zeros(6)
    args = [_f32(Rcurr), _f32(RcurrInv), _f32(Rlast), _f32(RlastInv), _f32(tcurr), _f32(tlast), _f32(K)]
    check("fb_rgb_step_static", _lib.load().fb_rgb_step_static(
        ctypes.byref(_img(gcurr, 1)), ctypes.byref(_img(glast, 1)), ctypes.byref(_img(vcurr, 16)),
        ctypes.byref(_img(vlast, 16)), ctypes.byref(_img(dx, 2)), ctypes.byref(_img(dy, 2)),
        *[_p(a) for a in args], _p(res), _p(A), _p(b), _stream(stream)))
    return res, A.reshape(6, 6), b


def step_scratch_bytes(cols, rows):
    return int(_lib.load().fb_step_scratch_bytes(cols, rows))


def track_reduction_grids(cfg):
    """The tracking kernels' grid at each pyramid level of cfg's camera
    (fb_track_reduction_grid): the summation order of the normal equations."""
    return tuple(int(_lib.load().fb_track_reduction_grid((cfg.width >> l) * (cfg.height >> l))) for l in range(3))


def pose_parts(T):
    """Matrix3f rotation, its transpose and translation of a 4x4 pose, as
    Frame::GpuRotation / GpuInvRotation / GpuTranslation round them."""
    T = np.asarray(T, np.float64)
    return (T[:3, :3].astype(np.float32), T[:3, :3].T.astype(np.float32), T[:3, 3].astype(np.float32))


def fuse_map_color(session, depth, rgb, nmap, T, K, stream=None):
    R, Ri, t = pose_parts(T)
    n = ctypes.c_uint32()
    check("fb_fuse_map_color", _lib.load().fb_fuse_map_color(
        session.h, ctypes.byref(_img(depth, 4)), ctypes.byref(_img(rgb, 3)), ctypes.byref(_img(nmap, 16)),
        _p(np.ascontiguousarray(R)), _p(np.ascontiguousarray(Ri)), _p(t), _p(_f32(K)), ctypes.byref(n),
        _stream(stream)))
    return n.value


def raycast(session, vmap, nmap, T, K, stream=None):
    R, Ri, t = pose_parts(T)
    rendered = ctypes.c_int()
    check("fb_raycast", _lib.load().fb_raycast(
        session.h, ctypes.byref(_img(vmap, 16)), ctypes.byref(_img(nmap, 16)), _p(np.ascontiguousarray(R)),
        _p(np.ascontiguousarray(Ri)), _p(t), _p(_f32(K)), ctypes.byref(rendered), _stream(stream)))
    return bool(rendered.value)


def render_top_down(session, dist, vmap, nmap, rgba, stream=None):
    """System::RenderTopDown (fb_render_top_down): the model from `dist`
    metres above, raycast into vmap/nmap (float4 device tensors) and shaded
    into rgba (uchar4).  Returns whether any block was in view."""
    rendered = ctypes.c_int()
    check("fb_render_top_down", _lib.load().fb_render_top_down(
        session.h, float(dist), ctypes.byref(_img(vmap, 16)), ctypes.byref(_img(nmap, 16)),
        ctypes.byref(_img(rgba, 4)), ctypes.byref(rendered), _stream(stream)))
    return bool(rendered.value)


def top_down_pose(dist):
    """The pose System::RenderTopDown renders from (4x4, double): rotation
    by pi/2 about -x (cos(pi/2) kept as computed), camera at (0, -dist, 0)."""
    c = np.cos(np.pi / 2)
    return np.array([[1, 0, 0, 0], [0, c, 1, -float(np.float32(dist))], [0, -1, c, 0], [0, 0, 0, 1]], np.float64)


def graph_exec_stats():
    """Frame-graph executables kept for reuse, and the captures served by an
    update of a kept one and by a new instantiation (fb_graph_exec_stats)."""
    v = [ctypes.c_longlong() for _ in range(3)]
    _lib.load().fb_graph_exec_stats(*[ctypes.byref(x) for x in v])
    return {"pooled": v[0].value, "updated": v[1].value, "instantiated": v[2].value}


def match_descriptors(query, train, stream=None):
    """Two nearest train descriptors of every query (fb_match_descriptors);
    CUDA float32 tensors [n, 64].  Returns (best int32 [nq, 2], dist [nq, 2])
    as tensors on the device."""
    import torch
    nq, nt = int(query.shape[0]), int(train.shape[0])
    best = torch.empty((nq, 2), dtype=torch.int32, device=query.device)
    dist = torch.empty((nq, 2), dtype=torch.float32, device=query.device)
    check("fb_match_descriptors", _lib.load().fb_match_descriptors(
        query.data_ptr() if nq else None, nq, train.data_ptr() if nt else None, nt,
        best.data_ptr() if nq else None, dist.data_ptr() if nq else None, _stream(stream)))
    return best, dist


def pose_estimate(src, ref, iterations=35, check_angle=True, seed=1):
    """Solver::PoseEstimate (fb_pose_estimate) on host arrays [n, 3]:
    (ok, T 4x4 mapping ref onto src, inlier mask)."""
    src = np.ascontiguousarray(src, np.float64)
    ref = np.ascontiguousarray(ref, np.float64)
    n = len(src)
    T = np.zeros((4, 4), np.float64)
    inl = np.zeros(max(n, 1), np.uint8)
    ok = ctypes.c_int()
    check("fb_pose_estimate", _lib.load().fb_pose_estimate(_p(src), _p(ref), n, int(iterations), 1 if check_angle else 0,
                                                           int(seed), _p(T), _p(inl), ctypes.byref(ok)))
    return bool(ok.value), T, inl[:n].astype(bool)


def mesh_case_table():
    """The marching-cubes case table of fb_mesh_scene: (tri int8 [256, 16]
    edge triples, -1 filled; counts int32 [256])."""
    tri = np.zeros((256, 16), np.int8)
    cnt = np.zeros(256, np.int32)
    check("fb_mesh_case_table", _lib.load().fb_mesh_case_table(_p(tri), _p(cnt)))
    return tri, cnt


def write_ply(path, vertex, normal, color):
    """The file writing of System::WriteMeshToDisk (fb_write_ply): ASCII PLY
    of a triangle soup (host arrays, three rows per triangle)."""
    V = np.ascontiguousarray(vertex, np.float32)
    N = np.ascontiguousarray(normal, np.float32)
    C = np.ascontiguousarray(color, np.uint8)
    if not (V.shape == N.shape == C.shape and V.ndim == 2 and V.shape[1] == 3 and V.shape[0] % 3 == 0):
        raise ValueError("vertex, normal and color must be [3T, 3] arrays of one shape")
    check("fb_write_ply", _lib.load().fb_write_ply(os.fsencode(path), _p(V), _p(N), _p(C), V.shape[0] // 3))


def render_image(vmap, nmap, light, rgba, stream=None):
    """RenderImage: Phong shading of a vertex/normal map into rgba (uchar4
    per pixel, device tensors)."""
    check("fb_render_image", _lib.load().fb_render_image(
        ctypes.byref(_img(vmap, 16)), ctypes.byref(_img(nmap, 16)), _p(_f32(light)), ctypes.byref(_img(rgba, 4)),
        _stream(stream)))


def depth_to_image(depth, rgba, stream=None):
    check("fb_depth_to_image", _lib.load().fb_depth_to_image(ctypes.byref(_img(depth, 4)),
                                                              ctypes.byref(_img(rgba, 4)), _stream(stream)))


def rgb_to_rgba(rgb, rgba, stream=None):
    check("fb_rgb_to_rgba", _lib.load().fb_rgb_to_rgba(ctypes.byref(_img(rgb, 3)), ctypes.byref(_img(rgba, 4)),
                                                        _stream(stream)))
