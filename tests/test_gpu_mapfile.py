"""The reference's map file (System::WriteMapToDisk / ReadMapFromDisk,
Core/System.cc:195-271) through fb_write_map_file / fb_read_map_file.

- Round trip in both forms: a session's map written and read into a fresh
  session of the same configuration gives the same hash table, counters,
  voxels and mesh; the file has the reference's size for those map sizes;
  as in the reference, the loaded session restarts its tracker and tracks
  without fusing until mapping is switched back on.
- Against the reference's own code (oracle/_ref): a map the reference's
  kernels built and the harness dumped in the reference's layout, loaded
  here, raycasts from the reference's last pose to the reference's vertex
  map (within 1e-5 m on 99.9 % of pixels) and meshes to the reference
  kernel's vertices; a map
  this library built, loaded into the reference's arrays, meshes there to
  this library's vertices.
"""
import os
import shutil

import numpy as np
import pytest

import rgbd_synth as synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _file_bytes(cfg):
    ns, nb, ne = cfg.num_blocks, cfg.num_buckets, cfg.num_excess
    return 16 + 12 + 4 * ns + 4 * nb + 8 * 512 * ns + 2 * 32 * (nb + ne) + 4 * 100000 + 288 * 500000


def _frames(cfg, seed, n):
    p = synth.params(cfg.width, cfg.height, seed, fx=cfg.fx, fy=cfg.fy, cx=cfg.cx, cy=cfg.cy,
                     depth_scale=cfg.depth_scale)
    d, c, _ = synth.render(p, 0, n)
    return d, c


def _same_map(a, b):
    ea, eb = a.entries(), b.entries()
    assert np.array_equal(ea, eb)
    sa, sb = a.stats(), b.stats()
    for k in ("heap_counter", "entry_ptr", "no_allocated", "no_visible"):
        assert sa[k] == sb[k], k
    assert sorted(a.visible().tolist()) == sorted(b.visible().tolist())
    ptrs = ea[ea[:, 3] >= 0][:, 3]
    (sa_, wa, ca), (sb_, wb, cb) = a.blocks(ptrs), b.blocks(ptrs)
    assert np.array_equal(wa, wb) and np.array_equal(ca, cb)
    assert np.array_equal(np.isnan(sa_), np.isnan(sb_))
    assert np.array_equal(sa_[~np.isnan(sa_)], sb_[~np.isnan(sb_)])


@pytest.mark.parametrize("form", ["reference", "precision"])
def test_map_file_round_trip(form, tmp_path):
    from fusion_b200 import Session, mixed_config
    from fusion_b200._lib import FB_FORM_PRECISION
    cfg = mixed_config(320, 240, 0.008)
    if form == "precision":
        cfg.form = FB_FORM_PRECISION
    d, c = _frames(cfg, synth.session_seed(4, 31), 9)
    a = Session(cfg)
    for k in range(5):
        a.grab(d[k], c[k])
    path = tmp_path / "map.bin"
    a.write_map_file(path)
    assert os.path.getsize(path) == _file_bytes(cfg)
    b = Session(cfg)
    b.read_map_file(path)
    _same_map(a, b)
    Va, Na, Ca = a.mesh()
    Vb, Nb, Cb = b.mesh()
    assert np.array_equal(Va, Vb) and np.array_equal(Na, Nb) and np.array_equal(Ca, Cb)
    # ReadMapFromDisk restarts the tracker and disables mapping
    e0 = b.entries()
    r = b.grab(d[5], c[5])
    assert r.tracker_state == 1 and not r.fused
    for k in range(6, 8):
        r = b.grab(d[k], c[k])
        assert not r.fused
    assert np.array_equal(b.entries(), e0)
    b.set_mapping(True)
    a.close()
    b.close()


def _ref():
    from oracle import refharness
    if not refharness.available():
        pytest.skip("reference kernels not built (make -C oracle ref)")
    return refharness


def _vertex_set(V, C):
    return np.unique(np.concatenate([np.ascontiguousarray(V).view(np.uint32), C.astype(np.uint32)], axis=1), axis=0)


def test_map_files_between_this_library_and_the_reference(tmp_path):
    rh = _ref()
    if shutil.disk_usage(tmp_path).free < 8e9:
        pytest.skip("not enough disk for two 3 GB map files")
    assert rh.sizeof_surf() == 288
    from fusion_b200 import Session
    from fusion_b200 import system as S
    cfg = S.reference_config(320, 240, fx=525.0, fy=525.0, depth_scale=5000.0, depth_cutoff=3.0)
    d, c = _frames(cfg, 0x5EEDF00D, 4)
    # the reference's map, here
    h = rh.RefHarness(320, 240, 525.0, 525.0, 160.0, 120.0, 5000.0, 3.0)
    for k in range(4):
        h.grab(d[k], c[k])
    path = tmp_path / "ref_map.bin"
    h.write_map(path)
    assert os.path.getsize(path) == _file_bytes(cfg)
    s = Session(cfg)
    s.read_map_file(path)
    os.remove(path)
    e_r, cnt = h.hash_entries()
    e_s = s.entries()
    assert np.array_equal(e_s, e_r)
    T = h.get_pose(0)
    ref_v = h.level(0, 0)["vmap"]
    K = np.array([cfg.fx, cfg.fy, cfg.cx, cfg.cy], np.float32)
    vm = torch.full((240, 320, 4), float("nan"), device="cuda")
    nm = torch.full((240, 320, 4), float("nan"), device="cuda")
    assert S.raycast(s, vm, nm, T, K)
    torch.cuda.synchronize()
    gv = vm.cpu().numpy()
    # fillBlocksKernel reads rendering-list entries past the tile count
    # (Mapping/RenderScene.cu:161-175, 269); with zeroed memory the
    # reference leaves the top-left 8 x 8 pixels unrendered on some runs
    gv[:8, :8] = np.nan
    ref_v = ref_v.copy()
    ref_v[:8, :8] = np.nan
    hit_g, hit_r = ~np.isnan(gv[..., 0]), ~np.isnan(ref_v[..., 0])
    both = hit_g & hit_r
    dv = np.abs(gv[both][:, :3] - ref_v[both][:, :3]).max(axis=1)
    print(f"reference map: raycast hits {hit_r.sum()} (reference) / {hit_g.sum()} (here), "
          f"same on {np.mean(hit_g == hit_r):.5f} of pixels; |dv| <= 1e-5 m on {np.mean(dv <= 1e-5):.5f}, "
          f"max {dv.max():.2e}")
    # the reference build contracts the ray march into FMAs: a rounding
    # difference can move a zero crossing by a step on a rare pixel
    assert np.mean(hit_g == hit_r) >= 0.999
    assert np.mean(dv <= 1e-5) >= 0.999 and np.mean(dv <= 1e-4) >= 0.9995
    Vr, Nr, Cr = h.mesh()
    Vs, Ns, Cs = s.mesh()
    assert np.array_equal(_vertex_set(Vs, Cs), _vertex_set(Vr, Cr))
    assert abs(len(Vs) - len(Vr)) <= 0.02 * len(Vr)
    s.close()
    h.close()
    # this library's map, in the reference
    s = Session(cfg)
    for k in range(3):
        s.grab(d[k], c[k])
    path = tmp_path / "our_map.bin"
    s.write_map_file(path)
    h = rh.RefHarness(320, 240, 525.0, 525.0, 160.0, 120.0, 5000.0, 3.0)
    h.read_map(path)
    os.remove(path)
    e_r, _ = h.hash_entries()
    assert np.array_equal(e_r, s.entries())
    Vr, Nr, Cr = h.mesh()
    Vs, Ns, Cs = s.mesh()
    assert np.array_equal(_vertex_set(Vs, Cs), _vertex_set(Vr, Cr))
    s.close()
    h.close()
