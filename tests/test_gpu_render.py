"""Headless rendering against the reference's own kernels (RenderImage,
DepthToImage, RgbImageToRgba, Tracking/Pyrdown.cu:322-428, built from the
reference's sources into oracle/_ref): the raycast vertex/normal maps of a
real session shaded by both, and the frame's depth and colour converted by
both, must give the same bytes (both use the same fast power function, so
an off-by-one byte from its rounding is allowed on a few pixels).

The top-down view (System::RenderTopDown, Core/System.cc:75-90) against the
oracle on the session's own map: the same visible blocks as the oracle's
visibility for a 640 x 480 camera at the top-down pose with the shifted
depth range, vertices within 1e-5 m of its raycast, and the image the
shading of those maps."""
import numpy as np
import pytest

import rgbd_synth as synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _ref():
    from oracle import refharness
    if not refharness.available():
        pytest.skip("reference kernels not built (make -C oracle ref)")
    return refharness


def test_render_depth_and_rgba_match_reference_kernels():
    rh = _ref()
    from fusion_b200 import Session, mixed_config
    from fusion_b200 import system as S
    cfg = mixed_config(320, 240, 0.007)
    p = synth.params(320, 240, synth.session_seed(4, 12), fx=cfg.fx, fy=cfg.fy, cx=cfg.cx, cy=cfg.cy,
                     depth_scale=5000.0)
    d, c, _ = synth.render(p, 0, 3)
    s = Session(cfg)
    for k in range(3):
        s.grab(d[k], c[k])
    lv = s.level(0, 0)                      # the last raycast (model) maps
    raw = s.raw(0)
    s.close()
    vm, nm = lv["vmap"], lv["nmap"]
    assert np.isfinite(vm[..., 0]).mean() > 0.5
    light = np.array([0.3, -0.2, 0.1], np.float32)
    ours = torch.zeros((240, 320, 4), dtype=torch.uint8, device="cuda")
    S.render_image(torch.from_numpy(vm).cuda(), torch.from_numpy(nm).cuda(), light, ours)
    ref = rh.render_image(vm, nm, light)
    diff = np.abs(ours.cpu().numpy().astype(int) - ref.astype(int))
    assert diff.max() <= 1 and (diff > 0).mean() <= 1e-3
    img = torch.zeros((240, 320, 4), dtype=torch.uint8, device="cuda")
    S.depth_to_image(torch.from_numpy(raw).cuda(), img)
    assert np.array_equal(img.cpu().numpy(), rh.depth_to_image(raw))
    S.rgb_to_rgba(torch.from_numpy(np.ascontiguousarray(c[2])).cuda(), img)
    assert np.array_equal(img.cpu().numpy(), rh.rgb_to_rgba(c[2]))


def test_top_down_render_matches_oracle():
    from fusion_b200 import Session, mixed_config
    from fusion_b200 import system as S
    from tests.test_gpu_mesh import _oracle_map
    cfg = mixed_config(640, 480, 0.01)
    p = synth.params(640, 480, synth.session_seed(4, 23), fx=cfg.fx, fy=cfg.fy, cx=cfg.cx, cy=cfg.cy,
                     depth_scale=5000.0)
    d, c, _ = synth.render(p, 0, 4)
    s = Session(cfg)
    for k in range(4):
        s.grab(d[k], c[k])
    dist = 8.0
    vm = torch.full((480, 640, 4), float("nan"), device="cuda")
    nm = torch.full((480, 640, 4), float("nan"), device="cuda")
    img = torch.zeros((480, 640, 4), dtype=torch.uint8, device="cuda")
    assert S.render_top_down(s, dist, vm, nm, img)
    n_vis = s.stats()["no_visible"]
    vis = sorted(s.visible().tolist())
    # the oracle on the session's map with the top-down camera: the depth
    # range shifted by dist in float, as the reference adds it
    e, st = s.entries(), s.stats()
    shifted = S.make_config(640, 480, cfg.voxel_size, 4, cfg.num_buckets, cfg.num_excess, cfg.num_blocks,
                            depth_min=float(np.float32(dist) + np.float32(cfg.depth_min)),
                            depth_max=float(np.float32(dist) + np.float32(cfg.depth_max)))
    shifted.trunc_dist = cfg.trunc_dist
    M = _oracle_map(e, s.blocks, shifted, st["heap_counter"], st["entry_ptr"])
    T = S.top_down_pose(dist)
    assert M.visibility(T) == n_vis > 0
    assert sorted(M.visible().tolist()) == vis
    vo, no, _, _, tiles = M.raycast(T)
    assert tiles > 0
    torch.cuda.synchronize()
    gv, gn = vm.cpu().numpy(), nm.cpu().numpy()
    vg, vo_ = ~np.isnan(gv[..., 0]), ~np.isnan(vo[..., 0])
    print(f"top-down: {n_vis} visible blocks, {vg.sum()} pixels hit, agree on {np.mean(vg == vo_):.5f}")
    assert vg.sum() > 1000
    assert np.array_equal(vg, vo_)
    assert np.abs(gv[vg] - vo[vg]).max() <= 1e-5
    assert np.abs(gn[vg] - no[vg]).max() <= 1e-4
    ref = torch.zeros_like(img)
    S.render_image(vm, nm, np.zeros(3, np.float32), ref)
    assert torch.equal(img, ref)
    M.close()
    s.close()
