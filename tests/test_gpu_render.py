"""Headless rendering against the reference's own kernels (RenderImage,
DepthToImage, RgbImageToRgba, Tracking/Pyrdown.cu:322-428, built from the
reference's sources into oracle/_ref): the raycast vertex/normal maps of a
real session shaded by both, and the frame's depth and colour converted by
both, must give the same bytes (both use the same fast power function, so
an off-by-one byte from its rounding is allowed on a few pixels)."""
import numpy as np
import pytest

from fusion_b200 import synth

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
