"""fb_rgb_step_static: the photometric step for callers that cannot allocate
device memory where they track a frame (frame loops that cannot wait for
cudaFree; plug-ins in hosts that keep all device memory to themselves).  It
takes no scratch argument and uses a fixed buffer inside the library instead.

Checked through the C ABI against fb_rgb_step with a caller-provided scratch
buffer, on two calls in a row (the fixed buffer keeps the previous call's
contents, so the second call shows that nothing stale leaks into the sums).
Both run the same kernels with the same grid and reduce in a fixed order, so
the results must be bit-identical: the tolerance is zero.  A frame larger
than the fixed buffer is refused.  This file is collected last so that a run stopping
at its first failure has run every other test already; it also passes alone.
"""
import numpy as np
import pytest

from tests import golden_util as G

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("pose", ["identity", "truth"])
def test_static_scratch_step_matches_step_with_caller_scratch(pose):
    from fusion_b200 import system as S
    pre = G.load("pre_128x96.npz")
    st = G.load("steps_128x96.npz")
    m = G.meta()
    Rc, Rci, tc = S.pose_parts(st[f"pose_{pose}"])
    Rl, Rli, tl = S.pose_parts(np.eye(4))
    for lv in range(3):
        s = 1 << lv
        K = np.array([m["fx"] / s, m["fy"] / s, m["cx"] / s, m["cy"] / s], np.float32)
        args = [dev(st[f"B_image{lv}"]), dev(pre[f"image{lv}"]), dev(st[f"B_vmap{lv}"]), dev(pre[f"vmap{lv}"]),
                dev(st[f"B_dx{lv}"]), dev(st[f"B_dy{lv}"]), Rc, Rci, Rl, Rli, tc, tl, K]
        h, w = pre[f"image{lv}"].shape
        scratch = torch.empty(S.step_scratch_bytes(w, h), dtype=torch.uint8, device="cuda")
        res_ref, A_ref, b_ref = S.rgb_step(*args, scratch)
        for _ in range(2):
            res, A, b = S.rgb_step_static(*args)
            assert np.array_equal(res, res_ref)               # count and residual, bit for bit
            assert np.array_equal(A, A_ref)
            assert np.array_equal(b, b_ref)


def test_static_scratch_step_refuses_frames_beyond_its_buffer():
    from fusion_b200 import _lib
    from fusion_b200 import system as S
    L = _lib.load()
    limit = int(L.fb_rgb_step_static_max_pixels())
    assert limit == 640 * 480
    H, W = 481, 640                                           # one row more than the buffer holds
    g = torch.zeros((H, W), dtype=torch.uint8, device="cuda")
    v = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    d = torch.zeros((H, W), dtype=torch.int16, device="cuda")
    eye = np.eye(3, dtype=np.float32)
    zero = np.zeros(3, np.float32)
    K = np.array([525.0, 525.0, 320.0, 240.0], np.float32)
    with pytest.raises(_lib.FusionError) as e:
        S.rgb_step_static(g, g, v, v, d, d, eye, eye, eye, eye, zero, zero, K)
    assert e.value.code == _lib.FB_EINVAL
    assert b"static scratch" in L.fb_last_error()
