"""Generate the golden vectors in tests/golden/ by running the REFERENCE'S OWN
CUDA kernels (oracle/_ref/libfusion_ref.so, built by `make -C oracle ref` from
the reference tree) on a GPU.  The oracle is pinned against these files by
tests/test_oracle_golden.py, which runs on CPU.

Workload ("ref-default"): the reference's compile-time map constants
(Mapping/DeviceMap.h:135-151: 6 mm voxels, 48 mm truncation, depth 0.1-3.0 m,
1e6 buckets, 5e5 excess entries, 7e5 blocks) on a 128x96 narrow-field camera
(fx = fy = 420, principal point at the centre) so that the fixtures stay small,
depth scale 5000 and depth cutoff 3.0 m.  Frames come from the seeded
generator in rgbd_synth.

    python tests/golden/make_golden.py --out tests/golden
"""
import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import rgbd_synth as synth  # noqa: E402
from oracle.refharness import RefHarness  # noqa: E402

W, H = 128, 96
FX = FY = 420.0
CX, CY = 64.0, 48.0
DEPTH_SCALE = 5000.0
DEPTH_CUTOFF = 3.0
SEED = 0x5EEDF00D
FRAME_A, FRAME_B = 20, 21
SEQ_FRAMES = 10
# the whole-loop sequence needs enough pixels at pyramid level 2 for the
# reference's minimum correspondence counts (Tracking/Tracking.h:102)
SEQ_W, SEQ_H, SEQ_F = 320, 240, 525.0


def camera_params():
    return synth.params(W, H, SEED, fx=FX, fy=FY, cx=CX, cy=CY)


def levels(ref, which):
    out = {}
    for lv in range(3):
        d = ref.level(which, lv)
        for k, v in d.items():
            out[f"{k}{lv}"] = v
    return out


def allocated(ref):
    e, cnt = ref.hash_entries()
    occ = np.nonzero(e[:, 3] >= 0)[0]
    rows = e[occ]
    order = np.lexsort((rows[:, 2], rows[:, 1], rows[:, 0]))
    return occ[order].astype(np.int32), rows[order], cnt


def sparse_voxels(ref, ptrs):
    sdf, w, rgb = ref.blocks(ptrs)
    bi, vi = np.nonzero(w > 0)
    return dict(vox_block=bi.astype(np.int32), vox_index=vi.astype(np.int16),
                vox_sdf=sdf[bi, vi], vox_weight=w[bi, vi], vox_rgb=rgb[bi, vi])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)

    p = camera_params()
    depth, rgb, gt = synth.render(p, 0, FRAME_B + 1)
    ref = RefHarness(W, H, FX, FY, CX, CY, DEPTH_SCALE, DEPTH_CUTOFF)
    consts = ref.constants()
    meta = dict(width=W, height=H, fx=FX, fy=FY, cx=CX, cy=CY, depth_scale=DEPTH_SCALE,
                depth_cutoff=DEPTH_CUTOFF, seed=SEED, frame_a=FRAME_A, frame_b=FRAME_B,
                seq_frames=SEQ_FRAMES, constants=consts)

    # 1. preprocessing of frame A (Frame::FillImages)
    ref.fill_images(1, depth[FRAME_A], rgb[FRAME_A])
    pre = levels(ref, 1)
    pre["range"] = ref.range(1)
    np.savez_compressed(os.path.join(args.out, "pre_128x96.npz"), depth_in=depth[FRAME_A],
                        rgb_in=rgb[FRAME_A], **pre)

    # 2. ResizeImages of frame A's own level-0 maps
    ref.resize_images(1)
    rs = {}
    for lv in (1, 2):
        d = ref.level(1, lv)
        rs[f"vmap{lv}"] = d["vmap"]
        rs[f"nmap{lv}"] = d["nmap"]
    np.savez_compressed(os.path.join(args.out, "resize_128x96.npz"), **rs)

    # 3. ICP / RGB normal equations: next = frame B, last = frame A
    ref.fill_images(1, depth[FRAME_A], rgb[FRAME_A])  # restore A's levels 1-2
    ref.swap()                                         # A becomes last
    ref.fill_images(1, depth[FRAME_B], rgb[FRAME_B])   # B is next
    preB = levels(ref, 1)
    T_last = np.eye(4)
    rel = np.linalg.inv(gt[FRAME_A]) @ gt[FRAME_B]     # true motion A -> B
    poses = {"identity": np.eye(4), "truth": rel}
    steps = {}
    for name, T_next in poses.items():
        ref.set_pose(0, T_last)
        ref.set_pose(1, T_next)
        for lv in range(3):
            A, b, res = ref.icp_step(lv)
            steps[f"icp_A_{name}{lv}"], steps[f"icp_b_{name}{lv}"], steps[f"icp_res_{name}{lv}"] = A, b, res
            A, b, res = ref.rgb_step(lv)
            steps[f"rgb_A_{name}{lv}"], steps[f"rgb_b_{name}{lv}"], steps[f"rgb_res_{name}{lv}"] = A, b, res
        steps[f"pose_{name}"] = T_next
    np.savez_compressed(os.path.join(args.out, "steps_128x96.npz"), depth_in=depth[FRAME_B],
                        rgb_in=rgb[FRAME_B], **{f"B_{k}": v for k, v in preB.items()}, **steps)

    # 4. allocation + integration + raycast from an empty map: frame A at the
    #    identity, then frame B at the true relative pose
    ref.reset_map()
    ref.swap()                                   # frame A is "next" again
    ref.set_pose(1, np.eye(4))
    fz = {}
    nvis = ref.fuse(1)
    slots, rows, cnt = allocated(ref)
    fz.update(a_slots=slots, a_entries=rows, a_counters=cnt, a_nvis=np.int64(nvis),
              a_visible=ref.visible(nvis))
    fz.update({f"a_{k}": v for k, v in sparse_voxels(ref, rows[:, 3]).items()})
    ref.raytrace(1, nvis)
    zmin, zmax = ref.zrange()
    lvA = ref.level(1, 0)
    fz.update(a_ray_vmap=lvA["vmap"], a_ray_nmap=lvA["nmap"], a_zmin=zmin, a_zmax=zmax)
    ref.swap()                                   # B is "next"
    ref.set_pose(1, rel)
    nvis = ref.fuse(1)
    slots, rows, cnt = allocated(ref)
    fz.update(b_slots=slots, b_entries=rows, b_counters=cnt, b_nvis=np.int64(nvis), b_pose=rel)
    fz.update({f"b_{k}": v for k, v in sparse_voxels(ref, rows[:, 3]).items()})
    ref.raytrace(1, nvis)
    lvB = ref.level(1, 0)
    fz.update(b_ray_vmap=lvB["vmap"], b_ray_nmap=lvB["nmap"])
    np.savez_compressed(os.path.join(args.out, "fuse_128x96.npz"), **fz)
    ref.close()

    # 5. the whole per-frame loop (System::GrabImage) on a fresh system at
    #    320x240 (fx = fy = 525, principal point at the centre)
    ps = synth.params(SEQ_W, SEQ_H, SEED, fx=SEQ_F, fy=SEQ_F, cx=SEQ_W / 2, cy=SEQ_H / 2)
    sdepth, srgb, _ = synth.render(ps, 0, SEQ_FRAMES)
    ref = RefHarness(SEQ_W, SEQ_H, SEQ_F, SEQ_F, SEQ_W / 2, SEQ_H / 2, DEPTH_SCALE, DEPTH_CUTOFF)
    infos, poses_out = [], []
    for k in range(SEQ_FRAMES):
        infos.append(ref.grab(sdepth[k], srgb[k]))
        poses_out.append(ref.get_pose(0))      # last frame = the one just tracked
    slots, rows, cnt = allocated(ref)
    sub = (rows[:, 0] + rows[:, 1] + rows[:, 2]) % 16 == 0
    sv = sparse_voxels(ref, rows[sub, 3])
    lv = ref.level(0, 0)
    np.savez_compressed(os.path.join(args.out, "seq_320x240.npz"), info=np.array(infos),
                        poses=np.array(poses_out), slots=slots, entries=rows, counters=cnt,
                        sub_blocks=rows[sub, :3], ray_z=lv["vmap"][..., 2],
                        ray_valid=~np.isnan(lv["vmap"][..., 0]),
                        ray_nmap16=lv["nmap"][..., :3].astype(np.float16),
                        **{f"s_{k}": v for k, v in sv.items()})
    ref.close()
    meta.update(seq_width=SEQ_W, seq_height=SEQ_H, seq_f=SEQ_F)
    with open(os.path.join(args.out, "golden_meta.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("golden vectors written to", args.out)


if __name__ == "__main__":
    main()
