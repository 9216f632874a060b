"""Loading of the golden vectors in tests/golden/ (made by make_golden.py from
the reference's own CUDA kernels) and the oracle configuration that matches
the reference build they came from."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def meta():
    with open(os.path.join(GOLDEN, "golden_meta.json")) as f:
        return json.load(f)


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def oracle_config(prec, width=None, height=None, f=None):
    from oracle import oracle as O
    m = meta()
    c = m["constants"]
    W = width or m["width"]
    H = height or m["height"]
    fx = f or m["fx"]
    return O.config(W, H, fx, fx, W / 2, H / 2, m["depth_scale"], m["depth_cutoff"],
                    voxel_size=c["voxel_size"], trunc_dist=c["trunc_dist"],
                    depth_min=c["depth_min"], depth_max=c["depth_max"],
                    num_buckets=int(c["num_buckets"]), num_excess=int(c["num_excess"]),
                    num_blocks=int(c["num_blocks"]), precision=prec)


def load_ref_state(M, fz, pfx):
    """Teacher forcing: put the reference's hash table and voxels into an
    oracle map."""
    ent, slots, cnt = fz[pfx + "entries"], fz[pfx + "slots"], fz[pfx + "counters"]
    M.set_entries(slots, ent, cnt[0], cnt[1])
    n = len(ent)
    sdf = np.full((n, 512), np.nan)
    w = np.zeros((n, 512), np.uint8)
    rgb = np.zeros((n, 512, 3), np.uint8)
    b, v = fz[pfx + "vox_block"], fz[pfx + "vox_index"]
    sdf[b, v] = fz[pfx + "vox_sdf"]
    w[b, v] = fz[pfx + "vox_weight"]
    rgb[b, v] = fz[pfx + "vox_rgb"]
    M.load_blocks(ent[:, 3], sdf, w, rgb)
    return ent, slots


def voxel_dict(ent, blocks, index, sdf, w, rgb):
    """{(bx, by, bz, voxel index): (sdf, weight, rgb)} of observed voxels."""
    keys = [(int(ent[b, 0]), int(ent[b, 1]), int(ent[b, 2]), int(v)) for b, v in zip(blocks, index)]
    return dict(zip(keys, zip(sdf, w, [tuple(int(c) for c in x) for x in rgb])))
