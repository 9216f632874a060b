"""Mesh extraction (fb_mesh_scene, fb_save_mesh) through the C ABI.

- Against the oracle's MeshScene restatement (Mapping/MeshScene.cu:20-295)
  run on the session's own map with the library's case table: the same
  triangles, positions, normals and colours bit for bit (compared as
  multisets; the oracle walks hash slots, the GPU the allocation order), in
  the reference and the precision form; two extractions give identical
  arrays (the order is deterministic).
- The oracle itself pinned against the reference's own MeshScene kernel
  (oracle/_ref, built from the reference's sources) on the reference's map,
  with the reference's table: positions and colours bit for bit, normals
  within 2e-6.
- On that map, the oracle with the library's table (the function the GPU
  kernel computes) gives exactly the reference kernel's vertices (position
  and colour); triangle counts agree within the ambiguous cases the two
  tables triangulate differently, and both wind the same way.
- fb_save_mesh writes what fb_write_ply writes for fb_mesh_scene's output.
"""
import numpy as np
import pytest

import rgbd_synth as synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _rows(V, N, C, with_normals=True):
    T = V.size // 9
    parts = [np.ascontiguousarray(V).reshape(T, 9).view(np.uint32)]
    if with_normals:
        parts.append(np.ascontiguousarray(N).reshape(T, 9).view(np.uint32))
    parts.append(C.reshape(T, 9).astype(np.uint32))
    return np.concatenate(parts, axis=1)


def _sorted(V, N, C):
    """Triangles in a canonical order: by vertex positions, then colours,
    then normals (triangles collapsed onto a voxel corner can share their
    positions)."""
    T = len(V) // 3
    key = _rows(V, N, C)[:, [*range(9), *range(18, 27), *range(9, 18)]]
    order = np.lexsort(key.T[::-1])
    return V.reshape(T, 9)[order], N.reshape(T, 9)[order], C.reshape(T, 9)[order]


def _report(a, b):
    """Which parts of the canonical triangle rows differ."""
    bad = np.nonzero((a != b).any(axis=1))[0]
    if not len(bad):
        return "identical"
    parts = {"positions": slice(0, 9), "normals": slice(9, 18), "colours": slice(18, 27)}
    out = [f"{len(bad)} of {len(a)} triangles differ"]
    for k, sl in parts.items():
        out.append(f"{k}: {int((a[bad, sl] != b[bad, sl]).any(axis=1).sum())}")
    i = bad[0]
    out.append(f"first: {a[i].view(np.float32)[:18].tolist()} vs {b[i].view(np.float32)[:18].tolist()}")
    return "; ".join(out)


def _oracle_map(entries, blocks_of, cfg, heap_counter=0, entry_ptr=1):
    """An oracle map holding `entries` ({x, y, z, ptr, offset} per slot) and
    the voxels blocks_of(ptrs) returns; the pool only as large as needed."""
    live = np.nonzero((entries[:, 3] >= 0) | (entries[:, 4] != 0))[0]
    occ = entries[:, 3] >= 0
    ptrs = entries[occ][:, 3]
    n_blocks = int(ptrs.max()) // 512 + 1 if len(ptrs) else 1
    oc = O.config(cfg.width, cfg.height, cfg.fx, cfg.fy, cfg.cx, cfg.cy, cfg.depth_scale, cfg.depth_cutoff,
                  voxel_size=cfg.voxel_size, trunc_dist=cfg.trunc_dist, depth_min=cfg.depth_min,
                  depth_max=cfg.depth_max, num_buckets=cfg.num_buckets, num_excess=cfg.num_excess,
                  num_blocks=n_blocks, precision=32)
    M = O.Map(oc)
    M.set_entries(live, entries[live], heap_counter, entry_ptr)
    sdf, w, rgb = blocks_of(ptrs)
    M.load_blocks(ptrs, sdf.astype(np.float64), w, rgb)
    return M


def _session_map(s):
    e = s.entries()
    st = s.stats()
    return _oracle_map(e, s.blocks, s.cfg, st["heap_counter"], st["entry_ptr"])


def _run(cfg, seed, n):
    from fusion_b200 import Session
    p = synth.params(cfg.width, cfg.height, seed, fx=cfg.fx, fy=cfg.fy, cx=cfg.cx, cy=cfg.cy,
                     depth_scale=cfg.depth_scale)
    depth, rgb, _ = synth.render(p, 0, n)
    s = Session(cfg)
    for k in range(n):
        s.grab(depth[k], rgb[k])
    return s


@pytest.mark.parametrize("form", ["reference", "precision"])
def test_mesh_matches_oracle_bit_for_bit(form):
    from fusion_b200 import mixed_config
    from fusion_b200._lib import FB_FORM_PRECISION
    from fusion_b200.system import mesh_case_table
    cfg = mixed_config(320, 240, 0.006)
    if form == "precision":
        cfg.form = FB_FORM_PRECISION
    s = _run(cfg, synth.session_seed(4, 21), 5)
    V, N, C = s.mesh()
    V2, N2, C2 = s.mesh()
    assert np.array_equal(V, V2) and np.array_equal(N, N2) and np.array_equal(C, C2)
    T = len(V) // 3
    assert T > 10000
    tri, cnt = mesh_case_table()
    M = _session_map(s)
    Vo, No, Co = M.mesh(tri, cnt, fused=1)
    print(f"{form}: {T} triangles")
    assert len(Vo) == len(V)
    a, b = _rows(*_sorted(Vo, No, Co)), _rows(*_sorted(V, N, C))
    assert np.array_equal(a, b), _report(a, b)
    # a capped extraction writes the first triangles of the same order
    Vc, Nc, Cc = s.mesh(max_triangles=T // 3)
    assert np.array_equal(Vc, V[:3 * (T // 3)]) and np.array_equal(Cc, C[:3 * (T // 3)])
    M.close()
    s.close()


def _ref():
    from oracle import refharness
    if not refharness.available():
        pytest.skip("reference kernels not built (make -C oracle ref)")
    return refharness


def _wound_inward(V, N):
    """Fraction of (non-degenerate) triangles whose right-hand normal points
    against their vertices' gradient normals."""
    T = len(V) // 3
    tv = V.reshape(T, 3, 3).astype(np.float64)
    g = np.cross(tv[:, 1] - tv[:, 0], tv[:, 2] - tv[:, 0])
    area = np.linalg.norm(g, axis=1)
    big = area > 1e-3 * np.median(area)
    return float(np.mean(np.einsum("ij,ij->i", g[big], N.reshape(T, 3, 3).sum(axis=1)[big]) < 0))


def _vertex_set(V, C):
    return np.unique(np.concatenate([np.ascontiguousarray(V).view(np.uint32), C.astype(np.uint32)], axis=1), axis=0)


def test_mesh_against_the_reference_kernel():
    """On the reference's own map (its kernels, its tracking, four frames):
    the oracle with the reference's table reproduces the reference kernel's
    triangles, and the oracle with this library's table -- the function the
    GPU kernel computes bit for bit (test above) -- gives the same vertices,
    nearly the same triangle count, and the same winding."""
    rh = _ref()
    from fusion_b200 import system as S
    from fusion_b200.system import mesh_case_table
    cfg = S.reference_config(320, 240, fx=525.0, fy=525.0, depth_scale=5000.0, depth_cutoff=3.0)
    p = synth.params(320, 240, 0x5EEDF00D, fx=525.0, fy=525.0, cx=160.0, cy=120.0, depth_scale=5000.0)
    depth, rgb, _ = synth.render(p, 0, 4)
    h = rh.RefHarness(320, 240, 525.0, 525.0, 160.0, 120.0, 5000.0, 3.0)
    for k in range(4):
        h.grab(depth[k], rgb[k])
    e, cnt = h.hash_entries()
    Vr, Nr, Cr = h.mesh()
    assert len(Vr) > 30000
    M = _oracle_map(e, h.blocks, cfg, cnt[0], cnt[1])
    tri_r, ntri_r = rh.mesh_tables()
    Vo, No, Co = M.mesh(tri_r, ntri_r, fused=1)
    assert len(Vo) == len(Vr)
    Vo, No, Co = _sorted(Vo, No, Co)
    Vs, Ns, Cs = _sorted(Vr, Nr, Cr)
    assert np.array_equal(Vo.view(np.uint32), Vs.view(np.uint32))
    assert np.array_equal(Co, Cs)
    d = np.abs(No - Ns)
    assert d.max() <= 2e-6
    tri, ntri = mesh_case_table()
    Vm, Nm, Cm = M.mesh(tri, ntri, fused=1)
    assert np.array_equal(_vertex_set(Vm, Cm), _vertex_set(Vr, Cr))
    wr, wm = _wound_inward(Vr, Nr), _wound_inward(Vm, Nm)
    print(f"reference kernel: {len(Vr) // 3} triangles, normals bit-equal to the fused oracle "
          f"{np.mean(d == 0):.4f} (max diff {d.max():.2e}); this library's table: {len(Vm) // 3} triangles; "
          f"wound against the normals: reference {wr:.4f}, this library {wm:.4f}")
    assert abs(len(Vm) - len(Vr)) <= 0.02 * len(Vr)
    assert abs(wr - wm) <= 0.02
    M.close()
    h.close()


def test_save_mesh_writes_the_extracted_mesh(tmp_path):
    from fusion_b200 import mixed_config
    from fusion_b200.system import write_ply
    s = _run(mixed_config(160, 120, 0.01), synth.session_seed(4, 22), 3)
    V, N, C = s.mesh()
    a, b = tmp_path / "a.ply", tmp_path / "b.ply"
    assert s.save_mesh(a) == len(V) // 3
    write_ply(b, V, N, C)
    assert a.read_bytes() == b.read_bytes()
    s.close()
