"""Marching-cubes case table, mesh oracle and PLY writer, on the CPU.

The library's case table (fb_mesh_case_table) is checked for what makes a
mesh closed and consistently wound: every case triangulates exactly its cut
edges with at most 5 triangles, each case's triangles form a surface whose
open edges lie on the cube's faces, and over a random field with every kind
of ambiguous face the triangles of neighbouring cubes join into a closed,
consistently oriented surface (every mesh edge inside the grid used twice,
in opposite directions).  The oracle's MeshScene restatement is run on a map
fused by the oracle from generated frames.  The PLY writer's output is
compared with the reference's format (System::WriteMeshToDisk,
Core/System.cc:140-193) built here with printf-style %g formatting.
"""
import collections

import numpy as np
import pytest

import rgbd_synth as synth
from fusion_b200.system import mesh_case_table, write_ply
from oracle import oracle as O

# corners and edges in MeshScene.cu's order (MeshScene.cu:105-256)
CORNER = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
EDGE = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]


def _faces_of(e):
    a, b = EDGE[e]
    return {(k, CORNER[a][k]) for k in range(3) if CORNER[a][k] == CORNER[b][k]}


def _tris(tri, cnt, ci):
    return [tuple(int(v) for v in tri[ci, 3 * t:3 * t + 3]) for t in range(cnt[ci])]


def test_every_case_triangulates_its_cut_edges():
    tri, cnt = mesh_case_table()
    assert cnt[0] == 0 and cnt[255] == 0
    for ci in range(1, 255):
        neg = [(ci >> i) & 1 for i in range(8)]
        cut = {e for e, (a, b) in enumerate(EDGE) if neg[a] != neg[b]}
        ts = _tris(tri, cnt, ci)
        assert 1 <= len(ts) <= 5, ci
        assert (tri[ci, 3 * len(ts):] == -1).all(), ci
        assert {e for t in ts for e in t} == cut, ci
        directed = collections.Counter()
        for t in ts:
            assert len(set(t)) == 3, ci
            for k in range(3):
                directed[(t[k], t[(k + 1) % 3])] += 1
        for (u, v), n in directed.items():
            assert n == 1, (ci, u, v)
            if (v, u) not in directed:
                # an open edge of the case's surface: on a face of the cube
                assert _faces_of(u) & _faces_of(v), (ci, u, v)


def _edge_key(x, y, z, e):
    """Lattice edge of cube (x, y, z)'s edge e: (axis, start point)."""
    a, b = EDGE[e]
    pa = np.add((x, y, z), CORNER[a])
    pb = np.add((x, y, z), CORNER[b])
    axis = int(np.nonzero(pa != pb)[0][0])
    start = np.minimum(pa, pb)
    return (axis, int(start[0]), int(start[1]), int(start[2]))


def test_random_fields_give_closed_consistently_wound_surfaces():
    tri, cnt = mesh_case_table()
    rng = np.random.default_rng(7)
    n = 9
    for trial in range(4):
        # signs at random (every ambiguous face pattern occurs many times);
        # magnitudes away from zero
        f = rng.choice([-1.0, 1.0], size=(n + 1, n + 1, n + 1)) * rng.uniform(0.2, 1.0, size=(n + 1,) * 3)
        directed = collections.Counter()
        wound = []
        for x in range(n):
            for y in range(n):
                for z in range(n):
                    s = [f[x + c[0], y + c[1], z + c[2]] for c in CORNER]
                    ci = sum(1 << i for i in range(8) if s[i] < 0)
                    for t in _tris(tri, cnt, ci):
                        keys = [_edge_key(x, y, z, e) for e in t]
                        pts, toward_neg = [], np.zeros(3)
                        for e in t:
                            a, b = EDGE[e]
                            va, vb = s[a], s[b]
                            u = va / (va - vb)
                            pa, pb = np.array(CORNER[a], float), np.array(CORNER[b], float)
                            pts.append(pa + u * (pb - pa))
                            toward_neg += (pa - pb) if va < 0 else (pb - pa)
                        nrm = np.cross(pts[1] - pts[0], pts[2] - pts[0])
                        wound.append(float(nrm @ toward_neg))
                        for k in range(3):
                            directed[(keys[k], keys[(k + 1) % 3])] += 1

        def on_boundary(k):
            axis, p = k[0], k[1:]
            return any(p[j] in (0, n) for j in range(3) if j != axis)

        for (u, v), c in directed.items():
            assert c == 1, (trial, u, v)
            if (v, u) not in directed:
                assert on_boundary(u) and on_boundary(v), (trial, u, v)
        # right-hand normals point to the negative side
        assert np.mean(np.array(wound) > 0) > 0.99


def _oracle_map(w=160, h=120, frames=3):
    cfg = O.config(w, h, 525.0 * w / 640.0, 525.0 * w / 640.0, w / 2.0, h / 2.0, depth_scale=5000.0,
                   depth_cutoff=3.0, voxel_size=0.01, trunc_dist=0.04, depth_min=0.1, depth_max=3.0,
                   num_buckets=1 << 15, num_excess=1 << 14, num_blocks=1 << 14, precision=32)
    p = synth.params(w, h, synth.session_seed(4, 3), fx=cfg.fx, fy=cfg.fy, cx=cfg.cx, cy=cfg.cy,
                     depth_scale=5000.0)
    depth, rgb, poses = synth.render(p, 0, frames)
    M = O.Map(cfg)
    for k in range(frames):
        raw, filt = O.filter_depth(depth[k], 5000.0, 3.0, 32)
        vm = O.vmap(filt.astype(np.float32), cfg.fx, cfg.fy, cfg.cx, cfg.cy, 3.0, 32)
        nm = O.nmap(vm, 32).astype(np.float32)
        M.fuse(raw.astype(np.float32), rgb[k], nm, poses[k])
    return M, cfg


def test_oracle_mesh_of_a_fused_map():
    tri, cnt = mesh_case_table()
    M, cfg = _oracle_map()
    V, N, C = M.mesh(tri, cnt, fused=1)
    T = len(V) // 3
    assert T > 1000
    assert np.isfinite(V).all() and np.isfinite(N).all()
    assert np.allclose(np.linalg.norm(N, axis=1), 1.0, atol=1e-5)
    # each vertex lies on a lattice edge: at least two coordinates on the grid
    g = V / np.float32(cfg.voxel_size)
    assert (np.sum(np.abs(g - np.round(g)) < 1e-3, axis=1) >= 2).all()
    # winding: right-hand normals point to the negative side, against the
    # gradient normals
    tv = V.reshape(T, 3, 3).astype(np.float64)
    geo = np.cross(tv[:, 1] - tv[:, 0], tv[:, 2] - tv[:, 0])
    area = np.linalg.norm(geo, axis=1)
    big = area > 1e-3 * np.median(area)
    agree = np.einsum("ij,ij->i", geo[big], N.reshape(T, 3, 3).sum(axis=1)[big]) < 0
    assert agree.mean() > 0.98
    assert C.any()
    # the unfused normal rounding differs from the fused one by a few ulps
    V0, N0, C0 = M.mesh(tri, cnt, fused=0)
    assert np.array_equal(V0, V) and np.array_equal(C0, C)
    assert np.abs(N0 - N).max() < 1e-5
    M.close()


def test_write_ply_matches_reference_format(tmp_path):
    rng = np.random.default_rng(3)
    V = rng.normal(size=(6, 3)).astype(np.float32)
    V[0, 0] = -0.0
    V[1, 1] = 1e-7
    V[2, 2] = 123456789.0
    N = rng.normal(size=(6, 3)).astype(np.float32)
    C = rng.integers(0, 256, size=(6, 3)).astype(np.uint8)
    path = tmp_path / "scene.ply"
    write_ply(path, V, N, C)
    header = ("ply\nformat ascii 1.0\nelement vertex 6\nproperty float x\nproperty float y\nproperty float z\n"
              "property float nx\nproperty float ny\nproperty float nz\nproperty uchar red\nproperty uchar green\n"
              "property uchar blue\nelement face 2\nproperty list uchar uint vertex_indices\nend_header\n")
    body = "".join("%g %g %g %g %g %g %d %d %d\n" % (*map(float, V[i]), *map(float, N[i]), *map(int, C[i]))
                   for i in range(6))
    faces = "3 0 1 2\n3 3 4 5\n"
    assert path.read_text() == header + body + faces
    write_ply(tmp_path / "empty.ply", np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 3)))
    assert "element vertex 0\n" in (tmp_path / "empty.ply").read_text()
    with pytest.raises(ValueError):
        write_ply(path, V[:4], N[:4], C[:4])
