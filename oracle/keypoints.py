"""ORACLE / TEST INFRASTRUCTURE ONLY.

numpy restatement of this library's key-point detector, descriptor,
back-projection and matcher (fusion_b200/csrc/keypoints.cu), used by the
tests to check the CUDA kernels.  The reference's key points come from
OpenCV's CUDA SURF, which is not available here, so this restates the
library's own implementation of the published SURF method (Bay et al., CVIU
2008) -- parity with the reference's key points is unpinned.  The
back-projection follows Frame::InterpDepth / InterpNormal / ExtractKeyPoints
(Core/Frame.cc:93-212) and the matcher cv::cuda BFMatcher knnMatch (k = 2).

Box sums are integers and the Hessian responses are float32 operations in
the kernels' order, so candidate sets and their ranking agree exactly; the
refinement, orientation and descriptor use library exp / atan2 / cos / sin
and agree to rounding.
"""
import math

import numpy as np

F = np.float32
OCTAVES, LAYERS, MAX_CAND = 4, 4, 16384


def filter_size(o, l):
    return 3 * ((2 << o) * (l + 1) + 1)


def margin(o):
    return filter_size(o, LAYERS - 1) // 2 + 1


def integral(gray):
    H, W = gray.shape
    I = np.zeros((H + 1, W + 1), np.int64)
    I[1:, 1:] = np.cumsum(np.cumsum(gray.astype(np.int64), axis=0), axis=1)
    return I


def box(I, x0, y0, x1, y1):
    """Sums over [x0, x1) x [y0, y1), clipped (arrays of corners)."""
    H, W = I.shape[0] - 1, I.shape[1] - 1
    x0, x1 = np.clip(x0, 0, W), np.clip(x1, 0, W)
    y0, y1 = np.clip(y0, 0, H), np.clip(y1, 0, H)
    s = I[y1, x1] - I[y0, x1] - I[y1, x0] + I[y0, x0]
    return np.where((x1 > x0) & (y1 > y0), s, 0)


def hessian(I, x, y, L):
    l, h, m = L // 3, (3 * (L // 3) - 1) // 2, (L // 3 - 1) // 2
    dyy = box(I, x - (l - 1), y - h, x + l, y + h + 1) - 3 * box(I, x - (l - 1), y - m, x + l, y + m + 1)
    dxx = box(I, x - h, y - (l - 1), x + h + 1, y + l) - 3 * box(I, x - m, y - (l - 1), x + m + 1, y + l)
    dxy = (box(I, x - l, y - l, x, y) + box(I, x + 1, y + 1, x + l + 1, y + l + 1) -
           box(I, x + 1, y - l, x + l + 1, y) - box(I, x - l, y + 1, x, y + l + 1))
    inv = F(1.0) / (F(L) * F(L))
    fxx, fyy, fxy = dxx.astype(F) * inv, dyy.astype(F) * inv, dxy.astype(F) * inv
    return fxx * fyy - (F(0.81) * fxy) * fxy


def det_maps(I, W, H):
    out = []
    for o in range(OCTAVES):
        ow, oh = W >> o, H >> o
        jj, ii = np.meshgrid(np.arange(oh), np.arange(ow), indexing="ij")
        x, y, mg = ii << o, jj << o, margin(o)
        inside = (x >= mg) & (y >= mg) & (x < W - mg) & (y < H - mg)
        maps = np.zeros((LAYERS, oh, ow), F)
        for l in range(LAYERS):
            maps[l] = np.where(inside, hessian(I, x, y, filter_size(o, l)), F(0))
        out.append(maps)
    return out


def candidates(maps, threshold):
    """(key, x, y, scale, response) of every refined extremum, key =
    response bits << 32 | sample index (the kernels' ranking key)."""
    out = []
    code0 = 0
    for o in range(OCTAVES):
        M = maps[o]
        _, oh, ow = M.shape
        mg = (margin(o) + (1 << o) - 1) >> o
        for l in range(1, LAYERS - 1):
            v = M[l]
            js, is_ = np.nonzero(v > threshold)
            for j, i in zip(js, is_):
                if i < mg + 1 or j < mg + 1 or i >= ow - mg - 1 or j >= oh - mg - 1:
                    continue
                c = v[j, i]
                nb = M[l - 1:l + 2, j - 1:j + 2, i - 1:i + 2].copy()
                nb[1, 1, 1] = -np.inf
                if not np.all(c > nb):
                    continue

                def at(dl, dj, di):
                    return M[l + dl, j + dj, i + di]
                gx = F(0.5) * (at(0, 0, 1) - at(0, 0, -1))
                gy = F(0.5) * (at(0, 1, 0) - at(0, -1, 0))
                gs = F(0.5) * (at(1, 0, 0) - at(-1, 0, 0))
                hxx = at(0, 0, 1) + at(0, 0, -1) - F(2) * c
                hyy = at(0, 1, 0) + at(0, -1, 0) - F(2) * c
                hss = at(1, 0, 0) + at(-1, 0, 0) - F(2) * c
                hxy = F(0.25) * (at(0, 1, 1) - at(0, 1, -1) - at(0, -1, 1) + at(0, -1, -1))
                hxs = F(0.25) * (at(1, 0, 1) - at(1, 0, -1) - at(-1, 0, 1) + at(-1, 0, -1))
                hys = F(0.25) * (at(1, 1, 0) - at(1, -1, 0) - at(-1, 1, 0) + at(-1, -1, 0))
                Hm = np.array([[hxx, hxy, hxs], [hxy, hyy, hys], [hxs, hys, hss]], np.float64)
                if not abs(np.linalg.det(Hm)) > 1e-30:
                    continue
                off = np.linalg.solve(Hm, -np.array([gx, gy, gs], np.float64))
                if not np.all(np.abs(off) < 0.5):
                    continue
                step = float(1 << o)
                L = F(filter_size(o, l)) + F(off[2]) * F(filter_size(o, l + 1) - filter_size(o, l))
                code = code0 + ((l - 1) * oh + j) * ow + i
                key = (int(np.array(c, F).view(np.uint32)) << 32) | code
                out.append((key, F((F(i) + F(off[0])) * F(step)), F((F(j) + F(off[1])) * F(step)),
                            F(F(1.2) * L / F(9)), c))
        code0 += (LAYERS - 2) * oh * ow
    return out


def even_size(v):
    return max(2, 2 * int(np.rint(0.5 * v)))


def haar(I, x, y, h):
    r = h // 2
    dx = box(I, x, y - r, x + r, y + r) - box(I, x - r, y - r, x, y + r)
    dy = box(I, x - r, y, x + r, y + r) - box(I, x - r, y - r, x + r, y)
    return dx.astype(np.float64), dy.astype(np.float64)


def describe(I, x, y, s):
    """(angle, 64 descriptor values) of a key point."""
    ab = [(a, b) for b in range(-5, 6) for a in range(-5, 6) if a * a + b * b < 36]
    a = np.array([p[0] for p in ab])
    b = np.array([p[1] for p in ab])
    dx, dy = haar(I, np.rint(x + a * s).astype(int), np.rint(y + b * s).astype(int), even_size(4 * s))
    g = np.exp(-(a * a + b * b) / 8.0)
    dx, dy = dx * g, dy * g
    ang = np.arctan2(dy, dx)
    ang = np.where(ang < 0, ang + 2 * math.pi, ang)
    best, bx, by = -1.0, 0.0, 0.0
    for w in range(72):
        d = ang - w * (2 * math.pi / 72)
        d = np.where(d < 0, d + 2 * math.pi, d)
        sel = d < math.pi / 3
        sx, sy = dx[sel].sum(), dy[sel].sum()
        if sx * sx + sy * sy > best:
            best, bx, by = sx * sx + sy * sy, sx, sy
    theta = math.atan2(by, bx)
    co, si = math.cos(theta), math.sin(theta)
    desc = np.zeros(64)
    h2 = even_size(2 * s)
    for sub in range(16):
        sr, sc = sub >> 2, sub & 3
        t = np.arange(25)
        kk, mm = sc * 5 + t % 5, sr * 5 + t // 5
        u, v = (kk - 9.5) * s, (mm - 9.5) * s
        px = np.rint(x + u * co - v * si).astype(int)
        py = np.rint(y + u * si + v * co).astype(int)
        ddx, ddy = haar(I, px, py, h2)
        g = np.exp(-((kk - 9.5) ** 2 + (mm - 9.5) ** 2) / (2 * 3.3 * 3.3))
        rx, ry = g * (ddx * co + ddy * si), g * (-ddx * si + ddy * co)
        desc[4 * sub:4 * sub + 4] = [rx.sum(), ry.sum(), np.abs(rx).sum(), np.abs(ry).sum()]
    n = np.sqrt((desc * desc).sum())
    return theta, (desc / n if n > 0 else desc)


def detect(gray, threshold=20.0):
    """Key points of a uint8 image: (kp [n, 4] = x, y, scale, angle; desc [n, 64])."""
    H, W = gray.shape
    I = integral(gray)
    maps = det_maps(I, W, H)
    thr = threshold
    for _ in range(8):
        cand = candidates(maps, thr)
        if len(cand) <= MAX_CAND:
            break
        thr *= 2.0
    cand.sort(key=lambda c: -c[0])
    cand = cand[:W * H // 100]
    kp = np.zeros((len(cand), 4), np.float32)
    desc = np.zeros((len(cand), 64), np.float32)
    for k, (_, x, y, s, _) in enumerate(cand):
        theta, d = describe(I, float(x), float(y), float(s))
        kp[k] = (x, y, s, theta)
        desc[k] = d
    return kp, desc


def interp_depth(depth, x, y, cutoff):
    """Frame::InterpDepth (its bounds test exchanges rows and columns; a
    second test keeps the reads in the image)."""
    H, W = depth.shape
    x, y = F(x), F(y)
    if x <= 1 or y <= 1 or y >= W - 1 or x >= H - 1:
        return np.nan
    cx, cy = x - F(math.floor(x)), y - F(math.floor(y))
    x0, x1, y0, y1 = int(math.floor(x)), int(math.ceil(x)), int(math.floor(y)), int(math.ceil(y))
    if x1 >= W or y1 >= H:
        return np.nan
    ds = [depth[y0, x0], depth[y1, x0], depth[y0, x1], depth[y1, x1]]
    for d in ds:
        if np.isnan(d) or d < 0.3 or d > cutoff:
            return np.nan
    d00, d10, d01, d11 = (F(d) for d in ds)
    d0 = d01 * cx + d00 * (F(1) - cx)
    d1 = d11 * cx + d10 * (F(1) - cx)
    fin = (F(1) - cy) * d0 + cy * d1
    return fin if abs(fin - d00) <= 0.005 else np.nan


def interp_normal(nmap, x, y):
    H, W = nmap.shape[:2]
    x, y = F(x), F(y)
    if x <= 1 or y <= 1 or y >= W - 1 or x >= H - 1:
        return None
    cx, cy = x - F(math.floor(x)), y - F(math.floor(y))
    x0, x1, y0, y1 = int(math.floor(x)), int(math.ceil(x)), int(math.floor(y)), int(math.ceil(y))
    if x1 >= W or y1 >= H:
        return None
    d00, d10, d01, d11 = nmap[y0, x0], nmap[y1, x0], nmap[y0, x1], nmap[y1, x1]
    d0 = d01 * cx + d00 * (F(1) - cx)
    d1 = d11 * cx + d10 * (F(1) - cx)
    f = d0 * (F(1) - cy) + d1 * cy
    e = f - d00
    return f if math.sqrt(float((e * e).sum())) <= 0.1 else None


def backproject(kp, desc, depth, nmap, fx, fy, cx, cy, cutoff):
    """Frame::ExtractKeyPoints' filter: (kp, pts, nrm, desc) of the key points
    with a depth in (0.3, cutoff) and a normal."""
    keep = []
    for k in range(len(kp)):
        x, y = kp[k, 0], kp[k, 1]
        d = interp_depth(depth, x, y, cutoff)
        if np.isnan(d) or not (d > 0.3 and d < cutoff):
            continue
        n = interp_normal(nmap, x, y)
        if n is None or np.isnan(n[0]):
            continue
        p = (F(d) * (F(x) - F(cx)) / F(fx), F(d) * (F(y) - F(cy)) / F(fy), F(d), F(1))
        keep.append((k, p, n))
    idx = [k for k, _, _ in keep]
    return (kp[idx], np.array([p for _, p, _ in keep], np.float32).reshape(-1, 4),
            np.array([n for _, _, n in keep], np.float32).reshape(-1, 4), desc[idx])


def match2(q, t):
    """Two nearest train rows of every query row (L2): (best [nq, 2], dist [nq, 2])."""
    d2 = ((q[:, None, :].astype(np.float64) - t[None, :, :]) ** 2).sum(-1)
    order = np.argsort(d2, axis=1, kind="stable")[:, :2]
    dist = np.sqrt(np.take_along_axis(d2, order, axis=1))
    return order, dist
