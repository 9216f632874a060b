// Seeded synthetic RGB-D sequence generator (see synth.h for the scene).
#include "synth.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kNumObjects = 20;
constexpr int kNumSegments = 256;      // spline segments with a fixed time scale
constexpr double kSegSeconds = 1.5;    // nominal duration of one spline segment

// Room bounds (world frame, y points down like the camera's y axis).
constexpr double kRoomMin[3] = {-2.0, -1.5, -2.0};
constexpr double kRoomMax[3] = {2.0, 1.5, 2.0};
// Free region the camera moves in.
constexpr double kCamHalf[3] = {0.6, 0.3, 0.6};

uint64_t splitmix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next() { s += 0x9E3779B97F4A7C15ull; return splitmix(s); }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform(double a, double b) { return a + (b - a) * uniform(); }
};

// Uniform in [0,1) from a counter (thread-order independent).
inline double hash_uniform(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t h = splitmix(a ^ splitmix(b ^ splitmix(c)));
    return (h >> 11) * (1.0 / 9007199254740992.0);
}

struct V3 { double x, y, z; };
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 normalise(V3 a) { double n = std::sqrt(dot(a, a)); return a * (1.0 / n); }

struct Object {
    int is_box;
    V3 c;            // centre
    double r;        // sphere radius / largest box half extent
    V3 half;         // box half extents (local frame)
    double cy, sy;   // box yaw (rotation about world y)
    double base[3];  // texture base colour
    V3 stripe;       // stripe direction
};

struct Scene {
    Object obj[kNumObjects];
    double wall_base[6][3];
    V3 wall_stripe[6];
};

// Control point of the camera spline.
struct Ctrl { double p[3]; double yaw, pitch, roll; };

struct Sequence {
    Scene scene;
    std::vector<Ctrl> ctrl;   // kNumSegments + 3 control points
    double time_scale;        // seconds of real time per nominal second
};

double dist_point_box(V3 c, const double* half) {
    double dx = std::max(0.0, std::fabs(c.x) - half[0]);
    double dy = std::max(0.0, std::fabs(c.y) - half[1]);
    double dz = std::max(0.0, std::fabs(c.z) - half[2]);
    return std::sqrt(dx * dx + dy * dy + dz * dz);
}

void build_scene(uint64_t seed, Scene* s) {
    Rng rng(splitmix(seed ^ 0x5CE9E5CE9Eull));
    for (int i = 0; i < kNumObjects; ++i) {
        Object& o = s->obj[i];
        for (int attempt = 0; attempt < 1000; ++attempt) {
            o.r = rng.uniform(0.1, 0.5);
            o.c.x = rng.uniform(kRoomMin[0] + o.r, kRoomMax[0] - o.r);
            o.c.y = rng.uniform(kRoomMin[1] + o.r, kRoomMax[1] - o.r);
            o.c.z = rng.uniform(kRoomMin[2] + o.r, kRoomMax[2] - o.r);
            if (dist_point_box(o.c, kCamHalf) > o.r * 1.8 + 0.45) break;
        }
        o.is_box = rng.uniform() < 0.5;
        o.half = {o.r, o.r * rng.uniform(0.5, 1.0), o.r * rng.uniform(0.5, 1.0)};
        double yaw = rng.uniform(0, 2 * kPi);
        o.cy = std::cos(yaw);
        o.sy = std::sin(yaw);
        for (int k = 0; k < 3; ++k) o.base[k] = rng.uniform(50, 230);
        o.stripe = normalise({rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(-1, 1)});
    }
    for (int w = 0; w < 6; ++w) {
        for (int k = 0; k < 3; ++k) s->wall_base[w][k] = rng.uniform(60, 220);
        s->wall_stripe[w] = normalise({rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(-1, 1)});
    }
}

double catmull(double p0, double p1, double p2, double p3, double t) {
    double t2 = t * t, t3 = t2 * t;
    return 0.5 * ((2 * p1) + (-p0 + p2) * t + (2 * p0 - 5 * p1 + 4 * p2 - p3) * t2 +
                  (-p0 + 3 * p1 - 3 * p2 + p3) * t3);
}

// Camera-to-world rotation from yaw (about y), pitch (about x), roll (about z).
void rotation(double yaw, double pitch, double roll, double R[9]) {
    double cy = std::cos(yaw), sy = std::sin(yaw);
    double cp = std::cos(pitch), sp = std::sin(pitch);
    double cr = std::cos(roll), sr = std::sin(roll);
    double Ry[9] = {cy, 0, sy, 0, 1, 0, -sy, 0, cy};
    double Rx[9] = {1, 0, 0, 0, cp, -sp, 0, sp, cp};
    double Rz[9] = {cr, -sr, 0, sr, cr, 0, 0, 0, 1};
    double T[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T[i * 3 + j] = 0;
            for (int k = 0; k < 3; ++k) T[i * 3 + j] += Ry[i * 3 + k] * Rx[k * 3 + j];
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            R[i * 3 + j] = 0;
            for (int k = 0; k < 3; ++k) R[i * 3 + j] += T[i * 3 + k] * Rz[k * 3 + j];
        }
}

// Pose at nominal spline time tau (seconds): position and rotation.
void eval_nominal(const std::vector<Ctrl>& c, double tau, double pos[3], double R[9]) {
    double u = tau / kSegSeconds;
    int seg = (int)std::floor(u);
    if (seg < 0) seg = 0;
    if (seg > kNumSegments - 1) seg = kNumSegments - 1;
    double t = u - seg;
    const Ctrl &a = c[seg], &b = c[seg + 1], &d = c[seg + 2], &e = c[seg + 3];
    for (int k = 0; k < 3; ++k) pos[k] = catmull(a.p[k], b.p[k], d.p[k], e.p[k], t);
    double yaw = catmull(a.yaw, b.yaw, d.yaw, e.yaw, t);
    double pitch = catmull(a.pitch, b.pitch, d.pitch, e.pitch, t);
    double roll = catmull(a.roll, b.roll, d.roll, e.roll, t);
    rotation(yaw, pitch, roll, R);
}

double rot_angle(const double A[9], const double B[9]) {
    double tr = 0;  // trace(A^T B)
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) tr += A[k * 3 + i] * B[k * 3 + i];
    double c = std::max(-1.0, std::min(1.0, (tr - 1) * 0.5));
    return std::acos(c);
}

void build_sequence(const fbs_params* p, Sequence* s) {
    build_scene(p->seed, &s->scene);
    Rng rng(splitmix(p->seed ^ 0x7AC70Aull));
    s->ctrl.resize(kNumSegments + 3);
    double yaw = rng.uniform(0, 2 * kPi);
    for (auto& c : s->ctrl) {
        for (int k = 0; k < 3; ++k) c.p[k] = rng.uniform(-kCamHalf[k], kCamHalf[k]);
        yaw += rng.uniform(-70, 70) * kPi / 180;
        c.yaw = yaw;
        c.pitch = rng.uniform(-20, 20) * kPi / 180;
        c.roll = rng.uniform(-5, 5) * kPi / 180;
    }
    // Time scale so that speed and angular rate stay within the limits.
    const double dt = 1.0 / 240.0;
    double vmax = 0, wmax = 0;
    double p0[3], R0[9], p1[3], R1[9];
    eval_nominal(s->ctrl, 0, p0, R0);
    for (double tau = dt; tau < kNumSegments * kSegSeconds; tau += dt) {
        eval_nominal(s->ctrl, tau, p1, R1);
        double dx = p1[0] - p0[0], dy = p1[1] - p0[1], dz = p1[2] - p0[2];
        vmax = std::max(vmax, std::sqrt(dx * dx + dy * dy + dz * dz) / dt);
        wmax = std::max(wmax, rot_angle(R0, R1) / dt);
        std::memcpy(p0, p1, sizeof p0);
        std::memcpy(R0, R1, sizeof R0);
    }
    double rate = p->max_rate_deg * kPi / 180;
    // 2 % margin for the sampling of the maxima
    s->time_scale = std::max(1.0, 1.02 * std::max(vmax / p->max_speed, wmax / rate));
}

struct Hit { double t; V3 n; int surf; };

// Ray o + t d (d unnormalised), nearest hit with t > 0.
Hit intersect(const Scene& sc, V3 o, V3 d) {
    Hit h{1e30, {0, 0, 0}, -1};
    // room: the ray starts inside; exit through the nearest wall
    const double* mn = kRoomMin;
    const double* mx = kRoomMax;
    double dv[3] = {d.x, d.y, d.z}, ov[3] = {o.x, o.y, o.z};
    for (int a = 0; a < 3; ++a) {
        if (dv[a] == 0) continue;
        double bound = dv[a] > 0 ? mx[a] : mn[a];
        double t = (bound - ov[a]) / dv[a];
        if (t > 0 && t < h.t) {
            h.t = t;
            double n[3] = {0, 0, 0};
            n[a] = dv[a] > 0 ? -1 : 1;
            h.n = {n[0], n[1], n[2]};
            h.surf = 100 + a * 2 + (dv[a] > 0);
        }
    }
    for (int i = 0; i < kNumObjects; ++i) {
        const Object& ob = sc.obj[i];
        V3 oc = o - ob.c;
        if (!ob.is_box) {
            double A = dot(d, d), B = 2 * dot(oc, d), C = dot(oc, oc) - ob.r * ob.r;
            double disc = B * B - 4 * A * C;
            if (disc < 0) continue;
            double sq = std::sqrt(disc);
            double t = (-B - sq) / (2 * A);
            if (t <= 1e-9) t = (-B + sq) / (2 * A);
            if (t > 1e-9 && t < h.t) {
                h.t = t;
                h.n = normalise(oc + d * t);
                h.surf = i;
            }
        } else {
            // local frame: rotate by -yaw about y
            V3 lo = {ob.cy * oc.x - ob.sy * oc.z, oc.y, ob.sy * oc.x + ob.cy * oc.z};
            V3 ld = {ob.cy * d.x - ob.sy * d.z, d.y, ob.sy * d.x + ob.cy * d.z};
            double lov[3] = {lo.x, lo.y, lo.z}, ldv[3] = {ld.x, ld.y, ld.z};
            double hv[3] = {ob.half.x, ob.half.y, ob.half.z};
            double tmin = -1e30, tmax = 1e30;
            int amin = -1;
            double smin = 0;
            bool miss = false;
            for (int a = 0; a < 3; ++a) {
                if (std::fabs(ldv[a]) < 1e-15) {
                    if (std::fabs(lov[a]) > hv[a]) { miss = true; break; }
                    continue;
                }
                double t1 = (-hv[a] - lov[a]) / ldv[a];
                double t2 = (hv[a] - lov[a]) / ldv[a];
                double s = -1;
                if (t1 > t2) { std::swap(t1, t2); s = 1; }
                if (t1 > tmin) { tmin = t1; amin = a; smin = s; }
                tmax = std::min(tmax, t2);
            }
            if (miss || tmin > tmax || tmin <= 1e-9 || amin < 0) continue;
            if (tmin < h.t) {
                double ln[3] = {0, 0, 0};
                ln[amin] = smin;
                // back to world: rotate by +yaw about y
                h.t = tmin;
                h.n = {ob.cy * ln[0] + ob.sy * ln[2], ln[1], -ob.sy * ln[0] + ob.cy * ln[2]};
                h.surf = i;
            }
        }
    }
    return h;
}

void shade(const Scene& sc, const Hit& h, V3 p, uint8_t out[3]) {
    const double* base;
    V3 stripe;
    if (h.surf >= 100) {
        base = sc.wall_base[h.surf - 100];
        stripe = sc.wall_stripe[h.surf - 100];
    } else {
        base = sc.obj[h.surf].base;
        stripe = sc.obj[h.surf].stripe;
    }
    const double cell = 0.08;
    int cx = (int)std::floor(p.x / cell), cy = (int)std::floor(p.y / cell),
        cz = (int)std::floor(p.z / cell);
    double checker = ((cx + cy + cz) & 1) ? 1.0 : 0.0;
    double wave = std::sin(2 * kPi * dot(p, stripe) / 0.13);
    V3 light = {0.0, -1.4, 0.0};
    V3 l = normalise(light - p);
    double lam = 0.65 + 0.35 * std::fabs(dot(h.n, l));
    double f = (0.5 + 0.32 * checker + 0.18 * wave) * lam;
    for (int k = 0; k < 3; ++k) {
        double v = base[k] * f + 12.0;
        v = std::max(0.0, std::min(255.0, v));
        out[k] = (uint8_t)std::lround(v);
    }
}

void pose_at(const Sequence& s, const fbs_params* p, int frame, double pos[3], double R[9]) {
    double t = frame / (double)p->fps;
    eval_nominal(s.ctrl, t / s.time_scale, pos, R);
}

}  // namespace

extern "C" {

uint64_t fbs_splitmix64(uint64_t x) { return splitmix(x); }

void fbs_default_params(fbs_params* p, int width, int height, uint64_t seed) {
    p->width = width;
    p->height = height;
    p->fx = p->fy = 525.0f * width / 640.0f;
    p->cx = width * 0.5f;
    p->cy = height * 0.5f;
    p->seed = seed;
    p->depth_scale = 5000.0f;
    p->min_range = 0.3f;
    p->max_range = 4.0f;
    p->dropout = 0.02f;
    p->noise = 1;
    p->fps = 30.0f;
    p->max_speed = 0.5f;
    p->max_rate_deg = 30.0f;
}

int fbs_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int fbs_render(const fbs_params* p, int first, int count, uint16_t* depth, uint8_t* rgb,
               double* poses) {
    if (!p || p->width <= 0 || p->height <= 0 || count < 0 || first < 0) return 1;
    if (p->fx <= 0 || p->fy <= 0 || p->fps <= 0 || p->max_speed <= 0 || p->max_rate_deg <= 0)
        return 1;
    Sequence seq;
    build_sequence(p, &seq);
    const int W = p->width, H = p->height;
    const size_t npx = (size_t)W * H;
    for (int f = 0; f < count; ++f) {
        int frame = first + f;
        double pos[3], R[9];
        pose_at(seq, p, frame, pos, R);
        if (poses) {
            double* T = poses + 16 * (size_t)f;
            for (int i = 0; i < 3; ++i) {
                for (int j = 0; j < 3; ++j) T[i * 4 + j] = R[i * 3 + j];
                T[i * 4 + 3] = pos[i];
            }
            T[12] = T[13] = T[14] = 0;
            T[15] = 1;
        }
        if (!depth && !rgb) continue;
        uint16_t* dout = depth ? depth + npx * f : nullptr;
        uint8_t* cout = rgb ? rgb + npx * 3 * f : nullptr;
        V3 o = {pos[0], pos[1], pos[2]};
#pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < H; ++y) {
            for (int x = 0; x < W; ++x) {
                V3 dc = {(x - p->cx) / p->fx, (y - p->cy) / p->fy, 1.0};
                V3 dw = {R[0] * dc.x + R[1] * dc.y + R[2] * dc.z,
                         R[3] * dc.x + R[4] * dc.y + R[5] * dc.z,
                         R[6] * dc.x + R[7] * dc.y + R[8] * dc.z};
                Hit h = intersect(seq.scene, o, dw);
                size_t idx = (size_t)y * W + x;
                double z = h.t;  // camera-frame depth (dc.z == 1)
                if (dout) {
                    double zn = z;
                    uint64_t key = (uint64_t)frame * 0x100000001ull;
                    if (p->noise) {
                        double sigma = 0.0012 + 0.0019 * (z - 0.4) * (z - 0.4);
                        double u1 = hash_uniform(p->seed, key, idx * 2 + 1);
                        double u2 = hash_uniform(p->seed, key, idx * 2 + 2);
                        if (u1 < 1e-300) u1 = 1e-300;
                        zn = z + sigma * std::sqrt(-2.0 * std::log(u1)) * std::cos(2 * kPi * u2);
                    }
                    double mm = std::nearbyint(zn * 1000.0);
                    double zq = mm / 1000.0;
                    uint16_t v = 0;
                    bool drop = hash_uniform(p->seed ^ 0xD809ull, key, idx) < p->dropout;
                    if (!drop && h.surf >= 0 && zq >= p->min_range && zq <= p->max_range) {
                        double u = std::nearbyint(zq * p->depth_scale);
                        v = (uint16_t)std::min(65535.0, u);
                    }
                    dout[idx] = v;
                }
                if (cout) {
                    uint8_t c[3] = {0, 0, 0};
                    if (h.surf >= 0) shade(seq.scene, h, o + dw * h.t, c);
                    cout[idx * 3 + 0] = c[0];
                    cout[idx * 3 + 1] = c[1];
                    cout[idx * 3 + 2] = c[2];
                }
            }
        }
    }
    return 0;
}

}  // extern "C"
