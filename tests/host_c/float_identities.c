/* Checks, on the host, the float identities the tracking and integration
 * kernels use in place of the reference's double arithmetic or of IEEE
 * division (fusion_b200/csrc/track.cu, fb_common.cuh fd_rcp).  Built and run
 * by tests/test_float_identities.py; prints one line per identity with the
 * number of mismatches (all must be 0). */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

static float f_of(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static uint32_t u_of(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static uint64_t rng = 0x9e3779b97f4a7c15ull;
static uint32_t next32(void) { rng ^= rng << 13; rng ^= rng >> 7; rng ^= rng << 17; return (uint32_t)(rng >> 16); }

/* float(a + b) rounded toward zero, a + b exact in double */
static float add_rz(float a, float b) {
    const double s = (double)a + (double)b;
    float r = (float)s;
    if (fabs((double)r) > fabs(s)) r = nextafterf(r, 0.0f);
    return r;
}

int main(void) {
    long long bad, n;
    /* 1. Markstein: q = a*y, r = fma(-q, b, a), q' = r == 0 ? q : fma(r, y, q)
     *    with y = RN(1/b) equals RN(a / b); every significand of b, 24 values
     *    of a each (random, and a = q*b +- 2 ulps near exact quotients). */
    bad = n = 0;
    for (uint32_t bm = 0; bm < (1u << 23); ++bm) {
        const float b = f_of(0x3f800000u | bm);
        const float y = (float)(1.0 / (double)b);
        for (int k = 0; k < 24; ++k) {
            uint32_t am;
            if (k < 8) {
                const float q = f_of(0x3f800000u | (next32() & 0x7fffffu));
                am = u_of(q * b) + (uint32_t)(k % 5) - 2u;
            } else {
                am = (0x3f800000u | (next32() & 0x7fffffu)) + ((k & 1) ? 0x00800000u : 0u);
            }
            const float a = f_of(am);
            const float want = (float)((double)a / (double)b);
            const float q = a * y;
            const float r = fmaf(-q, b, a);
            const float got = r == 0.0f ? q : fmaf(r, y, q);
            n++;
            if (u_of(got) != u_of(want)) bad++;
        }
    }
    printf("fd_rcp %lld %lld\n", n, bad);

    /* 2. (int)((double)f + 0.5) == trunc(RZ(f + 0.5f)), f over every 7th
     *    float bit pattern of [-8192, 8192] */
    bad = n = 0;
    for (uint32_t u = 0; u < 0x46000000u; u += 7) {
        for (int s = 0; s < 2; ++s) {
            const float f = f_of(u | (s ? 0x80000000u : 0u));
            const int want = (int)((double)f + 0.5);
            const int got = (int)add_rz(f, 0.5f);
            n++;
            if (got != want) bad++;
        }
    }
    printf("trunc_half_up %lld %lld\n", n, bad);

    /* 3. floorf((float)((double)p + 0.5)) == floorf(RN(p + 0.5f)) */
    bad = n = 0;
    for (uint32_t u = 0; u < 0x46000000u; u += 7) {
        for (int s = 0; s < 2; ++s) {
            const float p = f_of(u | (s ? 0x80000000u : 0u));
            const float want = floorf((float)((double)p + 0.5));
            const float got = floorf(p + 0.5f);
            n++;
            if (u_of(got) != u_of(want)) bad++;
        }
    }
    printf("floor_half_up %lld %lld\n", n, bad);

    /* 4. (double)x < c  <=>  x < threshold float, within 2^20 ulps of c */
    {
        const double cs[3] = {1e-3, 0.1, 1e-6};
        const float ts[3] = {0.001f, 0.1f, f_of(0x358637beu)};
        bad = n = 0;
        for (int i = 0; i < 3; ++i) {
            const uint32_t c = u_of((float)cs[i]);
            for (uint32_t u = c - (1u << 20); u < c + (1u << 20); ++u) {
                const float x = f_of(u);
                n++;
                if (((double)x < cs[i]) != (x < ts[i])) bad++;
            }
        }
        printf("thresholds %lld %lld\n", n, bad);
    }

    /* 5. (float)((double)d / 9.0) == RN(d / 9.0f) for every Sobel value and
     *    (float)(1.0 / (double)z) == RN(1.0f / z) on sampled z */
    bad = n = 0;
    for (int d = -1020; d <= 1020; ++d) {
        n++;
        if (u_of((float)((double)d / 9.0)) != u_of((float)d / 9.0f)) bad++;
    }
    for (uint32_t u = 0x3a000000u; u < 0x44000000u; u += 13) {
        const float z = f_of(u);
        n++;
        if (u_of((float)(1.0 / (double)z)) != u_of(1.0f / z)) bad++;
    }
    printf("quotients %lld %lld\n", n, bad);
    return 0;
}
