/*
 * Seeded synthetic RGB-D sequence generator.
 *
 * Stands in for the on-disk RGB-D sequence the reference reads frame by frame
 * (MainTum.cc:78-96: u16 depth PNG + RGB JPG per frame) and for its OpenNI
 * camera (Core/Camera.cc:117-144).  Frames have the reference's frame format:
 * u16 depth in 1/depth_scale metres (0 = no measurement) and packed RGB8.
 *
 * Scene: a 4 x 4 x 3 m room (axis-aligned box) holding 20 seeded spheres and
 * yaw-rotated boxes of radius 0.1-0.5 m, each surface with a procedural colour
 * texture.  Camera: a seeded Catmull-Rom spline through control points in the
 * free centre of the room, time-scaled so that speed <= max_speed and angular
 * rate <= max_rate at the given frame rate.  Depth noise is Kinect-like:
 * N(0, 0.0012 + 0.0019 (z - 0.4)^2) m, 1 mm quantisation, random dropouts,
 * valid range [min_range, max_range].
 *
 * Rendering casts one ray per pixel against the analytic primitives (exact
 * intersections, which is what a converged ray-march would return).
 */
#ifndef FB_SYNTH_H
#define FB_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fbs_params {
    int width, height;
    float fx, fy, cx, cy;
    uint64_t seed;          /* scene + trajectory + noise seed */
    float depth_scale;      /* u16 units per metre (5000 = 0.2 mm units) */
    float min_range, max_range;  /* valid depth range, metres */
    float dropout;          /* probability of a zero pixel */
    int noise;              /* 0: noise-free depth (still quantised to 1 mm) */
    float fps;              /* frames per second of the trajectory */
    float max_speed;        /* m/s */
    float max_rate_deg;     /* deg/s */
} fbs_params;

/* Fill p with the defaults of the benchmark generator for a width x height
 * camera (fx = fy = 525 * width / 640, principal point at the centre). */
void fbs_default_params(fbs_params* p, int width, int height, uint64_t seed);

/* splitmix64 of x: the seed derivation seed = splitmix64(config << 32 | id). */
uint64_t fbs_splitmix64(uint64_t x);

/* Render frames [first, first + count) of the sequence.
 * depth: count * height * width u16, rgb: count * height * width * 3 bytes,
 * poses: count * 16 doubles (camera-to-world, row-major) or NULL.
 * Any output may be NULL.  Returns 0 on success, nonzero on bad arguments. */
int fbs_render(const fbs_params* p, int first, int count,
               uint16_t* depth, uint8_t* rgb, double* poses);

/* Number of threads the renderer uses (OpenMP). */
int fbs_num_threads(void);

#ifdef __cplusplus
}
#endif

#endif
