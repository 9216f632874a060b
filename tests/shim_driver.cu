// TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's first-frame call sequence (System::GrabImage ->
// Frame / Tracker / Mapping, Core/System.cc:92-138) on the reference's own
// buffer types through include/fusion_b200_shim.hpp, so that the shim is
// exercised the way the reference's host classes would call it:
//   FilterDepth, ImageToIntensity, ComputeVMap, ComputeNMap, PyrDownGauss
//   (float and byte), ComputeDerivativeImage, ResetMap, FuseMapColor,
//   CheckBlockVisibility, CreateRenderingBlocks + Raycast, ResizeMap,
//   ICPStep, RGBStep, RenderImage.
// Built by `make -C oracle shim` against the reference's headers (never
// copied into this repository); tests/test_gpu_shim.py runs it and compares
// every output with the same calls made through the C ABI directly.
//
// usage: shim_driver W H fx fy cx cy depth_scale depth_cutoff depth_min
//        depth_max depth.u16 rgb.u8 out.bin
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "Reduction.h"
#include "fusion_b200_shim.hpp"

template <class T>
static void put(FILE* f, const DeviceArray2D<T>& a) {
    std::vector<T> h((size_t)a.cols * a.rows);
    a.download(h.data(), sizeof(T) * a.cols);
    fwrite(h.data(), sizeof(T), h.size(), f);
}

template <class T>
static std::vector<T> load(const char* path, size_t n) {
    std::vector<T> v(n);
    FILE* f = fopen(path, "rb");
    if (!f || fread(v.data(), sizeof(T), n, f) != n) {
        fprintf(stderr, "cannot read %s\n", path);
        exit(2);
    }
    fclose(f);
    return v;
}

int main(int argc, char** argv) {
    if (argc != 14) {
        fprintf(stderr, "usage: %s W H fx fy cx cy scale cutoff dmin dmax depth rgb out\n", argv[0]);
        return 2;
    }
    const int W = atoi(argv[1]), H = atoi(argv[2]);
    const float fx = (float)atof(argv[3]), fy = (float)atof(argv[4]), cx = (float)atof(argv[5]),
                cy = (float)atof(argv[6]), scale = (float)atof(argv[7]), cutoff = (float)atof(argv[8]),
                dmin = (float)atof(argv[9]), dmax = (float)atof(argv[10]);
    std::vector<unsigned short> hd = load<unsigned short>(argv[11], (size_t)W * H);
    std::vector<unsigned char> hc = load<unsigned char>(argv[12], (size_t)W * H * 3);

    DeviceArray2D<unsigned short> depth(W, H);
    DeviceArray2D<uchar3> color(W, H);
    depth.upload(hd.data(), sizeof(unsigned short) * W);
    color.upload(hc.data(), 3 * W);
    DeviceArray2D<float> raw(W, H), filt(W, H), depth1(W / 2, H / 2);
    DeviceArray2D<unsigned char> gray(W, H), gray1(W / 2, H / 2);
    DeviceArray2D<float4> vmap(W, H), nmap(W, H), rvmap(W, H), rnmap(W, H), rv1(W / 2, H / 2), rn1(W / 2, H / 2);
    DeviceArray2D<short> dx(W, H), dy(W, H);
    DeviceArray2D<uchar4> shaded(W, H);

    FilterDepth(depth, raw, filt, scale, cutoff);
    ImageToIntensity(color, gray);
    ComputeVMap(filt, vmap, fx, fy, cx, cy, cutoff);
    ComputeNMap(vmap, nmap);
    PyrDownGauss(filt, depth1);
    PyrDownGauss(gray, gray1);
    ComputeDerivativeImage(gray, dx, dy);

    Matrix3f I;
    I.rowx = make_float3(1, 0, 0);
    I.rowy = make_float3(0, 1, 0);
    I.rowz = make_float3(0, 0, 1);
    const float3 t0 = make_float3(0, 0, 0);
    DeviceMap map{};
    DeviceArray<uint> noVisible;
    ResetMap(map);   // before the first frame: no session yet
    uint fused = 0, visible = 0;
    FuseMapColor(raw, color, nmap, noVisible, I, I, t0, map, fx, fy, cx, cy, dmax, dmin, &fused);
    CheckBlockVisibility(map, noVisible, I, I, t0, W, H, fx, fy, cx, cy, dmax, dmin, &visible);
    DeviceArray<HashEntry> visibleEntries;
    DeviceArray2D<float> zX, zY;
    DeviceArray<RenderingBlock> blocks;
    DeviceArray<uint> noBlocks;
    int rendered = 0;
    if (CreateRenderingBlocks(visibleEntries, zX, zY, dmax, dmin, blocks, noBlocks, I, t0, visible, fx, fy, cx, cy)) {
        Raycast(map, rvmap, rnmap, zX, zY, I, I, t0, 1.0f / fx, 1.0f / fy, cx, cy);
        rendered = 1;
    }
    ResizeMap(rvmap, rnmap, rv1, rn1);

    // one Gauss-Newton step of the frame against its own raycast, identity poses
    Intrinsics K(fx, fy, cx, cy);
    DeviceArray2D<float> sum;
    DeviceArray<float> out;
    DeviceArray2D<int> sumRes;
    DeviceArray<int> outRes;
    float icp_res[2] = {0, 0}, rgb_res[2] = {0, 0};
    double icpA[36], icpb[6], rgbA[36], rgbb[6];
    ICPStep(vmap, rvmap, nmap, rnmap, I, t0, I, I, t0, K, sum, out, icp_res, icpA, icpb);
    RGBStep(gray, gray, vmap, rvmap, dx, dy, I, I, I, I, t0, t0, K, sum, out, sumRes, outRes, rgb_res, rgbA, rgbb);
    RenderImage(rvmap, rnmap, make_float3(0, 0, 0), shaded);
    cudaDeviceSynchronize();

    FILE* f = fopen(argv[13], "wb");
    if (!f) return 2;
    const int counts[3] = {(int)fused, (int)visible, rendered};
    fwrite(counts, sizeof(int), 3, f);
    put(f, raw);
    put(f, filt);
    put(f, gray);
    put(f, vmap);
    put(f, nmap);
    put(f, depth1);
    put(f, gray1);
    put(f, dx);
    put(f, dy);
    put(f, rvmap);
    put(f, rnmap);
    put(f, rv1);
    put(f, rn1);
    put(f, shaded);
    fwrite(icp_res, sizeof(float), 2, f);
    fwrite(icpA, sizeof(double), 36, f);
    fwrite(icpb, sizeof(double), 6, f);
    fwrite(rgb_res, sizeof(float), 2, f);
    fwrite(rgbA, sizeof(double), 36, f);
    fwrite(rgbb, sizeof(double), 6, f);
    fclose(f);
    printf("shim driver: fused %u visible %u rendered %d\n", fused, visible, rendered);
    return 0;
}
