// TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's first-frame call sequence (System::GrabImage ->
// Frame / Tracker / Mapping, Core/System.cc:92-138) on the reference's own
// buffer types through include/fusion_b200_shim.hpp, so that the shim is
// exercised the way the reference's host classes would call it:
//   FilterDepth, ImageToIntensity, ComputeVMap, ComputeNMap, PyrDownGauss
//   (float and byte), ComputeDerivativeImage, ResetMap, FuseMapColor,
//   CheckBlockVisibility, CreateRenderingBlocks + Raycast, ResizeMap,
//   ICPStep, RGBStep, RenderImage;
// then the mapping calls of a second frame at a given pose, with the map's
// buffers allocated as Mapping::Create does (Mapping/Mapping.cc:11-51) and
// passed as Mapping::operator DeviceMap does (Mapping.cc:311-325); then the
// reference's buffers are read back: the visible entries and counter after
// each frame, the z-range images, the whole map after ExportMap, and the map
// after a ResetMap of the populated map.
// Built by `make -C oracle shim` against the reference's headers (never
// copied into this repository); tests/test_gpu_shim.py runs it and compares
// every output with the same calls made through the C ABI directly.
//
// usage: shim_driver W H fx fy cx cy depth_scale depth_cutoff depth_min
//        depth_max depth.u16 rgb.u8 depth2.u16 rgb2.u8 pose2.f64 out.bin
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
    if (argc != 17) {
        fprintf(stderr, "usage: %s W H fx fy cx cy scale cutoff dmin dmax depth rgb depth2 rgb2 pose2 out\n",
                argv[0]);
        return 2;
    }
    const int W = atoi(argv[1]), H = atoi(argv[2]);
    const float fx = (float)atof(argv[3]), fy = (float)atof(argv[4]), cx = (float)atof(argv[5]),
                cy = (float)atof(argv[6]), scale = (float)atof(argv[7]), cutoff = (float)atof(argv[8]),
                dmin = (float)atof(argv[9]), dmax = (float)atof(argv[10]);
    std::vector<unsigned short> hd = load<unsigned short>(argv[11], (size_t)W * H);
    std::vector<unsigned char> hc = load<unsigned char>(argv[12], (size_t)W * H * 3);
    std::vector<unsigned short> hd2 = load<unsigned short>(argv[13], (size_t)W * H);
    std::vector<unsigned char> hc2 = load<unsigned char>(argv[14], (size_t)W * H * 3);
    std::vector<double> T2 = load<double>(argv[15], 16);

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
    // the map's buffers as Mapping::Create allocates them, and the DeviceMap
    // view Mapping::operator DeviceMap passes
    DeviceArray<int> heapCounter(1), hashCounter(1), heap(DeviceMap::NumSdfBlocks),
        bucketMutex(DeviceMap::NumBuckets);
    DeviceArray<uint> noVisible(1), noBlocks(1);
    DeviceArray<Voxel> sdfBlock(DeviceMap::NumVoxels);
    DeviceArray<HashEntry> hashEntries(DeviceMap::NumEntries), visibleEntries(DeviceMap::NumEntries);
    DeviceArray2D<float> zX(80, 60), zY(80, 60);
    DeviceArray<RenderingBlock> blocks(DeviceMap::MaxRenderingBlocks);
    DeviceMap map;
    map.heapMem = heap;
    map.heapCounter = heapCounter;
    map.noVisibleBlocks = noVisible;
    map.bucketMutex = bucketMutex;
    map.hashEntries = hashEntries;
    map.visibleEntries = visibleEntries;
    map.voxelBlocks = sdfBlock;
    map.entryPtr = hashCounter;
    ResetMap(map);   // before the first frame: no session yet
    uint fused = 0, visible = 0;
    FuseMapColor(raw, color, nmap, noVisible, I, I, t0, map, fx, fy, cx, cy, dmax, dmin, &fused);
    CheckBlockVisibility(map, noVisible, I, I, t0, W, H, fx, fy, cx, cy, dmax, dmin, &visible);
    int rendered = 0;
    if (CreateRenderingBlocks(visibleEntries, zX, zY, dmax, dmin, blocks, noBlocks, I, t0, visible, fx, fy, cx, cy)) {
        Raycast(map, rvmap, rnmap, zX, zY, I, I, t0, 1.0f / fx, 1.0f / fy, cx, cy);
        rendered = 1;
    }
    // frame 1 as the reference's buffers hold it
    std::vector<uint> h_nvis1(1), h_tiles1(1);
    noVisible.download(h_nvis1.data());
    noBlocks.download(h_tiles1.data());
    std::vector<HashEntry> h_vis1(visible);
    if (visible) cudaMemcpy(h_vis1.data(), visibleEntries.data, sizeof(HashEntry) * visible, cudaMemcpyDeviceToHost);
    std::vector<float> h_zx1(80 * 60), h_zy1(80 * 60);
    zX.download(h_zx1.data(), sizeof(float) * 80);
    zY.download(h_zy1.data(), sizeof(float) * 80);
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

    // frame 2: its preprocessing and the mapping calls at pose T2
    depth.upload(hd2.data(), sizeof(unsigned short) * W);
    color.upload(hc2.data(), 3 * W);
    DeviceArray2D<float> raw2(W, H), filt2(W, H);
    DeviceArray2D<float4> vmap2(W, H), nmap2(W, H), rvmap2(W, H), rnmap2(W, H);
    FilterDepth(depth, raw2, filt2, scale, cutoff);
    ComputeVMap(filt2, vmap2, fx, fy, cx, cy, cutoff);
    ComputeNMap(vmap2, nmap2);
    Matrix3f R2, R2inv;
    R2.rowx = make_float3((float)T2[0], (float)T2[1], (float)T2[2]);
    R2.rowy = make_float3((float)T2[4], (float)T2[5], (float)T2[6]);
    R2.rowz = make_float3((float)T2[8], (float)T2[9], (float)T2[10]);
    R2inv.rowx = make_float3((float)T2[0], (float)T2[4], (float)T2[8]);
    R2inv.rowy = make_float3((float)T2[1], (float)T2[5], (float)T2[9]);
    R2inv.rowz = make_float3((float)T2[2], (float)T2[6], (float)T2[10]);
    const float3 t2 = make_float3((float)T2[3], (float)T2[7], (float)T2[11]);
    uint fused2 = 0, visible2 = 0;
    FuseMapColor(raw2, color, nmap2, noVisible, R2, R2inv, t2, map, fx, fy, cx, cy, dmax, dmin, &fused2);
    CheckBlockVisibility(map, noVisible, R2, R2inv, t2, W, H, fx, fy, cx, cy, dmax, dmin, &visible2);
    int rendered2 = 0;
    if (CreateRenderingBlocks(visibleEntries, zX, zY, dmax, dmin, blocks, noBlocks, R2inv, t2, visible2, fx, fy, cx,
                              cy)) {
        Raycast(map, rvmap2, rnmap2, zX, zY, R2, R2inv, t2, 1.0f / fx, 1.0f / fy, cx, cy);
        rendered2 = 1;
    }
    std::vector<uint> h_nvis2(1), h_tiles2(1);
    noVisible.download(h_nvis2.data());
    noBlocks.download(h_tiles2.data());
    std::vector<HashEntry> h_vis2(visible2);
    if (visible2)
        cudaMemcpy(h_vis2.data(), visibleEntries.data, sizeof(HashEntry) * visible2, cudaMemcpyDeviceToHost);
    std::vector<float> h_zx2(80 * 60), h_zy2(80 * 60);
    zX.download(h_zx2.data(), sizeof(float) * 80);
    zY.download(h_zy2.data(), sizeof(float) * 80);
    // the whole map in the reference's buffers, then the visible blocks' voxels
    fusion_b200_shim::ExportMap(map);
    std::vector<HashEntry> h_table(DeviceMap::NumEntries);
    hashEntries.download(h_table.data());
    std::vector<int> h_hc(1), h_ep(1), h_heap(DeviceMap::NumSdfBlocks);
    heapCounter.download(h_hc.data());
    hashCounter.download(h_ep.data());
    heap.download(h_heap.data());
    std::vector<Voxel> h_vox((size_t)visible2 * 512);
    for (uint i = 0; i < visible2; ++i)
        cudaMemcpy(h_vox.data() + (size_t)i * 512, (const Voxel*)sdfBlock.data + h_vis2[i].ptr, 512 * sizeof(Voxel),
                   cudaMemcpyDeviceToHost);   // DeviceArray::data is a void pointer
    // ResetMap of the populated map: the exported map is empty again
    ResetMap(map);
    uint visible3 = 0;
    CheckBlockVisibility(map, noVisible, R2, R2inv, t2, W, H, fx, fy, cx, cy, dmax, dmin, &visible3);
    fusion_b200_shim::ExportMap(map);
    std::vector<HashEntry> h_table3(DeviceMap::NumEntries);
    hashEntries.download(h_table3.data());
    std::vector<int> h_hc3(1), h_ep3(1);
    heapCounter.download(h_hc3.data());
    hashCounter.download(h_ep3.data());
    int occupied3 = 0;
    for (const HashEntry& e : h_table3) occupied3 += e.ptr >= 0;

    FILE* f = fopen(argv[16], "wb");
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
    // the reference's buffers: frame 1, frame 2, the exported map, after ResetMap
    const int more[10] = {(int)h_nvis1[0], (int)h_tiles1[0], (int)fused2, (int)visible2, rendered2,
                          (int)h_nvis2[0], (int)h_tiles2[0], h_hc[0], h_ep[0], (int)visible3};
    fwrite(more, sizeof(int), 10, f);
    fwrite(h_vis1.data(), sizeof(HashEntry), h_vis1.size(), f);
    fwrite(h_zx1.data(), sizeof(float), h_zx1.size(), f);
    fwrite(h_zy1.data(), sizeof(float), h_zy1.size(), f);
    fwrite(h_vis2.data(), sizeof(HashEntry), h_vis2.size(), f);
    fwrite(h_zx2.data(), sizeof(float), h_zx2.size(), f);
    fwrite(h_zy2.data(), sizeof(float), h_zy2.size(), f);
    fwrite(h_table.data(), sizeof(HashEntry), h_table.size(), f);
    fwrite(h_heap.data(), sizeof(int), h_heap.size(), f);
    fwrite(h_vox.data(), sizeof(Voxel), h_vox.size(), f);
    put(f, rvmap2);
    put(f, rnmap2);
    const int reset[3] = {occupied3, h_hc3[0], h_ep3[0]};
    fwrite(reset, sizeof(int), 3, f);
    fclose(f);
    printf("shim driver: fused %u visible %u rendered %d; frame 2: fused %u visible %u rendered %d\n", fused,
           visible, rendered, fused2, visible2, rendered2);
    return 0;
}
