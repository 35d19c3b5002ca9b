// ORACLE -- test infrastructure only.
//
// C entry points over the reference's own BVHRT-Core code compiled for the
// host execution model (simt.h) by oracle/build.py into
// oracle/_ref/libbvhrt_ref_host.so.  ref_host_run follows the call sequence
// of gpu-ray-traversal/src/rt/cuda/Renderer.cpp:164-228: SceneWrapper ->
// LBVHBuilder::BuildTree -> (TRBVH | Agglomerative)TreeletOptimizer::Optimize
// -> BVHTreeCollapser::Collapse -> BVHTreeInstanceManager::DeviceToHost*Tree.
// The ref_host_* helpers call the reference's __host__ __device__ arithmetic
// (BVHRT-Core/src/Commons.cuh) and SoABVHTree::SAH directly.

#include <chrono>
#include <cstring>
#include <iostream>
#include <sstream>

#include "AgglomerativeTreeletOptimizer.h"
#include "BVHCollapsedTree.h"
#include "BVHTreeCollapser.h"
#include "BVHTreeInstanceManager.h"
#include "Commons.cuh"
#include "CubWrapper.h"
#include "LBVH.h"
#include "LBVHBuilder.h"
#include "SceneWrapper.h"
#include "TRBVHOptimizer.h"

using namespace BVHRT;

namespace {

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

float4 f4(const float* p) { return float4{p[0], p[1], p[2], p[3]}; }
float3 f3(const float* p) { return float3{p[0], p[1], p[2]}; }

struct Quiet {
    std::ostringstream sink;
    std::streambuf* old;
    explicit Quiet(bool on) : old(on ? std::cout.rdbuf(sink.rdbuf()) : nullptr) {}
    ~Quiet() {
        if (old) std::cout.rdbuf(old);
    }
};

}  // namespace

extern "C" {

// optimizer: 0 none, 1 ATRBVH, 2 TRBVH.  Tree outputs (2n-1 entries, boxes as
// float4) and collapsed outputs may be NULL.  times_ms[0..2] = build,
// optimise, collapse host times.  Returns 0.
int ref_host_run(const float* vertices, unsigned int n, const float* bbmin, const float* bbmax, int use64,
                 int optimizer, int treelet, int iterations, int collapse, int quiet, int* parent, int* left,
                 int* right, int* data, float* bmin4, float* bmax4, float* area, int* c_parent, int* c_left,
                 int* c_right, int* c_data, int* c_count, float* c_bmin4, float* c_bmax4, int* c_tri,
                 float* collapse_sah, double* times_ms) {
    Quiet q(quiet != 0);
    float4* v = new float4[3 * (size_t)n];
    std::memcpy(v, vertices, sizeof(float4) * 3 * (size_t)n);
    SceneWrapper* sw = new SceneWrapper(n, v, f3(bbmin), f3(bbmax));  // takes ownership of v
    const double t0 = now_ms();
    LBVHBuilder builder(use64 != 0);
    BVHTree* dt = builder.BuildTree(sw);
    const double t1 = now_ms();
    if (optimizer == 1) {
        AgglomerativeTreeletOptimizer opt(treelet, iterations);
        opt.Optimize(dt);
    } else if (optimizer == 2) {
        TRBVHOptimizer opt(treelet, iterations);
        opt.Optimize(dt);
    }
    const double t2 = now_ms();
    BVHTreeInstanceManager mgr;
    BVHTree* ht = mgr.DeviceToHostTree(dt);
    const size_t nn = 2 * (size_t)n - 1;
    for (size_t i = 0; i < nn; ++i) {
        if (parent) parent[i] = ht->ParentIndex((int)i);
        if (left) left[i] = ht->LeftIndex((int)i);
        if (right) right[i] = ht->RightIndex((int)i);
        if (data) data[i] = ht->DataIndex((int)i);
        if (bmin4) {
            const float4 b = ht->BoundingBoxMin((int)i);
            std::memcpy(bmin4 + 4 * i, &b, 16);
        }
        if (bmax4) {
            const float4 b = ht->BoundingBoxMax((int)i);
            std::memcpy(bmax4 + 4 * i, &b, 16);
        }
        if (area) area[i] = ht->Area((int)i);
    }
    delete ht;
    double t3 = t2;
    if (collapse) {
        float sah = 0.0f;
        BVHTreeCollapser collapser;
        BVHCollapsedTree* dc = collapser.Collapse(dt, &sah);
        t3 = now_ms();
        if (collapse_sah) *collapse_sah = sah;
        BVHCollapsedTree* hc = mgr.DeviceToHostCollapsedTree(dc);
        for (size_t i = 0; i < nn; ++i) {
            if (c_parent) c_parent[i] = hc->nodes.parentIndices[i];
            if (c_left) c_left[i] = hc->nodes.leftIndices[i];
            if (c_right) c_right[i] = hc->nodes.rightIndices[i];
            if (c_data) c_data[i] = hc->nodes.dataIndices[i];
            if (c_count) c_count[i] = hc->nodes.triangleCount[i];
            if (c_bmin4) std::memcpy(c_bmin4 + 4 * i, &hc->nodes.boundingBoxMin[i], 16);
            if (c_bmax4) std::memcpy(c_bmax4 + 4 * i, &hc->nodes.boundingBoxMax[i], 16);
        }
        if (c_tri) std::memcpy(c_tri, hc->triangleIndices, sizeof(int) * n);
        delete hc;
        mgr.FreeDeviceCollapsedTree(dc);
    }
    mgr.FreeDeviceTree(dt);
    delete sw;
    if (times_ms) {
        times_ms[0] = t1 - t0;
        times_ms[1] = t2 - t1;
        times_ms[2] = t3 - t2;
    }
    return 0;
}

// The reference's Morton kernel (LBVH.cu:53-97) through DeviceGenerateMortonCodes:
// keys (30-bit into keys32, or 63-bit into keys64) and the index array it fills.
int ref_host_morton(const float* vertices, unsigned int n, const float* bbmin, const float* bbmax, int use64,
                    unsigned int* keys32, unsigned long long int* keys64, unsigned int* indices) {
    float4* v = new float4[3 * (size_t)n];
    std::memcpy(v, vertices, sizeof(float4) * 3 * (size_t)n);
    SceneWrapper sw(n, v, f3(bbmin), f3(bbmax));
    unsigned int* idx = nullptr;
    cudaMalloc(&idx, n * sizeof(unsigned int));
    if (use64) {
        unsigned long long int* k = nullptr;
        cudaMalloc(&k, n * sizeof(unsigned long long int));
        DeviceGenerateMortonCodes(n, sw.DeviceScene(), k, idx);
        std::memcpy(keys64, k, n * sizeof(unsigned long long int));
        cudaFree(k);
    } else {
        unsigned int* k = nullptr;
        cudaMalloc(&k, n * sizeof(unsigned int));
        DeviceGenerateMortonCodes(n, sw.DeviceScene(), k, idx);
        std::memcpy(keys32, k, n * sizeof(unsigned int));
        cudaFree(k);
    }
    if (indices) std::memcpy(indices, idx, n * sizeof(unsigned int));
    cudaFree(idx);
    return 0;
}

// The reference's triangle-splitting LBVH kernels (no builder of the
// reference calls them): LBVH.cu:99-161 DeviceGenerateMortonCodes over
// primitive boxes, the sort into the *Out buffers, LBVH.cu:320-428
// DeviceBuildTree with data and routing indices, LBVH.cu:572-669
// DeviceCalculateInternalNodeBoundingBoxes with counters preset to 0xFF as
// LBVHBuilder.cpp:90-94 does for the other path.  pbmin4 / pbmax4: n float4;
// pdata: n triangle indices; the scene box comes from bbmin / bbmax.
int ref_host_lbvh_ts(unsigned int n, const float* pbmin4, const float* pbmax4, const unsigned int* pdata,
                     const float* bbmin, const float* bbmax, int use64, int* parent, int* left, int* right,
                     int* data, float* bmin4, float* bmax4, float* area) {
    // A scene holding the box: the primitive-box Morton kernel reads only
    // scene->boundingBoxMin/Max (one placeholder triangle).
    float4* v = new float4[3];
    for (int k = 0; k < 3; ++k) v[k] = float4{0.0f, 0.0f, 0.0f, 0.0f};
    SceneWrapper sw(1, v, f3(bbmin), f3(bbmax));
    float4 *bmn = nullptr, *bmx = nullptr;
    unsigned int *route = nullptr, *route_out = nullptr, *dind = nullptr, *counters = nullptr;
    cudaMalloc(&bmn, n * sizeof(float4));
    cudaMalloc(&bmx, n * sizeof(float4));
    cudaMalloc(&route, n * sizeof(unsigned int));
    cudaMalloc(&route_out, n * sizeof(unsigned int));
    cudaMalloc(&dind, n * sizeof(unsigned int));
    cudaMalloc(&counters, (n - 1) * sizeof(unsigned int));
    std::memcpy(bmn, pbmin4, n * sizeof(float4));
    std::memcpy(bmx, pbmax4, n * sizeof(float4));
    std::memcpy(dind, pdata, n * sizeof(unsigned int));
    BVHTreeInstanceManager mgr;
    SoABVHTree* dt = mgr.CreateDeviceTree(n);
    if (use64) {
        unsigned long long int *k = nullptr, *ko = nullptr;
        cudaMalloc(&k, n * sizeof(unsigned long long int));
        cudaMalloc(&ko, n * sizeof(unsigned long long int));
        DeviceGenerateMortonCodes(n, sw.DeviceScene(), bmn, bmx, k, route);
        DeviceSort(n, &k, &ko, &route, &route_out);
        DeviceBuildTree(n, ko, dind, dt, route_out);
        cudaFree(k);
        cudaFree(ko);
    } else {
        unsigned int *k = nullptr, *ko = nullptr;
        cudaMalloc(&k, n * sizeof(unsigned int));
        cudaMalloc(&ko, n * sizeof(unsigned int));
        DeviceGenerateMortonCodes(n, sw.DeviceScene(), bmn, bmx, k, route);
        DeviceSort(n, &k, &ko, &route, &route_out);
        DeviceBuildTree(n, ko, dind, dt, route_out);
        cudaFree(k);
        cudaFree(ko);
    }
    cudaMemset(counters, 0xFF, (n - 1) * sizeof(unsigned int));
    DeviceCalculateInternalNodeBoundingBoxes(n, dt, counters, bmn, bmx, route_out);
    BVHTree* ht = mgr.DeviceToHostTree(dt);
    for (size_t i = 0; i < 2 * (size_t)n - 1; ++i) {
        if (parent) parent[i] = ht->ParentIndex((int)i);
        if (left) left[i] = ht->LeftIndex((int)i);
        if (right) right[i] = ht->RightIndex((int)i);
        if (data) data[i] = ht->DataIndex((int)i);
        if (bmin4) {
            const float4 b = ht->BoundingBoxMin((int)i);
            std::memcpy(bmin4 + 4 * i, &b, 16);
        }
        if (bmax4) {
            const float4 b = ht->BoundingBoxMax((int)i);
            std::memcpy(bmax4 + 4 * i, &b, 16);
        }
        if (area) area[i] = ht->Area((int)i);
    }
    delete ht;
    mgr.FreeDeviceTree(dt);
    cudaFree(bmn);
    cudaFree(bmx);
    cudaFree(route);
    cudaFree(route_out);
    cudaFree(dind);
    cudaFree(counters);
    return 0;
}

// Commons.cuh:481-510 and 606-662 on a point of the unit cube.
unsigned int ref_host_morton30_point(float x, float y, float z) { return calculateMortonCode(float3{x, y, z}); }
unsigned long long int ref_host_morton63_point(float x, float y, float z) {
    return calculateMortonCode64(float3{x, y, z});
}
unsigned int ref_host_expand_bits(unsigned int v) { return expandBits(v); }

// Commons.cuh:99-135 (float3, float4 and array overloads) and 156-194.
float ref_host_box_area3(const float* mn, const float* mx) { return calculateBoundingBoxSurfaceArea(f3(mn), f3(mx)); }
float ref_host_box_area4(const float* mn, const float* mx) { return calculateBoundingBoxSurfaceArea(f4(mn), f4(mx)); }
float ref_host_box_area_arr(const float* mn, const float* mx) { return calculateBoundingBoxSurfaceArea(mn, mx); }
float ref_host_union_area4(const float* mn1, const float* mx1, const float* mn2, const float* mx2) {
    return calculateBoundingBoxAndSurfaceArea(f4(mn1), f4(mx1), f4(mn2), f4(mx2));
}
float ref_host_union_area3(const float* mn1, const float* mx1, const float* mn2, const float* mx2) {
    return calculateBoundingBoxAndSurfaceArea(f3(mn1), f3(mx1), f3(mn2), f3(mx2));
}

// SoABVHTree::SAH (SoABVHTree.cpp:50-74) of a tree given by its area array;
// the root is node 0.
float ref_host_sah(unsigned int n, const float* area, float ci, float ct) {
    BVHTreeInstanceManager mgr;
    BVHTree* dt = mgr.CreateDeviceTree(n);
    for (size_t i = 0; i < 2 * (size_t)n - 1; ++i) dt->SetArea((int)i, area[i]);
    dt->SetRootIndex(0);
    BVHTree* ht = mgr.DeviceToHostTree(dt);
    const float s = ht->SAH(ci, ct);
    delete ht;
    mgr.FreeDeviceTree(dt);
    return s;
}

}  // extern "C"
