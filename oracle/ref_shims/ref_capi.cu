// ORACLE -- test infrastructure only.
//
// A C entry point over the reference's own BVHRT-Core classes, compiled from
// the reference sources by oracle/build.py into oracle/_ref/.  It follows the
// call sequence of gpu-ray-traversal/src/rt/cuda/Renderer.cpp:164-228:
// SceneWrapper -> LBVHBuilder::BuildTree -> (TRBVHOptimizer |
// AgglomerativeTreeletOptimizer)::Optimize -> BVHTreeCollapser::Collapse ->
// BVHTreeInstanceManager::DeviceToHost*Tree, and copies the arrays out.

#include <chrono>
#include <cstring>
#include <iostream>
#include <sstream>

#include "AgglomerativeTreeletOptimizer.h"
#include "BVHCollapsedTree.h"
#include "BVHTreeCollapser.h"
#include "BVHTreeInstanceManager.h"
#include "LBVHBuilder.h"
#include "SceneWrapper.h"
#include "TRBVHOptimizer.h"

using namespace BVHRT;

namespace {
double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

extern "C" {

// optimizer: 0 none, 1 ATRBVH, 2 TRBVH.  Tree outputs (2n-1 entries, boxes as
// float4) and collapsed outputs may be NULL.  times_ms[0..2] = build,
// optimize, collapse wall times (device synchronised).  Returns 0 on success.
int ref_run(const float* vertices, unsigned int n, const float* bbmin, const float* bbmax, int use64,
            int optimizer, int treelet, int iterations, int collapse, int quiet, int* parent, int* left,
            int* right, int* data, float* bmin4, float* bmax4, float* area, int* c_parent, int* c_left,
            int* c_right, int* c_data, int* c_count, float* c_bmin4, float* c_bmax4, int* c_tri,
            float* collapse_sah, double* times_ms) {
    std::ostringstream sink;
    std::streambuf* old = nullptr;
    if (quiet) old = std::cout.rdbuf(sink.rdbuf());
    float4* v = new float4[3 * (size_t)n];
    std::memcpy(v, vertices, sizeof(float4) * 3 * (size_t)n);
    float3 mn = make_float3(bbmin[0], bbmin[1], bbmin[2]);
    float3 mx = make_float3(bbmax[0], bbmax[1], bbmax[2]);
    SceneWrapper* sw = new SceneWrapper(n, v, mn, mx);  // takes ownership of v
    cudaDeviceSynchronize();
    double t0 = now_ms();
    LBVHBuilder builder(use64 != 0);
    BVHTree* dt = builder.BuildTree(sw);
    cudaDeviceSynchronize();
    double t1 = now_ms();
    if (optimizer == 1) {
        AgglomerativeTreeletOptimizer opt(treelet, iterations);
        opt.Optimize(dt);
    } else if (optimizer == 2) {
        TRBVHOptimizer opt(treelet, iterations);
        opt.Optimize(dt);
    }
    cudaDeviceSynchronize();
    double t2 = now_ms();
    BVHTreeInstanceManager mgr;
    BVHTree* ht = mgr.DeviceToHostTree(dt);
    const size_t nn = 2 * (size_t)n - 1;
    for (size_t i = 0; i < nn; ++i) {
        if (parent) parent[i] = ht->ParentIndex((int)i);
        if (left) left[i] = ht->LeftIndex((int)i);
        if (right) right[i] = ht->RightIndex((int)i);
        if (data) data[i] = ht->DataIndex((int)i);
        if (bmin4) { float4 b = ht->BoundingBoxMin((int)i); std::memcpy(bmin4 + 4 * i, &b, 16); }
        if (bmax4) { float4 b = ht->BoundingBoxMax((int)i); std::memcpy(bmax4 + 4 * i, &b, 16); }
        if (area) area[i] = ht->Area((int)i);
    }
    delete ht;
    double t3 = t2;
    if (collapse) {
        float sah = 0.0f;
        BVHTreeCollapser collapser;
        double tc0 = now_ms();
        BVHCollapsedTree* dc = collapser.Collapse(dt, &sah);
        cudaDeviceSynchronize();
        t3 = now_ms() - tc0 + t2;
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
    if (times_ms) { times_ms[0] = t1 - t0; times_ms[1] = t2 - t1; times_ms[2] = t3 - t2; }
    if (old) std::cout.rdbuf(old);
    cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : (int)e;
}

}  // extern "C"
