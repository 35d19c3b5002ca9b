// Box refit that allocates no device memory.
//
// atr_refit takes its per-node arrival counters from the stream-ordered pool.
// Some callers cannot allocate on the device at the point where they refit:
// a frame loop or a serving path that runs under a fixed memory budget with
// every buffer reserved up front, code that must not touch the allocator
// while another component owns the device's memory, or host code that may
// only enqueue work on a stream it was handed.  This entry point serves them:
// the caller passes the tree arrays (device pointers) and a stream, and the
// counters live in one file-scope __device__ array of fixed size.
//
// Limits and sharing:
//   * meshes of at most kNoAllocMaxTriangles triangles (the array holds one
//     counter per internal node); larger meshes are rejected with an error;
//   * the array exists once per device that loads this library and stays
//     allocated until the process exits;
//   * every call on a device uses the same array: each call clears the
//     counters it needs before its kernel runs, and two calls whose work
//     overlaps on the GPU (different streams, no ordering between them) race
//     on the array and give wrong boxes.  Serialise calls on one stream or
//     order them with events.
//   * every call made outside stream capture looks up the array's device
//     address (cudaGetSymbolAddress, a host-side lookup that allocates
//     nothing) with the caller's device current, so a device reset, which
//     reloads the module and can move the array, never leaves a stale
//     address behind.  A call made while its stream is being captured uses
//     the address the last uncaptured call on that device found; make one
//     uncaptured call on a device (after any reset) before capturing.

#include <mutex>

#include "common.cuh"
#include "internal.h"

namespace atr {
namespace {

constexpr uint32_t kNoAllocMaxTriangles = 1u << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint32_t g_refit_counters[kNoAllocMaxTriangles - 1];

std::mutex g_addr_mutex;
uint32_t* g_addr[kMaxDevices] = {};

// Device address of g_refit_counters on the current device.  Outside stream
// capture it is looked up afresh (the module, and with it the array, moves
// when the device's primary context is reset and recreated); inside a capture
// the address from the last uncaptured call on this device is used.
int counters_address(cudaStream_t s, uint32_t** out) {
    int dev = 0;
    ATR_CUDA(cudaGetDevice(&dev));
    ATR_REQUIRE(dev >= 0 && dev < kMaxDevices, ATR_ERR_NO_DEVICE, "atr_refit_noalloc: device %d", dev);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    ATR_CUDA(cudaStreamIsCapturing(s, &cap));
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (cap == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_refit_counters);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_refit_counters)", __FILE__, __LINE__);
        g_addr[dev] = static_cast<uint32_t*>(p);
    }
    ATR_REQUIRE(g_addr[dev] != nullptr, ATR_ERR_INVALID_ARG,
                "atr_refit_noalloc: first call on device %d made during stream capture; make one call outside "
                "capture first", dev);
    *out = g_addr[dev];
    return ATR_OK;
}

// Same computation as k_refit in lbvh.cu: leaf boxes from the triangle's three
// vertices, then one thread climbs while it is the second child to arrive.
__global__ void __launch_bounds__(256) k_refit_noalloc(const float4* __restrict__ verts, uint32_t n,
                                                        const int32_t* __restrict__ parent,
                                                        const int32_t* __restrict__ left,
                                                        const int32_t* __restrict__ right,
                                                        const int32_t* __restrict__ data,
                                                        float4* __restrict__ bmin, float4* __restrict__ bmax,
                                                        float* __restrict__ area, uint32_t* __restrict__ counters) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int leaf = (int)i + (int)n - 1;
    const uint32_t tri = (uint32_t)data[leaf];
    const float4 a = __ldg(verts + 3 * (size_t)tri), b = __ldg(verts + 3 * (size_t)tri + 1),
                 c = __ldg(verts + 3 * (size_t)tri + 2);
    float4 mn = make_float4(fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z), 0.0f);
    float4 mx = make_float4(fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z), 0.0f);
    bmin[leaf] = mn;
    bmax[leaf] = mx;
    area[leaf] = box_area(mn, mx);
    int cur = parent[leaf];
    while (cur >= 0) {
        __threadfence();
        if (atomicAdd(&counters[cur], 1u) == 0u) return;
        __threadfence();
        const int l = left[cur], r = right[cur];
        const float4 lm = ld_cg(bmin + l), lx = ld_cg(bmax + l), rm = ld_cg(bmin + r), rx = ld_cg(bmax + r);
        mn = make_float4(fminf(lm.x, rm.x), fminf(lm.y, rm.y), fminf(lm.z, rm.z), 0.0f);
        mx = make_float4(fmaxf(lx.x, rx.x), fmaxf(lx.y, rx.y), fmaxf(lx.z, rx.z), 0.0f);
        bmin[cur] = mn;
        bmax[cur] = mx;
        area[cur] = box_area(mn, mx);
        cur = parent[cur];
    }
}

}  // namespace
}  // namespace atr

using namespace atr;

extern "C" int atr_refit_noalloc(void* stream, uint32_t num_triangles, const float* vertices, const int32_t* parent,
                                 const int32_t* left, const int32_t* right, const int32_t* data, float* bbox_min,
                                 float* bbox_max, float* area) {
    ATR_REQUIRE(vertices && parent && left && right && data && bbox_min && bbox_max && area, ATR_ERR_INVALID_ARG,
                "atr_refit_noalloc: NULL argument");
    ATR_REQUIRE(num_triangles >= 2, ATR_ERR_INVALID_ARG, "atr_refit_noalloc: %u triangles (need at least 2)",
                num_triangles);
    ATR_REQUIRE(num_triangles <= kNoAllocMaxTriangles, ATR_ERR_INVALID_ARG,
                "atr_refit_noalloc: %u triangles exceed the fixed maximum of %u; use atr_refit", num_triangles,
                kNoAllocMaxTriangles);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* counters = nullptr;
    ATR_TRY(counters_address(s, &counters));
    ATR_CUDA(cudaMemsetAsync(counters, 0, (size_t)(num_triangles - 1) * 4, s));
    k_refit_noalloc<<<(num_triangles + 255) / 256, 256, 0, s>>>(
        reinterpret_cast<const float4*>(vertices), num_triangles, parent, left, right, data,
        reinterpret_cast<float4*>(bbox_min), reinterpret_cast<float4*>(bbox_max), area, counters);
    ATR_CUDA(cudaGetLastError());
    return ATR_OK;
}
