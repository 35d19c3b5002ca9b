// Context, scene and tree objects; error reporting; host-side views.

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "internal.h"

namespace atr {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    set_error("%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    if (e == cudaErrorMemoryAllocation) return ATR_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return ATR_ERR_NO_DEVICE;
    return ATR_ERR_CUDA;
}

int tree_alloc(atr_ctx* ctx, uint32_t n, atr_tree** out) {
    const size_t nn = 2 * (size_t)n - 1;
    const size_t b4 = align256(nn * 4), b16 = align256(nn * 16), b8 = align256((size_t)(n - 1) * 8);
    atr_tree* t = new atr_tree();
    t->ctx = ctx;
    t->n = n;
    int s = ctx->alloc(&t->block, 5 * b4 + 2 * b16 + b8);
    if (s != ATR_OK) { delete t; return s; }
    char* p = static_cast<char*>(t->block);
    t->parent = reinterpret_cast<int32_t*>(p); p += b4;
    t->left = reinterpret_cast<int32_t*>(p); p += b4;
    t->right = reinterpret_cast<int32_t*>(p); p += b4;
    t->data = reinterpret_cast<int32_t*>(p); p += b4;
    t->area = reinterpret_cast<float*>(p); p += b4;
    t->bmin = reinterpret_cast<float4*>(p); p += b16;
    t->bmax = reinterpret_cast<float4*>(p); p += b16;
    t->range = reinterpret_cast<int2*>(p);
    *out = t;
    return ATR_OK;
}

}  // namespace atr

int atr_ctx::alloc(void** p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) return ATR_OK;
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, pool, stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        return atr::cuda_fail(e, "cudaMallocAsync", __FILE__, __LINE__);
    }
    return ATR_OK;
}

void atr_ctx::release(void* p) {
    if (p) cudaFreeAsync(p, stream);
}

void atr_ctx::phase_begin(const char* name) {
    if (!timing) return;
    Phase ph;
    ph.name = name;
    cudaEventCreate(&ph.a);
    cudaEventCreate(&ph.b);
    if (capture_marks) cudaEventRecordWithFlags(ph.a, stream, cudaEventRecordExternal);
    else cudaEventRecord(ph.a, stream);
    phases.push_back(ph);
}

void atr_ctx::phase_end() {
    if (!timing || phases.empty()) return;
    if (capture_marks) cudaEventRecordWithFlags(phases.back().b, stream, cudaEventRecordExternal);
    else cudaEventRecord(phases.back().b, stream);
}

extern "C" {

const char* atr_last_error(void) { return atr::g_err; }
const char* atr_version(void) { return "atrbvh-b200 0.1 (sm_100a)"; }

int atr_ctx_create(int device, void* stream, atr_ctx** out) {
    ATR_REQUIRE(out, ATR_ERR_INVALID_ARG, "atr_ctx_create: out is NULL");
    *out = nullptr;
    int count = 0;
    ATR_CUDA(cudaGetDeviceCount(&count));
    ATR_REQUIRE(device >= 0 && device < count, ATR_ERR_NO_DEVICE, "atr_ctx_create: device %d of %d", device, count);
    ATR_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    ATR_CUDA(cudaGetDeviceProperties(&prop, device));
    ATR_REQUIRE(prop.major == 10 && prop.minor == 0, ATR_ERR_NO_DEVICE,
                "atr_ctx_create: device %d is sm_%d%d, this build targets sm_100a", device, prop.major,
                prop.minor);
    atr_ctx* c = new atr_ctx();
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    if (stream) {
        c->stream = static_cast<cudaStream_t>(stream);
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { delete c; return atr::cuda_fail(e, "cudaStreamCreate", __FILE__, __LINE__); }
        c->own_stream = true;
    }
    // The context's own stream-ordered pool; freed memory stays cached in it
    // for the next build.
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaError_t e = cudaMemPoolCreate(&c->pool, &props);
    if (e == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        e = cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    if (e != cudaSuccess) {
        if (c->pool) cudaMemPoolDestroy(c->pool);
        if (c->own_stream) cudaStreamDestroy(c->stream);
        delete c;
        return atr::cuda_fail(e, "cudaMemPoolCreate", __FILE__, __LINE__);
    }
    e = cudaMalloc(&c->d_error, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(c->d_error, 0, sizeof(uint32_t));
    if (e == cudaSuccess && atr::lbvh_prepare() != ATR_OK) e = cudaErrorInvalidValue;
    if (e == cudaSuccess && atr::atrbvh_prepare() != ATR_OK) e = cudaErrorInvalidValue;
    if (e != cudaSuccess) {
        cudaMemPoolDestroy(c->pool);
        if (c->own_stream) cudaStreamDestroy(c->stream);
        delete c;
        return atr::cuda_fail(e, "cudaMalloc(error word)", __FILE__, __LINE__);
    }
    *out = c;
    return ATR_OK;
}

int atr_ctx_destroy(atr_ctx* ctx) {
    if (!ctx) return ATR_OK;
    cudaStreamSynchronize(ctx->stream);
    for (auto& p : ctx->phases) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    cudaFree(ctx->d_error);
    // Memory still allocated from the pool (objects the caller has not yet
    // destroyed) stays valid; the pool goes once the last of it is freed.
    cudaMemPoolDestroy(ctx->pool);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return ATR_OK;
}

int atr_ctx_synchronize(atr_ctx* ctx) {
    ATR_REQUIRE(ctx, ATR_ERR_INVALID_ARG, "atr_ctx_synchronize: ctx is NULL");
    ATR_CUDA(cudaStreamSynchronize(ctx->stream));
    uint32_t err = 0;
    ATR_CUDA(cudaMemcpy(&err, ctx->d_error, sizeof(err), cudaMemcpyDeviceToHost));
    if (err) {
        cudaMemset(ctx->d_error, 0, sizeof(uint32_t));
        atr::set_error("device-side bounded wait gave up (error bits 0x%x)", err);
        return ATR_ERR_DEVICE_WAIT;
    }
    return ATR_OK;
}

int atr_ctx_launch_count(atr_ctx* ctx, uint64_t* count) {
    ATR_REQUIRE(ctx && count, ATR_ERR_INVALID_ARG, "atr_ctx_launch_count: NULL argument");
    *count = ctx->launches;
    return ATR_OK;
}

int atr_ctx_get_stream(atr_ctx* ctx, void** stream) {
    ATR_REQUIRE(ctx && stream, ATR_ERR_INVALID_ARG, "atr_ctx_get_stream: NULL argument");
    *stream = ctx->stream;
    return ATR_OK;
}

int atr_ctx_set_tuning(atr_ctx* ctx, int knob, int value) {
    ATR_REQUIRE(ctx, ATR_ERR_INVALID_ARG, "atr_ctx_set_tuning: ctx is NULL");
    switch (knob) {
        case ATR_TUNE_ATR_WARPS:
            ATR_REQUIRE(value == 2 || value == 4 || value == 8, ATR_ERR_INVALID_ARG,
                        "atr_ctx_set_tuning: ATRBVH warps per block %d (2, 4 or 8)", value);
            ctx->atr_warps = value;
            return ATR_OK;
        case ATR_TUNE_ATR_GROUP_MIN:
            ATR_REQUIRE(value >= 2 && value <= 33, ATR_ERR_INVALID_ARG,
                        "atr_ctx_set_tuning: group threshold %d outside [2, 33]", value);
            ctx->atr_group_min = value;
            return ATR_OK;
        case ATR_TUNE_SORT_BITS:
            ATR_REQUIRE(value == 8 || value == 10, ATR_ERR_INVALID_ARG,
                        "atr_ctx_set_tuning: sort digit width %d (8 or 10)", value);
            ctx->sort_bits = value;
            return ATR_OK;
        case ATR_TUNE_ATR_LEVELS:
            ATR_REQUIRE(value >= 0 && value <= 64, ATR_ERR_INVALID_ARG,
                        "atr_ctx_set_tuning: level passes %d outside [0, 64]", value);
            ctx->atr_levels = value;
            return ATR_OK;
        case ATR_TUNE_QUAD_MIN:
            ATR_REQUIRE(value >= -1, ATR_ERR_INVALID_ARG, "atr_ctx_set_tuning: quad threshold %d below -1", value);
            ctx->atr_quad_min = value;
            return ATR_OK;
        case ATR_TUNE_WARP_MAX:
            ATR_REQUIRE(value >= 0, ATR_ERR_INVALID_ARG, "atr_ctx_set_tuning: whole-warp threshold %d below 0", value);
            ctx->atr_warp_max = value;
            return ATR_OK;
        default:
            break;
    }
    ATR_REQUIRE(false, ATR_ERR_INVALID_ARG, "atr_ctx_set_tuning: unknown knob %d", knob);
}

int atr_ctx_get_tuning(atr_ctx* ctx, int knob, int* value) {
    ATR_REQUIRE(ctx && value, ATR_ERR_INVALID_ARG, "atr_ctx_get_tuning: NULL argument");
    switch (knob) {
        case ATR_TUNE_ATR_WARPS: *value = ctx->atr_warps; return ATR_OK;
        case ATR_TUNE_ATR_GROUP_MIN: *value = ctx->atr_group_min; return ATR_OK;
        case ATR_TUNE_SORT_BITS: *value = ctx->sort_bits; return ATR_OK;
        case ATR_TUNE_ATR_LEVELS: *value = ctx->atr_levels; return ATR_OK;
        case ATR_TUNE_QUAD_MIN: *value = ctx->atr_quad_min; return ATR_OK;
        case ATR_TUNE_WARP_MAX: *value = ctx->atr_warp_max; return ATR_OK;
        default: break;
    }
    ATR_REQUIRE(false, ATR_ERR_INVALID_ARG, "atr_ctx_get_tuning: unknown knob %d", knob);
}

int atr_ctx_set_timing(atr_ctx* ctx, int enable) {
    ATR_REQUIRE(ctx, ATR_ERR_INVALID_ARG, "atr_ctx_set_timing: ctx is NULL");
    ATR_CUDA(cudaStreamSynchronize(ctx->stream));
    for (auto& p : ctx->phases) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    ctx->phases.clear();
    ctx->timing = enable != 0;
    return ATR_OK;
}

int atr_ctx_phase_times(atr_ctx* ctx, float* ms, int capacity, int* count) {
    ATR_REQUIRE(ctx && count, ATR_ERR_INVALID_ARG, "atr_ctx_phase_times: NULL argument");
    ATR_CUDA(cudaStreamSynchronize(ctx->stream));
    int k = 0;
    ctx->phase_names.clear();
    for (auto& p : ctx->phases) {
        float t = 0.0f;
        ATR_CUDA(cudaEventElapsedTime(&t, p.a, p.b));
        if (ms && k < capacity) ms[k] = t;
        if (!ctx->phase_names.empty()) ctx->phase_names += ",";
        ctx->phase_names += p.name;
        ++k;
    }
    *count = k;
    for (auto& p : ctx->phases) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    ctx->phases.clear();
    return ATR_OK;
}

const char* atr_ctx_phase_names(atr_ctx* ctx) { return ctx ? ctx->phase_names.c_str() : ""; }

int atr_scene_destroy(atr_scene* s) {
    if (!s) return ATR_OK;
    s->ctx->release(s->verts);
    s->ctx->release(s->d_bounds);
    delete s;
    return ATR_OK;
}

int atr_scene_device_vertices(const atr_scene* s, float** vertices, uint32_t* n) {
    ATR_REQUIRE(s, ATR_ERR_INVALID_ARG, "atr_scene_device_vertices: scene is NULL");
    if (vertices) *vertices = reinterpret_cast<float*>(s->verts);
    if (n) *n = s->n;
    return ATR_OK;
}

int atr_scene_bounds(atr_ctx* ctx, const atr_scene* s, float* bmin, float* bmax) {
    ATR_REQUIRE(ctx && s && bmin && bmax, ATR_ERR_INVALID_ARG, "atr_scene_bounds: NULL argument");
    float h[6];
    ATR_CUDA(cudaMemcpyAsync(h, s->d_bounds, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    ATR_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < 3; ++k) { bmin[k] = h[k]; bmax[k] = h[3 + k]; }
    return ATR_OK;
}

int atr_tree_destroy(atr_tree* t) {
    if (!t) return ATR_OK;
    atr::refit_plan_free(t->ctx, t->refit_plan);
    t->ctx->release(t->block);
    t->ctx->release(t->prepass_block);
    t->ctx->release(t->sorted_keys);
    t->ctx->release(t->sorted_idx);
    delete t;
    return ATR_OK;
}

int atr_tree_view_get(const atr_tree* t, atr_tree_view* v) {
    ATR_REQUIRE(t && v, ATR_ERR_INVALID_ARG, "atr_tree_view_get: NULL argument");
    v->num_triangles = t->n;
    v->root = 0;
    v->parent = t->parent;
    v->left = t->left;
    v->right = t->right;
    v->data = t->data;
    v->bbox_min = reinterpret_cast<float*>(t->bmin);
    v->bbox_max = reinterpret_cast<float*>(t->bmax);
    v->area = t->area;
    return ATR_OK;
}

int atr_tree_download(atr_ctx* ctx, const atr_tree* t, int32_t* parent, int32_t* left, int32_t* right,
                      int32_t* data, float* bmin, float* bmax, float* area) {
    ATR_REQUIRE(ctx && t, ATR_ERR_INVALID_ARG, "atr_tree_download: NULL argument");
    const size_t nn = 2 * (size_t)t->n - 1;
    cudaStream_t s = ctx->stream;
    if (parent) ATR_CUDA(cudaMemcpyAsync(parent, t->parent, nn * 4, cudaMemcpyDeviceToHost, s));
    if (left) ATR_CUDA(cudaMemcpyAsync(left, t->left, nn * 4, cudaMemcpyDeviceToHost, s));
    if (right) ATR_CUDA(cudaMemcpyAsync(right, t->right, nn * 4, cudaMemcpyDeviceToHost, s));
    if (data) ATR_CUDA(cudaMemcpyAsync(data, t->data, nn * 4, cudaMemcpyDeviceToHost, s));
    if (bmin) ATR_CUDA(cudaMemcpyAsync(bmin, t->bmin, nn * 16, cudaMemcpyDeviceToHost, s));
    if (bmax) ATR_CUDA(cudaMemcpyAsync(bmax, t->bmax, nn * 16, cudaMemcpyDeviceToHost, s));
    if (area) ATR_CUDA(cudaMemcpyAsync(area, t->area, nn * 4, cudaMemcpyDeviceToHost, s));
    return atr_ctx_synchronize(ctx);
}

int atr_tree_sah(atr_ctx* ctx, const atr_tree* t, float ci, float ct, float* sah) {
    ATR_REQUIRE(ctx && t && sah, ATR_ERR_INVALID_ARG, "atr_tree_sah: NULL argument");
    const uint32_t n = t->n;
    std::vector<float> area(2 * (size_t)n - 1);
    ATR_CUDA(cudaMemcpyAsync(area.data(), t->area, area.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
    ATR_TRY(atr_ctx_synchronize(ctx));
    // SoABVHTree::SAH: root area first, then internal nodes in index order, then leaves.
    const float total = area[0];
    float si = total, sl = 0.0f;
    for (uint32_t i = 1; i < n - 1; ++i) si += area[i];
    for (size_t i = n - 1; i < area.size(); ++i) sl += area[i];
    *sah = (ci * si + ct * sl) / total;
    return ATR_OK;
}

int atr_tree_sorted_keys(atr_ctx* ctx, const atr_tree* t, uint64_t* keys, uint32_t* idx) {
    ATR_REQUIRE(ctx && t, ATR_ERR_INVALID_ARG, "atr_tree_sorted_keys: NULL argument");
    ATR_REQUIRE(t->sorted_keys && t->sorted_idx, ATR_ERR_INVALID_ARG,
                "atr_tree_sorted_keys: tree keeps no sort output");
    const uint32_t n = t->n;
    if (keys) {
        if (t->morton_bits == 30) {
            std::vector<uint32_t> k(n);
            ATR_CUDA(cudaMemcpyAsync(k.data(), t->sorted_keys, n * 4ull, cudaMemcpyDeviceToHost, ctx->stream));
            ATR_TRY(atr_ctx_synchronize(ctx));
            for (uint32_t i = 0; i < n; ++i) keys[i] = k[i];
        } else {
            ATR_CUDA(cudaMemcpyAsync(keys, t->sorted_keys, n * 8ull, cudaMemcpyDeviceToHost, ctx->stream));
        }
    }
    if (idx) ATR_CUDA(cudaMemcpyAsync(idx, t->sorted_idx, n * 4ull, cudaMemcpyDeviceToHost, ctx->stream));
    return atr_ctx_synchronize(ctx);
}

}  // extern "C"
