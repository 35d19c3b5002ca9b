// bvhrt.hpp -- the reference's BVHRT-Core builder classes over the C ABI.
//
// Same class names, constructor defaults and call sequence as
// leonardo-domingues/atrbvh BVHRT-Core/src (SceneWrapper.h, LBVHBuilder.h,
// AgglomerativeTreeletOptimizer.h, TRBVHOptimizer.h, BVHTreeCollapser.h,
// BVHTreeInstanceManager.h, SoABVHTree.h, BVHCollapsedTree.h), so that the
// reference's caller (gpu-ray-traversal/src/rt/cuda/Renderer.cpp:164-228)
// compiles against it unchanged.  Differences: failures throw
// BVHRT::Error (the reference prints and exit()s), and device trees are
// opaque handles (the reference hands out a device pointer to a device-side
// struct of device pointers).  All calls of a thread share one context on
// the current CUDA device.
#pragma once

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "atrbvh.h"

#if defined(__has_include)
#if __has_include(<vector_types.h>)
#include <vector_types.h>
#define BVHRT_HAVE_VECTOR_TYPES 1
#endif
#endif

namespace BVHRT {

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& what) : std::runtime_error(what), status(s) {}
};

inline void check(int status) {
    if (status != ATR_OK) throw Error(status, atr_last_error());
}

// One context (stream + scratch pool) per host thread.
inline atr_ctx* context() {
    struct Holder {
        atr_ctx* ctx = nullptr;
        ~Holder() { if (ctx) atr_ctx_destroy(ctx); }
    };
    thread_local Holder h;
    if (!h.ctx) check(atr_ctx_create(0, nullptr, &h.ctx));
    return h.ctx;
}

#ifdef BVHRT_HAVE_VECTOR_TYPES
using ::float3;
using ::float4;
#else
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
#endif

struct Scene {
    unsigned int numberOfTriangles;
    float4* vertices;
    float3 boundingBoxMin;
    float3 boundingBoxMax;
};

// BVHRT::SceneWrapper: takes ownership of the host vertex array (delete[] in
// the destructor, SceneWrapper.cpp:35) and keeps a device copy.
class SceneWrapper {
public:
    SceneWrapper(unsigned int numberOfTriangles, float4* vertices, float3 boundingBoxMin, float3 boundingBoxMax) {
        host_.numberOfTriangles = numberOfTriangles;
        host_.vertices = vertices;
        host_.boundingBoxMin = boundingBoxMin;
        host_.boundingBoxMax = boundingBoxMax;
        const float mn[3] = {boundingBoxMin.x, boundingBoxMin.y, boundingBoxMin.z};
        const float mx[3] = {boundingBoxMax.x, boundingBoxMax.y, boundingBoxMax.z};
        check(atr_scene_create(context(), reinterpret_cast<const float*>(vertices), numberOfTriangles, mn, mx, 0,
                               &scene_));
    }
    ~SceneWrapper() {
        atr_scene_destroy(scene_);
        delete[] host_.vertices;
    }
    SceneWrapper(const SceneWrapper&) = delete;
    SceneWrapper& operator=(const SceneWrapper&) = delete;
    const Scene* HostScene() const { return &host_; }
    atr_scene* handle() const { return scene_; }

private:
    Scene host_{};
    atr_scene* scene_ = nullptr;
};

// Device tree handle (the reference's BVHTree* device pointer).
class BVHTree {
public:
    explicit BVHTree(atr_tree* t) : t_(t) {}
    ~BVHTree() { atr_tree_destroy(t_); }
    atr_tree* handle() const { return t_; }
    unsigned int NumberOfTriangles() const {
        atr_tree_view v;
        check(atr_tree_view_get(t_, &v));
        return v.num_triangles;
    }

private:
    atr_tree* t_;
};

// Host copy of a tree: SoABVHTree's accessors (SoABVHTree.h:53-273).
class SoABVHTree {
public:
    explicit SoABVHTree(unsigned int n) : n_(n), parent_(2 * n - 1), left_(2 * n - 1), right_(2 * n - 1),
                                          data_(2 * n - 1), bmin_(2 * n - 1), bmax_(2 * n - 1), area_(2 * n - 1) {}
    int RootIndex() const { return 0; }
    int ParentIndex(int i) const { return parent_[i]; }
    int LeftIndex(int i) const { return left_[i]; }
    int RightIndex(int i) const { return right_[i]; }
    int DataIndex(int i) const { return data_[i]; }
    float4 BoundingBoxMin(int i) const { return bmin_[i]; }
    float4 BoundingBoxMax(int i) const { return bmax_[i]; }
    float Area(int i) const { return area_[i]; }
    unsigned int NumberOfTriangles() const { return n_; }
    // SoABVHTree::SAH (SoABVHTree.cpp:50-74): sequential float sums.
    float SAH(float nodeTraversalCost = 1.2f, float triangleIntersectionCost = 1.0f) const {
        const float total = area_[0];
        float si = total, sl = 0.0f;
        for (unsigned int i = 1; i < n_ - 1; ++i) si += area_[i];
        for (unsigned int i = n_ - 1; i < 2 * n_ - 1; ++i) sl += area_[i];
        return (nodeTraversalCost * si + triangleIntersectionCost * sl) / total;
    }

private:
    friend class BVHTreeInstanceManager;
    unsigned int n_;
    std::vector<int32_t> parent_, left_, right_, data_;
    std::vector<float4> bmin_, bmax_;
    std::vector<float> area_;
};

// BVHCollapsedTree (BVHCollapsedTree.h:9-58) as a host copy.
struct BVHCollapsedNodes {
    int* parentIndices;
    int* leftIndices;
    int* rightIndices;
    int* dataIndices;
    int* triangleCount;
    float4* boundingBoxMin;
    float4* boundingBoxMax;
};

class BVHCollapsedTree {
public:
    int* triangleIndices = nullptr;
    BVHCollapsedNodes nodes{};
    int rootIndex = 0;
    explicit BVHCollapsedTree(atr_collapsed* c) : c_(c) {}
    ~BVHCollapsedTree() { if (c_) atr_collapsed_destroy(c_); }
    atr_collapsed* handle() const { return c_; }

private:
    friend class BVHTreeInstanceManager;
    atr_collapsed* c_ = nullptr;
    std::vector<int32_t> p_, l_, r_, d_, cnt_, tri_;
    std::vector<float4> mn_, mx_;
};

class BVHBuilder {
public:
    virtual ~BVHBuilder() = default;
    virtual BVHTree* BuildTree(const SceneWrapper* sceneWrapper) = 0;
};

class BVHOptimizer {
public:
    virtual ~BVHOptimizer() = default;
    virtual void Optimize(BVHTree* deviceTree) = 0;
};

class LBVHBuilder : public BVHBuilder {
public:
    explicit LBVHBuilder(bool use64BitMortonCodes = false) : bits_(use64BitMortonCodes ? 63 : 30) {}
    BVHTree* BuildTree(const SceneWrapper* sceneWrapper) override {
        atr_tree* t = nullptr;
        check(atr_build_lbvh(context(), sceneWrapper->handle(), bits_, &t));
        return new BVHTree(t);
    }

private:
    int bits_;
};

class AgglomerativeTreeletOptimizer : public BVHOptimizer {
public:
    explicit AgglomerativeTreeletOptimizer(int treeletSize = 9, int iterations = 2)
        : treeletSize_(treeletSize), iterations_(iterations) {}
    void Optimize(BVHTree* deviceTree) override {
        check(atr_optimize_atrbvh(context(), deviceTree->handle(), treeletSize_, iterations_, 1.2f, 1.0f));
    }

private:
    int treeletSize_, iterations_;
};

class TRBVHOptimizer : public BVHOptimizer {
public:
    explicit TRBVHOptimizer(int treeletSize = 7, int iterations = 3)
        : treeletSize_(treeletSize), iterations_(iterations) {}
    void Optimize(BVHTree* deviceTree) override {
        check(atr_optimize_trbvh(context(), deviceTree->handle(), treeletSize_, iterations_, 1.2f, 1.0f));
    }

private:
    int treeletSize_, iterations_;
};

class BVHTreeCollapser {
public:
    BVHCollapsedTree* Collapse(BVHTree* deviceTree, float* sah, float ci = 1.2f, float ct = 1.0f) {
        atr_collapsed* c = nullptr;
        check(atr_collapse(context(), deviceTree->handle(), ci, ct, 0, &c, sah));
        return new BVHCollapsedTree(c);
    }
};

class BVHTreeInstanceManager {
public:
    SoABVHTree* DeviceToHostTree(const BVHTree* deviceTree) const {
        auto* h = new SoABVHTree(deviceTree->NumberOfTriangles());
        check(atr_tree_download(context(), deviceTree->handle(), h->parent_.data(), h->left_.data(),
                                h->right_.data(), h->data_.data(), reinterpret_cast<float*>(h->bmin_.data()),
                                reinterpret_cast<float*>(h->bmax_.data()), h->area_.data()));
        return h;
    }
    void FreeDeviceTree(BVHTree* deviceTree) const { delete deviceTree; }
    BVHCollapsedTree* DeviceToHostCollapsedTree(const BVHCollapsedTree* deviceTree) const {
        atr_collapsed_view v;
        check(atr_collapsed_view_get(deviceTree->handle(), &v));
        const size_t nn = 2 * (size_t)v.num_triangles - 1;
        auto* h = new BVHCollapsedTree(nullptr);
        h->p_.resize(nn); h->l_.resize(nn); h->r_.resize(nn); h->d_.resize(nn); h->cnt_.resize(nn);
        h->mn_.resize(nn); h->mx_.resize(nn); h->tri_.resize(v.num_triangles);
        check(atr_collapsed_download(context(), deviceTree->handle(), h->p_.data(), h->l_.data(), h->r_.data(),
                                     h->d_.data(), h->cnt_.data(), reinterpret_cast<float*>(h->mn_.data()),
                                     reinterpret_cast<float*>(h->mx_.data()), h->tri_.data()));
        h->nodes = {h->p_.data(), h->l_.data(), h->r_.data(), h->d_.data(), h->cnt_.data(), h->mn_.data(),
                    h->mx_.data()};
        h->triangleIndices = h->tri_.data();
        h->rootIndex = 0;
        return h;
    }
    void FreeDeviceCollapsedTree(BVHCollapsedTree* deviceTree) const { delete deviceTree; }
};

}  // namespace BVHRT
