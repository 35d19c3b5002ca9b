// Serving loop: build/refit + trace requests with admission by device memory,
// resident BVHs, and continuous batching over several lanes.
//
// Each lane is a host thread with its own context (stream) and pinned staging
// buffers.  A lane that is free takes, under the queue lock, every waiting
// request that it can admit: builds up to the batch's triangle cap and refits
// of resident meshes that no other lane is using, as long as the estimated
// device memory of the taken work plus everything resident and in flight
// stays within the budget (idle resident batches are evicted oldest-use first
// when it would not).  It then runs, on its stream: one segmented build of all
// new meshes (sort, Karras build, ATRBVH, collapse, Compact2), the refits, and
// the traces of every taken request (one merged ray queue per batch), and
// copies the results back.  While one lane's batch is on the GPU the next
// arrivals are taken by another lane, so their work overlaps on the device.
//
// The build of a mesh does not depend on which other meshes share its batch
// (every stage of a segmented build works per mesh), so each result equals
// the result of the same request run alone.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Device bytes a build keeps per triangle (vertices 48, tree 104, collapsed
// tree 108, Compact2 upper bound 144) plus transient sort/treelet scratch.
constexpr uint64_t kBuildBytesPerTri = 460;
constexpr uint64_t kResidentBytesPerTri = 404;
constexpr uint64_t kRayBytes = 48;  // ray (32) + result (16)

struct BatchRec;

struct Request {
    uint64_t ticket = 0;
    atr_request req{};
    Clock::time_point t_submit, t_taken, t_done;
    bool done = false;
    bool waited = false;  // a thread is in atr_server_wait on this ticket
    int status = ATR_OK;
    float sah = 0.0f;
    uint32_t batch_requests = 0, lane = 0;
    uint64_t bytes = 0;  // admission estimate while in flight
    std::string error;
    std::shared_ptr<BatchRec> refit_rec;  // a refit: the resident batch it holds busy
    uint32_t refit_index = 0;             // and the mesh's index in it
    uint32_t refit_n = 0;                 // and its triangle count
};

struct BatchRec {
    atr_batch* batch = nullptr;
    uint64_t bytes = 0;
    uint32_t live = 0;   // resident meshes still referring to it
    uint32_t busy = 0;   // refits of its meshes in flight (on any lanes)
    uint64_t last_use = 0;
};

struct Resident {
    std::shared_ptr<BatchRec> rec;
    uint32_t index = 0;
    uint32_t n = 0;
    int busy_lane = -1;  // lane refitting this mesh, or -1
};

struct Lane {
    int id = 0;
    atr_ctx* ctx = nullptr;
    std::thread thread;
    // Pinned staging: vertices, rays, results.
    void* h_verts = nullptr;
    size_t h_verts_cap = 0;
    void* h_rays = nullptr;
    size_t h_rays_cap = 0;
    void* h_res = nullptr;
    size_t h_res_cap = 0;
    void* h_rverts = nullptr;  // refit vertices
    size_t h_rverts_cap = 0;
};

struct CopyJob {
    void* dst;
    const void* src;
    size_t bytes;
};

// Host copies between request buffers and pinned staging, cut into 4 MiB
// chunks spread over OpenMP threads: a lane batch moves hundreds of MB of
// vertices, rays and results, which one thread copies at a fraction of the
// host's memory bandwidth.
void par_copy(const std::vector<CopyJob>& jobs) {
    constexpr size_t kChunk = (size_t)4 << 20;
    std::vector<CopyJob> chunks;
    for (const CopyJob& j : jobs)
        for (size_t o = 0; o < j.bytes; o += kChunk)
            chunks.push_back({static_cast<char*>(j.dst) + o, static_cast<const char*>(j.src) + o,
                              std::min(kChunk, j.bytes - o)});
#pragma omp parallel for schedule(dynamic, 1) if (chunks.size() > 1)
    for (long i = 0; i < (long)chunks.size(); ++i) std::memcpy(chunks[i].dst, chunks[i].src, chunks[i].bytes);
}

int grow_pinned(void** p, size_t* cap, size_t need) {
    if (need <= *cap) return ATR_OK;
    // Grow by doubling: pinning host memory is slow, so reallocations must be rare.
    const size_t c = std::max({need, (size_t)1 << 20, 2 * *cap});
    if (*p) cudaFreeHost(*p);
    *p = nullptr;
    *cap = 0;
    ATR_CUDA(cudaHostAlloc(p, c, cudaHostAllocDefault));
    *cap = c;
    return ATR_OK;
}

// True for page-locked host memory (cudaHostAlloc'd or cudaHostRegister'ed):
// such request buffers are copied to and from the device directly, without
// the host staging copy.
bool is_pinned(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

struct atr_server {
    int device = 0;
    atr_server_config cfg{};
    uint8_t class_treelet[32] = {};
    uint8_t class_iters[32] = {};
    bool have_classes = false;

    std::mutex mu;
    std::condition_variable cv_work;  // lanes wait for requests / capacity
    std::condition_variable cv_done;  // waiters wait for completion
    std::deque<Request*> pending;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> tickets;
    std::unordered_map<uint64_t, Resident> resident;
    // Builds submitted but not finished, per mesh id kept resident: a refit
    // of that id waits for them.
    std::unordered_map<uint64_t, uint32_t> building;
    std::vector<std::shared_ptr<BatchRec>> batches;  // every live batch record
    uint64_t next_ticket = 1;
    uint64_t use_clock = 0;
    uint64_t inflight_bytes = 0;
    uint64_t resident_bytes = 0;
    bool stopping = false;
    std::vector<std::unique_ptr<Lane>> lanes;

    // Statistics.
    std::vector<double> latencies;
    atr_server_stats st{};
    uint32_t busy_lanes = 0;
    Clock::time_point busy_mark;
    double busy1_ms = 0, busy2_ms = 0;

    void account_busy(int delta) {  // caller holds mu
        const auto now = Clock::now();
        if (busy_lanes >= 1) busy1_ms += ms_between(busy_mark, now);
        if (busy_lanes >= 2) busy2_ms += ms_between(busy_mark, now);
        busy_mark = now;
        busy_lanes = (uint32_t)((int)busy_lanes + delta);
        st.max_lanes_busy = std::max(st.max_lanes_busy, busy_lanes);
    }

    void params_for(uint32_t n, uint8_t* ts, uint8_t* it) const {
        if (have_classes) {
            int c = 0;
            while ((2u << c) <= n && c < 31) ++c;  // floor(log2 n)
            *ts = class_treelet[c];
            *it = class_iters[c];
        } else {
            *ts = (uint8_t)cfg.treelet_size;
            *it = (uint8_t)cfg.iterations;
        }
    }

    // Drop one resident reference to rec; frees the batch when nothing refers
    // to it and no lane uses it.  Caller holds mu.
    void unref(const std::shared_ptr<BatchRec>& rec) {
        if (rec->live) --rec->live;
        maybe_free(rec);
    }
    void maybe_free(const std::shared_ptr<BatchRec>& rec) {
        if (rec->live || rec->busy || !rec->batch) return;
        atr_batch_destroy(rec->batch);
        rec->batch = nullptr;
        resident_bytes -= rec->bytes;
        batches.erase(std::remove(batches.begin(), batches.end(), rec), batches.end());
    }

    // Evict idle resident batches, oldest use first, that no waiting refit
    // needs, until `need` more bytes fit.  Caller holds mu.
    bool make_room(uint64_t need) {
        const uint64_t budget = cfg.hbm_budget_bytes;
        if (inflight_bytes + resident_bytes + need <= budget) return true;
        std::vector<std::shared_ptr<BatchRec>> idle;
        for (auto& b : batches)
            if (!b->busy && b->live) idle.push_back(b);
        std::sort(idle.begin(), idle.end(), [](auto& a, auto& b) { return a->last_use < b->last_use; });
        for (auto& b : idle) {
            bool wanted = false;
            for (Request* r : pending)
                if (r->req.kind == ATR_REQ_REFIT) {
                    auto it = resident.find(r->req.mesh_id);
                    if (it != resident.end() && it->second.rec == b) { wanted = true; break; }
                }
            if (wanted) continue;
            for (auto it = resident.begin(); it != resident.end();)
                if (it->second.rec == b) it = resident.erase(it); else ++it;
            b->live = 0;
            ++st.evictions;
            maybe_free(b);
            if (inflight_bytes + resident_bytes + need <= budget) return true;
        }
        return inflight_bytes + resident_bytes + need <= budget;
    }

    void finish(Request* r, int status, const char* msg) {  // caller holds mu
        if (r->req.kind == ATR_REQ_BUILD && r->req.keep_resident) {
            auto bld = building.find(r->req.mesh_id);
            if (bld != building.end() && --bld->second == 0) building.erase(bld);
        }
        r->status = status;
        if (msg) r->error = msg;
        r->t_done = Clock::now();
        r->done = true;
        if (status == ATR_OK) {
            ++st.completed;
            latencies.push_back(ms_between(r->t_submit, r->t_done));
        } else {
            ++st.failed;
        }
    }

    // Take admissible requests for `lane`.  Caller holds mu.
    std::vector<Request*> take(int lane) {
        std::vector<Request*> out;
        uint64_t tris = 0;
        for (auto it = pending.begin(); it != pending.end();) {
            if (out.size() >= cfg.max_batch_requests) break;
            Request* r = *it;
            uint64_t need = kRayBytes * r->req.num_rays;
            if (r->req.kind == ATR_REQ_REFIT) {
                auto bld = building.find(r->req.mesh_id);
                if (bld != building.end() && bld->second) { ++it; continue; }
                auto res = resident.find(r->req.mesh_id);
                if (res == resident.end()) {
                    finish(r, ATR_ERR_NOT_RESIDENT, "refit: mesh id is not resident");
                    it = pending.erase(it);
                    cv_done.notify_all();
                    continue;
                }
                // Refits of one mesh run on one lane at a time; refits of other
                // meshes of the same resident batch touch only their own slices
                // and may run on other lanes meanwhile.
                if (res->second.busy_lane >= 0 && res->second.busy_lane != lane) { ++it; continue; }
                need += 64ull * res->second.n;  // re-collapse / re-flatten scratch
            } else {
                if (!out.empty() && tris + r->req.num_triangles > cfg.max_batch_triangles) { ++it; continue; }
                need += kBuildBytesPerTri * r->req.num_triangles;
            }
            if (!make_room(need)) {
                if (out.empty() && inflight_bytes == 0 && batches.empty()) {
                    finish(r, ATR_ERR_OOM, "request does not fit the server's memory budget");
                    it = pending.erase(it);
                    cv_done.notify_all();
                    continue;
                }
                break;  // wait for memory to free up (keeps arrival order)
            }
            if (r->req.kind == ATR_REQ_REFIT) {
                Resident& res = resident.find(r->req.mesh_id)->second;
                res.busy_lane = lane;
                r->refit_rec = res.rec;
                r->refit_index = res.index;
                r->refit_n = res.n;
                ++res.rec->busy;
            } else {
                tris += r->req.num_triangles;
            }
            r->bytes = need;
            inflight_bytes += need;
            st.peak_bytes = std::max(st.peak_bytes, inflight_bytes + resident_bytes);
            r->t_taken = Clock::now();
            r->lane = (uint32_t)lane;
            out.push_back(r);
            it = pending.erase(it);
        }
        return out;
    }

    int run_batch(Lane& L, std::vector<Request*>& work, std::shared_ptr<BatchRec>* new_rec, std::vector<uint32_t>* build_index);
    void lane_loop(Lane* L);
};

namespace {

void set_msg(Request* r, int st) {
    if (st != ATR_OK) r->error = atr_last_error();
}

}  // namespace

int atr_server::run_batch(Lane& L, std::vector<Request*>& work, std::shared_ptr<BatchRec>* new_rec,
                          std::vector<uint32_t>* build_index) {
    atr_ctx* ctx = L.ctx;
    std::vector<Request*> builds, refits;
    for (Request* r : work) (r->req.kind == ATR_REQ_BUILD ? builds : refits).push_back(r);

    const Clock::time_point t_start = Clock::now();
    // Rays of every request into one device queue, in `work` order: a request
    // whose buffer is page-locked is copied from it directly, the others
    // through this lane's pinned staging buffer.
    // Staging holds only the pageable buffers, packed: stage_at[i] is request
    // i's offset (in rays) in the ray and result staging buffers.
    uint64_t total_rays = 0;
    for (Request* r : work) total_rays += r->req.num_rays;
    std::vector<uint64_t> ray_at(work.size() + 1, 0), stage_at(work.size(), 0);
    std::vector<char> rays_pinned(work.size(), 0), res_pinned(work.size(), 0), verts_pinned(work.size(), 0);
    uint64_t stage_rays = 0, stage_res = 0;
    for (size_t i = 0; i < work.size(); ++i) {
        ray_at[i + 1] = ray_at[i] + work[i]->req.num_rays;
        verts_pinned[i] = is_pinned(work[i]->req.vertices);
        if (!work[i]->req.num_rays) continue;
        rays_pinned[i] = is_pinned(work[i]->req.rays);
        res_pinned[i] = is_pinned(work[i]->req.results);
        stage_at[i] = std::max(stage_rays, stage_res);
        if (!rays_pinned[i]) stage_rays = stage_at[i] + work[i]->req.num_rays;
        if (!res_pinned[i]) stage_res = stage_at[i] + work[i]->req.num_rays;
    }
    if (stage_rays) ATR_TRY(grow_pinned(&L.h_rays, &L.h_rays_cap, stage_rays * 32));
    if (stage_res) ATR_TRY(grow_pinned(&L.h_res, &L.h_res_cap, stage_res * 16));
    std::vector<CopyJob> jobs;
    for (size_t i = 0; i < work.size(); ++i)
        if (work[i]->req.num_rays && !rays_pinned[i])
            jobs.push_back({static_cast<char*>(L.h_rays) + stage_at[i] * 32, work[i]->req.rays,
                            (size_t)work[i]->req.num_rays * 32});
    // Pageable refit vertices go to their own staging buffer (copied before any launch).
    uint64_t refit_tris = 0;
    std::vector<size_t> refit_at(work.size(), 0);
    for (size_t i = 0; i < work.size(); ++i) {
        if (work[i]->req.kind != ATR_REQ_REFIT || verts_pinned[i] || !work[i]->refit_rec) continue;
        refit_at[i] = refit_tris;
        refit_tris += work[i]->refit_n;
    }
    if (refit_tris) ATR_TRY(grow_pinned(&L.h_rverts, &L.h_rverts_cap, refit_tris * 48));
    for (size_t i = 0; i < work.size(); ++i) {
        if (work[i]->req.kind != ATR_REQ_REFIT || verts_pinned[i] || !work[i]->refit_rec) continue;
        jobs.push_back({static_cast<char*>(L.h_rverts) + refit_at[i] * 48, work[i]->req.vertices,
                        (size_t)work[i]->refit_n * 48});
    }
    par_copy(jobs);
    double copy_ms = ms_between(t_start, Clock::now());
    void* d_rays = nullptr;
    void* d_res = nullptr;
    if (total_rays) {
        ATR_TRY(ctx->alloc(&d_rays, total_rays * 32));
        int s = ctx->alloc(&d_res, total_rays * 16);
        if (s != ATR_OK) { ctx->release(d_rays); return s; }
        cudaError_t e = cudaSuccess;
        for (size_t i = 0; i < work.size() && e == cudaSuccess; ++i) {
            if (!work[i]->req.num_rays) continue;
            const void* src = rays_pinned[i] ? work[i]->req.rays
                                             : static_cast<const void*>(static_cast<char*>(L.h_rays) + stage_at[i] * 32);
            e = cudaMemcpyAsync(static_cast<char*>(d_rays) + ray_at[i] * 32, src, (size_t)work[i]->req.num_rays * 32,
                                cudaMemcpyHostToDevice, ctx->stream);
        }
        if (e != cudaSuccess) {
            ctx->release(d_rays);
            ctx->release(d_res);
            return atr::cuda_fail(e, "cudaMemcpyAsync(rays)", __FILE__, __LINE__);
        }
    }
    auto release_rays = [&]() {
        ctx->release(d_rays);
        ctx->release(d_res);
    };
    auto work_pos = [&](Request* r) {
        return (size_t)(std::find(work.begin(), work.end(), r) - work.begin());
    };
    for (size_t i = 0; i < builds.size(); ++i)
        if (work[i] != builds[i]) {
            release_rays();
            ATR_REQUIRE(false, ATR_ERR_INVALID_ARG, "server: builds must lead the lane batch");
        }

    // 1. One segmented build of every new mesh.
    if (!builds.empty()) {
        uint64_t tris = 0, stage_tris = 0;
        for (size_t m = 0; m < builds.size(); ++m) {
            tris += builds[m]->req.num_triangles;
            if (!verts_pinned[m]) stage_tris += builds[m]->req.num_triangles;
        }
        int s = stage_tris ? grow_pinned(&L.h_verts, &L.h_verts_cap, tris * 48) : ATR_OK;
        if (s != ATR_OK) { release_rays(); return s; }
        std::vector<uint32_t> off(builds.size() + 1, 0);
        std::vector<uint8_t> ts(builds.size()), it(builds.size());
        std::vector<CopyJob> vjobs;
        bool all_pinned = true;
        for (size_t m = 0; m < builds.size(); ++m) {
            const uint32_t n = builds[m]->req.num_triangles;
            if (!verts_pinned[m])
                vjobs.push_back({static_cast<char*>(L.h_verts) + (size_t)off[m] * 48, builds[m]->req.vertices,
                                 (size_t)n * 48});
            all_pinned = all_pinned && verts_pinned[m];
            off[m + 1] = off[m] + n;
            params_for(n, &ts[m], &it[m]);
        }
        const Clock::time_point tv = Clock::now();
        par_copy(vjobs);
        copy_ms += ms_between(tv, Clock::now());
        atr_batch* b = nullptr;
        if (all_pinned && builds.size() == 1) {
            s = atr_batch_create(ctx, static_cast<const float*>(builds[0]->req.vertices), off.data(), 1u, nullptr, 0,
                                 &b);
        } else if (all_pinned || vjobs.size() < builds.size()) {
            // Gather on the device: each mesh from its own pinned buffer or
            // from the staging buffer, then the batch copies the span.
            void* d_verts = nullptr;
            s = ctx->alloc(&d_verts, (size_t)tris * 48);
            cudaError_t e = cudaSuccess;
            for (size_t m = 0; s == ATR_OK && m < builds.size() && e == cudaSuccess; ++m) {
                const void* src = verts_pinned[m] ? builds[m]->req.vertices
                                                  : static_cast<const void*>(static_cast<char*>(L.h_verts) +
                                                                             (size_t)off[m] * 48);
                e = cudaMemcpyAsync(static_cast<char*>(d_verts) + (size_t)off[m] * 48, src,
                                    (size_t)builds[m]->req.num_triangles * 48, cudaMemcpyHostToDevice, ctx->stream);
            }
            if (s == ATR_OK && e != cudaSuccess) s = atr::cuda_fail(e, "cudaMemcpyAsync(vertices)", __FILE__, __LINE__);
            if (s == ATR_OK)
                s = atr_batch_create(ctx, static_cast<const float*>(d_verts), off.data(), (uint32_t)builds.size(),
                                     nullptr, 1, &b);
            ctx->release(d_verts);
        } else {
            s = atr_batch_create(ctx, static_cast<const float*>(L.h_verts), off.data(), (uint32_t)builds.size(),
                                 nullptr, 0, &b);
        }
        // Per-mesh parameters only with size classes; otherwise every mesh
        // takes the configuration's, passed to the build directly.
        if (s == ATR_OK && have_classes) s = atr_batch_set_params(ctx, b, ts.data(), it.data());
        if (s == ATR_OK) s = atr_batch_build(ctx, b, 1, cfg.treelet_size, cfg.iterations, 1.2f, 1.0f, 0);
        std::vector<float> sah(builds.size(), 0.0f);
        if (s == ATR_OK) s = atr_batch_collapse(ctx, b, 1.2f, 1.0f, cfg.max_leaf, sah.data());
        if (s == ATR_OK) s = atr_batch_flatten(ctx, b);
        if (s == ATR_OK) {
            // Merged queue over the builds' rays: `work` lists the builds
            // first, so their rays form the span [0, hi) of the ray buffer and
            // group m is build m's slice.
            std::vector<uint32_t> roff(1, 0), gm;
            for (size_t m = 0; m < builds.size(); ++m) {
                gm.push_back((uint32_t)m);
                roff.push_back((uint32_t)ray_at[m + 1]);
            }
            const uint64_t hi = ray_at[builds.size()];
            if (hi)
                s = atr_batch_trace(ctx, b, static_cast<const float*>(d_rays), (int64_t)hi, roff.data(), gm.data(),
                                    (uint32_t)gm.size(), 0, static_cast<int32_t*>(d_res));
        }
        if (s != ATR_OK) {
            for (Request* r : builds) set_msg(r, s);
            atr_batch_destroy(b);
            release_rays();
            return s;
        }
        for (size_t m = 0; m < builds.size(); ++m) builds[m]->sah = sah[m];
        auto rec = std::make_shared<BatchRec>();
        rec->batch = b;
        rec->bytes = kResidentBytesPerTri * tris;
        *new_rec = rec;
        build_index->resize(builds.size());
        for (size_t m = 0; m < builds.size(); ++m) (*build_index)[m] = (uint32_t)m;
    }

    // 2. Refits of resident meshes, each traced against its own batch.
    for (Request* r : refits) {
        // The batch taken for this refit, held busy (not evicted) until the
        // lane releases it.
        Resident res;
        if (!r->refit_rec || !r->refit_rec->batch) {
            r->status = ATR_ERR_NOT_RESIDENT;
            r->error = "refit: mesh was released";
            continue;
        }
        res.rec = r->refit_rec;
        res.index = r->refit_index;
        float sah = 0.0f;
        const size_t p = work_pos(r);
        const float* src = verts_pinned[p]
                               ? r->req.vertices
                               : reinterpret_cast<const float*>(static_cast<char*>(L.h_rverts) + refit_at[p] * 48);
        int s = atr::batch_refit_mesh(ctx, res.rec->batch, res.index, src, 0, &sah);
        if (s == ATR_OK && r->req.num_rays) {
            const uint32_t roff[2] = {0, r->req.num_rays};
            const uint32_t gm[1] = {res.index};
            s = atr_batch_trace(ctx, res.rec->batch, static_cast<const float*>(d_rays) + ray_at[p] * 8,
                                r->req.num_rays, roff, gm, 1, 0, static_cast<int32_t*>(d_res) + ray_at[p] * 4);
        }
        r->sah = sah;
        if (s != ATR_OK) { r->status = s; set_msg(r, s); }
    }

    // 3. Results back to host memory: straight into page-locked result
    // buffers, through the staging buffer for the others.
    for (size_t i = 0; i < work.size(); ++i) {
        if (!work[i]->req.num_rays) continue;
        void* dst = res_pinned[i] ? static_cast<void*>(work[i]->req.results)
                                  : static_cast<void*>(static_cast<char*>(L.h_res) + stage_at[i] * 16);
        cudaError_t e = cudaMemcpyAsync(dst, static_cast<char*>(d_res) + ray_at[i] * 16,
                                        (size_t)work[i]->req.num_rays * 16, cudaMemcpyDeviceToHost, ctx->stream);
        if (e != cudaSuccess) { release_rays(); return atr::cuda_fail(e, "cudaMemcpyAsync(results)", __FILE__, __LINE__); }
    }
    const int s = atr_ctx_synchronize(ctx);
    release_rays();
    const Clock::time_point t_done = Clock::now();
    ATR_TRY(s);
    std::vector<CopyJob> out;
    for (size_t i = 0; i < work.size(); ++i)
        if (work[i]->req.num_rays && work[i]->status == ATR_OK && !res_pinned[i])
            out.push_back({work[i]->req.results, static_cast<char*>(L.h_res) + stage_at[i] * 16,
                           (size_t)work[i]->req.num_rays * 16});
    par_copy(out);
    const double out_ms = ms_between(t_done, Clock::now());
    {
        std::lock_guard<std::mutex> lock(mu);
        st.host_copy_ms += copy_ms + out_ms;
        st.lane_batch_ms += ms_between(t_start, Clock::now());
    }
    return ATR_OK;
}

void atr_server::lane_loop(Lane* L) {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lock(mu);
    while (true) {
        std::vector<Request*> work;
        while (true) {
            if (!pending.empty()) {
                work = take(L->id);
                if (!work.empty()) break;
            }
            if (stopping && pending.empty()) return;
            cv_work.wait_for(lock, std::chrono::milliseconds(50));
        }
        // Builds first, so their rays form one span of the merged queue.
        std::stable_partition(work.begin(), work.end(),
                              [](Request* r) { return r->req.kind == ATR_REQ_BUILD; });
        account_busy(+1);
        ++st.lane_batches;
        st.max_batch_requests_seen = std::max(st.max_batch_requests_seen, (uint32_t)work.size());
        for (Request* r : work) r->batch_requests = (uint32_t)work.size();
        lock.unlock();

        std::shared_ptr<BatchRec> rec;
        std::vector<uint32_t> index;
        const int s = run_batch(*L, work, &rec, &index);
        const std::string msg = s == ATR_OK ? std::string() : std::string(atr_last_error());

        lock.lock();
        account_busy(-1);
        ++use_clock;
        // Resident bookkeeping for new meshes.
        if (rec && s != ATR_OK) {
            atr_batch_destroy(rec->batch);
            rec->batch = nullptr;
        }
        if (rec && s == ATR_OK) {
            size_t m = 0;
            for (Request* r : work) {
                if (r->req.kind != ATR_REQ_BUILD) continue;
                if (r->req.keep_resident) {
                    auto old = resident.find(r->req.mesh_id);
                    if (old != resident.end()) {
                        auto orec = old->second.rec;
                        resident.erase(old);
                        unref(orec);
                    }
                    resident[r->req.mesh_id] = Resident{rec, index[m], r->req.num_triangles};
                    ++rec->live;
                }
                ++m;
            }
            rec->last_use = use_clock;
            if (rec->live) {
                batches.push_back(rec);
                resident_bytes += rec->bytes;
            } else {
                atr_batch_destroy(rec->batch);
                rec->batch = nullptr;
            }
        }
        for (Request* r : work) {
            inflight_bytes -= r->bytes;
            if (r->req.kind == ATR_REQ_REFIT && r->refit_rec) {
                auto f = resident.find(r->req.mesh_id);
                if (f != resident.end() && f->second.busy_lane == L->id) f->second.busy_lane = -1;
                --r->refit_rec->busy;
                r->refit_rec->last_use = use_clock;
                r->refit_rec.reset();
            }
            if (s != ATR_OK) {
                finish(r, s, msg.c_str());
            } else {
                if (r->status == ATR_OK) {
                    if (r->req.kind == ATR_REQ_BUILD) {
                        ++st.builds;
                        st.triangles_built += r->req.num_triangles;
                    } else {
                        ++st.refits;
                        auto f = resident.find(r->req.mesh_id);
                        if (f != resident.end()) st.triangles_refit += f->second.n;
                    }
                    st.rays_traced += r->req.num_rays;
                }
                finish(r, r->status, r->status == ATR_OK ? nullptr : r->error.c_str());
            }
        }
        // Batches released while this lane used them.
        for (auto& b : std::vector<std::shared_ptr<BatchRec>>(batches)) maybe_free(b);
        cv_done.notify_all();
        cv_work.notify_all();
    }
}

extern "C" {

int atr_server_create(int device, const atr_server_config* cfg, atr_server** out) {
    ATR_REQUIRE(cfg && out, ATR_ERR_INVALID_ARG, "atr_server_create: NULL argument");
    ATR_REQUIRE(cfg->lanes >= 1 && cfg->lanes <= 8, ATR_ERR_INVALID_ARG, "atr_server_create: %u lanes", cfg->lanes);
    ATR_REQUIRE(cfg->max_batch_requests >= 1, ATR_ERR_INVALID_ARG, "atr_server_create: max_batch_requests 0");
    ATR_REQUIRE(cfg->max_batch_triangles >= 2 && cfg->max_batch_triangles < (1ull << 30), ATR_ERR_INVALID_ARG,
                "atr_server_create: max_batch_triangles %llu", (unsigned long long)cfg->max_batch_triangles);
    ATR_REQUIRE(cfg->treelet_size >= 3 && cfg->treelet_size <= 20 && cfg->iterations >= 0 && cfg->iterations <= 24,
                ATR_ERR_UNSUPPORTED, "atr_server_create: ATRBVH(%d, %d)", cfg->treelet_size, cfg->iterations);
    ATR_REQUIRE(cfg->max_leaf >= 0, ATR_ERR_INVALID_ARG, "atr_server_create: max_leaf %d", cfg->max_leaf);
    ATR_REQUIRE(!cfg->class_treelet == !cfg->class_iters, ATR_ERR_INVALID_ARG,
                "atr_server_create: give both size-class tables or neither");
    *out = nullptr;
    auto* s = new atr_server();
    s->device = device;
    s->cfg = *cfg;
    if (cfg->class_treelet) {
        for (int c = 0; c < 32; ++c) {
            if (cfg->class_treelet[c] < 3 || cfg->class_treelet[c] > 20 || cfg->class_iters[c] > 24) {
                delete s;
                ATR_REQUIRE(false, ATR_ERR_UNSUPPORTED, "atr_server_create: size class %d: ATRBVH(%d, %d)", c,
                            cfg->class_treelet[c], cfg->class_iters[c]);
            }
            s->class_treelet[c] = cfg->class_treelet[c];
            s->class_iters[c] = cfg->class_iters[c];
        }
        s->have_classes = true;
    }
    s->cfg.class_treelet = nullptr;
    s->cfg.class_iters = nullptr;
    s->busy_mark = Clock::now();
    for (uint32_t i = 0; i < cfg->lanes; ++i) {
        auto L = std::make_unique<Lane>();
        L->id = (int)i;
        const int st = atr_ctx_create(device, nullptr, &L->ctx);
        if (st != ATR_OK) {
            const std::string msg = atr_last_error();
            for (auto& l : s->lanes) atr_ctx_destroy(l->ctx);
            delete s;
            atr::set_error("%s", msg.c_str());
            return st;
        }
        // A lane's stream-ordered pool keeps what it frees.  Growing it maps
        // new device memory while the batch's requests wait (a few ms per GB,
        // measured): reserve up front what the lane's largest batch needs,
        // within half the budget's share per lane.
        const uint64_t prime = std::min<uint64_t>(cfg->max_batch_triangles * kBuildBytesPerTri,
                                                  cfg->hbm_budget_bytes / (2ull * cfg->lanes));
        void* p = nullptr;
        if (prime && L->ctx->alloc(&p, prime) == ATR_OK) {
            L->ctx->release(p);
            cudaStreamSynchronize(L->ctx->stream);
        }
        cudaGetLastError();
        s->lanes.push_back(std::move(L));
    }
    for (auto& L : s->lanes) L->thread = std::thread(&atr_server::lane_loop, s, L.get());
    *out = s;
    return ATR_OK;
}

int atr_server_submit(atr_server* s, const atr_request* req, uint64_t* ticket) {
    ATR_REQUIRE(s && req && ticket, ATR_ERR_INVALID_ARG, "atr_server_submit: NULL argument");
    ATR_REQUIRE(req->kind == ATR_REQ_BUILD || req->kind == ATR_REQ_REFIT, ATR_ERR_INVALID_ARG,
                "atr_server_submit: kind %d", req->kind);
    ATR_REQUIRE(req->vertices, ATR_ERR_INVALID_ARG, "atr_server_submit: no vertices");
    ATR_REQUIRE(req->kind == ATR_REQ_REFIT || req->num_triangles >= 2, ATR_ERR_INVALID_ARG,
                "atr_server_submit: %u triangles (need at least 2)", req->num_triangles);
    ATR_REQUIRE(req->kind == ATR_REQ_REFIT || req->num_triangles <= s->cfg.max_batch_triangles,
                ATR_ERR_INVALID_ARG, "atr_server_submit: %u triangles exceed the batch cap", req->num_triangles);
    ATR_REQUIRE(req->num_rays == 0 || (req->rays && req->results), ATR_ERR_INVALID_ARG,
                "atr_server_submit: rays without ray/result buffers");
    auto r = std::make_unique<Request>();
    r->req = *req;
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lock(s->mu);
    ATR_REQUIRE(!s->stopping, ATR_ERR_INVALID_ARG, "atr_server_submit: server is stopping");
    r->ticket = s->next_ticket++;
    *ticket = r->ticket;
    if (req->kind == ATR_REQ_BUILD && req->keep_resident) ++s->building[req->mesh_id];
    s->pending.push_back(r.get());
    s->tickets[r->ticket] = std::move(r);
    s->cv_work.notify_one();
    return ATR_OK;
}

int atr_server_wait(atr_server* s, uint64_t ticket, atr_request_result* out) {
    ATR_REQUIRE(s && out, ATR_ERR_INVALID_ARG, "atr_server_wait: NULL argument");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->tickets.find(ticket);
    ATR_REQUIRE(it != s->tickets.end(), ATR_ERR_INVALID_ARG, "atr_server_wait: unknown ticket %llu",
                (unsigned long long)ticket);
    Request* r = it->second.get();
    // The waiter erases the ticket (and frees the request) when it returns, so
    // a second concurrent waiter would read freed memory: refuse it.
    ATR_REQUIRE(!r->waited, ATR_ERR_INVALID_ARG, "atr_server_wait: ticket %llu already has a waiter",
                (unsigned long long)ticket);
    r->waited = true;
    s->cv_done.wait(lock, [&] { return r->done; });
    std::memset(out, 0, sizeof(*out));
    out->status = r->status;
    out->sah = r->sah;
    out->queue_ms = r->t_taken.time_since_epoch().count() ? ms_between(r->t_submit, r->t_taken) : 0.0;
    out->latency_ms = ms_between(r->t_submit, r->t_done);
    out->batch_requests = r->batch_requests;
    out->lane = r->lane;
    std::snprintf(out->error, sizeof(out->error), "%s", r->error.c_str());
    s->tickets.erase(it);
    return ATR_OK;
}

int atr_server_release(atr_server* s, uint64_t mesh_id) {
    ATR_REQUIRE(s, ATR_ERR_INVALID_ARG, "atr_server_release: NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->resident.find(mesh_id);
    ATR_REQUIRE(it != s->resident.end(), ATR_ERR_NOT_RESIDENT, "atr_server_release: mesh %llu is not resident",
                (unsigned long long)mesh_id);
    auto rec = it->second.rec;
    s->resident.erase(it);
    s->unref(rec);
    s->cv_work.notify_all();
    return ATR_OK;
}

int atr_server_stats_get(atr_server* s, atr_server_stats* out) {
    ATR_REQUIRE(s && out, ATR_ERR_INVALID_ARG, "atr_server_stats_get: NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    s->account_busy(0);
    *out = s->st;
    out->resident_meshes = (uint32_t)s->resident.size();
    out->resident_bytes = s->resident_bytes;
    out->busy_ms = s->busy1_ms;
    out->overlap_fraction = s->busy1_ms > 0 ? s->busy2_ms / s->busy1_ms : 0.0;
    std::vector<double> l = s->latencies;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) {
            const size_t i = (size_t)std::min<double>((double)l.size() - 1, std::ceil(q * (double)l.size()) - 1);
            return l[i];
        };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        double sum = 0;
        for (double x : l) sum += x;
        out->mean_ms = sum / (double)l.size();
        out->max_ms = l.back();
    }
    return ATR_OK;
}

int atr_server_destroy(atr_server* s) {
    if (!s) return ATR_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stopping = true;
    }
    s->cv_work.notify_all();
    for (auto& L : s->lanes)
        if (L->thread.joinable()) L->thread.join();
    for (auto& b : s->batches)
        if (b->batch) atr_batch_destroy(b->batch);
    s->batches.clear();
    for (auto& L : s->lanes) {
        if (L->h_verts) cudaFreeHost(L->h_verts);
        if (L->h_rays) cudaFreeHost(L->h_rays);
        if (L->h_res) cudaFreeHost(L->h_res);
        if (L->h_rverts) cudaFreeHost(L->h_rverts);
        atr_ctx_destroy(L->ctx);
    }
    delete s;
    return ATR_OK;
}

}  // extern "C"
