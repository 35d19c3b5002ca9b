// ATRBVH: agglomerative treelet restructuring on sm_100a.
//
// Semantics follow BVHRT-Core/src/AgglomerativeTreelet.cu:392-554 (bottom-up
// pass, one thread per leaf; the second child to arrive processes a node; a
// warp restructures the treelets of its lanes' nodes whose subtree holds at
// least gamma triangles) and AgglomerativeTreeletOptimizer.cpp:73-92 (gamma
// starts at the treelet size and doubles per iteration).
//
// Lane groups: the reference gives every treelet a whole warp although a
// treelet of n leaves keeps only n lanes busy.  Here a warp splits into
// 32/G groups of G >= n lanes (G = 8, 10, 16 or 32) and, when several of its
// lanes vote at once, restructures up to 32/G of their treelets together, one
// per group.  Treelets processed together root disjoint subtrees (a node is
// reached only after both of its subtrees are finished), so they touch
// disjoint nodes and the result does not depend on the order.  A single voter
// takes the whole warp.
//
// Per group, treelet formation keeps one treelet leaf per lane in registers;
// the merge phase keeps each treelet leaf's box, nodesSah and node id in
// shared memory (two float4 per leaf) beside the distance matrix, so a merge
// step reads the boxes it needs directly instead of broadcasting them.
//
// Ties resolve as in the reference.  formTreelet's argmax (Treelet.cuh:23-39)
// is a shuffle-down tree over the current leaves whose result on ties depends
// on its shape, so each group replays that exact tree on its own lanes.
// findMinimumDistance (AgglomerativeTreelet.cu:65-99) scans with lane stride 32
// (lane l keeps the first of its minima, j = l, l+32, ...) and then reduces
// with shuffle-down offsets 16, 8, 4, 2, 1 where the lower lane keeps ties.
// That tournament settles ties on lane bit 0 first (even lanes win), then
// bit 1, ..., bit 4, so it returns the minimum of the lexicographic key
// (distance, bit-reversed lane j mod 32, j); it is evaluated here as the
// minimum of a 64-bit key with those three fields.  Distances are surface
// areas, never negative, so their bit patterns order like the values; entries
// not below FLT_MAX are never chosen, as in the reference's strict comparison.
//
// Memory ordering: a node's data is published by the thread that finished it
// (plain stores, fence, atomic); the second arrival fences after its atomic
// and reads descendants through L2 (ld.cg), and __syncwarp orders the other
// lanes of the warp behind it.

#include "common.cuh"
#include "internal.h"
#include "treelet.cuh"

namespace atr {
namespace {

// Shared-memory layout of one lane group: distance matrix, then three float4
// per treelet leaf: (min.xyz, nodesSah), (max.xyz, node id bits) and
// (subtree count, next-iteration level, next-iteration nodesSah, unused).
template <int G>
struct GroupLayout {
    static constexpr int kGroups = 32 / G;
    static constexpr int kLeaves = G == 32 ? kMaxTreelet : G;
    static constexpr int kDist = kLeaves * (kLeaves - 1) / 2;
    static constexpr int kDistPad = (kDist + 3) & ~3;
    static constexpr int kFloats = kDistPad + 12 * kLeaves;
};

// The optimiser's per-node record, node-indexed in the batch layout (one
// 16-byte load gives a treelet leaf everything but its box):
//   x  subtree triangle count;
//   y  nodesSah of even iterations, z  nodesSah of odd iterations -- this
//      iteration's in component 1 + par (par = iteration & 1), the next
//      iteration's in the other;
//   w  big-node level: this iteration's until the node is finished, the next
//      iteration's after (only the level lists, built before any node is
//      finished, read this iteration's).
// The reference recomputes nodesSah bottom-up every iteration as
// (ci*A + left) + right, while a rewritten node stores the merge cost
// (left + right) + ci*A; the two can differ in the last bit, so the next
// iteration's values are kept in the recomputation's order.
__device__ __forceinline__ int rec_ns_cur(int par) { return 1 + par; }
__device__ __forceinline__ int rec_ns_next(int par) { return 2 - par; }
__device__ __forceinline__ float* rec_f(int4* r, int x, int c) { return reinterpret_cast<float*>(r + x) + c; }
__device__ __forceinline__ int* rec_i(int4* r, int x, int c) { return reinterpret_cast<int*>(r + x) + c; }
// A record from its fields, the nodesSah values placed by parity.
__device__ __forceinline__ int4 make_rec(int cnt, float ns_cur, float ns_next, int lvl, int par) {
    return par ? make_int4(cnt, __float_as_int(ns_next), __float_as_int(ns_cur), lvl)
               : make_int4(cnt, __float_as_int(ns_cur), __float_as_int(ns_next), lvl);
}

// What the treelet code keeps up to date, per mesh (rec starts at the mesh's
// first node): the records of the nodes it finishes or rewrites, the next
// iteration's gamma for their levels.
struct NextRefs {
    int4* rec;
    int par;
    int gamma;
    float ct;  // a triangle leaf's record is (1, ct * area, ct * area, 0), never rewritten
};

template <int G>
constexpr int warp_floats() {
    return GroupLayout<G>::kFloats * GroupLayout<G>::kGroups > GroupLayout<32>::kFloats
               ? GroupLayout<G>::kFloats * GroupLayout<G>::kGroups
               : GroupLayout<32>::kFloats;
}

// formTreelet's argmax tree (Treelet.cuh:23-39) over m lanes -- lane i takes
// lane i + floor(c/2) when that value is strictly larger, c halving upward --
// returns the largest value and, among equal largest values, the lane that
// comes first in a fixed order that depends only on m.  tree_winner replays
// the tree on a tie pattern; argmax_priority ranks the lanes by removing
// winners one at a time.  The full-warp path then needs two warp reductions:
// the maximum value, then the lowest rank among the lanes holding it.
struct ArgmaxPriority {
    uint8_t rank[kMaxTreelet + 1][32];
};

constexpr int tree_winner(int m, uint32_t tied) {
    int val[32] = {};
    int idx[32] = {};
    for (int i = 0; i < 32; ++i) {
        val[i] = (i < m && ((tied >> i) & 1u)) ? 1 : 0;
        idx[i] = i;
    }
    int c = m, sh = m / 2;
    while (c > 1) {
        for (int i = 0; i < c - sh; ++i)  // ascending: lane i + sh is read before it is updated
            if (val[i + sh] > val[i]) {
                val[i] = val[i + sh];
                idx[i] = idx[i + sh];
            }
        c = (c + 1) / 2;
        sh = c / 2;
    }
    return idx[0];
}

constexpr ArgmaxPriority argmax_priority() {
    ArgmaxPriority t{};
    for (int m = 0; m <= kMaxTreelet; ++m)
        for (int i = 0; i < 32; ++i) t.rank[m][i] = 255;
    for (int m = 1; m <= kMaxTreelet; ++m) {
        uint32_t rem = m == 32 ? 0xffffffffu : ((1u << m) - 1u);
        int k = 0;
        while (rem) {
            const int w = tree_winner(m, rem);
            t.rank[m][w] = (uint8_t)k++;
            rem &= ~(1u << w);
        }
    }
    return t;
}

__device__ const ArgmaxPriority g_argmax_priority = argmax_priority();

__device__ __forceinline__ float union_area3(float ax0, float ay0, float az0, float ax1, float ay1, float az1,
                                             float bx0, float by0, float bz0, float bx1, float by1, float bz1) {
    return sa3(__fsub_rn(fmaxf(ax1, bx1), fminf(ax0, bx0)), __fsub_rn(fmaxf(ay1, by1), fminf(ay0, by0)),
               __fsub_rn(fmaxf(az1, bz1), fminf(az0, bz0)));
}

// Treelets of at most kRegTreelet leaves on a whole warp (the dataflow
// pass's single treelets, whose latency is the pass's critical path): the
// merge and rewrite with every slot in its lane's registers and the distance
// matrix in two registers per lane (pair j in lane j % 32, register j / 32),
// exchanged by shuffles instead of shared memory.  Same choices, same
// arithmetic as the shared-memory merge below (AgglomerativeTreelet.cu:
// 101-212, 476-532); lane k < tsize enters holding leaf k.
constexpr int kRegTreelet = 11;  // 55 pairs fit two registers per lane

struct RegSlot {
    Box b;
    float sah;   // nodesSah, or the merge cost of a new node
    int node;    // node id; a retired slot's left child
    int cnt;     // subtree triangle count
    int nlv;     // next-iteration level
    float nsn;   // next-iteration nodesSah
    float area;  // the node's stored area; a retired slot's left child's
};

__device__ __forceinline__ RegSlot shfl_slot(const RegSlot& s, int src) {
    RegSlot o;
    o.b = shfl_box(s.b, src);
    o.sah = __shfl_sync(kFull, s.sah, src);
    o.node = __shfl_sync(kFull, s.node, src);
    o.cnt = __shfl_sync(kFull, s.cnt, src);
    o.nlv = __shfl_sync(kFull, s.nlv, src);
    o.nsn = __shfl_sync(kFull, s.nsn, src);
    o.area = __shfl_sync(kFull, s.area, src);
    return o;
}

__device__ __forceinline__ void merge_rewrite_regs(const TreeRefs& g, int nb, uint32_t n, int root, RegSlot sl,
                                                   int internal_node, int4* KD, const NextRefs& nx,
                                                   float root_sah, int tsize, float ci,
                                                   const uint16_t* __restrict__ s_rc) {
    const int lane = threadIdx.x & 31;
    int32_t* const P = g.parent + nb;
    int32_t* const Lf = g.left + nb;
    int32_t* const Rt = g.right + nb;
    float4* const BMN = g.bmin + nb;
    float4* const BMX = g.bmax + nb;
    float* const AR = g.area + nb;
    const int next_c = rec_ns_next(nx.par);
    // Pair coordinates (row > column) of this lane's two pairs.
    const uint32_t rc0 = s_rc[lane], rc1 = s_rc[lane + 32];
    const int r0 = (int)(rc0 >> 8), c0 = (int)(rc0 & 255u), r1 = (int)(rc1 >> 8), c1 = (int)(rc1 & 255u);
    float d0, d1;
    {
        const Box a0 = shfl_box(sl.b, r0), b0 = shfl_box(sl.b, c0);
        const Box a1 = shfl_box(sl.b, r1), b1 = shfl_box(sl.b, c1);
        d0 = union_area(a0, b0);
        d1 = union_area(a1, b1);
    }
    int right = 0;       // a retired slot's right child
    float right_area = 0.0f;  // and its stored area
    for (int last = tsize - 1; last >= 1; --last) {
        // The minimum distance over pairs j < last (last + 1) / 2, then the
        // lowest (brev5(j % 32), j) among the pairs holding it -- the lane-
        // strided scan's choice.
        const int msize = last * (last + 1) / 2;
        float bd = FLT_MAX;
        int bj = -1;
        if (lane < msize && d0 < bd) { bd = d0; bj = lane; }
        if (lane + 32 < msize && d1 < bd) { bd = d1; bj = lane + 32; }
        const uint32_t db = bj >= 0 ? __float_as_uint(bd) : 0xffffffffu;
        const uint32_t dmin = __reduce_min_sync(kFull, db);
        const uint32_t tk =
            (bj >= 0 && db == dmin) ? (((__brev((uint32_t)lane) >> 27) << 8) | (uint32_t)bj) : 0xffffffffu;
        const uint32_t kmin = __reduce_min_sync(kFull, tk);
        const int mi = dmin == 0xffffffffu ? 0 : (int)(kmin & 255u);
        const uint32_t rc = s_rc[mi];
        const int jr = (int)(rc >> 8), jc = (int)(rc & 255u);
        const RegSlot r = shfl_slot(sl, jr), c = shfl_slot(sl, jc), z = shfl_slot(sl, last);
        const int new_internal = __shfl_sync(kFull, internal_node, last - 1);
        // updateState (:101-150): the new node (rows jr and jc) takes slot jc,
        // slot `last` moves to slot jr, slot `last` retires holding the new
        // node (left child row jr's node, right child row jc's).
        RegSlot nw;
        nw.b.mnx = fminf(c.b.mnx, r.b.mnx); nw.b.mny = fminf(c.b.mny, r.b.mny); nw.b.mnz = fminf(c.b.mnz, r.b.mnz);
        nw.b.mxx = fmaxf(c.b.mxx, r.b.mxx); nw.b.mxy = fmaxf(c.b.mxy, r.b.mxy); nw.b.mxz = fmaxf(c.b.mxz, r.b.mxz);
        const float area_new = box_area(nw.b.mnx, nw.b.mny, nw.b.mnz, nw.b.mxx, nw.b.mxy, nw.b.mxz);
        nw.sah = __fadd_rn(__fadd_rn(r.sah, c.sah), __fmul_rn(ci, area_new));
        nw.cnt = r.cnt + c.cnt;
        nw.nlv = nw.cnt >= nx.gamma ? 1 + max(r.nlv, c.nlv) : 0;
        nw.nsn = __fadd_rn(__fadd_rn(__fmul_rn(ci, area_new), r.nsn), c.nsn);
        nw.node = new_internal;
        nw.area = area_new;  // what the rewrite stores: box_area of the same box
        if (lane == jc) sl = nw;
        if (lane == jr) sl = z;
        if (lane == last) {
            sl = nw;
            sl.node = r.node;
            sl.area = r.area;
            right = c.node;
            right_area = c.area;
        }
        // updateDistancesMatrix (:152-188): pairs (jc, k) take the union with
        // the new node (lane k computes it), pairs (jr, k) take the distance
        // of pair (last, k) as the step began.
        const float u = union_area(nw.b, sl.b);
        const int o0 = r0 + c0 - (r0 == jc || c0 == jc ? jc : jr);
        const int o1 = r1 + c1 - (r1 == jc || c1 == jc ? jc : jr);
        const int t0 = trm_idx(last, min(o0, last - 1)), t1 = trm_idx(last, min(o1, last - 1));
        const float u0 = __shfl_sync(kFull, u, o0 & 31), u1 = __shfl_sync(kFull, u, o1 & 31);
        const float m00 = __shfl_sync(kFull, d0, t0 & 31), m01 = __shfl_sync(kFull, d1, t0 & 31);
        const float m10 = __shfl_sync(kFull, d0, t1 & 31), m11 = __shfl_sync(kFull, d1, t1 & 31);
        if (r0 < last) {
            if (r0 == jc || c0 == jc) d0 = u0;
            else if (r0 == jr || c0 == jr) d0 = t0 >= 32 ? m01 : m00;
        }
        if (r1 < last) {
            if (r1 == jc || c1 == jc) d1 = u1;
            else if (r1 == jr || c1 == jr) d1 = t1 >= 32 ? m11 : m10;
        }
    }
    // ---- updateTreelet (:190-212): slot k >= 1 holds the k-th new node ----
    const int ni = __shfl_sync(kFull, internal_node, lane > 0 ? lane - 1 : 0);
    const bool accept = __shfl_sync(kFull, sl.sah, 1) < root_sah;
    const bool wr = accept && lane >= 1 && lane < tsize;
    if (wr) {
        Lf[ni] = sl.node;
        Rt[ni] = right;
        P[sl.node] = ni;
        P[right] = ni;
        const float4 mn = make_float4(sl.b.mnx, sl.b.mny, sl.b.mnz, 0.0f);
        const float4 mx = make_float4(sl.b.mxx, sl.b.mxy, sl.b.mxz, 0.0f);
        BMN[ni] = mn;
        BMX[ni] = mx;
        AR[ni] = box_area(mn, mx);
        nx.rec[ni] = make_rec(sl.cnt, sl.sah, sl.nsn, sl.nlv, nx.par);
    }
    // The rewritten nodes' child records: children and their stored areas
    // (new nodes' as just stored, the treelet leaves' as their parents'
    // records held them).
    if (wr) KD[ni] = make_int4(sl.node, right, __float_as_int(sl.area), __float_as_int(right_area));
    if (!accept && lane == 0) {
        const int lc = ld_cg(Lf + root), rc = ld_cg(Rt + root);
        const int4 rl = __ldcg(nx.rec + lc), rr = __ldcg(nx.rec + rc);
        const int a = is_internal(lc, n) ? rl.w : 0;
        const int b = is_internal(rc, n) ? rr.w : 0;
        *rec_i(nx.rec, root, 3) = ld_cg(rec_i(nx.rec, root, 0)) >= nx.gamma ? 1 + max(a, b) : 0;
        *rec_f(nx.rec, root, next_c) =
            __fadd_rn(__fadd_rn(__fmul_rn(ci, ld_cg(AR + root)), __int_as_float(next_c == 1 ? rl.y : rl.z)),
                      __int_as_float(next_c == 1 ? rr.y : rr.z));
    }
    __syncwarp();
}

// One treelet per lane group.  Lanes of a group hold the same root/mesh
// arguments; `active` is false for groups without a treelet (and for lanes
// outside every group).  maxts is the largest treelet size of the active
// groups of the warp: every lane runs the same number of loop trips so that
// the shuffles stay warp-wide.  sm is this group's shared memory.
template <int G>
__device__ __forceinline__ void process_group(const TreeRefs& g, bool active, int nb, uint32_t n, int root,
                                              int4 rk, int4* KD, const NextRefs& nx, float root_sah, int tsize,
                                              int maxts,
                                              float ci, float* sm, const uint16_t* __restrict__ s_rc,
                                              const uint8_t* __restrict__ s_prio, uint32_t* err) {
    using Lay = GroupLayout<G>;
    const int lane = threadIdx.x & 31;
    const int gb = G == 32 ? 0 : (lane / G) * G;
    const int gl = lane - gb;
    int32_t* const P = g.parent + nb;
    int32_t* const Lf = g.left + nb;
    int32_t* const Rt = g.right + nb;
    float4* const BMN = g.bmin + nb;
    float4* const BMX = g.bmax + nb;
    float* const AR = g.area + nb;
    const int cur_c = rec_ns_cur(nx.par), next_c = rec_ns_next(nx.par);

    // ---- formTreelet (Treelet.cuh:57-114) ----
    // Lane k holds treelet leaf k (node and area).  The child record of an
    // internal leaf (children and their areas) is copied into the lane's
    // shared slot with cp.async when the leaf joins; only the lane whose leaf
    // is expanded waits, for its own copy, so a step never waits for the
    // records of leaves that joined in the step before.  Boxes and nodesSah
    // are loaded once the treelet is complete.
    float* const dist = sm;
    float4* const lmn = reinterpret_cast<float4*>(sm + Lay::kDistPad);
    float4* const lmx = lmn + Lay::kLeaves;
    int4* const lcn = reinterpret_cast<int4*>(lmx + Lay::kLeaves);
    int4* const krec = lcn;  // child-record slots during formation
    int internal_node = gl == 0 ? root : -1;
    int s_node = -1;
    float s_area = 0.0f;
    auto join = [&](int node, float area) {
        s_node = node;
        s_area = area;
        if (is_internal(node, n)) cp_async16_cg(krec + gl, KD + node);
    };
    if (active && gl < 2) join(gl == 0 ? rk.x : rk.y, __int_as_float(gl == 0 ? rk.z : rk.w));
    bool ok = true;
    for (int it = 0; it < maxts - 2; ++it) {
        const bool act = active && ok && it < tsize - 2;
        const int m = 2 + it;
        int largest;
        if constexpr (G == 32) {
            // Largest value (internal nodes' areas as bits + 1, which order like
            // the areas; other leaves 0, the reference's -FLT_MAX), then, among
            // several lanes holding it, the first in the tree's tie order.
            const uint32_t ev = (gl < m && is_internal(s_node, n)) ? __float_as_uint(s_area) + 1u : 0u;
            const uint32_t vmax = __reduce_max_sync(kFull, ev);
            const uint32_t tied = __ballot_sync(kFull, gl < m && ev == vmax);
            if (__popc(tied) == 1) {
                largest = __ffs(tied) - 1;
            } else {
                const uint32_t pk = ((tied >> gl) & 1u) ? (uint32_t)s_prio[m * 32 + gl] : 255u;
                const uint32_t pmin = __reduce_min_sync(kFull, pk);
                largest = __ffs(__ballot_sync(kFull, pk == pmin)) - 1;
            }
        } else {
            float v = (gl < m && is_internal(s_node, n)) ? s_area : -FLT_MAX;
            int ix = gl;
            int c = m, sh = m >> 1;
            while (c > 1) {
                const float ov = __shfl_sync(kFull, v, lane + sh);
                const int oi = __shfl_sync(kFull, ix, lane + sh);
                if (gl < c - sh && ov > v) { v = ov; ix = oi; }
                c = (c + 1) >> 1;
                sh = c >> 1;
            }
            largest = __shfl_sync(kFull, ix, gb);
        }
        const int rep = __shfl_sync(kFull, s_node, gb + largest);
        const bool expand = act && is_internal(rep, n);
        if (expand && gl == largest) cp_async_wait_all();
        __syncwarp();
        int4 rk = make_int4(-1, -1, 0, 0);
        if (expand) rk = krec[largest];
        __syncwarp();
        if (act) {
            if (!expand) {
                ok = false;
            } else {
                if (gl == it + 1) internal_node = rep;
                if (gl == largest || gl == it + 2) {
                    const bool isl = gl == largest;
                    join(isl ? rk.x : rk.y, __int_as_float(isl ? rk.z : rk.w));
                }
            }
        }
    }
    const bool run = active && ok;
    if (active && !ok && gl == 0) set_error_bits(err, kErrTreeletClimb);
    float4 s_mn = make_float4(0.f, 0.f, 0.f, 0.f), s_mx = s_mn;
    float s_sah = 0.0f;
    int s_cnt = 0, s_nlv = 0;
    float s_nsn = 0.0f;
    if (run && gl < tsize) {
        s_mn = ld_cg(BMN + s_node);
        s_mx = ld_cg(BMX + s_node);
        if (is_internal(s_node, n)) {
            const int4 r = __ldcg(nx.rec + s_node);
            s_cnt = r.x;
            s_sah = __int_as_float(nx.par ? r.z : r.y);
            s_nsn = __int_as_float(nx.par ? r.y : r.z);
            s_nlv = r.w;
        } else {  // a triangle: its record follows from its area (the parent's child record's)
            s_cnt = 1;
            s_sah = s_nsn = __fmul_rn(nx.ct, s_area);
        }
    }
    // Records of leaves that were never expanded may still be in flight into
    // the slots the merge state reuses.
    cp_async_wait_all();
    __syncwarp();
    if constexpr (G == 32) {
        if (run && tsize <= kRegTreelet) {
            RegSlot sl;
            sl.b = Box{s_mn.x, s_mn.y, s_mn.z, s_mx.x, s_mx.y, s_mx.z};
            sl.sah = s_sah;
            sl.node = s_node;
            sl.cnt = s_cnt;
            sl.nlv = s_nlv;
            sl.nsn = s_nsn;
            sl.area = s_area;
            merge_rewrite_regs(g, nb, n, root, sl, internal_node, KD, nx, root_sah, tsize, ci, s_rc);
            return;
        }
    }

    // ---- distance matrix (AgglomerativeTreelet.cu:18-63) ----
    // Slot k: (min.xyz, nodesSah), (max.xyz, node), (count, next level,
    // next nodesSah, -).  When the merge retires slot k (step last = k) it
    // takes the new node instead: (min.xyz, cost), (max.xyz, left child),
    // (count, next level, next nodesSah, right child).
    if (run && gl < tsize) {
        lmn[gl] = make_float4(s_mn.x, s_mn.y, s_mn.z, s_sah);
        lmx[gl] = make_float4(s_mx.x, s_mx.y, s_mx.z, __int_as_float(s_node));
        lcn[gl] = make_int4(s_cnt, s_nlv, __float_as_int(s_nsn), 0);
    }
    __syncwarp();
    if (run) {
        const int np = tsize * (tsize - 1) / 2;
        for (int j = gl; j < np; j += G) {
            const uint32_t rc = s_rc[j];
            const float4 a0 = lmn[rc >> 8], a1 = lmx[rc >> 8], b0 = lmn[rc & 255u], b1 = lmx[rc & 255u];
            dist[j] = union_area3(a0.x, a0.y, a0.z, a1.x, a1.y, a1.z, b0.x, b0.y, b0.z, b1.x, b1.y, b1.z);
        }
    }
    __syncwarp();

    // ---- agglomerative merge (AgglomerativeTreelet.cu:476-532) ----
    float my0x = s_mn.x, my0y = s_mn.y, my0z = s_mn.z, my1x = s_mx.x, my1y = s_mx.y, my1z = s_mx.z;
    for (int step = 0; step < maxts - 1; ++step) {
        const int last = tsize - 1 - step;
        const bool act = run && last >= 1;
        int mi;
        if constexpr (G == 32) {
            // Lane l scans j = l, l + 32, ...; then the minimum distance, then
            // the lowest (brev5(l), j) among the lanes holding it.
            float bd = FLT_MAX;
            int bj = -1;
            if (act) {
                const int msize = last * (last + 1) / 2;
                for (int j = lane; j < msize; j += 32) {
                    const float d = dist[j];
                    if (d < bd) { bd = d; bj = j; }
                }
            }
            const uint32_t db = bj >= 0 ? __float_as_uint(bd) : 0xffffffffu;
            const uint32_t dmin = __reduce_min_sync(kFull, db);
            const uint32_t tk = (bj >= 0 && db == dmin) ? (((__brev((uint32_t)lane) >> 27) << 8) | (uint32_t)bj)
                                                        : 0xffffffffu;
            const uint32_t kmin = __reduce_min_sync(kFull, tk);
            mi = dmin == 0xffffffffu ? 0 : (int)(kmin & 255u);
        } else {
            // Fast path: the group minimum of the distances alone (32-bit), held
            // by one lane whose scan met it once, is the reference's choice.
            // Equal minima (two holders, or a holder that saw its minimum
            // twice) take the exact (distance, brev5(j), j) key reduction.
            const int msize = act ? last * (last + 1) / 2 : 0;
            uint32_t bd = 0xffffffffu;
            int bj = 0;
            bool tie = false;
            for (int j = gl; j < msize; j += G) {
                uint32_t d = __float_as_uint(dist[j]);
                d = d < 0x7f7fffffu ? d : 0xffffffffu;  // not below FLT_MAX: never chosen
                if (d < bd) {
                    bd = d;
                    bj = j;
                    tie = false;
                } else if (d == bd) {
                    tie = true;
                }
            }
            uint32_t dmin = bd;
            if ((G & (G - 1)) == 0) {
#pragma unroll
                for (int o = G >> 1; o > 0; o >>= 1) dmin = min(dmin, __shfl_xor_sync(kFull, dmin, o));
            } else {
                int c = G, sh = G >> 1;
                while (c > 1) {
                    const uint32_t od = __shfl_sync(kFull, dmin, lane + sh);
                    if (gl < c - sh) dmin = min(dmin, od);
                    c = (c + 1) >> 1;
                    sh = c >> 1;
                }
                dmin = __shfl_sync(kFull, dmin, gb);
            }
            const uint32_t gmask = (G == 32 ? kFull : ((1u << G) - 1u)) << gb;
            const bool holds = bd == dmin && dmin != 0xffffffffu;
            const uint32_t holders = __ballot_sync(kFull, holds) & gmask;
            const bool tied = (__ballot_sync(kFull, holds && tie) & gmask) != 0u || __popc(holders) > 1;
            mi = __shfl_sync(kFull, bj, holders ? __ffs(holders) - 1 : gb);
            if (!holders) mi = 0;
            if (__any_sync(kFull, tied)) {
                unsigned long long best = ~0ull;
                for (int j = gl; j < msize; j += G) {
                    const float d = dist[j];
                    if (d < FLT_MAX) {
                        const unsigned long long k = ((unsigned long long)__float_as_uint(d) << 32) |
                                                     (uint32_t)(((__brev((uint32_t)j) >> 27) << 8) | (uint32_t)j);
                        best = k < best ? k : best;
                    }
                }
                if ((G & (G - 1)) == 0) {
#pragma unroll
                    for (int o = G >> 1; o > 0; o >>= 1) {
                        const unsigned long long ob = __shfl_xor_sync(kFull, best, o);
                        best = ob < best ? ob : best;
                    }
                } else {
                    int c = G, sh = G >> 1;
                    while (c > 1) {
                        const unsigned long long ob = __shfl_sync(kFull, best, lane + sh);
                        if (gl < c - sh && ob < best) best = ob;
                        c = (c + 1) >> 1;
                        sh = c >> 1;
                    }
                    best = __shfl_sync(kFull, best, gb);
                }
                if (tied) mi = best == ~0ull ? 0 : (int)(best & 255u);
            }
        }
        const int new_internal = __shfl_sync(kFull, internal_node, gb + (last >= 1 ? last - 1 : 0));
        // updateState (:101-150): the new node (union of rows jr and jc) takes
        // slot jc, the last leaf moves to slot jr, slot `last` retires with
        // the new node for the final rewrite.
        int jr = 0, jc = 0;
        float a0x = 0.f, a0y = 0.f, a0z = 0.f, a1x = 0.f, a1y = 0.f, a1z = 0.f;
        float4 z0 = make_float4(0.f, 0.f, 0.f, 0.f), z1 = z0, nw0 = z0, nw1 = z0;
        int4 z2 = make_int4(0, 0, 0, 0), nw2 = z2;
        if (act) {
            const uint32_t rc = s_rc[mi];
            jr = (int)(rc >> 8);
            jc = (int)(rc & 255u);
            const float4 r0 = lmn[jr], r1 = lmx[jr], c0 = lmn[jc], c1 = lmx[jc];
            const int4 r2 = lcn[jr], c2 = lcn[jc];
            z0 = lmn[last];
            z1 = lmx[last];
            z2 = lcn[last];
            a0x = fminf(c0.x, r0.x); a0y = fminf(c0.y, r0.y); a0z = fminf(c0.z, r0.z);
            a1x = fmaxf(c1.x, r1.x); a1y = fmaxf(c1.y, r1.y); a1z = fmaxf(c1.z, r1.z);
            const float area_new = box_area(a0x, a0y, a0z, a1x, a1y, a1z);
            const float la = __fadd_rn(__fadd_rn(r0.w, c0.w), __fmul_rn(ci, area_new));
            const int cnt = r2.x + c2.x;
            // Next iteration's nodesSah of the new node (left = row jr).
            const float nsn = __fadd_rn(__fadd_rn(__fmul_rn(ci, area_new), __int_as_float(r2.z)), __int_as_float(c2.z));
            nw0 = make_float4(a0x, a0y, a0z, la);
            nw1 = make_float4(a1x, a1y, a1z, r1.w);  // left child: row jr's node
            nw2 = make_int4(cnt, cnt >= nx.gamma ? 1 + max(r2.y, c2.y) : 0, __float_as_int(nsn),
                            __float_as_int(c1.w));  // right child: row jc's node
        }
        __syncwarp();
        if (act) {
            if (gl == jc) {
                lmn[jc] = nw0;
                lmx[jc] = make_float4(a1x, a1y, a1z, __int_as_float(new_internal));
                lcn[jc] = make_int4(nw2.x, nw2.y, nw2.z, 0);
                my0x = a0x; my0y = a0y; my0z = a0z; my1x = a1x; my1y = a1y; my1z = a1z;
            }
            if (gl == jr) {
                lmn[jr] = z0;
                lmx[jr] = z1;
                lcn[jr] = z2;
                my0x = z0.x; my0y = z0.y; my0z = z0.z; my1x = z1.x; my1y = z1.y; my1z = z1.z;
            }
            if (gl == last) {
                lmn[last] = nw0;
                lmx[last] = nw1;
                lcn[last] = nw2;
            }
        }
        // updateDistancesMatrix (:152-188): row `last` moves to row jr, then the
        // distances to the new node at jc are recomputed.
        const bool du = act && last > 1;
        const bool mv = du && gl < last && gl != jr;
        float moved = 0.0f;
        if (mv) moved = dist[trm_idx(last, gl)];
        __syncwarp();
        if (mv) dist[trm_idx(max(jr, gl), min(jr, gl))] = moved;
        __syncwarp();
        if (du && gl < last && gl != jc)
            dist[trm_idx(max(jc, gl), min(jc, gl))] =
                union_area3(a0x, a0y, a0z, a1x, a1y, a1z, my0x, my0y, my0z, my1x, my1y, my1z);
        __syncwarp();
    }

    // ---- updateTreelet (:190-212) ----
    const int ni = __shfl_sync(kFull, internal_node, gb + (gl > 0 ? gl - 1 : 0));
    const bool accept = run && lmn[1].w < root_sah;
    const bool wr = accept && gl >= 1 && gl < tsize;
    int fl = 0, fr = 0;
    if (wr) {
        const float4 f0 = lmn[gl], f1 = lmx[gl];
        const int4 f2 = lcn[gl];
        fl = __float_as_int(f1.w);
        fr = f2.w;
        Lf[ni] = fl;
        Rt[ni] = fr;
        P[fl] = ni;
        P[fr] = ni;
        const float4 mn = make_float4(f0.x, f0.y, f0.z, 0.0f);
        const float4 mx = make_float4(f1.x, f1.y, f1.z, 0.0f);
        BMN[ni] = mn;
        BMX[ni] = mx;
        AR[ni] = box_area(mn, mx);
        nx.rec[ni] = make_rec(f2.x, f0.w, __int_as_float(f2.z), f2.y, nx.par);
    }
    __syncwarp();
    // The rewritten nodes' child records, once every new area is stored.
    if (wr) KD[ni] = make_int4(fl, fr, __float_as_int(__ldcg(AR + fl)), __float_as_int(__ldcg(AR + fr)));
    // A treelet left as it was: its root's next level and next nodesSah from
    // its children.
    if (run && !accept && gl == 0) {
        const int lc = ld_cg(Lf + root), rc = ld_cg(Rt + root);
        const int4 rl = __ldcg(nx.rec + lc), rr = __ldcg(nx.rec + rc);
        const int a = is_internal(lc, n) ? rl.w : 0;
        const int b = is_internal(rc, n) ? rr.w : 0;
        *rec_i(nx.rec, root, 3) = ld_cg(rec_i(nx.rec, root, 0)) >= nx.gamma ? 1 + max(a, b) : 0;
        *rec_f(nx.rec, root, next_c) =
            __fadd_rn(__fadd_rn(__fmul_rn(ci, ld_cg(AR + root)), __int_as_float(next_c == 1 ? rl.y : rl.z)),
                      __int_as_float(next_c == 1 ? rr.y : rr.z));
    }
    __syncwarp();
    (void)cur_c;
}

// One iteration over every mesh of `segs`: thread i starts at the i-th sorted
// leaf of the batch.  Each mesh has its own treelet size and iteration count
// when `seg_tsize`/`seg_iters` are given; a mesh whose iterations are done
// sits this launch out.
template <int G, int W>
__global__ void __launch_bounds__(W * 32, 16 / W) k_atrbvh(TreeRefs g, Segs segs, int4* __restrict__ rec,
                                                   uint32_t* __restrict__ counters, int4* __restrict__ kids,
                                                   int tsize_all,
                                                   const uint8_t* __restrict__ seg_tsize,
                                                   const uint8_t* __restrict__ seg_iters, int iteration, float ci,
                                                   float ct, int group_min, const uint2* __restrict__ start,
                                                   const uint32_t* __restrict__ start_count, uint32_t* err) {
    constexpr int kWarpFloats = warp_floats<G>();
    __shared__ __align__(16) float s_mem[W][kWarpFloats];
    __shared__ uint16_t s_rc[kMaxDist];
    __shared__ __align__(4) uint8_t s_prio[(kMaxTreelet + 1) * 32];
    if (start && blockIdx.x * W >= *start_count) return;  // no frontier node for this block
    for (int k = threadIdx.x; k < kMaxDist; k += blockDim.x) {
        int r, c;
        trm_rc(k, r, c);
        s_rc[k] = (uint16_t)((r << 8) | c);
    }
    for (int k = threadIdx.x; k < (kMaxTreelet + 1) * 8; k += blockDim.x)
        reinterpret_cast<uint32_t*>(s_prio)[k] = reinterpret_cast<const uint32_t*>(&g_argmax_priority.rank[0][0])[k];
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    int cur = -1, base = 0, cbase = 0, tsize = tsize_all;
    uint32_t nm = 2;
    // Frontier mode: climb from the frontier below the nodes the level passes
    // left over (everything under a start node is final); a thread takes the
    // next start whenever its climb ends, so any frontier size fits the grid.
    // Starts go to lane 0 of every warp first, then lane 1, ...: a warp
    // restructures the treelets its lanes reach one after another, so a small
    // frontier is spread over as many warps as possible.
    const uint32_t n_start = start ? *start_count : 0u;
    const uint32_t nwarps = gridDim.x * W;
    uint32_t next = (uint32_t)lane * nwarps + blockIdx.x * W + (uint32_t)w;
    auto take_start = [&]() {
        const uint2 e = start[next];
        next += 32u * nwarps;
        const uint32_t s0 = segs.tri_begin(e.x);
        nm = segs.tri_end(e.x) - s0;
        base = segs.node_base(e.x);
        cbase = segs.inner_base(e.x);
        tsize = seg_tsize ? (int)seg_tsize[e.x] : tsize_all;
        cur = g.parent[base + (int)e.y];
    };
    if (start) {
        if (next < n_start) take_start();
    } else if (i < segs.n) {
        const uint32_t m = segs.seg_of_tri(i);
        const uint32_t s0 = segs.tri_begin(m);
        nm = segs.tri_end(m) - s0;
        base = segs.node_base(m);
        cbase = segs.inner_base(m);
        if (seg_tsize) tsize = seg_tsize[m];
        if (!seg_iters || iteration < (int)seg_iters[m]) {
            const int leaf = base + (int)(i - s0) + (int)nm - 1;
            const float ls = __fmul_rn(ct, g.area[leaf]);
            rec[leaf] = make_int4(1, __float_as_int(ls), __float_as_int(ls), 0);
            cur = g.parent[leaf];
        }
    }
    // The arrival atomic is acquire-release; after a treelet rewrite, whose
    // stores other lanes of the warp made, a fence first publishes those too.
    bool rewrote = false;
    while (__any_sync(kFull, cur >= 0 || next < n_start)) {
        if (cur < 0 && next < n_start) take_start();
        const int gamma = tsize << iteration;
        bool second = false;
        // A node's links, area and parent stay as they are until it is
        // reached (only a treelet rooted at it or above rewrites them), so
        // they are loaded before the arrival atomic.
        int lc = 0, rc = 0, up = -1;
        float a = 0.0f;
        if (cur >= 0) {
            const int x = base + cur;
            lc = ld_cg(g.left + x);
            rc = ld_cg(g.right + x);
            up = ld_cg(g.parent + x);
            a = ld_cg(g.area + x);
            if (rewrote) fence_acq_rel_gpu();
            if (atomic_add_acq_rel_gpu(&counters[cbase + cur], 1u) == 0u) cur = -1;
            else second = true;
        }
        int cnt = 0;
        float my_sah = 0.0f;
        int4 myk = make_int4(-1, -1, 0, 0);
        if (second) {
            const int x = base + cur;
            const int l = base + lc, r = base + rc;
            const int cc = rec_ns_cur(iteration & 1);
            const int4 rl = __ldcg(rec + l), rr = __ldcg(rec + r);
            cnt = rl.x + rr.x;
            my_sah = __fadd_rn(__fadd_rn(__fmul_rn(ci, a), __int_as_float(cc == 1 ? rl.y : rl.z)),
                               __int_as_float(cc == 1 ? rr.y : rr.z));
            // Child record for treelet formation: one load yields both
            // children and their areas.
            myk = make_int4(lc, rc, __float_as_int(ld_cg(g.area + l)), __float_as_int(ld_cg(g.area + r)));
            kids[cbase + cur] = myk;
            if (cnt < gamma) {  // not a treelet root now, nor next iteration
                rec[x] = make_int4(cnt, __float_as_int(my_sah), __float_as_int(my_sah), 0);
            } else {  // the treelet writes the rest
                *rec_i(rec, x, 0) = cnt;
                *rec_f(rec, x, cc) = my_sah;
            }
        }
        unsigned vote = __ballot_sync(kFull, cnt >= gamma);
        rewrote = vote != 0;
        if (vote) __syncwarp();
        while (vote) {
            if (G < 32 && __popc(vote) >= group_min) {
                constexpr int NG = GroupLayout<G>::kGroups;
                const int grp = lane / G;
                unsigned v = vote;
                for (int k = 0; k < grp && v; ++k) v &= v - 1;
                const bool has = grp < NG && v != 0;
                const int rl = has ? __ffs(v) - 1 : 0;
                const int root = __shfl_sync(kFull, cur, rl);
                const float rsah = __shfl_sync(kFull, my_sah, rl);
                const int rbase = __shfl_sync(kFull, base, rl);
                const int rcb = __shfl_sync(kFull, cbase, rl);
                const uint32_t rn = __shfl_sync(kFull, nm, rl);
                const int rts = __shfl_sync(kFull, tsize, rl);
                const int maxts = (int)__reduce_max_sync(kFull, has ? (unsigned)rts : 0u);
                const int4 rk = make_int4(__shfl_sync(kFull, myk.x, rl), __shfl_sync(kFull, myk.y, rl),
                                          __shfl_sync(kFull, myk.z, rl), __shfl_sync(kFull, myk.w, rl));
                const NextRefs nx{rec + rbase, iteration & 1, rts << (iteration + 1), ct};
                process_group<G>(g, has, rbase, rn, root, rk, kids + rcb, nx, rsah, rts, maxts, ci,
                                 &s_mem[w][0] + (grp < NG ? grp : NG - 1) * GroupLayout<G>::kFloats, s_rc, s_prio, err);
#pragma unroll
                for (int k = 0; k < NG; ++k) vote &= vote - 1;
            } else {
                const int rl = __ffs(vote) - 1;
                const int root = __shfl_sync(kFull, cur, rl);
                const float rsah = __shfl_sync(kFull, my_sah, rl);
                const int rbase = __shfl_sync(kFull, base, rl);
                const int rcb = __shfl_sync(kFull, cbase, rl);
                const uint32_t rn = __shfl_sync(kFull, nm, rl);
                const int rts = __shfl_sync(kFull, tsize, rl);
                const int4 rk = make_int4(__shfl_sync(kFull, myk.x, rl), __shfl_sync(kFull, myk.y, rl),
                                          __shfl_sync(kFull, myk.z, rl), __shfl_sync(kFull, myk.w, rl));
                const NextRefs nx{rec + rbase, iteration & 1, rts << (iteration + 1), ct};
                process_group<32>(g, true, rbase, rn, root, rk, kids + rcb, nx, rsah, rts, rts, ci, &s_mem[w][0],
                                  s_rc, s_prio, err);
                vote &= vote - 1;
            }
        }
        if (cur >= 0) cur = up;
    }
}

template <int G>
cudaError_t launch_atrbvh_g(int warps, uint32_t blocks, cudaStream_t s, const TreeRefs& g, const Segs& segs,
                            int4* rec, uint32_t* counters, int4* kids, int tsize, const uint8_t* seg_tsize,
                            const uint8_t* seg_iters, int it, float ci, float ct, int gmin, const uint2* start,
                            const uint32_t* start_count, uint32_t* err) {
    switch (warps) {
        case 2: k_atrbvh<G, 2><<<blocks, 64, 0, s>>>(g, segs, rec, counters, kids, tsize, seg_tsize, seg_iters, it, ci, ct, gmin, start, start_count, err); break;
        case 8: k_atrbvh<G, 8><<<blocks, 256, 0, s>>>(g, segs, rec, counters, kids, tsize, seg_tsize, seg_iters, it, ci, ct, gmin, start, start_count, err); break;
        default: k_atrbvh<G, 4><<<blocks, 128, 0, s>>>(g, segs, rec, counters, kids, tsize, seg_tsize, seg_iters, it, ci, ct, gmin, start, start_count, err); break;
    }
    return cudaGetLastError();
}

// ---- level passes ---------------------------------------------------------------
// A node whose subtree holds at least gamma triangles ("big") is a treelet
// root; its results depend only on its subtree, so any order that finishes a
// node's big descendants first gives the reference's result.  The level of a
// big node is 1 + the largest level of its big children (0 for the others).
// Phase A finishes every node that is not big (subtree count, nodesSah, child
// record) and levels the big ones: k_levels climbs once from every leaf;
// k_levels_pp and k_levels_pp_hist take counts, nodesSah (and levels) from
// the LBVH build.  Phase B files big nodes of levels 1..L into per-level
// lists (in the same pass as the level counts: k_levels_pp_hist for the first
// iteration, k_level_hist for the others); phase C restructures each level's
// treelets in one launch, several per warp in lane groups; the dataflow kernel
// then climbs from the frontier below the levels above L.

constexpr int kMaxLevels = 64;  // largest L (ATR_TUNE_ATR_LEVELS)
constexpr int kListPer = 8;                  // nodes per thread of the level-list kernels
constexpr int kListBlock = 256 * kListPer;  // nodes per block of those kernels

struct LevelRefs {
    int4* rec;             // per node (node-indexed): count, nodesSah x 2, level (see NextRefs)
    int par;               // iteration & 1
    float ct;              // the leaf cost constant (triangle leaves' records)
    uint32_t* counters;
    int4* kids;
    uint32_t* cursor;      // [L + 2]: entries filed per level (the level's count)
    uint2* order;          // (mesh, local node) of big nodes: level l's list at (l - 1) * cap
    uint32_t cap;          // entries per level list (at most n / gamma nodes share a level)
    uint2* frontier;       // climb starts of the dataflow pass
    uint32_t* n_frontier;
    uint32_t* err;
};

constexpr int kLvBlock = 512;  // threads (leaves) per block of the phase-A climb

// Phase A of the first iteration: one climb from every leaf (sorted order)
// that finishes the nodes that are not treelet roots and levels the roots.
// With the radix tree's leaf ranges (a tree straight from the LBVH build), a
// node whose range lies inside the block's leaves is reached only by threads
// of the block, so its arrival counter and the first child's summary live in
// shared memory under block-scope ordering; only nodes whose range crosses a
// block boundary use a device-scope acquire-release atomic in global memory.
// Without ranges every node takes the global path.
__global__ void __launch_bounds__(kLvBlock) k_levels(TreeRefs g, Segs segs, LevelRefs lv, int tsize_all,
                                                     const uint8_t* __restrict__ seg_tsize,
                                                     const uint8_t* __restrict__ seg_iters, int iteration, float ci,
                                                     float ct, int L, const int2* __restrict__ ranges) {
    __shared__ uint32_t s_ctr[kLvBlock];
    __shared__ int4 s_rec[kLvBlock][2];  // per local node and side: (count, level, nodesSah, area)
    for (int k = threadIdx.x; k < kLvBlock; k += blockDim.x) s_ctr[k] = 0;
    __syncthreads();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= segs.n) return;
    const uint32_t m = segs.seg_of_tri(i);
    if (seg_iters && iteration >= (int)seg_iters[m]) return;
    const uint32_t s0 = segs.tri_begin(m);
    const uint32_t n = segs.tri_end(m) - s0;
    const int base = segs.node_base(m), cb = segs.inner_base(m);
    const int gamma = (seg_tsize ? (int)seg_tsize[m] : tsize_all) << iteration;
    const int64_t blo = (int64_t)blockIdx.x * blockDim.x, bhi = blo + blockDim.x - 1;
    const int li = (int)(i - s0);
    const int leaf = base + li + (int)n - 1;
    // Summary of the subtree this thread has just finished (the leaf first).
    const float la = g.area[leaf];
    int my_cnt = 1, my_lvl = 0, my_first = li, child = li + (int)n - 1;
    float my_nsah = __fmul_rn(ct, la), my_area = la;
    lv.rec[leaf] = make_int4(1, __float_as_int(my_nsah), __float_as_int(my_nsah), 0);
    const int cur_c = rec_ns_cur(lv.par);
    int cur = g.parent[leaf];
    while (cur >= 0) {
        const int x = base + cur;
        int sib_cnt, sib_lvl;
        float sib_nsah, sib_area;
        bool local = false;
        if (ranges) {
            const int2 rg = ranges[cb + cur];
            local = (int64_t)s0 + rg.x >= blo && (int64_t)s0 + rg.y <= bhi;
            if (local) {
                // Internal node cur covers [rg.x, rg.y] and is numbered by one
                // of its ends, so its slot lies inside the block.
                const int slot = (int)((int64_t)s0 + cur - blo);
                const int side = my_first == rg.x ? 0 : 1;
                s_rec[slot][side] = make_int4(my_cnt, my_lvl, __float_as_int(my_nsah), __float_as_int(my_area));
                __threadfence_block();
                if (atomicAdd(&s_ctr[slot], 1u) == 0u) return;
                __threadfence_block();
                const int4 r = s_rec[slot][side ^ 1];
                sib_cnt = r.x;
                sib_lvl = r.y;
                sib_nsah = __int_as_float(r.z);
                sib_area = __int_as_float(r.w);
                my_first = rg.x;
            }
        }
        const int lc = ld_cg(g.left + x), rc = ld_cg(g.right + x);
        const int sib = lc == child ? rc : lc;
        if (!local) {
            if (atomic_add_acq_rel_gpu(&lv.counters[cb + cur], 1u) == 0u) return;
            const int4 sr = __ldcg(lv.rec + base + sib);
            sib_cnt = sr.x;
            sib_lvl = is_internal(sib, n) ? sr.w : 0;
            sib_nsah = __int_as_float(cur_c == 1 ? sr.y : sr.z);
            sib_area = ld_cg(g.area + base + sib);
            if (ranges) my_first = min(my_first, ranges[cb + cur].x);
        }
        const bool mine_left = lc == child;
        const int cnt = my_cnt + sib_cnt;
        const float a = ld_cg(g.area + x);
        lv.kids[cb + cur] = make_int4(lc, rc, __float_as_int(mine_left ? my_area : sib_area),
                                      __float_as_int(mine_left ? sib_area : my_area));
        int lvl = 0;
        float ns = 0.0f;
        if (cnt < gamma) {
            ns = __fadd_rn(__fadd_rn(__fmul_rn(ci, a), mine_left ? my_nsah : sib_nsah), mine_left ? sib_nsah : my_nsah);
            lv.rec[x] = make_int4(cnt, __float_as_int(ns), __float_as_int(ns), 0);
        } else {
            lvl = 1 + max(my_lvl, sib_lvl);
            *rec_i(lv.rec, x, 0) = cnt;
            *rec_i(lv.rec, x, 3) = lvl;
        }
        my_cnt = cnt;
        my_lvl = lvl;
        my_nsah = ns;  // only read while the climb stays below the treelet roots (cnt < gamma)
        my_area = a;
        child = cur;
        cur = g.parent[x];
    }
}

// Phase A of the first iteration on a tree straight from the LBVH build,
// which left every node's nodesSah for the default constants: subtree counts
// come from the radix tree's leaf ranges, so a streaming pass (one thread per
// leaf and internal node) writes counts and child records, finishes the nodes
// that are not treelet roots, and starts a climb at every treelet root whose
// children are not roots (level 1).  The climbs visit treelet roots only and
// wait at a root only when both of its children are roots.
__global__ void __launch_bounds__(256) k_levels_pp(TreeRefs g, Segs segs, LevelRefs lv, const int2* __restrict__ ranges,
                                                   int tsize_all, const uint8_t* __restrict__ seg_tsize,
                                                   const uint8_t* __restrict__ seg_iters, int iteration,
                                                   bool levels_known) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= segs.n) return;
    const uint32_t m = segs.seg_of_tri(i);
    if (seg_iters && iteration >= (int)seg_iters[m]) return;
    const uint32_t s0 = segs.tri_begin(m);
    const uint32_t n = segs.tri_end(m) - s0;
    const int base = segs.node_base(m), cb = segs.inner_base(m);
    const int gamma = (seg_tsize ? (int)seg_tsize[m] : tsize_all) << iteration;
    const int li = (int)(i - s0);
    // Leaves: the build's records are final (count 1, both nodesSah, level 0).
    if (li >= (int)n - 1) return;
    auto count = [&](int c) {
        if (!is_internal(c, n)) return 1;
        const int2 r = ranges[cb + c];
        return r.y - r.x + 1;
    };
    int x = li;
    const int lc = g.left[base + x], rc = g.right[base + x];
    const int cnt = count(x);
    lv.kids[cb + x] = make_int4(lc, rc, __float_as_int(g.area[base + lc]), __float_as_int(g.area[base + rc]));
    if (cnt < gamma) {
        const int ns = *rec_i(lv.rec, base + x, 1);  // the build's nodesSah (even iterations)
        lv.rec[base + x] = make_int4(cnt, ns, ns, 0);
        return;
    }
    if (levels_known) return;  // the build left every level in the records
    if (count(lc) >= gamma || count(rc) >= gamma) return;  // not a level-1 root: reached by a climb
    int lvl = 1;
    while (true) {
        *rec_i(lv.rec, base + x, 3) = lvl;
        const int p = g.parent[base + x];
        if (p < 0) return;
        const int pl = g.left[base + p];
        const int o = pl == x ? g.right[base + p] : pl;
        int olvl = 0;
        if (count(o) >= gamma) {
            if (atomic_add_acq_rel_gpu(&lv.counters[cb + p], 1u) == 0u) return;
            olvl = ld_cg(rec_i(lv.rec, base + o, 3));
        }
        lvl = 1 + max(lvl, olvl);
        x = p;
    }
}

// Phase A of the first iteration when the LBVH build left the levels too:
// one streaming pass writes the counts, child records and next-iteration
// values of the nodes that are not big, counts the levels 1..L and lists
// the frontier below the levels above L (k_level_hist's work as well).
// Files a block's nodes of levels 1..L into the level lists: thread-held
// levels me[q] (0: none) and entries ent[q].  Ranks within the block come from
// one shared atomic per level present in a warp (__match_any_sync), then one
// global reservation per level per block on lv.cursor (which ends as the
// level's count).  Nodes of one level have disjoint subtrees of at least gamma
// triangles each, so a list holds at most lv.cap of them; a reservation past
// that sets kErrLevelList and writes nothing.  Every thread of the block calls
// it; s_cnt holds L + 2 zeroed counters.
__device__ __forceinline__ void file_levels(const LevelRefs& lv, int L, const int (&me)[kListPer],
                                            const uint2 (&ent)[kListPer], uint32_t* s_cnt, uint32_t* s_base) {
    const int lane = threadIdx.x & 31;
    uint32_t key[kListPer];
#pragma unroll
    for (int q = 0; q < kListPer; ++q) {
        const uint32_t peers = __match_any_sync(kFull, me[q]);
        const int leader = __ffs(peers) - 1;
        uint32_t b = 0;
        if (lane == leader && me[q] > 0) b = atomicAdd(&s_cnt[me[q]], (uint32_t)__popc(peers));
        b = __shfl_sync(kFull, b, leader) + (uint32_t)__popc(peers & ((1u << lane) - 1u));
        key[q] = me[q] > 0 ? ((uint32_t)me[q] << 16) | b : 0u;  // rank < kListBlock
    }
    __syncthreads();
    for (int k = threadIdx.x; k < L + 2; k += blockDim.x)
        s_base[k] = s_cnt[k] ? atomicAdd(&lv.cursor[k], s_cnt[k]) : 0u;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kListPer; ++q)
        if (key[q]) {
            const uint32_t l = key[q] >> 16;
            const uint32_t at = s_base[l] + (key[q] & 0xffffu);
            if (at < lv.cap) lv.order[(size_t)(l - 1) * lv.cap + at] = ent[q];
            else set_error_bits(lv.err, kErrLevelList);
        }
}

__global__ void __launch_bounds__(256) k_levels_pp_hist(TreeRefs g, Segs segs, LevelRefs lv,
                                                        const int2* __restrict__ ranges, int tsize_all,
                                                        const uint8_t* __restrict__ seg_tsize,
                                                        const uint8_t* __restrict__ seg_iters, int L) {
    __shared__ uint32_t s_cnt[kMaxLevels + 2];
    __shared__ uint32_t s_base[kMaxLevels + 2];
    for (int k = threadIdx.x; k < L + 2; k += blockDim.x) s_cnt[k] = 0;
    __syncthreads();
    int lvl[kListPer];
    uint2 lent[kListPer];
#pragma unroll
    for (int q = 0; q < kListPer; ++q) {
        const uint32_t i = blockIdx.x * kListBlock + q * 256 + threadIdx.x;
        int push = 0;
        uint2 ent[2];
        lvl[q] = 0;
        lent[q] = make_uint2(0u, 0u);
        if (i < segs.n) {
            const uint32_t m = segs.seg_of_tri(i);
            const uint32_t s0 = segs.tri_begin(m);
            const uint32_t n = segs.tri_end(m) - s0;
            if (!seg_iters || 0 < (int)seg_iters[m]) {
                const int base = segs.node_base(m), cb = segs.inner_base(m);
                const int gamma = seg_tsize ? (int)seg_tsize[m] : tsize_all;
                const int li = (int)(i - s0);
                // The build's records are final for every node below gamma (count,
                // both nodesSah, level 0) and hold the level of the others.
                if (li < (int)n - 1) {
                    const int x = li;
                    const int lc = g.left[base + x], rc = g.right[base + x];
                    const int2 r = ranges[cb + x];
                    const int cnt = r.y - r.x + 1;
                    lv.kids[cb + x] =
                        make_int4(lc, rc, __float_as_int(g.area[base + lc]), __float_as_int(g.area[base + rc]));
                    if (cnt >= gamma) {
                        const int me = *rec_i(lv.rec, base + x, 3);
                        if (me <= L) {
                            lvl[q] = me;
                            lent[q] = make_uint2(m, (uint32_t)x);
                        } else {
                            if ((is_internal(lc, n) ? *rec_i(lv.rec, base + lc, 3) : 0) <= L)
                                ent[push++] = make_uint2(m, (uint32_t)lc);
                            if ((is_internal(rc, n) ? *rec_i(lv.rec, base + rc, 3) : 0) <= L)
                                ent[push++] = make_uint2(m, (uint32_t)rc);
                        }
                    }
                }
            }
        }
        // Frontier entries: one atomic per warp.
        uint32_t incl = push;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, incl, o);
            if ((threadIdx.x & 31) >= o) incl += y;
        }
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        uint32_t at = 0;
        if ((threadIdx.x & 31) == 31 && total) at = atomicAdd(lv.n_frontier, total);
        at = __shfl_sync(kFull, at, 31) + incl - push;
        for (int k = 0; k < push; ++k) lv.frontier[at + k] = ent[k];
    }
    file_levels(lv, L, lvl, lent, s_cnt, s_base);
}

// Phase A of iterations after the first: the previous iteration left every
// internal node's level for this one (next levels of the nodes it finished,
// kept current by treelet rewrites), and subtree counts, nodesSah and child
// records that are already final for nodes that are not treelet roots now.
// Count the levels, mark this iteration's non-roots as non-roots for the next
// one too, and list the frontier below the levels above L.
__global__ void __launch_bounds__(256) k_level_hist(Segs segs, LevelRefs lv, const uint8_t* __restrict__ seg_iters,
                                                    int iteration, int L) {
    __shared__ uint32_t s_cnt[kMaxLevels + 2];
    __shared__ uint32_t s_base[kMaxLevels + 2];
    for (int k = threadIdx.x; k < L + 2; k += blockDim.x) s_cnt[k] = 0;
    __syncthreads();
    int lvl[kListPer];
    uint2 lent[kListPer];
#pragma unroll
    for (int q = 0; q < kListPer; ++q) {
        const uint32_t i = blockIdx.x * kListBlock + q * 256 + threadIdx.x;
        int push = 0;
        uint32_t m = 0;
        uint2 ent[2];
        lvl[q] = 0;
        lent[q] = make_uint2(0u, 0u);
        if (i < segs.n) {
            m = segs.seg_of_tri(i);
            const uint32_t s0 = segs.tri_begin(m);
            const uint32_t n = segs.tri_end(m) - s0;
            const uint32_t li = i - s0;
            if ((!seg_iters || iteration < (int)seg_iters[m]) && li < n - 1) {
                const int cb = segs.inner_base(m), nb = segs.node_base(m);
                const int me = *rec_i(lv.rec, nb + (int)li, 3);
                if (me == 0) {
                    // Not a treelet root: its next nodesSah is this one (the level
                    // stays 0).
                    *rec_f(lv.rec, nb + (int)li, rec_ns_next(lv.par)) = *rec_f(lv.rec, nb + (int)li, rec_ns_cur(lv.par));
                } else if (me <= L) {
                    lvl[q] = me;
                    lent[q] = make_uint2(m, li);
                } else {
                    const int4 kd = lv.kids[cb + (int)li];
                    if ((is_internal(kd.x, n) ? *rec_i(lv.rec, nb + kd.x, 3) : 0) <= L)
                        ent[push++] = make_uint2(m, (uint32_t)kd.x);
                    if ((is_internal(kd.y, n) ? *rec_i(lv.rec, nb + kd.y, 3) : 0) <= L)
                        ent[push++] = make_uint2(m, (uint32_t)kd.y);
                }
            }
        }
        // Frontier entries: one atomic per warp.
        uint32_t incl = push;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, incl, o);
            if ((threadIdx.x & 31) >= o) incl += y;
        }
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        uint32_t at = 0;
        if ((threadIdx.x & 31) == 31 && total) at = atomicAdd(lv.n_frontier, total);
        at = __shfl_sync(kFull, at, 31) + incl - push;
        for (int k = 0; k < push; ++k) lv.frontier[at + k] = ent[k];
    }
    file_levels(lv, L, lvl, lent, s_cnt, s_base);
}

// ---- quads: eight treelets per warp ----------------------------------------
// The first levels hold most treelets (a quarter of a million in the first
// level of a four-million-triangle scene) and the level pass is bound by
// instruction issue.  There a group of four lanes restructures a treelet of
// up to KL leaves, lane l owning leaves l, l + 4, ...: the searches and
// updates are strided over four lanes and the reductions are two butterfly
// steps, so a warp instruction serves eight treelets instead of three.  Same
// operations, operands and order as process_group (same tie rules), hence the
// same results bit for bit.
template <int KL>
struct QuadLayout {
    static constexpr int kDist = KL * (KL - 1) / 2;
    static constexpr int kDistPad = (kDist + 3) & ~3;
    // dist, then per leaf slot three float4 (as GroupLayout), then the
    // treelet's internal nodes.
    static constexpr int kFloats = kDistPad + 12 * KL + ((KL + 3) & ~3);
};
constexpr int kQuadLeaves = 10;  // largest treelet the quad path takes

template <int KL>
__device__ __forceinline__ void process_quad(const TreeRefs& g, bool active, int nb, uint32_t n, int root,
                                             int4 rk, int4* KD, const NextRefs& nx, float root_sah, int tsize,
                                             int maxts,
                                             float ci, float* sm, const uint16_t* __restrict__ s_rc,
                                             const uint8_t* __restrict__ s_prio, uint32_t* err) {
    using Lay = QuadLayout<KL>;
    const int lane = threadIdx.x & 31;
    const int gb = lane & ~3;
    const int gl = lane & 3;
    const uint32_t gmask = 0xfu << gb;
    int32_t* const P = g.parent + nb;
    int32_t* const Lf = g.left + nb;
    int32_t* const Rt = g.right + nb;
    float4* const BMN = g.bmin + nb;
    float4* const BMX = g.bmax + nb;
    float* const AR = g.area + nb;
    const int next_c = rec_ns_next(nx.par);
    float* const dist = sm;
    float4* const lmn = reinterpret_cast<float4*>(sm + Lay::kDistPad);
    float4* const lmx = lmn + KL;
    int4* const lcn = reinterpret_cast<int4*>(lmx + KL);
    int* const inner = reinterpret_cast<int*>(lcn + KL);
    int4* const krec = lcn;  // child-record slots during formation

    // ---- formTreelet (Treelet.cuh:57-114) ----
    // Slot k's node and area sit in lmx[k].w and lmn[k].w while the treelet
    // grows; the owner lane (k mod 4) copies an internal leaf's child record
    // into krec[k] with cp.async and is the only lane that waits for it.
    auto join = [&](int k, int node, float area) {
        lmx[k].w = __int_as_float(node);
        lmn[k].w = area;
        if (is_internal(node, n)) cp_async16_cg(krec + k, KD + node);
    };
    if (active) {
        if (gl == 0) {
            join(0, rk.x, __int_as_float(rk.z));
            inner[0] = root;
        }
        if (gl == 1) join(1, rk.y, __int_as_float(rk.w));
    }
    __syncwarp();
    bool ok = true;
    for (int it = 0; it < maxts - 2; ++it) {
        const bool act = active && ok && it < tsize - 2;
        const int m = 2 + it;
        // Largest area among internal leaves (others -FLT_MAX), ties to the
        // lowest rank of the reference's reduction tree over m lanes.
        float bv = -FLT_MAX;
        int bk = gl < m ? gl : 0, brk = 255;
        for (int k = gl; k < m; k += 4) {
            const float v = is_internal(__float_as_int(lmx[k].w), n) ? lmn[k].w : -FLT_MAX;
            const int rk = s_prio[m * 32 + k];
            if (brk == 255 || v > bv || (v == bv && rk < brk)) {
                bv = v;
                bk = k;
                brk = rk;
            }
        }
#pragma unroll
        for (int o = 1; o <= 2; o <<= 1) {
            const float ov = __shfl_xor_sync(kFull, bv, o);
            const int opk = __shfl_xor_sync(kFull, (brk << 8) | bk, o);
            const int ork = opk >> 8;
            if (ov > bv || (ov == bv && ork < brk)) {
                bv = ov;
                bk = opk & 255;
                brk = ork;
            }
        }
        const int largest = bk;
        const int rep = act ? __float_as_int(lmx[largest].w) : -1;
        const bool expand = act && is_internal(rep, n);
        if (expand && gl == (largest & 3)) cp_async_wait_all();
        __syncwarp();
        int4 rk = make_int4(-1, -1, 0, 0);
        if (expand) rk = krec[largest];
        __syncwarp();
        if (act) {
            if (!expand) {
                ok = false;
            } else {
                if (gl == 0) inner[it + 1] = rep;
                if (gl == (largest & 3)) join(largest, rk.x, __int_as_float(rk.z));
                if (gl == (m & 3)) join(m, rk.y, __int_as_float(rk.w));
            }
        }
        __syncwarp();
    }
    const bool run = active && ok;
    if (active && !ok && gl == 0) set_error_bits(err, kErrTreeletClimb);
    cp_async_wait_all();
    __syncwarp();

    // ---- leaf data and distance matrix (AgglomerativeTreelet.cu:18-63) ----
    // Slot k: (min.xyz, nodesSah), (max.xyz, node), (count, next level,
    // next nodesSah, -); a retired slot holds the new node of its step:
    // (min.xyz, cost), (max.xyz, left child), (count, next level, next
    // nodesSah, right child).
    // A lane's leaves arrive by cp.async, all in flight at once: boxes into
    // lmn/lmx and the node's record into lcn, which the lane then rearranges
    // (this iteration's nodesSah to lmn.w).  Nothing else in this level pass
    // writes a treelet leaf's records.
    {
        int node[3];
        float area[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const int k = gl + 4 * q;
            node[q] = run && k < tsize ? __float_as_int(lmx[k].w) : -1;
            area[q] = node[q] >= 0 ? lmn[k].w : 0.0f;
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            if (node[q] < 0) continue;
            const int k = gl + 4 * q;
            cp_async16_cg(lmn + k, BMN + node[q]);
            cp_async16_cg(lmx + k, BMX + node[q]);
            // A triangle's record follows from its area: not fetched.
            if (is_internal(node[q], n)) cp_async16_cg(lcn + k, nx.rec + node[q]);
        }
        cp_async_wait_all();
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            if (node[q] < 0) continue;
            const int k = gl + 4 * q;
            lmx[k].w = __int_as_float(node[q]);
            if (is_internal(node[q], n)) {
                const int4 r = lcn[k];
                lmn[k].w = __int_as_float(nx.par ? r.z : r.y);
                lcn[k] = make_int4(r.x, r.w, nx.par ? r.y : r.z, 0);
            } else {
                const float ns = __fmul_rn(nx.ct, area[q]);
                lmn[k].w = ns;
                lcn[k] = make_int4(1, 0, __float_as_int(ns), 0);
            }
        }
    }
    __syncwarp();
    if (run) {
        const int np = tsize * (tsize - 1) / 2;
        for (int j = gl; j < np; j += 4) {
            const uint32_t rc = s_rc[j];
            const float4 a0 = lmn[rc >> 8], a1 = lmx[rc >> 8], b0 = lmn[rc & 255u], b1 = lmx[rc & 255u];
            dist[j] = union_area3(a0.x, a0.y, a0.z, a1.x, a1.y, a1.z, b0.x, b0.y, b0.z, b1.x, b1.y, b1.z);
        }
    }
    __syncwarp();

    // ---- agglomerative merge (AgglomerativeTreelet.cu:476-532) ----
    for (int step = 0; step < maxts - 1; ++step) {
        const int last = tsize - 1 - step;
        const bool act = run && last >= 1;
        const int msize = act ? last * (last + 1) / 2 : 0;
        // findMinimumDistance as in process_group: distances alone unless the
        // group minimum is held twice; then the exact key.
        uint32_t bd = 0xffffffffu;
        int bj = 0;
        bool tie = false;
        for (int j = gl; j < msize; j += 4) {
            uint32_t d = __float_as_uint(dist[j]);
            d = d < 0x7f7fffffu ? d : 0xffffffffu;
            if (d < bd) {
                bd = d;
                bj = j;
                tie = false;
            } else if (d == bd) {
                tie = true;
            }
        }
        uint32_t dmin = min(bd, __shfl_xor_sync(kFull, bd, 1));
        dmin = min(dmin, __shfl_xor_sync(kFull, dmin, 2));
        const bool holds = bd == dmin && dmin != 0xffffffffu;
        const uint32_t holders = __ballot_sync(kFull, holds) & gmask;
        const bool tied = (__ballot_sync(kFull, holds && tie) & gmask) != 0u || __popc(holders) > 1;
        int mi = __shfl_sync(kFull, bj, holders ? __ffs(holders) - 1 : gb);
        if (!holders) mi = 0;
        if (__any_sync(kFull, tied)) {
            unsigned long long best = ~0ull;
            for (int j = gl; j < msize; j += 4) {
                const float d = dist[j];
                if (d < FLT_MAX) {
                    const unsigned long long k = ((unsigned long long)__float_as_uint(d) << 32) |
                                                 (uint32_t)(((__brev((uint32_t)j) >> 27) << 8) | (uint32_t)j);
                    best = k < best ? k : best;
                }
            }
#pragma unroll
            for (int o = 1; o <= 2; o <<= 1) {
                const unsigned long long ob = __shfl_xor_sync(kFull, best, o);
                best = ob < best ? ob : best;
            }
            if (tied) mi = best == ~0ull ? 0 : (int)(best & 255u);
        }
        // updateState (:101-150): the new node takes slot jc, the last leaf
        // moves to slot jr, slot `last` retires with the new node.  Lanes 0,
        // 1 and 2 of the group write those three slots.
        int jr = 0, jc = 0;
        float a0x = 0.f, a0y = 0.f, a0z = 0.f, a1x = 0.f, a1y = 0.f, a1z = 0.f;
        float4 w0 = make_float4(0.f, 0.f, 0.f, 0.f), w1 = w0;
        int4 w2 = make_int4(0, 0, 0, 0);
        int wslot = -1;
        float ral = 0.f, rar = 0.f;
        if (act) {
            const uint32_t rc = s_rc[mi];
            jr = (int)(rc >> 8);
            jc = (int)(rc & 255u);
            const int new_internal = inner[last - 1];
            const float4 r0 = lmn[jr], r1 = lmx[jr], c0 = lmn[jc], c1 = lmx[jc];
            const int4 r2 = lcn[jr], c2 = lcn[jc];
            a0x = fminf(c0.x, r0.x); a0y = fminf(c0.y, r0.y); a0z = fminf(c0.z, r0.z);
            a1x = fmaxf(c1.x, r1.x); a1y = fmaxf(c1.y, r1.y); a1z = fmaxf(c1.z, r1.z);
            const float area_new = box_area(a0x, a0y, a0z, a1x, a1y, a1z);
            const float la = __fadd_rn(__fadd_rn(r0.w, c0.w), __fmul_rn(ci, area_new));
            const int cnt = r2.x + c2.x;
            const float nsn = __fadd_rn(__fadd_rn(__fmul_rn(ci, area_new), __int_as_float(r2.z)), __int_as_float(c2.z));
            const int nlv = cnt >= nx.gamma ? 1 + max(r2.y, c2.y) : 0;
            if (gl == 0) {  // slot jc: the new node
                wslot = jc;
                w0 = make_float4(a0x, a0y, a0z, la);
                w1 = make_float4(a1x, a1y, a1z, __int_as_float(new_internal));
                w2 = make_int4(cnt, nlv, __float_as_int(nsn), 0);
            } else if (gl == 1) {  // slot jr: the last leaf (nothing when jr is last)
                if (jr != last) {
                    wslot = jr;
                    w0 = lmn[last];
                    w1 = lmx[last];
                    w2 = lcn[last];
                }
            } else if (gl == 2) {  // slot last: retired, left = row jr, right = column jc
                wslot = last;
                w0 = make_float4(a0x, a0y, a0z, la);
                w1 = make_float4(a1x, a1y, a1z, r1.w);
                w2 = make_int4(cnt, nlv, __float_as_int(nsn), __float_as_int(c1.w));
                // The children's areas (their boxes' surface areas, as the
                // area array holds them) for the child record at the rewrite.
                ral = box_area(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z);
                rar = box_area(c0.x, c0.y, c0.z, c1.x, c1.y, c1.z);
            }
        }
        // updateDistancesMatrix (:152-188): row `last` moves to row jr, then
        // the distances to the new node at jc are recomputed.
        const bool du = act && last > 1;
        float mv[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const int c = gl + 4 * q;
            if (du && c < last && c != jr) mv[q] = dist[trm_idx(last, c)];
        }
        __syncwarp();
        if (wslot >= 0) {
            lmn[wslot] = w0;
            lmx[wslot] = w1;
            lcn[wslot] = w2;
        }

#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const int c = gl + 4 * q;
            if (du && c < last && c != jr) dist[trm_idx(max(jr, c), min(jr, c))] = mv[q];
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const int c = gl + 4 * q;
            if (du && c < last && c != jc) {
                const float4 b0 = lmn[c], b1 = lmx[c];
                dist[trm_idx(max(jc, c), min(jc, c))] =
                    union_area3(a0x, a0y, a0z, a1x, a1y, a1z, b0.x, b0.y, b0.z, b1.x, b1.y, b1.z);
            }
        }
        // The retired node's child areas for the rewrite: in row `last` of the
        // matrix, dead now (slot 1's, the final step's, in slot 0, which the
        // rewrite does not read).
        if (act && gl == 2) {
            float* const ca = last >= 2 ? dist + trm_idx(last, 0) : reinterpret_cast<float*>(lmn);
            ca[0] = ral;
            ca[1] = rar;
        }
        __syncwarp();
    }

    // ---- updateTreelet (:190-212) ----
    const bool accept = run && lmn[1].w < root_sah;
    int fls[3], frs[3], nis[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const int sl = 1 + gl + 4 * q;
        nis[q] = -1;
        if (accept && sl < tsize) {
            const float4 f0 = lmn[sl], f1 = lmx[sl];
            const int4 f2 = lcn[sl];
            const int ni = inner[sl - 1];
            const int fl = __float_as_int(f1.w), fr = f2.w;
            nis[q] = ni;
            fls[q] = fl;
            frs[q] = fr;
            Lf[ni] = fl;
            Rt[ni] = fr;
            P[fl] = ni;
            P[fr] = ni;
            const float4 mn = make_float4(f0.x, f0.y, f0.z, 0.0f);
            const float4 mx = make_float4(f1.x, f1.y, f1.z, 0.0f);
            BMN[ni] = mn;
            BMX[ni] = mx;
            AR[ni] = box_area(mn, mx);
            nx.rec[ni] = make_rec(f2.x, f0.w, __int_as_float(f2.z), f2.y, nx.par);
        }
    }
    __syncwarp();
    // The rewritten nodes' child records, with the child areas kept in the
    // dead matrix rows.
#pragma unroll
    for (int q = 0; q < 3; ++q)
        if (nis[q] >= 0) {
            const int sl = 1 + gl + 4 * q;
            const float* const ca = sl >= 2 ? dist + trm_idx(sl, 0) : reinterpret_cast<const float*>(lmn);
            KD[nis[q]] = make_int4(fls[q], frs[q], __float_as_int(ca[0]), __float_as_int(ca[1]));
        }
    // A treelet left as it was: its root's next level and next nodesSah.
    if (run && !accept && gl == 0) {
        const int lc = ld_cg(Lf + root), rc = ld_cg(Rt + root);
        const int4 rl = __ldcg(nx.rec + lc), rr = __ldcg(nx.rec + rc);
        const int a = is_internal(lc, n) ? rl.w : 0;
        const int b = is_internal(rc, n) ? rr.w : 0;
        *rec_i(nx.rec, root, 3) = ld_cg(rec_i(nx.rec, root, 0)) >= nx.gamma ? 1 + max(a, b) : 0;
        *rec_f(nx.rec, root, next_c) =
            __fadd_rn(__fadd_rn(__fmul_rn(ci, ld_cg(AR + root)), __int_as_float(next_c == 1 ? rl.y : rl.z)),
                      __int_as_float(next_c == 1 ? rr.y : rr.z));
    }
    __syncwarp();
}

// Phase C: every treelet root of level `lev`.  Each warp takes `per` roots
// at a time: 32/G in lane groups of G, or (QUADS) eight in four-lane groups.
template <int G, int W, bool QUADS>
__global__ void __launch_bounds__(W * 32, (G == 32 ? 16 : 32) / W) k_level_groups(TreeRefs g, Segs segs, LevelRefs lv, int lev,
                                                                 int tsize_all, const uint8_t* __restrict__ seg_tsize,
                                                                 int iteration, float ci, uint32_t* err) {
    constexpr int per = QUADS ? 8 : GroupLayout<G>::kGroups;
    constexpr int kGroupFloats = QUADS ? QuadLayout<kQuadLeaves>::kFloats : GroupLayout<G>::kFloats;
    __shared__ __align__(16) float s_mem[W][kGroupFloats * per];
    __shared__ uint16_t s_rc[kMaxDist];
    __shared__ __align__(4) uint8_t s_prio[(kMaxTreelet + 1) * 32];
    const uint32_t beg = (uint32_t)(lev - 1) * lv.cap;
    const uint32_t end = beg + min(lv.cursor[lev], lv.cap);
    if (beg + blockIdx.x * (uint32_t)(W * per) >= end) return;  // no root for this block
    for (int k = threadIdx.x; k < kMaxDist; k += blockDim.x) {
        int r, c;
        trm_rc(k, r, c);
        s_rc[k] = (uint16_t)((r << 8) | c);
    }
    for (int k = threadIdx.x; k < (kMaxTreelet + 1) * 8; k += blockDim.x)
        reinterpret_cast<uint32_t*>(s_prio)[k] = reinterpret_cast<const uint32_t*>(&g_argmax_priority.rank[0][0])[k];
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int gw = QUADS ? 4 : G;
    const int grp = lane / gw;
    const uint32_t warp = blockIdx.x * W + w, nwarps = gridDim.x * W;
    for (uint32_t e0 = beg + warp * per; e0 < end; e0 += nwarps * per) {
        const uint32_t e = e0 + (uint32_t)grp;
        const bool has = grp < per && e < end;
        int nb = 0, x = 0, tsize = 0;
        uint32_t n = 2;
        int4* kd = lv.kids;
        float root_sah = 0.0f;
        int4 rk = make_int4(-1, -1, 0, 0);
        const int cur_c = rec_ns_cur(lv.par);
        if (has) {
            const uint2 q = lv.order[e];
            const uint32_t s0 = segs.tri_begin(q.x);
            n = segs.tri_end(q.x) - s0;
            nb = segs.node_base(q.x);
            kd = lv.kids + segs.inner_base(q.x);
            x = (int)q.y;
            tsize = seg_tsize ? (int)seg_tsize[q.x] : tsize_all;
            rk = __ldcg(kd + x);
            root_sah = __fadd_rn(__fadd_rn(__fmul_rn(ci, __ldcg(g.area + nb + x)), ld_cg(rec_f(lv.rec, nb + rk.x, cur_c))),
                                 ld_cg(rec_f(lv.rec, nb + rk.y, cur_c)));
            if (lane == grp * gw) *rec_f(lv.rec, nb + x, cur_c) = root_sah;
        }
        const int maxts = (int)__reduce_max_sync(kFull, has ? (unsigned)tsize : 0u);
        __syncwarp();
        const NextRefs nx{lv.rec + nb, lv.par, tsize << (iteration + 1), lv.ct};
        float* const sm = &s_mem[w][0] + (grp < per ? grp : per - 1) * kGroupFloats;
        if constexpr (QUADS)
            process_quad<kQuadLeaves>(g, has, nb, n, x, rk, kd, nx, root_sah, tsize, maxts, ci, sm, s_rc, s_prio,
                                      err);
        else
            process_group<G>(g, has, nb, n, x, rk, kd, nx, root_sah, tsize, maxts, ci, sm, s_rc, s_prio, err);
    }
}

template <int G, bool QUADS>
void launch_level_g(int warps, unsigned blocks, cudaStream_t s, const TreeRefs& g, const Segs& segs,
                    const LevelRefs& lv, int lev, int tsize, const uint8_t* seg_tsize, int it, float ci,
                    uint32_t* err) {
    switch (warps) {
        case 2: k_level_groups<G, 2, QUADS><<<blocks, 64, 0, s>>>(g, segs, lv, lev, tsize, seg_tsize, it, ci, err); break;
        case 8: k_level_groups<G, 8, QUADS><<<blocks, 256, 0, s>>>(g, segs, lv, lev, tsize, seg_tsize, it, ci, err); break;
        default: k_level_groups<G, 4, QUADS><<<blocks, 128, 0, s>>>(g, segs, lv, lev, tsize, seg_tsize, it, ci, err); break;
    }
}

}  // namespace

// Lane-group width for treelets of at most max_tsize leaves.
int atrbvh_group_width(int max_tsize) {
    return max_tsize <= 8 ? 8 : max_tsize <= 10 ? 10 : max_tsize <= 16 ? 16 : 32;
}

// ATRBVH over every mesh of `segs` (total_nodes = sum of 2n_m - 1).  tsize and
// iterations apply to all meshes unless per-mesh arrays are given, in which
// case `iterations` is their maximum and max_tsize the largest per-mesh size.
int atrbvh_run(atr_ctx* ctx, const TreeRefs& g_in, const Segs& segs, size_t total_nodes, int tsize,
               int max_tsize, int iterations, const uint8_t* seg_tsize, const uint8_t* seg_iters, float ci,
               float ct, const int2* karras_ranges, const BuildPrepass* prepass) {
    if (iterations <= 0) return ATR_OK;
    const size_t inner = segs.n - segs.count;
    const int max_ts = seg_tsize ? max_tsize : tsize;
    const int L = ctx->atr_levels;
    void* scratch = nullptr;
    const size_t b_rec = align256(total_nodes * 16), b_ctr = align256(inner * 4);
    const size_t b_kid = align256(inner * 16);
    // Big nodes of one level root disjoint subtrees of at least gamma
    // triangles (the first iteration's gamma, the smallest; 3 bounds per-mesh
    // sizes), so each level's list holds at most n / gamma; frontier nodes
    // root disjoint subtrees too, so they number at most the triangles.
    const uint32_t gamma0 = seg_tsize ? 3u : (uint32_t)tsize;
    const uint32_t cap = (segs.n + gamma0 - 1) / gamma0;
    const size_t b_ord = L ? align256((size_t)L * cap * 8) : 0;
    const size_t b_front = L ? align256((size_t)segs.n * 8) : 0;
    const size_t b_small = L ? align256((size_t)((L + 2) + 1) * 4) : 0;
    // The build's prepass records (counts, first nodesSah, levels) serve as
    // the optimiser's records when its constants are this pass's.
    const bool use_pp = prepass && prepass->rec && karras_ranges && L > 0 && ci == kPrepassCi && ct == kPrepassCt;
    // ... and its levels serve as the first iteration's when its gamma is this
    // pass's treelet size (per mesh, when the sizes are per mesh).
    const bool use_pp_levels = use_pp && (seg_tsize ? prepass->seg_gamma == seg_tsize
                                                    : !prepass->seg_gamma && tsize == prepass->gamma);
    ATR_TRY(ctx->alloc(&scratch, (use_pp ? 0 : b_rec) + b_kid + b_ctr + b_ord + b_front + b_small));
    char* p = static_cast<char*>(scratch);
    TreeRefs g = g_in;
    int4* rec;
    if (use_pp) {
        rec = prepass->rec;
    } else {
        rec = reinterpret_cast<int4*>(p);
        p += b_rec;
    }
    int4* kids = reinterpret_cast<int4*>(p); p += b_kid;
    uint32_t* counters = reinterpret_cast<uint32_t*>(p); p += b_ctr;
    LevelRefs lv{};
    lv.rec = rec;
    lv.counters = counters;
    lv.kids = kids;
    if (L) {
        lv.order = reinterpret_cast<uint2*>(p); p += b_ord;
        lv.cap = cap;
        lv.err = ctx->d_error;
        lv.frontier = reinterpret_cast<uint2*>(p); p += b_front;
        lv.cursor = reinterpret_cast<uint32_t*>(p);
        lv.n_frontier = lv.cursor + (L + 2);
    }
    const int warps = ctx->atr_warps == 2 || ctx->atr_warps == 4 ? ctx->atr_warps : 8;
    const int threads = warps * 32;
    const uint32_t leaf_blocks = (segs.n + threads - 1) / threads;
    const uint32_t front_blocks = (uint32_t)ctx->num_sms * (256 / threads) * 4;  // grid-stride over the frontier
    const int gw = atrbvh_group_width(max_ts);
    const int gmin = ctx->atr_group_min < 2 ? 2 : ctx->atr_group_min;
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaSuccess;
    ctx->phase_begin("atrbvh");
    for (int it = 0; it < iterations && e == cudaSuccess; ++it) {
        lv.par = it & 1;
        lv.ct = ct;
        const bool hist_done = L && it == 0 && use_pp_levels;
        // Arrival counters: for the first iteration's climbs, else only for
        // the dataflow pass (cleared again below).
        if (!L || (it == 0 && !hist_done)) e = cudaMemsetAsync(counters, 0, inner * 4, st);
        const uint2* start = nullptr;
        const uint32_t* start_count = nullptr;
        uint32_t blocks = leaf_blocks;
        if (L && e == cudaSuccess) {
            if (zero_words_async(ctx, lv.cursor, b_small / 4) != ATR_OK) e = cudaErrorLaunchFailure;
            const unsigned gb = (segs.n + 255) / 256;
            const unsigned gbl = (segs.n + kListBlock - 1) / kListBlock;
            if (hist_done)
                k_levels_pp_hist<<<gbl, 256, 0, st>>>(g, segs, lv, karras_ranges, tsize, seg_tsize, seg_iters, L);
            else if (it == 0 && use_pp)
                k_levels_pp<<<gb, 256, 0, st>>>(g, segs, lv, karras_ranges, tsize, seg_tsize, seg_iters, it,
                                                use_pp_levels);
            else if (it == 0)
                k_levels<<<(segs.n + kLvBlock - 1) / kLvBlock, kLvBlock, 0, st>>>(g, segs, lv, tsize, seg_tsize,
                                                                                  seg_iters, it, ci, ct, L,
                                                                                  karras_ranges);
            if (it == 0) ++ctx->launches;
            // Level counts and the frontier of the dataflow pass (after the
            // first iteration's climb, or from the levels the previous
            // iteration left).
            if (!hist_done) {
                k_level_hist<<<gbl, 256, 0, st>>>(segs, lv, seg_iters, it, L);
                ++ctx->launches;
            }
            const unsigned lg = (unsigned)ctx->num_sms * (256 / threads) * 4;
            // Roots per level fall by about 0.62 per level from n / (1.5 gamma)
            // at level 1 (gamma = tsize << it); levels expected to hold at
            // least atr_quad_min roots run in four-lane groups, levels expected
            // to hold at most atr_warp_max one treelet per warp (the shortest
            // latency per treelet, for levels too narrow to fill the GPU).
            const double gamma = (double)(tsize << it);
            double expect = (double)segs.n / (1.5 * gamma);
            for (int lev = 1; lev <= L; ++lev, expect *= 0.62) {
                const bool quads = max_ts <= kQuadLeaves && ctx->atr_quad_min >= 0 && expect >= ctx->atr_quad_min;
                const bool whole = !quads && max_ts <= kRegTreelet && expect <= (double)ctx->atr_warp_max;
                if (quads) {
                    launch_level_g<8, true>(warps, lg, st, g, segs, lv, lev, tsize, seg_tsize, it, ci, ctx->d_error);
                } else if (whole) {
                    launch_level_g<32, false>(warps, lg, st, g, segs, lv, lev, tsize, seg_tsize, it, ci, ctx->d_error);
                } else {
                    switch (gw) {
                        case 8: launch_level_g<8, false>(warps, lg, st, g, segs, lv, lev, tsize, seg_tsize, it, ci, ctx->d_error); break;
                        case 10: launch_level_g<10, false>(warps, lg, st, g, segs, lv, lev, tsize, seg_tsize, it, ci, ctx->d_error); break;
                        case 16: launch_level_g<16, false>(warps, lg, st, g, segs, lv, lev, tsize, seg_tsize, it, ci, ctx->d_error); break;
                        default: launch_level_g<32, false>(warps, lg, st, g, segs, lv, lev, tsize, seg_tsize, it, ci, ctx->d_error); break;
                    }
                }
                ++ctx->launches;
            }
            if (e == cudaSuccess) e = cudaMemsetAsync(counters, 0, inner * 4, st);
            start = lv.frontier;
            start_count = lv.n_frontier;
            blocks = front_blocks;
        }
        if (e != cudaSuccess) break;
        switch (gw) {
            case 8: e = launch_atrbvh_g<8>(warps, blocks, st, g, segs, rec, counters, kids, tsize, seg_tsize, seg_iters, it, ci, ct, gmin, start, start_count, ctx->d_error); break;
            case 10: e = launch_atrbvh_g<10>(warps, blocks, st, g, segs, rec, counters, kids, tsize, seg_tsize, seg_iters, it, ci, ct, gmin, start, start_count, ctx->d_error); break;
            case 16: e = launch_atrbvh_g<16>(warps, blocks, st, g, segs, rec, counters, kids, tsize, seg_tsize, seg_iters, it, ci, ct, gmin, start, start_count, ctx->d_error); break;
            default: e = launch_atrbvh_g<32>(warps, blocks, st, g, segs, rec, counters, kids, tsize, seg_tsize, seg_iters, it, ci, ct, gmin, start, start_count, ctx->d_error); break;
        }
        ++ctx->launches;
    }
    ctx->phase_end();
    ctx->release(scratch);
    if (e != cudaSuccess) return cuda_fail(e, "k_atrbvh launch", __FILE__, __LINE__);
    return ATR_OK;
}

// Kernel attributes (once per context); none are needed at present.
int atrbvh_prepare() { return ATR_OK; }

}  // namespace atr

using namespace atr;

extern "C" int atr_optimize_atrbvh(atr_ctx* ctx, atr_tree* tree, int tsize, int iterations, float ci, float ct) {
    ATR_REQUIRE(ctx && tree, ATR_ERR_INVALID_ARG, "atr_optimize_atrbvh: NULL argument");
    ATR_REQUIRE(tsize >= 3 && tsize <= kMaxTreelet, ATR_ERR_UNSUPPORTED,
                "atr_optimize_atrbvh: treelet size %d outside [3, %d]", tsize, kMaxTreelet);
    ATR_REQUIRE(iterations >= 0 && iterations <= 24, ATR_ERR_INVALID_ARG, "atr_optimize_atrbvh: iterations %d",
                iterations);
    const uint32_t n = tree->n;
    TreeRefs g{n, tree->parent, tree->left, tree->right, tree->bmin, tree->bmax, tree->area, nullptr};
    Segs segs{nullptr, nullptr, 1u, n};
    const int2* ranges = tree->karras ? tree->range : nullptr;
    const BuildPrepass* pp = tree->prepass_block ? &tree->prepass : nullptr;
    if (iterations <= 0) return ATR_OK;
    tree->karras = false;
    tree_topology_changed(tree);
    const int st = atrbvh_run(ctx, g, segs, 2 * (size_t)n - 1, tsize, tsize, iterations, nullptr, nullptr, ci, ct,
                              ranges, pp);
    // The prepass arrays served as this pass's scratch; they are stale now.
    ctx->release(tree->prepass_block);
    tree->prepass_block = nullptr;
    tree->prepass = BuildPrepass{};
    return st;
}
