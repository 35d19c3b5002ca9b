// ORACLE -- test infrastructure only.
//
// Fibers and the block scheduler of the host execution model declared in
// simt.h, and the subset of the CUDA runtime API the reference's host code
// calls, over host memory.

#include "simt.h"

#include <sys/mman.h>

#include <chrono>

#include "cuda_runtime.h"

// Saves the callee-saved registers and the stack pointer of the running
// context into *save_sp and resumes the context whose stack pointer is load_sp
// (System V x86-64).
extern "C" void simt_switch(void** save_sp, void* load_sp);
asm(R"(
    .text
    .globl simt_switch
    .type simt_switch, @function
simt_switch:
    pushq %rbp
    pushq %rbx
    pushq %r12
    pushq %r13
    pushq %r14
    pushq %r15
    movq %rsp, (%rdi)
    movq %rsi, %rsp
    popq %r15
    popq %r14
    popq %r13
    popq %r12
    popq %rbx
    popq %rbp
    ret
    .size simt_switch, .-simt_switch
)");

namespace simt {
namespace {

enum State { kReady, kInCollective, kAtBarrier, kDone };

struct Thread {
    void* sp = nullptr;
    char* stack = nullptr;
    uint3 tid{0, 0, 0};
    int state = kDone;
    int kind = 0;
    int arg = 0;
    uint64_t value = 0;
    uint64_t result = 0;
};

// Lanes wait in the same collective when they wait in collectives of the same
// kind (and, for inserted warp syncs, the same id).  Code addresses cannot
// tell this: an optimising compiler may duplicate one source-level
// collective into several code paths.
bool same_collective(const Thread& a, const Thread& b) {
    return a.kind == b.kind && (a.kind != kWarpSync || a.arg == b.arg);
}

constexpr size_t kStackBytes = 256 * 1024;

struct Runner {
    std::vector<Thread> threads;
    std::vector<char*> stacks;
    void* sched_sp = nullptr;
    Thread* cur = nullptr;
    const std::function<void()>* body = nullptr;
    uint3 block{0, 0, 0};
    dim3 bdim, gdim;
    std::vector<unsigned char> shared;
    Stats stats{};
};

Runner g;

[[noreturn]] void fail(const char* what) {
    std::fprintf(stderr, "simt: %s\n", what);
    std::abort();
}

void fiber_main() {
    (*g.body)();
    g.cur->state = kDone;
    simt_switch(&g.cur->sp, g.sched_sp);
    fail("a finished fiber was resumed");
}

char* stack_for(size_t i) {
    while (g.stacks.size() <= i) {
        void* p = mmap(nullptr, kStackBytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
        if (p == MAP_FAILED) fail("cannot map a fiber stack");
        g.stacks.push_back(static_cast<char*>(p));
    }
    return g.stacks[i];
}

// Initial frame: six zeroed callee-saved registers, then fiber_main as the
// return address of simt_switch, then a dummy return address so that
// fiber_main starts with the stack alignment of a called function.
void* initial_sp(char* stack) {
    uintptr_t top = (reinterpret_cast<uintptr_t>(stack) + kStackBytes) & ~uintptr_t(15);
    void** sp = reinterpret_cast<void**>(top);
    *--sp = nullptr;
    *--sp = reinterpret_cast<void*>(&fiber_main);
    for (int r = 0; r < 6; ++r) *--sp = nullptr;
    return sp;
}

void resume(Thread* t) {
    g.cur = t;
    simt_switch(&g.sched_sp, t->sp);
    g.cur = nullptr;
}

void yield() {
    Thread* t = g.cur;
    if (!t) fail("a device intrinsic was called outside a kernel");
    simt_switch(&t->sp, g.sched_sp);
}

// Return addresses of a suspended thread's frames, outermost first (frame
// pointers are kept in every object of the host model).
std::vector<const void*> call_chain(const Thread& t) {
    std::vector<const void*> chain;
    void* const* regs = static_cast<void* const*>(t.sp);
    chain.push_back(regs[6]);
    const char* lo = t.stack;
    const char* hi = t.stack + kStackBytes;
    const char* fp = static_cast<const char*>(regs[5]);
    while (fp && fp >= lo && fp + 16 <= hi) {
        chain.push_back(reinterpret_cast<void* const*>(fp)[1]);
        fp = static_cast<const char*>(reinterpret_cast<void* const*>(fp)[0]);
    }
    std::reverse(chain.begin(), chain.end());
    return chain;
}

// True when a's call chain lies before b's in program order: compared at the
// first frame where they differ, by code address.
bool chain_before(const std::vector<const void*>& a, const std::vector<const void*>& b) {
    const size_t m = std::min(a.size(), b.size());
    for (size_t k = 0; k < m; ++k)
        if (a[k] != b[k]) return a[k] < b[k];
    return a.size() < b.size();
}

// All live lanes of [lo, hi) wait in collectives.  When they wait in the same
// one, all take part.  When they wait in different ones (a collective inside
// a branch some lanes skipped), the lanes furthest back in program order (by
// call chain; the code concerned keeps source order in its layout) take part
// and the others keep waiting: the divergent path runs to its reconvergence
// point first, as on a warp of the pre-Volta SIMT model.  Each lane taking
// part gets its result from the operands as deposited; a source lane that
// takes no part gives the reader its own operand.
void complete_collective(size_t lo, size_t hi) {
    std::vector<char> part(hi - lo, 0);
    bool one_site = true;
    const Thread* ref = nullptr;
    for (size_t i = lo; i < hi; ++i) {
        const Thread& t = g.threads[i];
        if (t.state != kInCollective) continue;
        if (!ref) ref = &t;
        else if (!same_collective(t, *ref)) one_site = false;
    }
    if (one_site) {
        for (size_t i = lo; i < hi; ++i) part[i - lo] = g.threads[i].state == kInCollective;
    } else {
        std::vector<std::vector<const void*>> chains(hi - lo);
        std::vector<const void*>* best = nullptr;
        for (size_t i = lo; i < hi; ++i) {
            if (g.threads[i].state != kInCollective) continue;
            chains[i - lo] = call_chain(g.threads[i]);
            if (!best || chain_before(chains[i - lo], *best)) best = &chains[i - lo];
        }
        for (size_t i = lo; i < hi; ++i)
            part[i - lo] = g.threads[i].state == kInCollective && chains[i - lo] == *best;
        ++g.stats.divergent;
    }
    int first_kind = -1;
    for (size_t i = lo; i < hi; ++i) {
        if (!part[i - lo]) continue;
        const Thread& t = g.threads[i];
        if (first_kind < 0) first_kind = t.kind;
        if (t.kind != first_kind) fail("lanes at one call site wait in different kinds of collective");
    }
    auto lane_live = [&](size_t i) { return i < hi && part[i - lo]; };
    uint32_t ballot = 0;
    if (first_kind == kBallot)
        for (size_t i = lo; i < hi; ++i)
            if (lane_live(i) && g.threads[i].value) ballot |= 1u << (i - lo);
    for (size_t i = lo; i < hi; ++i) {
        Thread& t = g.threads[i];
        if (!part[i - lo]) continue;
        switch (first_kind) {
            case kShfl: {
                const size_t src = lo + ((unsigned)t.arg & 31u);
                if (lane_live(src)) {
                    t.result = g.threads[src].value;
                } else {
                    t.result = t.value;
                    ++g.stats.inactive_sources;
                }
                break;
            }
            case kShflDown: {
                const size_t lane = i - lo;
                const size_t src = i + (size_t)t.arg;
                if (lane + (size_t)t.arg < 32 && lane_live(src)) {
                    t.result = g.threads[src].value;
                } else {
                    t.result = t.value;
                    if (lane + (size_t)t.arg < 32) ++g.stats.inactive_sources;
                }
                break;
            }
            case kBallot:
                t.result = ballot;
                break;
            default:
                t.result = 0;
        }
    }
    for (size_t i = lo; i < hi; ++i)
        if (part[i - lo]) g.threads[i].state = kReady;
    ++g.stats.collectives;
}

void run_block() {
    const size_t n = (size_t)g.bdim.x * g.bdim.y * g.bdim.z;
    g.threads.assign(n, Thread{});
    for (size_t i = 0; i < n; ++i) {
        Thread& t = g.threads[i];
        t.tid = uint3{(unsigned)(i % g.bdim.x), (unsigned)((i / g.bdim.x) % g.bdim.y),
                      (unsigned)(i / ((size_t)g.bdim.x * g.bdim.y))};
        t.state = kReady;
        t.stack = stack_for(i);
        t.sp = initial_sp(t.stack);
    }
    const size_t warps = (n + 31) / 32;
    while (true) {
        bool progress = false;
        for (size_t w = 0; w < warps; ++w) {
            const size_t lo = 32 * w, hi = std::min(n, lo + 32);
            for (size_t i = lo; i < hi; ++i) {
                if (g.threads[i].state == kReady) {
                    resume(&g.threads[i]);
                    progress = true;
                }
            }
            bool live = false, all_waiting = true;
            for (size_t i = lo; i < hi; ++i) {
                const int s = g.threads[i].state;
                if (s == kDone) continue;
                live = true;
                if (s != kInCollective) all_waiting = false;
            }
            if (live && all_waiting) {
                complete_collective(lo, hi);
                progress = true;
            }
        }
        if (progress) continue;
        size_t live = 0, barrier = 0;
        for (const Thread& t : g.threads) {
            if (t.state == kDone) continue;
            ++live;
            if (t.state == kAtBarrier) ++barrier;
        }
        if (live == 0) break;
        if (barrier != live) fail("deadlock: threads wait in a warp collective and at a block barrier at once");
        for (Thread& t : g.threads)
            if (t.state == kAtBarrier) t.state = kReady;
        ++g.stats.barriers;
    }
    g.stats.threads += n;
    ++g.stats.blocks;
}

}  // namespace

const uint3& thread_index() {
    if (!g.cur) fail("threadIdx read outside a kernel");
    return g.cur->tid;
}
const uint3& block_index() { return g.block; }
const dim3& block_dim() { return g.bdim; }
const dim3& grid_dim() { return g.gdim; }
void* dynamic_shared() { return g.shared.data(); }

__attribute__((noinline)) uint64_t warp_collective(int kind, uint64_t value, int arg) {
    Thread* t = g.cur;
    if (!t) fail("warp intrinsic called outside a kernel");
    t->kind = kind;
    t->value = value;
    t->arg = arg;
    t->state = kInCollective;
    yield();
    return t->result;
}

void block_barrier() {
    Thread* t = g.cur;
    if (!t) fail("__syncthreads outside a kernel");
    t->state = kAtBarrier;
    yield();
}

void run(const Launch& cfg, const std::function<void()>& body) {
    if (g.body) fail("kernel launched from inside a kernel");
    g.stats = Stats{};
    g.body = &body;
    g.bdim = cfg.block;
    g.gdim = cfg.grid;
    g.shared.assign(cfg.shared + 16, 0);
    for (unsigned z = 0; z < cfg.grid.z; ++z)
        for (unsigned y = 0; y < cfg.grid.y; ++y)
            for (unsigned x = 0; x < cfg.grid.x; ++x) {
                g.block = uint3{x, y, z};
                run_block();
            }
    g.body = nullptr;
}

Stats last_stats() { return g.stats; }

}  // namespace simt

// ---- CUDA runtime API over host memory ---------------------------------------

namespace {
cudaError_t g_last = cudaSuccess;
}

struct simt_event {
    std::chrono::steady_clock::time_point t;
};

cudaError_t cudaMalloc(void** p, size_t bytes) {
    const size_t sz = (bytes + 255) & ~size_t(255);
    *p = std::aligned_alloc(256, sz ? sz : 256);
    if (!*p) return g_last = cudaErrorMemoryAllocation;
    std::memset(*p, 0, sz ? sz : 256);
    return cudaSuccess;
}
cudaError_t cudaFree(void* p) {
    std::free(p);
    return cudaSuccess;
}
cudaError_t cudaMemcpy(void* dst, const void* src, size_t bytes, cudaMemcpyKind) {
    if (bytes) std::memmove(dst, src, bytes);
    return cudaSuccess;
}
cudaError_t cudaMemset(void* p, int value, size_t bytes) {
    std::memset(p, value, bytes);
    return cudaSuccess;
}
cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
cudaError_t cudaGetLastError() {
    const cudaError_t e = g_last;
    g_last = cudaSuccess;
    return e;
}
const char* cudaGetErrorString(cudaError_t e) { return e == cudaSuccess ? "no error" : "host model error"; }
cudaError_t cudaEventCreate(cudaEvent_t* e) {
    *e = new simt_event{};
    return cudaSuccess;
}
cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t) {
    e->t = std::chrono::steady_clock::now();
    return cudaSuccess;
}
cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t a, cudaEvent_t b) {
    *ms = std::chrono::duration<float, std::milli>(b->t - a->t).count();
    return cudaSuccess;
}
cudaError_t cudaEventDestroy(cudaEvent_t e) {
    delete e;
    return cudaSuccess;
}
