// mpx_engine.cu -- host engine and C ABI (include/mpx.h) of the B200 propagation engine.
//
// The engine owns one CUDA stream and a device-resident term store. A propagate call uploads the
// circuit once as per-gate descriptors, then issues two kernels per gate with no host round trip per
// gate: the sweep kernel refuses to start a gate that could overflow the store (it records the step and
// every later launch becomes a no-op), and the host, which checks the counters once per chunk of gates,
// grows the store and re-issues from that step. Truncation semantics follow the reference's fused
// ContractImmediately path (MonomialPropagator.inl:594-618).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/mpx.h"
#include "mpx_kernels.cuh"
#include "mpx_small.cuh"

using namespace mpx;

namespace {

thread_local std::string g_create_error;

}  // namespace

struct mpx_circuit {
    mpx::GateDesc *d_desc = nullptr;
    uint64_t id = 0;         // unique per uploaded circuit (keys the engine's graph cache)
    bool persistent = false; // uploaded by mpx_circuit_upload (worth a CUDA graph)
    uint64_t n = 0;
    std::vector<uint64_t> words; // host copy of the generators, for mpx_circuit_set_angles
    std::vector<double> angles;  // host copy of the current angles (a cloned engine re-uploads the circuit)
    int W = 1;
    int device = 0;
    bool any_cos_zero = false; // some gate has cos(2 angle) == 0 exactly (needs the pre-gate copy `aux`)
};
using CircuitDev = mpx_circuit;

// Gradient state between mpx_adjoint_forward and mpx_adjoint_backward: coefficient checkpoints at
// segment starts (keys are append-only, so a prefix of the final store plus its coefficients restores
// any earlier state), the final coefficients, and the forward pass's per-gate counters.
struct AdjointState {
    const mpx_circuit *circuit = nullptr;
    uint64_t L = 0;
    std::vector<uint64_t> seg_lo; // first step of each segment
    std::vector<uint64_t> ck_n;   // store size at each segment start
    std::vector<double *> ck_coef;
    double *final_coef = nullptr;
    uint64_t n_final = 0;
    std::vector<uint64_t> stats; // [L][4] n_g, a_g, e_g, (unused) per step
    uint32_t *w_anti = nullptr;   // [L][sweep warps] anticommuting terms per sweep warp and step
    // pairs recorded by the forward pass (valid when rec_ok: the log did not overflow)
    uint32_t *r_src = nullptr, *r_tgt = nullptr;
    int8_t *r_code = nullptr;
    uint64_t *r_begin = nullptr;
    uint64_t r_total = 0;
    bool rec_ok = false;
    // only_rotate_len_k of the forward pass (0: none) and its outside-set bits over the final store
    uint32_t len_k = 0;
    uint32_t *longb = nullptr;
    // a forward pass that logged everything the reverse sweep needs (log_ok: nothing overflowed): both
    // pre-gate values of every recorded pair and the undo log; f_ubegin[st] = first undo record of step st
    double *r_vs = nullptr, *r_vt = nullptr;
    uint32_t *f_uidx = nullptr;
    double *f_uval = nullptr;
    unsigned long long *f_utotal = nullptr;
    uint64_t *f_ubegin = nullptr;
    uint64_t f_ucap = 0;
    bool log_ok = false;
};

// A frozen structure (the surrogate "graph" of the reference's variational loop): every gate's rotated
// and appended pairs of the build, plus what re-deriving the anticommuting sets needs.
struct FrozenGraph {
    uint64_t circuit_id = 0, L = 0, n_final = 0;
    uint32_t *src = nullptr, *tgt = nullptr;
    int8_t *code = nullptr;
    uint64_t *p_begin = nullptr;            // [L] device
    unsigned long long *p_count = nullptr;  // [L] device
    std::vector<uint64_t> n0, anti, count;  // per step (host)
    uint32_t *w_anti = nullptr;             // [L][sweep warps] anticommuting terms per sweep warp (build)
    uint32_t *done = nullptr;               // [ceil(n_final / 32)] scratch bitmap
    int32_t *last = nullptr;                // paring (mpx_graph_pare): [n_final] last relevant step per term
    bool pared = false;                     // the frozen kernels skip pared terms
    double last_for = -1.0;                 // threshold `last` was computed for (< 0: none yet)
    // the device view the frozen kernels take
    uint32_t *longb = nullptr;              // only_rotate_len_k of the build: terms outside its set (bits)
    // A built graph replays as the reference's graph does: its cos set is recomputed from the fold over all
    // terms below the post-insert count, with no length filter (MonomialPropagator.inl:872-895), so terms
    // outside the only_rotate_len_k set are scaled there and a pair's partner outside it is a plain pair.
    // The recorded view of a propagation (the adjoint of that propagation) keeps the forward semantics:
    // such terms and partners are never scaled.
    bool forward_len_k = false;
    Frozen view() const {
        return Frozen{src, tgt, code, p_begin, p_count, pared ? last : nullptr, forward_len_k ? longb : nullptr};
    }
};

struct mpx_engine {
    mpx_config cfg{};
    int W = 1;
    Trunc tr{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    int grid = 0;
    int table_shift = 1;
    bool aux_on = false; // the store carries `aux` (only circuits with an exact cos == 0 gate need it)
    Store st{};
    Scratch sc{};
    Counters *d_cnt = nullptr;
    Counters *h_cnt = nullptr; // pinned
    Counters *h_snap = nullptr; // pinned, two per-chunk snapshots
    cudaEvent_t ev[2] = {nullptr, nullptr};
    StateMask mask{};
    double core = 0.0;
    uint64_t *d_init_keys = nullptr;
    double *d_init_coef = nullptr;
    uint64_t n_init = 0;
    uint64_t *d_stats = nullptr;
    uint64_t stats_cap = 0;
    uint64_t last_gates = 0;
    std::vector<uint64_t> h_stats;
    double *d_partial = nullptr;
    double *d_out = nullptr;
    double *h_out = nullptr; // pinned
    uint64_t launches = 0;
    uint64_t graph_replays = 0; // gate ranges run as one captured CUDA graph
    // Per-kernel event timing (mpx_set_profiling): start/stop events around every sweep and resolve
    // launch of the last propagate call, summed on the host afterwards.
    int profile = 0;
    std::vector<cudaEvent_t> pev;
    double t_sweep_ms = 0.0, t_resolve_ms = 0.0, t_columns_ms = 0.0;
    uint64_t n_sweep = 0;
    AdjointState adj;
    FrozenGraph fg;
    Tape fwd_tape{}; // tape fields the forward sweep fills (w_anti while recording a gradient)
    // CUDA graphs of whole gate ranges of persistent circuits: captured after a propagation that did not
    // grow the store, replayed while the store, its scratch and the truncation settings are unchanged.
    struct GraphEntry {
        uint64_t circuit_id, lo, hi, gen;
        const uint32_t *w_anti;
        const uint32_t *r_src;
        uint64_t r_cap;
        cudaGraphExec_t exec;
    };
    std::vector<GraphEntry> graphs;
    uint64_t store_gen = 0;
    uint64_t rec_hint = 0; // pair records the last recording forward pass needed (sizes the next log)
    uint64_t undo_hint = 0; // undo records (anticommuting terms over all gates) of the last gradient forward pass
    int64_t pair_log = -1; // mpx_set_pair_log: < 0 automatic, 0 off, > 0 fixed capacity
    uint64_t *d_basis = nullptr; // basis_change rows [2T][W] (tr.basis_rows points here when set)
    // Re-weighted initial operator (mpx_update_initial_operator): store indices and coefficients that
    // graph evaluations start from instead of the constructor's operator.
    uint32_t *d_start_idx = nullptr;
    double *d_start_val = nullptr;
    uint64_t n_start = 0;
    bool start_on = false;
    // Schrodinger picture: the store holds the evolved state; the observable is kept apart for <O>
    bool schr = false;
    uint64_t *d_obs_keys = nullptr;
    double *d_obs_coef = nullptr;
    uint32_t *d_obs_idx = nullptr;
    uint64_t n_obs = 0;
    // Large blocks through the kept-block cache (dev_alloc). The batch runner turns it off for its
    // engines: with several engines growing at once, power-of-two classes and idle kept blocks crowd
    // the device, and a 96-instance gradient batch took 2x longer with them.
    bool keep_blocks = true;
    bool use_pdl = true; // programmatic dependent launch of the per-gate kernels
    bool use_graphs = true;
    bool small_path = true; // run small stores in one shared-memory block (mpx_small.cuh)
    std::string err;
};

namespace {

std::atomic<uint64_t> g_circuit_ids{1};

// Largest initial Schrodinger state the engine builds (paired monomials; 8W + 8 bytes each on the device).
constexpr uint64_t kMaxPairedTerms = uint64_t(1) << 28;

#define MPX_CUDA(call)                                                                                              \
    do {                                                                                                            \
        cudaError_t e_ = (call);                                                                                    \
        if (e_ != cudaSuccess) {                                                                                    \
            /* out of memory is MPX_ERR_NOMEM (callers may retry once memory is released) */                      \
            if (e_ == cudaErrorMemoryAllocation) cudaGetLastError();                                              \
            return fail(eng, e_ == cudaErrorMemoryAllocation ? MPX_ERR_NOMEM : MPX_ERR_CUDA,                       \
                        std::string(#call ": ") + cudaGetErrorString(e_));                                          \
        }                                                                                                           \
    } while (0)

mpx_status fail(mpx_engine *eng, mpx_status st, const std::string &msg) {
    if (eng != nullptr) eng->err = msg;
    else g_create_error = msg;
    return st;
}

// Device memory of every engine on a device comes from one library-owned stream-ordered pool whose
// release threshold is unbounded: freed blocks stay mapped for the next allocation (a new engine, a
// regrown store) instead of being unmapped and re-mapped, which for multi-GB stores costs far more than
// the kernels. mpx_trim_device_memory hands the cached memory back.
cudaMemPool_t engine_pool(int device) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    uint64_t threshold = ~0ULL;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    pools[device] = pool;
    return pool;
}

uint64_t next_pow2(uint64_t x) {
    uint64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

// Large blocks (>= 1 MiB) are not handed back to the pool when freed but kept, per device and
// power-of-two size class, for the next request of that class: a store that regrows, or the next
// engine of the same workload, gets the very same mapped block back. Asking the pool for a multi-GB
// block instead can cost a second or more when it has to assemble the block from freed pieces. A kept
// block carries an event recorded on the stream that freed it, which the next user's stream waits on.
// When an allocation fails, every kept block of the device goes back to the pool and it is retried;
// mpx_trim_device_memory does the same and then trims the pool.
struct KeptBlock {
    void *ptr;
    cudaEvent_t ready;
};
struct BlockCache {
    std::mutex mu;
    std::map<std::pair<int, size_t>, std::vector<KeptBlock>> idle; // (device, class) -> blocks
    std::unordered_map<void *, size_t> live;                        // block -> class, while in use
};
BlockCache &block_cache() {
    static BlockCache *c = new BlockCache; // never destroyed: engines may outlive static destruction
    return *c;
}
constexpr size_t kKeepMin = size_t(1) << 20;

// Returns every kept block of `device` to the pool (the caller has made `device` current).
void release_kept_blocks(int device) {
    BlockCache &c = block_cache();
    std::vector<KeptBlock> out;
    {
        std::lock_guard<std::mutex> lock(c.mu);
        for (auto it = c.idle.begin(); it != c.idle.end();) {
            if (it->first.first == device) {
                out.insert(out.end(), it->second.begin(), it->second.end());
                it = c.idle.erase(it);
            }
            else {
                ++it;
            }
        }
    }
    for (const KeptBlock &b : out) {
        cudaEventSynchronize(b.ready);
        cudaEventDestroy(b.ready);
        cudaFreeAsync(b.ptr, nullptr);
    }
    if (!out.empty()) cudaStreamSynchronize(nullptr);
    cudaGetLastError();
}

// Device bytes an allocation of this engine can still get: the device's free memory, the pool's reserved
// but unused bytes (freed blocks stay reserved: the release threshold is unbounded) and the idle kept
// blocks of the device (cudaMemGetInfo counts both as used).
size_t device_available(mpx_engine *e) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    uint64_t reserved = 0, used = 0; // the pool attributes are 64-bit values
    if (e->pool != nullptr && cudaMemPoolGetAttribute(e->pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(e->pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
        free_b += static_cast<size_t>(reserved - used);
    cudaGetLastError();
    BlockCache &c = block_cache();
    std::lock_guard<std::mutex> lock(c.mu);
    for (const auto &[key, blocks] : c.idle)
        if (key.first == e->device) free_b += key.second * blocks.size();
    return free_b;
}

cudaError_t dev_alloc(mpx_engine *e, void **ptr, size_t bytes) {
    BlockCache &c = block_cache();
    if (bytes < kKeepMin || !e->keep_blocks) {
        const cudaError_t ce = cudaMallocFromPoolAsync(ptr, bytes, e->pool, e->stream);
        if (ce == cudaSuccess) { // an address is never on record as a kept class while it is a small block
            std::lock_guard<std::mutex> lock(c.mu);
            c.live.erase(*ptr);
        }
        return ce;
    }
    const size_t cls = next_pow2(bytes);
    {
        std::lock_guard<std::mutex> lock(c.mu);
        auto it = c.idle.find({e->device, cls});
        if (it != c.idle.end() && !it->second.empty()) {
            const KeptBlock b = it->second.back();
            it->second.pop_back();
            c.live[b.ptr] = cls;
            *ptr = b.ptr;
            const cudaError_t ce = cudaStreamWaitEvent(e->stream, b.ready, 0);
            cudaEventDestroy(b.ready);
            return ce;
        }
    }
    cudaError_t ce = cudaMallocFromPoolAsync(ptr, cls, e->pool, e->stream);
    if (ce == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        release_kept_blocks(e->device);
        ce = cudaMallocFromPoolAsync(ptr, cls, e->pool, e->stream);
    }
    if (ce == cudaSuccess) {
        std::lock_guard<std::mutex> lock(c.mu);
        c.live[*ptr] = cls;
    }
    return ce;
}

// Frees a block from dev_alloc, stream-ordered on `stream` of `device` (the current device). Every block
// from dev_alloc must come back through here: a block of a kept class freed any other way would leave
// its class on record for an address the pool may hand out again at another size.
void dev_release(int device, cudaStream_t stream, void *ptr) {
    if (ptr == nullptr) return;
    BlockCache &c = block_cache();
    size_t cls = 0;
    {
        std::lock_guard<std::mutex> lock(c.mu);
        auto it = c.live.find(ptr);
        if (it != c.live.end()) {
            cls = it->second;
            c.live.erase(it);
        }
    }
    cudaEvent_t ev = nullptr;
    if (cls == 0 || cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventRecord(ev, stream) != cudaSuccess) {
        cudaGetLastError();
        if (ev != nullptr) cudaEventDestroy(ev);
        cudaFreeAsync(ptr, stream);
        return;
    }
    std::lock_guard<std::mutex> lock(c.mu);
    c.idle[{device, cls}].push_back({ptr, ev});
}

void dev_free(mpx_engine *e, void *ptr) { dev_release(e->device, e->stream, ptr); }

// Small pinned host buffers (counter snapshots, results) are reused across engines: cudaFreeHost waits
// for the whole device, which in a batch would stall every other engine's stream once per instance.
struct PinnedCache {
    std::mutex mu;
    std::map<size_t, std::vector<void *>> idle;
};
PinnedCache &pinned_cache() {
    static PinnedCache *c = new PinnedCache; // never destroyed: engines may outlive static destruction
    return *c;
}
cudaError_t pinned_get(void **ptr, size_t bytes) {
    PinnedCache &c = pinned_cache();
    {
        std::lock_guard<std::mutex> lock(c.mu);
        auto it = c.idle.find(bytes);
        if (it != c.idle.end() && !it->second.empty()) {
            *ptr = it->second.back();
            it->second.pop_back();
            return cudaSuccess;
        }
    }
    return cudaMallocHost(ptr, bytes);
}
void pinned_put(void *ptr, size_t bytes) {
    if (ptr == nullptr) return;
    PinnedCache &c = pinned_cache();
    std::lock_guard<std::mutex> lock(c.mu);
    c.idle[bytes].push_back(ptr);
}

// ----- kernel dispatch over (W, basis) ------------------------------------------------------------------

// Launches `kernel` on the engine stream, with programmatic dependent launch unless profiling (the
// kernel waits with griddepcontrol.wait before reading what the previous kernel wrote).
template <typename... KArgs, typename... Args>
void launch_dep_on(mpx_engine *e, unsigned grid, unsigned block, void (*kernel)(KArgs...), Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = e->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    const bool pdl = e->use_pdl && !e->profile;
    cfg.attrs = pdl ? attr : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    if (cudaLaunchKernelEx(&cfg, kernel, args...) != cudaSuccess && pdl) {
        // the attribute was refused: launch plainly from now on (a failed launch of the kernel itself
        // fails again here and is reported by the caller's error check)
        cudaGetLastError();
        e->use_pdl = false;
        cfg.attrs = nullptr;
        cfg.numAttrs = 0;
        cudaLaunchKernelEx(&cfg, kernel, args...);
    }
}

// The per-gate grid of the engine (one resident wave of kBlock-thread blocks).
template <typename... KArgs, typename... Args>
void launch_dep(mpx_engine *e, void (*kernel)(KArgs...), Args... args) {
    launch_dep_on(e, static_cast<unsigned>(e->grid), kBlock, kernel, args...);
}

template <int W, int B, int EXT>
void launch_gate_ext(mpx_engine *e, const GateDesc *d_desc, uint32_t gate, uint32_t step, cudaEvent_t *ev) {
    if (ev) cudaEventRecord(ev[0], e->stream);
    launch_dep(e, &k_sweep<W, B, false, EXT>, e->st, e->sc, e->d_cnt, d_desc, gate, step, e->tr, e->fwd_tape,
               e->d_stats);
    if (ev) cudaEventRecord(ev[1], e->stream);
    launch_dep(e, &k_resolve<W, B, false, (EXT & 1) != 0>, e->st, e->sc, e->d_cnt, d_desc, gate, step, e->tr,
               e->fwd_tape);
    if (ev) cudaEventRecord(ev[2], e->stream);
}

// One gate: the sweep/resolve variant of the engine's options (only_rotate_len_k; basis_change, which only
// Majorana engines accept).
template <int W, int B>
void launch_gate(mpx_engine *e, const GateDesc *d_desc, uint32_t gate, uint32_t step) {
    cudaEvent_t *ev = e->profile ? &e->pev[4 * static_cast<size_t>(step)] : nullptr;
    const int ext = (e->tr.has_len_k ? 1 : 0) | (e->tr.basis_rows != nullptr ? 2 : 0);
    if constexpr (B == 0) {
        switch (ext) {
        case 0: launch_gate_ext<W, B, 0>(e, d_desc, gate, step, ev); break;
        case 1: launch_gate_ext<W, B, 1>(e, d_desc, gate, step, ev); break;
        case 2: launch_gate_ext<W, B, 2>(e, d_desc, gate, step, ev); break;
        default: launch_gate_ext<W, B, 3>(e, d_desc, gate, step, ev); break;
        }
    }
    else {
        if (ext & 1) launch_gate_ext<W, B, 1>(e, d_desc, gate, step, ev);
        else launch_gate_ext<W, B, 0>(e, d_desc, gate, step, ev);
    }
}

template <int W, int B, int EXT>
void launch_replay_ext(mpx_engine *e, const GateDesc *d_desc, uint32_t gate, uint32_t step, const Tape &tp) {
    launch_dep(e, &k_sweep<W, B, true, EXT>, e->st, e->sc, e->d_cnt, d_desc, gate, step, e->tr, tp, e->d_stats);
    launch_dep(e, &k_resolve<W, B, true, (EXT & 1) != 0>, e->st, e->sc, e->d_cnt, d_desc, gate, step, e->tr, tp);
    launch_dep_on(e, 1, 32, &k_replay_advance, e->d_cnt, tp.n_next, step);
}

// A gate replayed for the gradient: same sweep and resolve, logging to the tape; no appends. The variant
// follows the engine's options (only_rotate_len_k; basis_change, which changes only the emit decisions).
template <int W, int B>
void launch_replay(mpx_engine *e, const GateDesc *d_desc, uint32_t gate, uint32_t step, const Tape &tp) {
    const int ext = (e->tr.has_len_k ? 1 : 0) | (B == 0 && e->tr.basis_rows != nullptr ? 2 : 0);
    if constexpr (B == 0) {
        switch (ext) {
        case 0: launch_replay_ext<W, B, 0>(e, d_desc, gate, step, tp); break;
        case 1: launch_replay_ext<W, B, 1>(e, d_desc, gate, step, tp); break;
        case 2: launch_replay_ext<W, B, 2>(e, d_desc, gate, step, tp); break;
        default: launch_replay_ext<W, B, 3>(e, d_desc, gate, step, tp); break;
        }
    }
    else {
        if (ext & 1) launch_replay_ext<W, B, 1>(e, d_desc, gate, step, tp);
        else launch_replay_ext<W, B, 0>(e, d_desc, gate, step, tp);
    }
}

// Shared-memory capacity of the single-block path per key width: the largest power-of-two-friendly size
// whose store, query list, hash table (load <= 1/2) and bitmap fit in 227 KB.
constexpr uint32_t kSmallCap[5] = {0, 8192, 6144, 4096, 4096};
constexpr uint32_t kSmallTableBits[5] = {0, 14, 14, 13, 13};

template <int W, int B>
cudaError_t launch_small(mpx_engine *e, const GateDesc *d_desc, uint32_t L, uint32_t lo, uint32_t hi) {
    const uint32_t cap = kSmallCap[W], tbits = kSmallTableBits[W];
    const size_t bytes = small_smem_bytes(W, cap, tbits);
    static bool configured = false; // per instantiation; the attribute is per function
    if (!configured) {
        const cudaError_t ce = cudaFuncSetAttribute(k_small<W, B>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    static_cast<int>(bytes));
        if (ce != cudaSuccess) return ce;
        configured = true;
    }
    k_small<W, B><<<1, kSmallThreads, bytes, e->stream>>>(e->st, e->d_cnt, d_desc, L, lo, hi, e->tr, e->d_stats, cap,
                                                         tbits);
    return cudaGetLastError();
}

using SmallFn = cudaError_t (*)(mpx_engine *, const GateDesc *, uint32_t, uint32_t, uint32_t);
SmallFn pick_small(int W, int basis) {
    switch (W) {
    case 1: return basis == 1 ? &launch_small<1, 1> : &launch_small<1, 0>;
    case 2: return basis == 1 ? &launch_small<2, 1> : &launch_small<2, 0>;
    case 3: return basis == 1 ? &launch_small<3, 1> : &launch_small<3, 0>;
    case 4: return basis == 1 ? &launch_small<4, 1> : &launch_small<4, 0>;
    default: return nullptr;
    }
}

template <int W, bool LOG>
void launch_frozen(mpx_engine *e, const GateDesc *d_desc, const Frozen &fz, uint32_t gate, uint32_t step, uint64_t n0,
                   uint32_t *done, const Tape &tp) {
    launch_dep(e, &k_frozen_pairs<LOG>, e->st.coef, fz, d_desc, gate, step, done, tp);
    launch_dep(e, &k_frozen_scan<W, LOG>, e->st, d_desc, gate, step, n0, done, tp, fz.last, fz.longb);
}

using FrozenFn = void (*)(mpx_engine *, const GateDesc *, const Frozen &, uint32_t, uint32_t, uint64_t, uint32_t *,
                          const Tape &);
template <bool LOG>
FrozenFn pick_frozen(int W) {
    switch (W) {
    case 1: return &launch_frozen<1, LOG>;
    case 2: return &launch_frozen<2, LOG>;
    case 3: return &launch_frozen<3, LOG>;
    case 4: return &launch_frozen<4, LOG>;
    case 5: return &launch_frozen<5, LOG>;
    case 6: return &launch_frozen<6, LOG>;
    case 7: return &launch_frozen<7, LOG>;
    default: return &launch_frozen<8, LOG>;
    }
}

// out[i] = the reference-state score of stored term i, for i in [lo, hi)
template <int W, int B>
void launch_adj_init(mpx_engine *e, double *out, uint64_t lo, uint64_t hi) {
    const uint64_t n = hi - lo;
    const uint64_t blocks = std::min<uint64_t>((n + kBlock - 1) / kBlock + 1, static_cast<uint64_t>(e->grid) * 4);
    k_adj_init<W, B><<<static_cast<unsigned>(blocks), kBlock, 0, e->stream>>>(e->st.keys + lo * W, n, e->mask,
                                                                              out + lo);
}

template <int W, int B>
void launch_expect(mpx_engine *e) {
    k_expect<W, B><<<e->grid, kBlock, 0, e->stream>>>(e->st, e->d_cnt, e->mask, e->d_partial);
}

// Hash table and bit-columns of terms [lo, hi).
template <int W>
void launch_table(mpx_engine *e, uint64_t lo, uint64_t hi) {
    if (hi <= lo) return;
    const uint64_t blocks = std::min<uint64_t>((hi - lo + 255) / 256, static_cast<uint64_t>(e->grid) * 4);
    k_build_table<W><<<static_cast<unsigned>(blocks), 256, 0, e->stream>>>(e->st, e->d_cnt, lo, hi);
}

template <int W>
void launch_build(mpx_engine *e, uint64_t lo, uint64_t hi) {
    if (hi <= lo) return;
    launch_table<W>(e, lo, hi);
    const uint64_t cblocks = std::min<uint64_t>((hi - lo + 32 * kBlock - 1) / (32 * kBlock) + 1,
                                                static_cast<uint64_t>(e->grid));
    k_columns<W><<<static_cast<unsigned>(cblocks), kBlock, 0, e->stream>>>(e->st, e->d_cnt, lo, hi, 0);
}

using GateFn = void (*)(mpx_engine *, const GateDesc *, uint32_t, uint32_t);
using ReplayFn = void (*)(mpx_engine *, const GateDesc *, uint32_t, uint32_t, const Tape &);
using AdjInitFn = void (*)(mpx_engine *, double *, uint64_t, uint64_t);
using ExpFn = void (*)(mpx_engine *);
using BuildFn = void (*)(mpx_engine *, uint64_t, uint64_t);

template <int W>
GateFn gate_fn(int basis) {
    return basis == 1 ? &launch_gate<W, 1> : &launch_gate<W, 0>;
}
template <int W>
ExpFn exp_fn(int basis) {
    return basis == 1 ? &launch_expect<W, 1> : &launch_expect<W, 0>;
}
template <int W>
ReplayFn replay_fn(int basis) {
    return basis == 1 ? &launch_replay<W, 1> : &launch_replay<W, 0>;
}
template <int W>
AdjInitFn adj_init_fn(int basis) {
    return basis == 1 ? &launch_adj_init<W, 1> : &launch_adj_init<W, 0>;
}

GateFn pick_gate(int W, int basis) {
    switch (W) {
    case 1: return gate_fn<1>(basis);
    case 2: return gate_fn<2>(basis);
    case 3: return gate_fn<3>(basis);
    case 4: return gate_fn<4>(basis);
    case 5: return gate_fn<5>(basis);
    case 6: return gate_fn<6>(basis);
    case 7: return gate_fn<7>(basis);
    default: return gate_fn<8>(basis);
    }
}
ExpFn pick_exp(int W, int basis) {
    switch (W) {
    case 1: return exp_fn<1>(basis);
    case 2: return exp_fn<2>(basis);
    case 3: return exp_fn<3>(basis);
    case 4: return exp_fn<4>(basis);
    case 5: return exp_fn<5>(basis);
    case 6: return exp_fn<6>(basis);
    case 7: return exp_fn<7>(basis);
    default: return exp_fn<8>(basis);
    }
}
ReplayFn pick_replay(int W, int basis) {
    switch (W) {
    case 1: return replay_fn<1>(basis);
    case 2: return replay_fn<2>(basis);
    case 3: return replay_fn<3>(basis);
    case 4: return replay_fn<4>(basis);
    case 5: return replay_fn<5>(basis);
    case 6: return replay_fn<6>(basis);
    case 7: return replay_fn<7>(basis);
    default: return replay_fn<8>(basis);
    }
}
AdjInitFn pick_adj_init(int W, int basis) {
    switch (W) {
    case 1: return adj_init_fn<1>(basis);
    case 2: return adj_init_fn<2>(basis);
    case 3: return adj_init_fn<3>(basis);
    case 4: return adj_init_fn<4>(basis);
    case 5: return adj_init_fn<5>(basis);
    case 6: return adj_init_fn<6>(basis);
    case 7: return adj_init_fn<7>(basis);
    default: return adj_init_fn<8>(basis);
    }
}
template <int W>
void launch_lookup(mpx_engine *e, const uint64_t *qkeys, uint64_t nq, uint64_t n_live, uint32_t *out) {
    const uint64_t blocks = std::min<uint64_t>((nq + 255) / 256, 4096);
    k_lookup<W><<<static_cast<unsigned>(std::max<uint64_t>(blocks, 1)), 256, 0, e->stream>>>(e->st, qkeys, nq, n_live,
                                                                                          out, e->d_cnt);
}
using LookupFn = void (*)(mpx_engine *, const uint64_t *, uint64_t, uint64_t, uint32_t *);
LookupFn pick_lookup(int W) {
    switch (W) {
    case 1: return &launch_lookup<1>;
    case 2: return &launch_lookup<2>;
    case 3: return &launch_lookup<3>;
    case 4: return &launch_lookup<4>;
    case 5: return &launch_lookup<5>;
    case 6: return &launch_lookup<6>;
    case 7: return &launch_lookup<7>;
    default: return &launch_lookup<8>;
    }
}

template <int W>
void launch_long_bits(mpx_engine *e, uint64_t n, uint32_t len_k, uint32_t *out, unsigned blocks) {
    k_long_bits<W><<<blocks, 256, 0, e->stream>>>(e->st.keys, n, len_k, out);
}
using LongBitsFn = void (*)(mpx_engine *, uint64_t, uint32_t, uint32_t *, unsigned);
LongBitsFn pick_long_bits(int W) {
    switch (W) {
    case 1: return &launch_long_bits<1>;
    case 2: return &launch_long_bits<2>;
    case 3: return &launch_long_bits<3>;
    case 4: return &launch_long_bits<4>;
    case 5: return &launch_long_bits<5>;
    case 6: return &launch_long_bits<6>;
    case 7: return &launch_long_bits<7>;
    default: return &launch_long_bits<8>;
    }
}

BuildFn pick_table(int W) {
    switch (W) {
    case 1: return &launch_table<1>;
    case 2: return &launch_table<2>;
    case 3: return &launch_table<3>;
    case 4: return &launch_table<4>;
    case 5: return &launch_table<5>;
    case 6: return &launch_table<6>;
    case 7: return &launch_table<7>;
    default: return &launch_table<8>;
    }
}
BuildFn pick_build(int W) {
    switch (W) {
    case 1: return &launch_build<1>;
    case 2: return &launch_build<2>;
    case 3: return &launch_build<3>;
    case 4: return &launch_build<4>;
    case 5: return &launch_build<5>;
    case 6: return &launch_build<6>;
    case 7: return &launch_build<7>;
    default: return &launch_build<8>;
    }
}

// ----- store management ---------------------------------------------------------------------------------

// Store buffers come from the engine's memory pool and go back to it stream-ordered (a plain cudaFree
// would bypass the pool's bookkeeping, and the next engine would map fresh memory instead of reusing it).
void free_store(mpx_engine *e) {
    dev_free(e, e->st.keys);
    dev_free(e, e->st.coef);
    dev_free(e, e->st.table);
    dev_free(e, e->st.cols);
    dev_free(e, e->sc.q_src);
    dev_free(e, e->sc.q_flag);
    dev_free(e, e->sc.q_val);
    dev_free(e, e->sc.emit_bits);
    dev_free(e, e->sc.aux);
    e->st = Store{};
    e->sc.q_src = nullptr;
    e->sc.q_flag = nullptr;
    e->sc.q_val = nullptr;
    e->sc.emit_bits = nullptr;
    e->sc.aux = nullptr;
}

void clear_graphs(mpx_engine *e) {
    for (auto &g : e->graphs) cudaGraphExecDestroy(g.exec);
    e->graphs.clear();
}

// (Re)allocates the store for capacity `cap`, keeping the first n terms, and rebuilds the hash table.
mpx_status alloc_store(mpx_engine *eng, uint64_t cap, uint64_t n_keep) {
    mpx_engine *e = eng;
    clear_graphs(e);
    ++e->store_gen;
    const int W = e->W;
    if (cap >= 0xFFFFFFF0ULL) return fail(eng, MPX_ERR_CAPACITY, "term capacity exceeds the 32-bit term index");
    uint64_t *keys = nullptr;
    double *coef = nullptr;
    unsigned long long *table = nullptr;
    uint32_t *cols = nullptr;
    const uint64_t tcap = next_pow2(std::max<uint64_t>(cap << e->table_shift, 64));
    const uint64_t q_cap = cap + (static_cast<uint64_t>(e->grid) * kWarps + 2) * 1024; // + region slack
    const uint64_t cstride = ((cap + 31) / 32 + 31) / 32 * 32; // 128-byte aligned columns
    Scratch nsc = e->sc;
    cudaError_t ce = cudaSuccess;
    auto A = [&](void **p, size_t bytes) {
        if (ce == cudaSuccess) ce = dev_alloc(e, p, bytes);
    };
    A(reinterpret_cast<void **>(&keys), cap * W * sizeof(uint64_t));
    A(reinterpret_cast<void **>(&coef), cap * sizeof(double));
    A(reinterpret_cast<void **>(&table), tcap * sizeof(unsigned long long));
    A(reinterpret_cast<void **>(&cols), (64 * W + 1) * cstride * sizeof(uint32_t));
    A(reinterpret_cast<void **>(&nsc.q_src), q_cap * sizeof(uint32_t));
    A(reinterpret_cast<void **>(&nsc.q_flag), q_cap * sizeof(uint8_t));
    A(reinterpret_cast<void **>(&nsc.q_val), q_cap * sizeof(double));
    A(reinterpret_cast<void **>(&nsc.emit_bits), cstride * sizeof(uint32_t));
    if (e->aux_on) A(reinterpret_cast<void **>(&nsc.aux), cap * sizeof(double));
    else nsc.aux = nullptr;
    if (ce != cudaSuccess) {
        dev_free(e, keys);
        dev_free(e, coef);
        dev_free(e, table);
        dev_free(e, cols);
        dev_free(e, nsc.q_src == e->sc.q_src ? nullptr : nsc.q_src);
        dev_free(e, nsc.q_flag == e->sc.q_flag ? nullptr : nsc.q_flag);
        dev_free(e, nsc.q_val == e->sc.q_val ? nullptr : nsc.q_val);
        dev_free(e, nsc.emit_bits == e->sc.emit_bits ? nullptr : nsc.emit_bits);
        dev_free(e, nsc.aux == e->sc.aux ? nullptr : nsc.aux);
        cudaGetLastError();
        return fail(eng, MPX_ERR_NOMEM, std::string("device allocation failed: ") + cudaGetErrorString(ce));
    }
    // Bit-column words of the kept terms are copied as they are (the bits of terms not yet stored are
    // zero in them); the words above start at zero, for the appends to OR into.
    const uint64_t wk = std::min<uint64_t>((n_keep + 31) / 32, cstride);
    if (n_keep > 0) {
        MPX_CUDA(cudaMemcpyAsync(keys, e->st.keys, n_keep * W * sizeof(uint64_t), cudaMemcpyDeviceToDevice, e->stream));
        MPX_CUDA(cudaMemcpyAsync(coef, e->st.coef, n_keep * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
        MPX_CUDA(cudaMemcpy2DAsync(cols, cstride * sizeof(uint32_t), e->st.cols, e->st.cstride * sizeof(uint32_t),
                                   wk * sizeof(uint32_t), 64 * W + 1, cudaMemcpyDeviceToDevice, e->stream));
    }
    if (wk < cstride)
        MPX_CUDA(cudaMemset2DAsync(cols + wk, cstride * sizeof(uint32_t), 0, (cstride - wk) * sizeof(uint32_t),
                                   64 * W + 1, e->stream));
    dev_free(e, e->st.keys);
    dev_free(e, e->st.coef);
    dev_free(e, e->st.table);
    dev_free(e, e->st.cols);
    dev_free(e, e->sc.q_src);
    dev_free(e, e->sc.q_flag);
    dev_free(e, e->sc.q_val);
    dev_free(e, e->sc.emit_bits);
    dev_free(e, e->sc.aux);
    e->st.keys = keys;
    e->st.coef = coef;
    e->st.table = table;
    e->st.cols = cols;
    e->st.cstride = cstride;
    e->st.cap = cap;
    e->st.tmask = tcap - 1;
    nsc.q_cap = q_cap;
    e->sc = nsc;
    MPX_CUDA(cudaMemsetAsync(table, 0xFF, tcap * sizeof(unsigned long long), e->stream));
    pick_table(W)(e, 0, n_keep);
    e->launches += n_keep > 0 ? 1 : 0;
    MPX_CUDA(cudaGetLastError());
    return MPX_OK;
}

mpx_status ensure_stats(mpx_engine *eng, uint64_t n) {
    mpx_engine *e = eng;
    if (n <= e->stats_cap) return MPX_OK;
    clear_graphs(e); // the counters buffer is a kernel argument of every captured graph
    dev_free(e, e->d_stats);
    e->d_stats = nullptr;
    const uint64_t c = std::max<uint64_t>(n, 1024);
    MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&e->d_stats), c * 4 * sizeof(uint64_t)));
    e->stats_cap = c;
    return MPX_OK;
}

void pair_swap_words(const uint64_t *g, uint64_t *out, int W) {
    for (int w = 0; w < W; ++w) out[w] = ((g[w] & kEven) << 1) | ((g[w] >> 1) & kEven);
}

void interleave_words(const uint64_t *g, uint64_t *out, int W) {
    int above = 0;
    for (int w = 0; w < W; ++w) out[w] = 0;
    for (int c = 64 * W - 1; c >= 0; --c) {
        if (above & 1) out[c / 64] |= 1ULL << (c % 64);
        above += static_cast<int>((g[c / 64] >> (c % 64)) & 1ULL);
    }
}

void make_desc(const mpx_engine *e, const uint64_t *g, double angle, GateDesc &d) {
    const int W = e->W;
    std::memset(&d, 0, sizeof(d));
    int gpop = 0, gy = 0;
    for (int w = 0; w < W; ++w) {
        d.g[w] = g[w];
        gpop += __builtin_popcountll(g[w]);
        const uint64_t v = g[w] & kEven, u = (g[w] >> 1) & kEven;
        gy += __builtin_popcountll(v & ~u);
    }
    d.gpop = gpop;
    d.gy = gy;
    if (e->cfg.basis == MPX_BASIS_PAULI) {
        pair_swap_words(g, d.fold, W);
        d.g_odd = 0;
    }
    else {
        for (int w = 0; w < W; ++w) d.fold[w] = g[w];
        d.g_odd = gpop & 1;
        interleave_words(g, d.wmask, W);
    }
    d.pivot_word = 0;
    d.pivot_bit = 0;
    for (int w = 0; w < W; ++w) {
        if (g[w] != 0) {
            d.pivot_word = w;
            d.pivot_bit = g[w] & (~g[w] + 1);
            d.pivot_col = 64 * w + __builtin_ctzll(g[w]);
            break;
        }
    }
    d.empty = gpop == 0;
    d.n_fold = 0;
    for (int w = 0; w < W; ++w) d.n_fold += __builtin_popcountll(d.fold[w]);
    int f = 0;
    for (int w = 0; w < W && d.n_fold <= kMaxFoldCols; ++w)
        for (uint64_t x = d.fold[w]; x != 0; x &= x - 1) d.fold_cols[f++] = static_cast<uint16_t>(64 * w + __builtin_ctzll(x));
    // The same libm calls and argument as the reference (Engine.h:555-560, FusedApply.h:45-46).
    const double c = std::cos(2.0 * angle);
    const double s = std::sin(2.0 * angle);
    d.cosv = c;
    d.sinv = s;
    d.abs_sin = std::fabs(s);
    d.cos_zero = c == 0.0;
    d.inv_cos = c != 0.0 ? 1.0 / c : 1.0;
}

// Device descriptors of a circuit, in the order the kernels take them: the gates are applied from the
// last descriptor to the first. Heisenberg applies the circuit's last gate first (MonomialPropagator.inl:
// 720-733), so descriptor l is gate l. The Schrodinger picture applies the first gate first at the negated
// angle (MonomialPropagator.inl:595-620, parameters mapped with phase -1, MPFunctions.cpp:186-193), so
// descriptor l is gate n-1-l with angle -angle.
void make_descs(const mpx_engine *e, const uint64_t *gen_words, const double *angles, uint64_t n,
                std::vector<GateDesc> &h) {
    h.resize(n);
    for (uint64_t l = 0; l < n; ++l) {
        const uint64_t gi = e->schr ? n - 1 - l : l;
        make_desc(e, gen_words + gi * e->W, e->schr ? -angles[gi] : angles[gi], h[l]);
    }
}

mpx_status upload_circuit(mpx_engine *eng, const uint64_t *gen_words, const double *angles, uint64_t n,
                          CircuitDev &cd) {
    mpx_engine *e = eng;
    std::vector<GateDesc> h;
    make_descs(e, gen_words, angles, n, h);
    MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&cd.d_desc), std::max<uint64_t>(n, 1) * sizeof(GateDesc)));
    if (n > 0) {
        MPX_CUDA(cudaMemcpyAsync(cd.d_desc, h.data(), n * sizeof(GateDesc), cudaMemcpyHostToDevice, e->stream));
    }
    MPX_CUDA(cudaStreamSynchronize(e->stream)); // h goes out of scope
    cd.n = n;
    cd.W = e->W;
    cd.id = g_circuit_ids.fetch_add(1);
    cd.any_cos_zero = false;
    for (const GateDesc &g : h) cd.any_cos_zero = cd.any_cos_zero || g.cos_zero;
    cd.device = e->device;
    cd.words.assign(gen_words, gen_words + n * e->W);
    cd.angles.assign(angles, angles + n);
    return MPX_OK;
}

// Applies the uploaded gates last to first (Heisenberg; MonomialPropagator.inl:720-733). Gates are
// issued in chunks; the counters after chunk k are inspected while chunk k+1 already runs, so the GPU
// is never idle on a healthy run. A stalled step makes the rest of the queue no-ops; the host waits,
// grows the store and re-issues from that step.
mpx_status run_range(mpx_engine *eng, const CircuitDev &cd, uint64_t lo, uint64_t hi) {
    mpx_engine *e = eng;
    const uint64_t L = cd.n;
    if (L == 0) return MPX_OK;
    mpx_status s = ensure_stats(e, L);
    if (s != MPX_OK) return s;
    // the sweeps add their blocks' counts into the per-gate counters of the range
    MPX_CUDA(cudaMemsetAsync(e->d_stats + 4 * lo, 0, 4 * (hi - lo) * sizeof(uint64_t), e->stream));
    if ((cd.any_cos_zero || e->tr.has_len_k) && !e->aux_on) {
        clear_graphs(e);
        e->aux_on = true;
        MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&e->sc.aux), e->st.cap * sizeof(double)));
    }
    if (e->profile) {
        while (e->pev.size() < 4 * L) {
            cudaEvent_t ev = nullptr;
            MPX_CUDA(cudaEventCreate(&ev));
            e->pev.push_back(ev);
        }
    }
    const GateFn gate = pick_gate(e->W, e->cfg.basis);
    constexpr uint64_t kChunk = 48;
    uint64_t step = lo;
    uint64_t chunk_id = 0;
    bool pending = false;
    uint64_t pending_slot = 0;
    // Small store: run gates in one shared-memory block until the store outgrows it (or the range ends).

    if (e->small_path && e->W <= 4 && !e->profile && !cd.any_cos_zero && !e->tr.has_len_k && e->tr.basis_rows == nullptr &&
        e->fwd_tape.w_anti == nullptr &&
        hi - lo >= 8) {
        MPX_CUDA(cudaMemcpyAsync(e->h_cnt, e->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, e->stream));
        MPX_CUDA(cudaStreamSynchronize(e->stream));
        const uint64_t n_now = e->h_cnt->n;
        const uint32_t cap_small = kSmallCap[e->W];
        if (e->h_cnt->stall == kNoStall && n_now * 2 <= cap_small) {
            if (e->st.cap < cap_small) {
                s = alloc_store(e, 2 * cap_small, n_now);
                if (s != MPX_OK) return s;
            }
            MPX_CUDA(pick_small(e->W, e->cfg.basis)(e, cd.d_desc, static_cast<uint32_t>(L), static_cast<uint32_t>(lo),
                                                   static_cast<uint32_t>(hi)));
            e->launches += 1;
            MPX_CUDA(cudaMemcpyAsync(e->h_cnt, e->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, e->stream));
            MPX_CUDA(cudaStreamSynchronize(e->stream));
            const uint64_t n = e->h_cnt->n;
            const uint64_t resume = e->h_cnt->stall == kNoStall ? hi : e->h_cnt->stall;
            // the streaming kernels need the hash table and bit-columns of the store the block wrote back
            MPX_CUDA(cudaMemsetAsync(e->st.table, 0xFF, (e->st.tmask + 1) * sizeof(unsigned long long), e->stream));
            MPX_CUDA(cudaMemsetAsync(e->st.cols, 0, (64 * e->W + 1) * e->st.cstride * sizeof(uint32_t), e->stream));
            pick_build(e->W)(e, 0, n);
            e->launches += 2;
            Counters c{};
            c.n = n;
            c.n0 = n;
            c.stall = kNoStall;
            c.err = e->h_cnt->err; // a table inconsistency of the shared-memory path is reported below
            MPX_CUDA(cudaMemcpyAsync(e->d_cnt, &c, sizeof(Counters), cudaMemcpyHostToDevice, e->stream));
            step = resume;

        }
    }
    const uint64_t gen0 = e->store_gen;
    // A gradient's forward pass is not captured: its tape buffers are allocated per call, so a captured
    // range would rarely match the next call's pointers and each miss would pay a new capture.
    // The streaming part of the range, [glo, hi): after the shared-memory path, from the gate it handed
    // over at (the same gate on every call with the same circuit, angles and initial operator).
    const uint64_t glo = step;
    const bool graphable = e->use_graphs && !e->profile && cd.persistent && e->fwd_tape.w_anti == nullptr && glo < hi;
    bool replayed = false;
    if (graphable) {
        for (const auto &g : e->graphs) {
            if (g.circuit_id != cd.id || g.lo != glo || g.hi != hi || g.gen != gen0 || g.w_anti != e->fwd_tape.w_anti ||
                g.r_src != e->fwd_tape.r_src || g.r_cap != e->fwd_tape.r_cap)
                continue;
            // One launch for the whole range; a gate that would overflow stalls the rest (no-ops), and the
            // host resumes from it below exactly as after a chunk.
            MPX_CUDA(cudaGraphLaunch(g.exec, e->stream));
            e->launches += 2 * (hi - glo);
            ++e->graph_replays;
            MPX_CUDA(cudaMemcpyAsync(&e->h_snap[0], e->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, e->stream));
            MPX_CUDA(cudaEventRecord(e->ev[0], e->stream));
            step = hi;
            pending = true;
            pending_slot = 0;
            chunk_id = 1;
            replayed = true;
            break;
        }
    }
    for (;;) {
        bool issued = false;
        if (step < hi) {
            const uint64_t stop = std::min(hi, step + kChunk);
            for (uint64_t st = step; st < stop; ++st) {
                gate(e, cd.d_desc, static_cast<uint32_t>(L - 1 - st), static_cast<uint32_t>(st));
            }
            e->launches += 2 * (stop - step);
            MPX_CUDA(cudaGetLastError());
            const uint64_t slot = chunk_id & 1;
            MPX_CUDA(cudaMemcpyAsync(&e->h_snap[slot], e->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, e->stream));
            MPX_CUDA(cudaEventRecord(e->ev[slot], e->stream));
            step = stop;
            issued = true;
        }
        if (pending) {
            MPX_CUDA(cudaEventSynchronize(e->ev[pending_slot]));
            const Counters snap = e->h_snap[pending_slot];
            if (snap.stall != kNoStall) {
                MPX_CUDA(cudaStreamSynchronize(e->stream));
                const uint64_t at = snap.stall;
                const uint64_t n = e->h_snap[pending_slot].n;
                // room for the worst case of the stalled gate (2n) with headroom: four times the capacity
                // (fewer regrowths), or, if that does not fit, at least double
                const uint64_t cap0 = e->st.cap;
                s = alloc_store(e, std::max<uint64_t>(3 * n, 4 * cap0), n);
                if (s == MPX_ERR_NOMEM) s = alloc_store(e, std::max<uint64_t>(3 * n, 2 * cap0), n);
                if (s != MPX_OK) return s;
                Counters fresh{};
                fresh.n = n;
                fresh.n0 = n;
                fresh.stall = kNoStall;
                fresh.err = snap.err;
                fresh.rec_total = snap.rec_total; // a recording pass keeps its log offsets
                MPX_CUDA(cudaMemcpyAsync(e->d_cnt, &fresh, sizeof(Counters), cudaMemcpyHostToDevice, e->stream));
                MPX_CUDA(cudaStreamSynchronize(e->stream));
                step = at;
                pending = false;
                ++chunk_id;
                continue;
            }
        }
        if (!issued) break;
        pending = true;
        pending_slot = chunk_id & 1;
        ++chunk_id;
    }
    MPX_CUDA(cudaMemcpyAsync(e->h_cnt, e->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, e->stream));
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    e->last_gates = L;
    if (graphable && !replayed && e->store_gen == gen0 && e->h_cnt->err == 0) {
        // the range ran without growing the store: capture it for the next call
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        bool ok = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            for (uint64_t st = glo; st < hi; ++st) gate(e, cd.d_desc, static_cast<uint32_t>(L - 1 - st), static_cast<uint32_t>(st));
            ok = cudaStreamEndCapture(e->stream, &graph) == cudaSuccess && graph != nullptr;
        }
        ok = ok && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
        if (graph != nullptr) cudaGraphDestroy(graph);
        if (ok) {
            if (e->graphs.size() >= 16) {
                cudaGraphExecDestroy(e->graphs.front().exec);
                e->graphs.erase(e->graphs.begin());
            }
            e->graphs.push_back({cd.id, glo, hi, gen0, e->fwd_tape.w_anti, e->fwd_tape.r_src, e->fwd_tape.r_cap, exec});
        }
        else {
            e->use_graphs = false; // capture unavailable here: keep issuing kernels directly
        }
        cudaGetLastError();
    }
    if (e->profile) {
        e->t_sweep_ms = e->t_resolve_ms = e->t_columns_ms = 0.0;
        for (uint64_t st = lo; st < hi; ++st) {
            float a = 0.f, b = 0.f, c = 0.f;
            MPX_CUDA(cudaEventElapsedTime(&a, e->pev[4 * st], e->pev[4 * st + 1]));
            MPX_CUDA(cudaEventElapsedTime(&b, e->pev[4 * st + 1], e->pev[4 * st + 2]));
            c = 0.0f; // no per-gate column launch: the resolve ORs the appended terms' bits
            e->t_sweep_ms += a;
            e->t_resolve_ms += b;
            e->t_columns_ms += c;
        }
        e->n_sweep = hi - lo;
    }
    if (e->h_cnt->err != 0)
        return fail(eng, MPX_ERR_STATE, "hash table probe limit reached (internal error); the store is invalid");
    return MPX_OK;
}

mpx_status run_circuit(mpx_engine *e, const CircuitDev &cd) {
    e->adj.circuit = nullptr; // a plain propagation invalidates a pending gradient
    return run_range(e, cd, 0, cd.n);
}

mpx_status load_initial(mpx_engine *eng) {
    mpx_engine *e = eng;
    const int W = e->W;
    if (e->n_init > 0) {
        MPX_CUDA(cudaMemcpyAsync(e->st.keys, e->d_init_keys, e->n_init * W * sizeof(uint64_t),
                                 cudaMemcpyDeviceToDevice, e->stream));
        MPX_CUDA(cudaMemcpyAsync(e->st.coef, e->d_init_coef, e->n_init * sizeof(double), cudaMemcpyDeviceToDevice,
                                 e->stream));
    }
    MPX_CUDA(cudaMemsetAsync(e->st.table, 0xFF, (e->st.tmask + 1) * sizeof(unsigned long long), e->stream));
    {
        // clear the column bits of the terms the previous propagation appended
        const uint64_t w0 = (e->n_init + 31) / 32;
        if (w0 < e->st.cstride)
            MPX_CUDA(cudaMemset2DAsync(e->st.cols + w0, e->st.cstride * sizeof(uint32_t), 0,
                                       (e->st.cstride - w0) * sizeof(uint32_t), 64 * W + 1, e->stream));
    }
    pick_build(W)(e, 0, e->n_init);
    e->launches += e->n_init > 0 ? 2 : 0;
    Counters c{};
    c.n = e->n_init;
    c.n0 = e->n_init;
    c.stall = kNoStall;
    c.err = 0;
    MPX_CUDA(cudaMemcpyAsync(e->d_cnt, &c, sizeof(Counters), cudaMemcpyHostToDevice, e->stream));
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    e->last_gates = 0;
    return MPX_OK;
}

// ----- gradient (adjoint) -------------------------------------------------------------------------------

void free_adjoint(mpx_engine *e) {
    for (double *p : e->adj.ck_coef)
        dev_free(e, p);
    dev_free(e, e->adj.final_coef);
    dev_free(e, e->adj.w_anti);
    dev_free(e, e->adj.r_src);
    dev_free(e, e->adj.r_tgt);
    dev_free(e, e->adj.r_code);
    dev_free(e, e->adj.r_begin);
    dev_free(e, e->adj.longb);
    for (void *p : {static_cast<void *>(e->adj.r_vs), static_cast<void *>(e->adj.r_vt),
                    static_cast<void *>(e->adj.f_uidx), static_cast<void *>(e->adj.f_uval),
                    static_cast<void *>(e->adj.f_utotal), static_cast<void *>(e->adj.f_ubegin)})
        dev_free(e, p);
    e->adj = AdjointState{};
    e->fwd_tape = Tape{};
}

// Forward pass for the gradient: resets the store to the initial operator, propagates the circuit
// segment by segment (segment_gates gates each) and saves the coefficient array at every segment start
// and at the end. With log_all, and when the previous gradient forward pass of this engine says how many
// undo records the circuit needs and they fit in free device memory, the pass also logs everything the
// reverse sweep needs (undo log, both values of every pair), so the backward pass replays nothing.
mpx_status adjoint_forward(mpx_engine *eng, const CircuitDev &cd, uint64_t segment_gates, bool log_all = false) {
    mpx_engine *e = eng;
    free_adjoint(e);
    mpx_status s = load_initial(e);
    if (s != MPX_OK) return s;
    const uint64_t L = cd.n;
    const uint64_t K = segment_gates == 0 ? std::max<uint64_t>(L, 1) : segment_gates;
    uint64_t n = e->n_init;
    const uint64_t n_warps = static_cast<uint64_t>(e->grid) * kWarps;
    MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&e->adj.w_anti), std::max<uint64_t>(L, 1) * n_warps * sizeof(uint32_t)));
    e->fwd_tape.w_anti = e->adj.w_anti;
    // The pair log: sized by what the last recording pass needed (or the store capacity), checked after.
    if (e->pair_log != 0) {
        uint64_t r_cap = e->pair_log > 0 ? static_cast<uint64_t>(e->pair_log)
                                         : std::max<uint64_t>({e->rec_hint + e->rec_hint / 4, e->st.cap, 1ULL << 16});
        // at most half of the free device memory, so that the store, the checkpoints and the backward
        // tape still fit (9 bytes per record)
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) r_cap = std::min<uint64_t>(r_cap, free_b / 2 / 9);
        cudaError_t ce = dev_alloc(e, reinterpret_cast<void **>(&e->adj.r_src), r_cap * sizeof(uint32_t));
        if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&e->adj.r_tgt), r_cap * sizeof(uint32_t));
        if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&e->adj.r_code), r_cap * sizeof(int8_t));
        if (ce == cudaSuccess)
            ce = dev_alloc(e, reinterpret_cast<void **>(&e->adj.r_begin), std::max<uint64_t>(L, 1) * sizeof(uint64_t));
        if (ce == cudaSuccess) {
            e->fwd_tape.r_src = e->adj.r_src;
            e->fwd_tape.r_tgt = e->adj.r_tgt;
            e->fwd_tape.r_code = e->adj.r_code;
            e->fwd_tape.r_begin = e->adj.r_begin;
            e->fwd_tape.r_cap = r_cap;
        }
        else {
            cudaGetLastError(); // no room for a log: the backward pass replays with the streaming kernels
        }
    }
    if (log_all && e->fwd_tape.r_src != nullptr && e->undo_hint > 0) {
        AdjointState &A = e->adj;
        const uint64_t u_cap = e->undo_hint + e->undo_hint / 16 + (1ULL << 16);
        const uint64_t r_cap = e->fwd_tape.r_cap;
        // large blocks come from power-of-two classes (dev_alloc)
        const size_t need = next_pow2(u_cap * sizeof(uint32_t)) + next_pow2(u_cap * sizeof(double)) +
                            2 * next_pow2(r_cap * sizeof(double)) + (L + 2) * sizeof(uint64_t);
        // headroom for the store's growth and the backward pass's adjoint arrays
        const size_t reserve = (size_t{4} << 30) + static_cast<size_t>(e->st.cap) * 24;
        if (need + reserve <= device_available(e)) {
            cudaError_t ce = dev_alloc(e, reinterpret_cast<void **>(&A.f_uidx), u_cap * sizeof(uint32_t));
            if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&A.f_uval), u_cap * sizeof(double));
            if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&A.r_vs), r_cap * sizeof(double));
            if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&A.r_vt), r_cap * sizeof(double));
            if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&A.f_utotal), sizeof(unsigned long long));
            if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&A.f_ubegin), (L + 1) * sizeof(uint64_t));
            if (ce == cudaSuccess) ce = cudaMemsetAsync(A.f_utotal, 0, sizeof(unsigned long long), e->stream);
            if (ce == cudaSuccess) ce = cudaMemsetAsync(A.f_ubegin, 0, (L + 1) * sizeof(uint64_t), e->stream);
            if (ce == cudaSuccess) {
                A.f_ucap = u_cap;
                e->fwd_tape.r_vs = A.r_vs;
                e->fwd_tape.r_vt = A.r_vt;
                e->fwd_tape.f_uidx = A.f_uidx;
                e->fwd_tape.f_uval = A.f_uval;
                e->fwd_tape.f_utotal = A.f_utotal;
                e->fwd_tape.f_ubegin = A.f_ubegin;
                e->fwd_tape.f_ucap = u_cap;
            }
            else {
                cudaGetLastError(); // no room after all: the backward pass replays segments
                for (void *p : {static_cast<void *>(A.r_vs), static_cast<void *>(A.r_vt),
                                static_cast<void *>(A.f_uidx), static_cast<void *>(A.f_uval),
                                static_cast<void *>(A.f_utotal), static_cast<void *>(A.f_ubegin)})
                    dev_free(e, p);
                A.r_vs = A.r_vt = nullptr;
                A.f_uidx = nullptr;
                A.f_uval = nullptr;
                A.f_utotal = nullptr;
                A.f_ubegin = nullptr;
            }
        }
    }
    for (uint64_t lo = 0; lo < L; lo += K) {
        double *ck = nullptr;
        MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&ck), std::max<uint64_t>(n, 1) * sizeof(double)));
        e->adj.ck_coef.push_back(ck);
        if (n > 0) MPX_CUDA(cudaMemcpyAsync(ck, e->st.coef, n * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
        e->adj.seg_lo.push_back(lo);
        e->adj.ck_n.push_back(n);
        s = run_range(e, cd, lo, std::min(L, lo + K));
        if (s != MPX_OK) {
            free_adjoint(e);
            return s;
        }
        n = e->h_cnt->n;
    }
    if (e->fwd_tape.r_src != nullptr) {
        e->adj.r_total = e->h_cnt->rec_total;
        e->adj.rec_ok = e->adj.r_total <= e->fwd_tape.r_cap;
        e->rec_hint = std::max(e->rec_hint, e->adj.r_total);
    }
    if (e->fwd_tape.f_utotal != nullptr) {
        unsigned long long u_total = 0;
        MPX_CUDA(cudaMemcpyAsync(&u_total, e->fwd_tape.f_utotal, sizeof(u_total), cudaMemcpyDeviceToHost, e->stream));
        MPX_CUDA(cudaStreamSynchronize(e->stream));
        e->adj.log_ok = e->adj.rec_ok && u_total <= e->adj.f_ucap;
    }
    e->fwd_tape = Tape{};
    if (e->tr.has_len_k) {
        // only_rotate_len_k: which terms of the final store lie outside every gate's rotation set
        e->adj.len_k = e->tr.len_k;
        const uint64_t words = std::max<uint64_t>((n + 31) / 32, 1);
        MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&e->adj.longb), words * sizeof(uint32_t)));
        if (n > 0) {
            const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 4096));
            pick_long_bits(e->W)(e, n, e->tr.len_k, e->adj.longb, blocks);
            ++e->launches;
        }
    }
    MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&e->adj.final_coef), std::max<uint64_t>(n, 1) * sizeof(double)));
    if (n > 0)
        MPX_CUDA(cudaMemcpyAsync(e->adj.final_coef, e->st.coef, n * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
    e->adj.n_final = n;
    e->adj.L = L;
    e->adj.stats.assign(4 * L, 0);
    if (L > 0)
        MPX_CUDA(cudaMemcpyAsync(e->adj.stats.data(), e->d_stats, 4 * L * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                 e->stream));
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    e->last_gates = L;
    e->adj.circuit = &cd;
    // undo records the circuit needs (every anticommuting term of every gate): sizes the next pass's log
    uint64_t undo = 0;
    for (uint64_t st = 0; st < L; ++st) undo += e->adj.stats[4 * st + 1];
    if (log_all) e->undo_hint = undo;
    return MPX_OK;
}

// Reverse sweep over the logs of a forward pass that logged everything (AdjointState::log_ok): no
// checkpoint, no replay. Pair members keep their undo records (the sweep wrote them before the resolve
// knew the pairs), so each gate runs the pairs kernel, which marks them done, then the undo kernel.
mpx_status adjoint_backward_logged(mpx_engine *eng, const CircuitDev &cd, double *grad_angles) {
    mpx_engine *e = eng;
    AdjointState &A = e->adj;
    const uint64_t L = A.L, nf = A.n_final;
    std::vector<uint64_t> ub(L + 1), rb(L);
    MPX_CUDA(cudaMemcpyAsync(ub.data(), A.f_ubegin, (L + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, e->stream));
    MPX_CUDA(cudaMemcpyAsync(rb.data(), A.r_begin, L * sizeof(uint64_t), cudaMemcpyDeviceToHost, e->stream));
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    std::vector<unsigned long long> cnts(2 * L);
    for (uint64_t st = 0; st < L; ++st) {
        cnts[st] = ub[st + 1] - ub[st];
        cnts[L + st] = (st + 1 < L ? rb[st + 1] : A.r_total) - rb[st];
    }
    unsigned long long *d_cnts = nullptr; // u_cnt | p_cnt
    double *lam = nullptr, *grad = nullptr, *gpart = nullptr;
    uint32_t *done = nullptr;
    cudaError_t ce = cudaSuccess;
    auto A_ = [&](void **ptr, size_t bytes) {
        if (ce == cudaSuccess) ce = dev_alloc(e, ptr, std::max<size_t>(bytes, 16));
    };
    A_(reinterpret_cast<void **>(&d_cnts), 2 * L * sizeof(unsigned long long));
    A_(reinterpret_cast<void **>(&lam), nf * sizeof(double));
    A_(reinterpret_cast<void **>(&grad), L * sizeof(double));
    A_(reinterpret_cast<void **>(&done), ((nf + 31) / 32) * sizeof(uint32_t));
    A_(reinterpret_cast<void **>(&gpart), (2 * static_cast<size_t>(e->grid) + 1) * sizeof(double));
    auto release = [&]() {
        for (void *ptr : {static_cast<void *>(d_cnts), static_cast<void *>(lam), static_cast<void *>(grad),
                          static_cast<void *>(done), static_cast<void *>(gpart)})
            dev_free(e, ptr);
    };
    if (ce != cudaSuccess) {
        cudaGetLastError();
        release();
        return fail(eng, MPX_ERR_NOMEM, std::string("gradient allocation failed: ") + cudaGetErrorString(ce));
    }
#define MPX_CUDA_REL(call)                                                                                          \
    do {                                                                                                            \
        cudaError_t e2_ = (call);                                                                                   \
        if (e2_ != cudaSuccess) {                                                                                   \
            release();                                                                                              \
            return fail(eng, MPX_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e2_));                     \
        }                                                                                                           \
    } while (0)
    MPX_CUDA_REL(cudaMemcpyAsync(d_cnts, cnts.data(), 2 * L * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                                 e->stream));
    MPX_CUDA_REL(cudaMemsetAsync(grad, 0, L * sizeof(double), e->stream));
    MPX_CUDA_REL(cudaMemsetAsync(done, 0, std::max<uint64_t>((nf + 31) / 32, 1) * sizeof(uint32_t), e->stream));
    const GradPartials gp{gpart, reinterpret_cast<unsigned int *>(gpart + 2 * static_cast<size_t>(e->grid))};
    MPX_CUDA_REL(cudaMemsetAsync(gp.arrivals, 0, sizeof(unsigned int), e->stream));
    if (e->schr) {
        MPX_CUDA_REL(cudaMemsetAsync(lam, 0, std::max<uint64_t>(nf, 1) * sizeof(double), e->stream));
        if (e->n_obs > 0 && nf > 0) {
            pick_lookup(e->W)(e, e->d_obs_keys, e->n_obs, nf, e->d_obs_idx);
            k_scatter<<<static_cast<unsigned>(std::min<uint64_t>((e->n_obs + 255) / 256, 4096)), 256, 0, e->stream>>>(
                lam, e->d_obs_idx, e->d_obs_coef, e->n_obs);
        }
    }
    else {
        pick_adj_init(e->W, e->cfg.basis)(e, lam, 0, nf);
    }
    Tape tp{};
    tp.u_idx = A.f_uidx;
    tp.u_val = A.f_uval;
    tp.u_base = A.f_ubegin;
    tp.u_cnt = d_cnts;
    tp.p_src = A.r_src;
    tp.p_tgt = A.r_tgt;
    tp.p_code = A.r_code;
    tp.p_vs = A.r_vs;
    tp.p_vt = A.r_vt;
    tp.p_base = A.r_begin;
    tp.p_cnt = d_cnts + L;
    for (uint64_t st = L; st-- > 0;) {
        const uint32_t gate = static_cast<uint32_t>(L - 1 - st);
        launch_dep(e, &k_adj_pairs, tp, static_cast<const GateDesc *>(cd.d_desc), gate, static_cast<uint32_t>(st), lam,
                   done, gp);
        launch_dep(e, &k_adj_undo, tp, static_cast<const GateDesc *>(cd.d_desc), gate, static_cast<uint32_t>(st), lam,
                   done, gp, grad);
    }
    e->launches += 2 * L + 1;
    MPX_CUDA_REL(cudaGetLastError());
    MPX_CUDA_REL(cudaMemcpyAsync(grad_angles, grad, L * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    MPX_CUDA_REL(cudaStreamSynchronize(e->stream));
#undef MPX_CUDA_REL
    release();
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    return MPX_OK;
}

// Values the replay starts terms [lo, hi) of the final store from: the reference-state score in the
// Schrodinger picture; otherwise 0, and with `with_start` the re-weighted initial operator's terms in that
// range (mpx_update_initial_operator; frozen_forward starts from them). A segment's checkpoint holds the
// terms that existed at its start; the frozen pair kernel reads an appended partner's slot at its gate, so
// the later slots must hold these values again before the segment is replayed.
mpx_status replay_start_tail(mpx_engine *eng, uint64_t lo, uint64_t hi, bool with_start) {
    mpx_engine *e = eng;
    if (hi <= lo) return MPX_OK;
    if (e->schr) {
        pick_adj_init(e->W, e->cfg.basis)(e, e->st.coef, lo, hi);
    }
    else {
        MPX_CUDA(cudaMemsetAsync(e->st.coef + lo, 0, (hi - lo) * sizeof(double), e->stream));
        if (with_start && e->start_on && e->n_start > 0)
            k_scatter<<<static_cast<unsigned>(std::min<uint64_t>((e->n_start + 255) / 256, 4096)), 256, 0, e->stream>>>(
                e->st.coef, e->d_start_idx, e->d_start_val, e->n_start, static_cast<uint32_t>(lo));
    }
    MPX_CUDA(cudaGetLastError());
    return MPX_OK;
}

// Reverse sweep: per segment (last first) restore its checkpoint, replay it logging the tape, then walk
// its gates backwards. grad_angles[l] = dE/d(angle_l) for circuit layer l (angle = theta[map] * g).
// With fg == nullptr: the gradient of the last mpx_adjoint_forward (segments replayed with the
// streaming kernels). With fg: the gradient of the frozen structure fg at the circuit's current angles
// (segments replayed with the frozen kernels, whose pair counts are fixed).
mpx_status adjoint_backward(mpx_engine *eng, const CircuitDev &cd, double *grad_angles, const FrozenGraph *fg = nullptr) {
    mpx_engine *e = eng;
    AdjointState &A = e->adj;
    const uint64_t L = A.L;
    const uint64_t nf = A.n_final;
    const size_t S = A.seg_lo.size();
    // per-step bases of the tape (prefix sums within each segment) and store sizes after each step
    std::vector<uint64_t> u_base(L), p_base(L), n_next(L);
    uint64_t u_max = 1, p_max = 1;
    for (size_t sg = 0; sg < S; ++sg) {
        const uint64_t lo = A.seg_lo[sg], hi = sg + 1 < S ? A.seg_lo[sg + 1] : L;
        uint64_t u = 0, p = 0;
        for (uint64_t st = lo; st < hi; ++st) {
            u_base[st] = u;
            p_base[st] = p;
            u += A.stats[4 * st + 1];
            p += A.stats[4 * st + 2];
            n_next[st] = st + 1 < L ? A.stats[4 * (st + 1)] : nf;
        }
        u_max = std::max(u_max, u);
        p_max = std::max(p_max, p);
    }
    Tape tp{};
    uint64_t *d_steps = nullptr;  // u_base | p_base | n_next
    unsigned long long *d_cnts = nullptr; // u_cnt | p_cnt
    double *lam = nullptr, *grad = nullptr;
    double *gpart = nullptr; // per-block partials of dE/dangle, then the arrival counter (GradPartials)
    uint32_t *done = nullptr;
    cudaError_t ce = cudaSuccess;
    auto A_ = [&](void **ptr, size_t bytes) {
        if (ce == cudaSuccess) ce = dev_alloc(e, ptr, std::max<size_t>(bytes, 16));
    };
    A_(reinterpret_cast<void **>(&tp.u_idx), u_max * sizeof(uint32_t));
    A_(reinterpret_cast<void **>(&tp.u_val), u_max * sizeof(double));
    A_(reinterpret_cast<void **>(&tp.p_src), p_max * sizeof(uint32_t));
    A_(reinterpret_cast<void **>(&tp.p_tgt), p_max * sizeof(uint32_t));
    A_(reinterpret_cast<void **>(&tp.p_code), p_max * sizeof(int8_t));
    A_(reinterpret_cast<void **>(&tp.p_vs), p_max * sizeof(double));
    A_(reinterpret_cast<void **>(&tp.p_vt), p_max * sizeof(double));
    A_(reinterpret_cast<void **>(&d_steps), 3 * L * sizeof(uint64_t));
    A_(reinterpret_cast<void **>(&d_cnts), 2 * L * sizeof(unsigned long long));
    A_(reinterpret_cast<void **>(&lam), nf * sizeof(double));
    A_(reinterpret_cast<void **>(&grad), L * sizeof(double));
    A_(reinterpret_cast<void **>(&done), ((nf + 31) / 32) * sizeof(uint32_t));
    A_(reinterpret_cast<void **>(&gpart), (2 * static_cast<size_t>(e->grid) + 1) * sizeof(double));
    auto release = [&]() {
        for (void *ptr : {static_cast<void *>(tp.u_idx), static_cast<void *>(tp.u_val), static_cast<void *>(tp.p_src),
                          static_cast<void *>(tp.p_tgt), static_cast<void *>(tp.p_code), static_cast<void *>(tp.p_vs),
                          static_cast<void *>(tp.p_vt), static_cast<void *>(d_steps), static_cast<void *>(d_cnts),
                          static_cast<void *>(lam), static_cast<void *>(grad), static_cast<void *>(done),
                          static_cast<void *>(gpart)})
            dev_free(e, ptr);
    };
    if (ce != cudaSuccess) {
        cudaGetLastError();
        release();
        return fail(eng, MPX_ERR_NOMEM, std::string("gradient tape allocation failed (use shorter segments): ") +
                                            cudaGetErrorString(ce));
    }
    tp.u_base = d_steps;
    tp.p_base = d_steps + L;
    tp.n_next = d_steps + 2 * L;
    tp.u_cnt = d_cnts;
    tp.p_cnt = d_cnts + L;
#define MPX_CUDA_REL(call)                                                                                          \
    do {                                                                                                            \
        cudaError_t e2_ = (call);                                                                                   \
        if (e2_ != cudaSuccess) {                                                                                   \
            release();                                                                                              \
            if (e2_ == cudaErrorMemoryAllocation) cudaGetLastError();                                             \
            return fail(eng, e2_ == cudaErrorMemoryAllocation ? MPX_ERR_NOMEM : MPX_ERR_CUDA,                      \
                        std::string(#call ": ") + cudaGetErrorString(e2_));                                         \
        }                                                                                                           \
    } while (0)
    MPX_CUDA_REL(cudaMemcpyAsync(d_steps, u_base.data(), L * sizeof(uint64_t), cudaMemcpyHostToDevice, e->stream));
    MPX_CUDA_REL(cudaMemcpyAsync(d_steps + L, p_base.data(), L * sizeof(uint64_t), cudaMemcpyHostToDevice, e->stream));
    MPX_CUDA_REL(cudaMemcpyAsync(d_steps + 2 * L, n_next.data(), L * sizeof(uint64_t), cudaMemcpyHostToDevice, e->stream));
    MPX_CUDA_REL(cudaMemsetAsync(d_cnts, 0, 2 * L * sizeof(unsigned long long), e->stream));
    if (fg != nullptr)
        MPX_CUDA_REL(cudaMemcpyAsync(d_cnts + L, fg->p_count, L * sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                     e->stream));
    const uint32_t n_warps = static_cast<uint32_t>(e->grid) * kWarps;
    uint64_t max_seg = 1;
    for (size_t sg = 0; sg < S; ++sg) max_seg = std::max<uint64_t>(max_seg, (sg + 1 < S ? A.seg_lo[sg + 1] : L) - A.seg_lo[sg]);
    uint64_t *u_off = nullptr;
    MPX_CUDA_REL(dev_alloc(e, reinterpret_cast<void **>(&u_off), max_seg * n_warps * sizeof(uint64_t)));
    tp.w_anti = A.w_anti;
    tp.u_off = u_off;
    MPX_CUDA_REL(cudaMemsetAsync(grad, 0, L * sizeof(double), e->stream));
    MPX_CUDA_REL(cudaMemsetAsync(done, 0, ((nf + 31) / 32) * sizeof(uint32_t), e->stream));
    const GradPartials gp{gpart, reinterpret_cast<unsigned int *>(gpart + 2 * static_cast<size_t>(e->grid))};
    MPX_CUDA_REL(cudaMemsetAsync(gp.arrivals, 0, sizeof(unsigned int), e->stream));
    if (e->schr) {
        // Schrodinger: <O> = core + sum_t o_t state[idx_t], so the adjoint of the final state is the
        // observable at its terms' store rows (0 elsewhere)
        MPX_CUDA_REL(cudaMemsetAsync(lam, 0, std::max<uint64_t>(nf, 1) * sizeof(double), e->stream));
        if (e->n_obs > 0 && nf > 0) {
            pick_lookup(e->W)(e, e->d_obs_keys, e->n_obs, nf, e->d_obs_idx);
            k_scatter<<<static_cast<unsigned>(std::min<uint64_t>((e->n_obs + 255) / 256, 4096)), 256, 0, e->stream>>>(
                lam, e->d_obs_idx, e->d_obs_coef, e->n_obs);
        }
    }
    else {
        pick_adj_init(e->W, e->cfg.basis)(e, lam, 0, nf);
    }
    const ReplayFn replay = pick_replay(e->W, e->cfg.basis);
    const FrozenFn frozen_replay = pick_frozen<true>(e->W);
    Frozen fz{};
    if (fg != nullptr) fz = fg->view();
    for (size_t sg = S; sg-- > 0;) {
        const uint64_t lo = A.seg_lo[sg], hi = sg + 1 < S ? A.seg_lo[sg + 1] : L;
        const uint64_t n = A.ck_n[sg];
        if (n > 0)
            MPX_CUDA_REL(cudaMemcpyAsync(e->st.coef, A.ck_coef[sg], n * sizeof(double), cudaMemcpyDeviceToDevice,
                                         e->stream));
        if (fg != nullptr && nf > n) {
            const mpx_status ts = replay_start_tail(e, n, nf, fg == &e->fg);
            if (ts != MPX_OK) {
                release();
                return ts;
            }
        }
        Counters c{};
        c.n = n;
        c.n0 = n;
        c.stall = kNoStall;
        MPX_CUDA_REL(cudaMemcpyAsync(e->d_cnt, &c, sizeof(Counters), cudaMemcpyHostToDevice, e->stream));
        k_undo_offsets<<<static_cast<unsigned>(hi - lo), 1024, 0, e->stream>>>(tp, n_warps, lo, u_off);
        tp.u_off_step0 = lo;
        for (uint64_t st = lo; st < hi; ++st) {
            if (fg != nullptr)
                frozen_replay(e, cd.d_desc, fz, static_cast<uint32_t>(L - 1 - st), static_cast<uint32_t>(st), fg->n0[st],
                              done, tp);
            else
                replay(e, cd.d_desc, static_cast<uint32_t>(L - 1 - st), static_cast<uint32_t>(st), tp);
        }
        for (uint64_t st = hi; st-- > lo;) {
            const uint32_t gate = static_cast<uint32_t>(L - 1 - st);
            if (fg != nullptr) {
                // frozen replay: pair members carry the skip index in the undo log, one launch per step
                launch_dep(e, &k_adj_step, tp, static_cast<const GateDesc *>(cd.d_desc), gate, static_cast<uint32_t>(st),
                           lam, gp, grad);
            }
            else {
                launch_dep(e, &k_adj_pairs, tp, static_cast<const GateDesc *>(cd.d_desc), gate, static_cast<uint32_t>(st),
                           lam, done, gp);
                launch_dep(e, &k_adj_undo, tp, static_cast<const GateDesc *>(cd.d_desc), gate, static_cast<uint32_t>(st),
                           lam, done, gp, grad);
            }
        }
        e->launches += (fg != nullptr ? 3 : 5) * (hi - lo) + 1;
        MPX_CUDA_REL(cudaGetLastError());
    }
    e->launches += 1;
    // the engine keeps the evolved operator of the forward pass (a single segment replayed from the start
    // has just left it in the store)
    if (nf > 0 && A.final_coef != nullptr)
        MPX_CUDA_REL(cudaMemcpyAsync(e->st.coef, A.final_coef, nf * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
    MPX_CUDA_REL(cudaMemcpyAsync(e->h_cnt, e->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, e->stream));
    MPX_CUDA_REL(cudaMemcpyAsync(grad_angles, grad, L * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    MPX_CUDA_REL(cudaStreamSynchronize(e->stream));
    const uint32_t err = e->h_cnt->err;
    Counters c{};
    c.n = nf;
    c.n0 = nf;
    c.stall = kNoStall;
    MPX_CUDA_REL(cudaMemcpyAsync(e->d_cnt, &c, sizeof(Counters), cudaMemcpyHostToDevice, e->stream));
    release();
    dev_free(e, u_off);
    MPX_CUDA(cudaStreamSynchronize(e->stream));
#undef MPX_CUDA_REL
    if (err != 0) return fail(eng, MPX_ERR_STATE, "gradient replay diverged from the forward pass (internal error)");
    return MPX_OK;
}

// ----- frozen structure (graph) -----------------------------------------------------------------------

// The pairs a recording forward pass logged, as a frozen structure over the adjoint state's arrays (the
// view owns only p_count, filled here).
mpx_status recorded_view(mpx_engine *eng, FrozenGraph &v) {
    mpx_engine *e = eng;
    const AdjointState &A = e->adj;
    const uint64_t L = A.L;
    std::vector<uint64_t> begin(L);
    if (L > 0)
        MPX_CUDA(cudaMemcpyAsync(begin.data(), A.r_begin, L * sizeof(uint64_t), cudaMemcpyDeviceToHost, e->stream));
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    v = FrozenGraph{};
    v.L = L;
    v.n_final = A.n_final;
    v.src = A.r_src;
    v.tgt = A.r_tgt;
    v.code = A.r_code;
    v.p_begin = A.r_begin;
    v.w_anti = A.w_anti;
    v.longb = A.longb;
    v.forward_len_k = true;
    v.n0.resize(L);
    v.anti.resize(L);
    v.count.resize(L);
    for (uint64_t st = 0; st < L; ++st) {
        v.n0[st] = A.stats[4 * st];
        v.anti[st] = A.stats[4 * st + 1];
        v.count[st] = (st + 1 < L ? begin[st + 1] : A.r_total) - begin[st];
    }
    MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&v.p_count), std::max<uint64_t>(L, 1) * sizeof(unsigned long long)));
    if (L > 0)
        MPX_CUDA(cudaMemcpyAsync(v.p_count, v.count.data(), L * sizeof(uint64_t), cudaMemcpyHostToDevice, e->stream));
    return MPX_OK;
}

void free_graph(mpx_engine *e) {
    FrozenGraph &g = e->fg;
    for (void *p : {static_cast<void *>(g.src), static_cast<void *>(g.tgt), static_cast<void *>(g.code),
                    static_cast<void *>(g.p_begin), static_cast<void *>(g.p_count), static_cast<void *>(g.w_anti),
                    static_cast<void *>(g.done), static_cast<void *>(g.last), static_cast<void *>(g.longb)})
        dev_free(e, p);
    g = FrozenGraph{};
}

template <int W>
void launch_pare_init(mpx_engine *e, uint64_t n, int32_t keep_paired, int32_t last_step, int32_t *last) {
    const uint64_t blocks = std::min<uint64_t>((n + kBlock - 1) / kBlock, static_cast<uint64_t>(e->grid) * 4);
    k_pare_init<W><<<static_cast<unsigned>(std::max<uint64_t>(blocks, 1)), kBlock, 0, e->stream>>>(e->st.keys, n,
                                                                                                 keep_paired, last_step,
                                                                                                 last);
}
using PareInitFn = void (*)(mpx_engine *, uint64_t, int32_t, int32_t, int32_t *);
PareInitFn pick_pare_init(int W) {
    switch (W) {
    case 1: return &launch_pare_init<1>;
    case 2: return &launch_pare_init<2>;
    case 3: return &launch_pare_init<3>;
    case 4: return &launch_pare_init<4>;
    case 5: return &launch_pare_init<5>;
    case 6: return &launch_pare_init<6>;
    case 7: return &launch_pare_init<7>;
    default: return &launch_pare_init<8>;
    }
}

// Pares the frozen graph at `threshold` (the reference's pare_graph, PareGraph.cpp:103-141): last[i] from
// the driving vector (the reference state's scores; in the Schrodinger picture the observable), then one
// backward step per layer over its pairs.
mpx_status graph_pare(mpx_engine *eng, double threshold) {
    mpx_engine *e = eng;
    FrozenGraph &g = e->fg;
    if (threshold < 0.0) { // a negative threshold keeps every term (indices_above): no paring
        g.pared = false;
        return MPX_OK;
    }
    if (g.last != nullptr && g.last_for == threshold) {
        g.pared = true;
        return MPX_OK;
    }
    if (g.last == nullptr)
        MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&g.last), std::max<uint64_t>(g.n_final, 1) * sizeof(int32_t)));
    if (e->schr) {
        // Schrodinger: the driving vector is the observable (MonomialPropagator.inl:960-962): its terms
        // above the threshold are the ones kept after the last step
        MPX_CUDA(cudaMemsetAsync(g.last, 0xFF, std::max<uint64_t>(g.n_final, 1) * sizeof(int32_t), e->stream));
        if (e->n_obs > 0 && g.n_final > 0) {
            pick_lookup(e->W)(e, e->d_obs_keys, e->n_obs, g.n_final, e->d_obs_idx);
            k_pare_seed<<<static_cast<unsigned>(std::min<uint64_t>((e->n_obs + 255) / 256, 4096)), 256, 0, e->stream>>>(
                e->d_obs_idx, e->d_obs_coef, e->n_obs, threshold, static_cast<int32_t>(g.L) - 1, g.last);
        }
    }
    else {
        // |weight| = 1 on fully paired terms: kept iff 1 > threshold
        pick_pare_init(e->W)(e, g.n_final, 1.0 > threshold ? 1 : 0, static_cast<int32_t>(g.L) - 1, g.last);
    }
    const Frozen fz = Frozen{g.src, g.tgt, g.code, g.p_begin, g.p_count, nullptr, nullptr};
    for (uint64_t st = g.L; st-- > 0;) {
        const uint64_t cnt = g.count[st];
        if (cnt == 0) continue;
        const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((cnt + kBlock - 1) / kBlock,
                                                                         static_cast<uint64_t>(e->grid)));
        k_pare_step<<<blocks, kBlock, 0, e->stream>>>(fz, static_cast<uint32_t>(st), g.last);
        ++e->launches;
    }
    MPX_CUDA(cudaGetLastError());
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    g.pared = true;
    g.last_for = threshold;
    return MPX_OK;
}

// Build: the gradient forward pass (checkpoints, per-warp counts), then every segment replayed once with
// the streaming kernels to collect each gate's pairs into the graph.
// Drops a re-weighted initial operator (mpx_update_initial_operator): reset and graph builds start from
// the constructor's operator again.
void clear_start(mpx_engine *e) {
    dev_free(e, e->d_start_idx);
    dev_free(e, e->d_start_val);
    e->d_start_idx = nullptr;
    e->d_start_val = nullptr;
    e->n_start = 0;
    e->start_on = false;
}

mpx_status graph_build(mpx_engine *eng, const CircuitDev &cd, uint64_t segment_gates) {
    mpx_engine *e = eng;
    free_graph(e);
    clear_start(e);
    mpx_status s = adjoint_forward(e, cd, segment_gates);
    if (s != MPX_OK) return s;
    AdjointState &A = e->adj;
    FrozenGraph &g = e->fg;
    const uint64_t L = A.L, nf = A.n_final;
    if (A.rec_ok) {
        // The forward pass logged every gate's pairs: the graph takes the log over, no replay needed.
        s = recorded_view(e, g);
        if (s != MPX_OK) return s;
        g.forward_len_k = false; // a built graph replays as the reference's graph (no length filter)
        g.circuit_id = cd.id;
        MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&g.done), std::max<uint64_t>((nf + 31) / 32, 4) * sizeof(uint32_t)));
        MPX_CUDA(cudaMemsetAsync(g.done, 0, ((nf + 31) / 32) * sizeof(uint32_t), e->stream));
        A.r_src = nullptr;
        A.r_tgt = nullptr;
        A.r_code = nullptr;
        A.r_begin = nullptr;
        A.longb = nullptr; // owned by the graph now
        A.w_anti = nullptr;
        free_adjoint(e);
        MPX_CUDA(cudaStreamSynchronize(e->stream));
        return MPX_OK;
    }
    const size_t S = A.seg_lo.size();
    std::vector<uint64_t> begin(L), u_base(L), n_next(L);
    uint64_t total_e = 0, u_max = 1;
    for (size_t sg = 0; sg < S; ++sg) {
        const uint64_t lo = A.seg_lo[sg], hi = sg + 1 < S ? A.seg_lo[sg + 1] : L;
        uint64_t u = 0;
        for (uint64_t st = lo; st < hi; ++st) {
            u_base[st] = u;
            u += A.stats[4 * st + 1];
            n_next[st] = st + 1 < L ? A.stats[4 * (st + 1)] : nf;
        }
        u_max = std::max(u_max, u);
    }
    for (uint64_t st = 0; st < L; ++st) {
        begin[st] = total_e;
        total_e += A.stats[4 * st + 2];
    }
    Tape tp{};
    uint64_t *d_steps = nullptr, *u_off = nullptr;
    unsigned long long *u_cnt = nullptr;
    cudaError_t ce = cudaSuccess;
    auto A_ = [&](void **ptr, size_t bytes) {
        if (ce == cudaSuccess) ce = dev_alloc(e, ptr, std::max<size_t>(bytes, 16));
    };
    const uint32_t n_warps = static_cast<uint32_t>(e->grid) * kWarps;
    uint64_t max_seg = 1;
    for (size_t sg = 0; sg < S; ++sg) max_seg = std::max<uint64_t>(max_seg, (sg + 1 < S ? A.seg_lo[sg + 1] : L) - A.seg_lo[sg]);
    A_(reinterpret_cast<void **>(&g.src), total_e * sizeof(uint32_t));
    A_(reinterpret_cast<void **>(&g.tgt), total_e * sizeof(uint32_t));
    A_(reinterpret_cast<void **>(&g.code), total_e * sizeof(int8_t));
    A_(reinterpret_cast<void **>(&g.p_begin), L * sizeof(uint64_t));
    A_(reinterpret_cast<void **>(&g.p_count), L * sizeof(unsigned long long));
    A_(reinterpret_cast<void **>(&g.done), ((nf + 31) / 32) * sizeof(uint32_t));
    A_(reinterpret_cast<void **>(&tp.p_vs), total_e * sizeof(double));
    A_(reinterpret_cast<void **>(&tp.p_vt), total_e * sizeof(double));
    A_(reinterpret_cast<void **>(&tp.u_idx), u_max * sizeof(uint32_t));
    A_(reinterpret_cast<void **>(&tp.u_val), u_max * sizeof(double));
    A_(reinterpret_cast<void **>(&d_steps), 2 * L * sizeof(uint64_t));
    A_(reinterpret_cast<void **>(&u_cnt), L * sizeof(unsigned long long));
    A_(reinterpret_cast<void **>(&u_off), max_seg * n_warps * sizeof(uint64_t));
    auto release = [&]() {
        for (void *ptr : {static_cast<void *>(tp.p_vs), static_cast<void *>(tp.p_vt), static_cast<void *>(tp.u_idx),
                          static_cast<void *>(tp.u_val), static_cast<void *>(d_steps), static_cast<void *>(u_cnt),
                          static_cast<void *>(u_off)})
            dev_free(e, ptr);
    };
    if (ce != cudaSuccess) {
        cudaGetLastError();
        release();
        free_graph(e);
        return fail(eng, MPX_ERR_NOMEM, std::string("graph allocation failed: ") + cudaGetErrorString(ce));
    }
    MPX_CUDA(cudaMemcpyAsync(g.p_begin, begin.data(), L * sizeof(uint64_t), cudaMemcpyHostToDevice, e->stream));
    MPX_CUDA(cudaMemsetAsync(g.p_count, 0, L * sizeof(unsigned long long), e->stream));
    MPX_CUDA(cudaMemsetAsync(g.done, 0, ((nf + 31) / 32) * sizeof(uint32_t), e->stream));
    MPX_CUDA(cudaMemcpyAsync(d_steps, u_base.data(), L * sizeof(uint64_t), cudaMemcpyHostToDevice, e->stream));
    MPX_CUDA(cudaMemcpyAsync(d_steps + L, n_next.data(), L * sizeof(uint64_t), cudaMemcpyHostToDevice, e->stream));
    tp.p_src = g.src;
    tp.p_tgt = g.tgt;
    tp.p_code = g.code;
    tp.p_base = g.p_begin;
    tp.p_cnt = g.p_count;
    tp.u_base = d_steps;
    tp.n_next = d_steps + L;
    tp.u_cnt = u_cnt;
    tp.w_anti = A.w_anti;
    tp.u_off = u_off;
    const ReplayFn replay = pick_replay(e->W, e->cfg.basis);
    for (size_t sg = 0; sg < S; ++sg) {
        const uint64_t lo = A.seg_lo[sg], hi = sg + 1 < S ? A.seg_lo[sg + 1] : L;
        const uint64_t n = A.ck_n[sg];
        if (n > 0)
            MPX_CUDA(cudaMemcpyAsync(e->st.coef, A.ck_coef[sg], n * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
        Counters c{};
        c.n = n;
        c.n0 = n;
        c.stall = kNoStall;
        MPX_CUDA(cudaMemcpyAsync(e->d_cnt, &c, sizeof(Counters), cudaMemcpyHostToDevice, e->stream));
        k_undo_offsets<<<static_cast<unsigned>(hi - lo), 1024, 0, e->stream>>>(tp, n_warps, lo, u_off);
        tp.u_off_step0 = lo;
        for (uint64_t st = lo; st < hi; ++st) replay(e, cd.d_desc, static_cast<uint32_t>(L - 1 - st), static_cast<uint32_t>(st), tp);
        e->launches += 3 * (hi - lo) + 1;
        MPX_CUDA(cudaGetLastError());
    }
    // the engine keeps the evolved operator of the build
    if (nf > 0) MPX_CUDA(cudaMemcpyAsync(e->st.coef, A.final_coef, nf * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
    MPX_CUDA(cudaMemcpyAsync(e->h_cnt, e->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, e->stream));
    g.count.assign(L, 0);
    MPX_CUDA(cudaMemcpyAsync(g.count.data(), g.p_count, L * sizeof(uint64_t), cudaMemcpyDeviceToHost, e->stream));
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    const uint32_t err = e->h_cnt->err;
    Counters c{};
    c.n = nf;
    c.n0 = nf;
    c.stall = kNoStall;
    MPX_CUDA(cudaMemcpyAsync(e->d_cnt, &c, sizeof(Counters), cudaMemcpyHostToDevice, e->stream));
    release();
    g.circuit_id = cd.id;
    g.L = L;
    g.n_final = nf;
    g.n0.resize(L);
    g.anti.resize(L);
    for (uint64_t st = 0; st < L; ++st) {
        g.n0[st] = A.stats[4 * st];
        g.anti[st] = A.stats[4 * st + 1];
    }
    g.w_anti = A.w_anti; // the graph keeps the per-warp counts and the outside-set bits
    g.longb = A.longb;
    A.longb = nullptr;
    A.w_anti = nullptr;
    free_adjoint(e);
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    if (err != 0) {
        free_graph(e);
        return fail(eng, MPX_ERR_STATE, "graph build replay diverged from the forward pass (internal error)");
    }
    return MPX_OK;
}

// The frozen structure at the circuit's current angles, from the initial operator; with segment_gates
// > 0 the coefficient array is saved at segment starts (for the frozen gradient).
// The values a replay of the frozen structure starts every term of the final store from.
mpx_status frozen_start(mpx_engine *eng) {
    mpx_engine *e = eng;
    FrozenGraph &g = e->fg;
    const uint64_t nf = g.n_final;
    if (e->schr) {
        // Schrodinger: the replay starts from the dense reference state, every stored term at its
        // reference-state score, appended terms included (MPOperator.h:169-181)
        if (nf > 0) pick_adj_init(e->W, e->cfg.basis)(e, e->st.coef, 0, nf);
    }
    else if (e->start_on) {
        // the re-weighted initial operator (mpx_update_initial_operator), in store positions
        if (nf > 0) MPX_CUDA(cudaMemsetAsync(e->st.coef, 0, nf * sizeof(double), e->stream));
        if (e->n_start > 0)
            k_scatter<<<static_cast<unsigned>(std::min<uint64_t>((e->n_start + 255) / 256, 4096)), 256, 0, e->stream>>>(
                e->st.coef, e->d_start_idx, e->d_start_val, e->n_start);
    }
    else {
        if (e->n_init > 0)
            MPX_CUDA(cudaMemcpyAsync(e->st.coef, e->d_init_coef, e->n_init * sizeof(double), cudaMemcpyDeviceToDevice,
                                     e->stream));
        if (nf > e->n_init)
            MPX_CUDA(cudaMemsetAsync(e->st.coef + e->n_init, 0, (nf - e->n_init) * sizeof(double), e->stream));
    }
    MPX_CUDA(cudaMemsetAsync(g.done, 0, ((nf + 31) / 32) * sizeof(uint32_t), e->stream));
    return MPX_OK;
}

// The frozen gradient as one segment whose forward pass is the reverse sweep's own logging replay: only
// the replay's starting coefficients are saved, and the replay leaves the final state in the store (no
// separate forward pass).
mpx_status frozen_single_segment(mpx_engine *eng) {
    mpx_engine *e = eng;
    FrozenGraph &g = e->fg;
    const uint64_t L = g.L, nf = g.n_final;
    free_adjoint(e);
    mpx_status s = frozen_start(e);
    if (s != MPX_OK) return s;
    const uint64_t n = L > 0 ? g.n0[0] : nf;
    double *ck = nullptr;
    MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&ck), std::max<uint64_t>(n, 1) * sizeof(double)));
    e->adj.ck_coef.push_back(ck);
    if (n > 0) MPX_CUDA(cudaMemcpyAsync(ck, e->st.coef, n * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
    e->adj.seg_lo.push_back(0);
    e->adj.ck_n.push_back(n);
    e->adj.n_final = nf;
    e->adj.L = L;
    e->adj.stats.assign(4 * L, 0);
    for (uint64_t st = 0; st < L; ++st) {
        e->adj.stats[4 * st] = g.n0[st];
        e->adj.stats[4 * st + 1] = g.anti[st];
        e->adj.stats[4 * st + 2] = g.count[st];
    }
    e->adj.w_anti = g.w_anti; // borrowed: released before free_adjoint can see it
    return MPX_OK;
}

mpx_status frozen_forward(mpx_engine *eng, const CircuitDev &cd, uint64_t segment_gates) {
    mpx_engine *e = eng;
    FrozenGraph &g = e->fg;
    const uint64_t L = g.L, nf = g.n_final;
    free_adjoint(e);
    mpx_status s0 = frozen_start(e);
    if (s0 != MPX_OK) return s0;
    const Frozen fz = g.view();
    const FrozenFn run = pick_frozen<false>(e->W);
    const uint64_t K = segment_gates == 0 ? std::max<uint64_t>(L, 1) : segment_gates;
    for (uint64_t st = 0; st < L; ++st) {
        if (segment_gates > 0 && st % K == 0) {
            const uint64_t n = g.n0[st];
            double *ck = nullptr;
            MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&ck), std::max<uint64_t>(n, 1) * sizeof(double)));
            e->adj.ck_coef.push_back(ck);
            if (n > 0) MPX_CUDA(cudaMemcpyAsync(ck, e->st.coef, n * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
            e->adj.seg_lo.push_back(st);
            e->adj.ck_n.push_back(n);
        }
        run(e, cd.d_desc, fz, static_cast<uint32_t>(L - 1 - st), static_cast<uint32_t>(st), g.n0[st], g.done, Tape{});
    }
    e->launches += 2 * L;
    MPX_CUDA(cudaGetLastError());
    Counters c{};
    c.n = nf;
    c.n0 = nf;
    c.stall = kNoStall;
    MPX_CUDA(cudaMemcpyAsync(e->d_cnt, &c, sizeof(Counters), cudaMemcpyHostToDevice, e->stream));
    if (segment_gates > 0) {
        MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&e->adj.final_coef), std::max<uint64_t>(nf, 1) * sizeof(double)));
        if (nf > 0)
            MPX_CUDA(cudaMemcpyAsync(e->adj.final_coef, e->st.coef, nf * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
        e->adj.n_final = nf;
        e->adj.L = L;
        e->adj.stats.assign(4 * L, 0);
        for (uint64_t st = 0; st < L; ++st) {
            e->adj.stats[4 * st] = g.n0[st];
            e->adj.stats[4 * st + 1] = g.anti[st];
            e->adj.stats[4 * st + 2] = g.count[st];
        }
        e->adj.w_anti = g.w_anti; // borrowed: released before free_adjoint can see it
    }
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    return MPX_OK;
}

mpx_status validate_cfg(const mpx_config *c) {
    if (c == nullptr) return fail(nullptr, MPX_ERR_INVALID, "config is NULL");
    if (c->num_modes < 1 || c->num_modes > 256)
        return fail(nullptr, MPX_ERR_INVALID, "logical_num_modes must be in the range [1, 256].");
    if (c->basis != MPX_BASIS_PAULI && c->basis != MPX_BASIS_MAJORANA)
        return fail(nullptr, MPX_ERR_INVALID, "basis must be 'majorana' or 'pauli'");
    if (c->cutoff_type != MPX_CUTOFF_LENGTH && c->cutoff_type != MPX_CUTOFF_SUPPORT)
        return fail(nullptr, MPX_ERR_INVALID, "cutoff_type must be 'length' or 'support'");
    if (c->basis == MPX_BASIS_PAULI && c->cutoff_type != MPX_CUTOFF_SUPPORT)
        return fail(nullptr, MPX_ERR_INVALID,
                    "Pauli basis requires cutoff_type == Support (Length has no Pauli-weight meaning under the "
                    "Pauli encoding).");
    if (c->has_lower_atol && c->has_upper_atol && c->upper_atol < c->lower_atol)
        return fail(nullptr, MPX_ERR_STATE, "upper_atol must be greater than or equal to lower_atol.");
    if (c->logical_num_modes < 0 || c->logical_num_modes > c->num_modes)
        return fail(nullptr, MPX_ERR_INVALID, "logical_num_modes must be in the range [0, num_modes].");
    if (c->has_schrodinger && c->schrodinger_cutoff < 0)
        return fail(nullptr, MPX_ERR_INVALID, "schrodinger_cutoff must be non-negative.");
    return MPX_OK;
}

}  // namespace

// ----- C ABI ------------------------------------------------------------------------------------------------

extern "C" {

}  // extern "C"

namespace {

// mpx_create; `shared`: the engine shares the GPU with the other engines of a batch, so from its first
// buffer on it allocates straight from the pool (no kept-block cache) and launches without programmatic
// dependent launch (a kernel scheduled early would hold SM slots at its dependency wait that another
// engine's ready kernel could use).
// The Schrodinger picture's initial state (MonomialPropagator.inl:162-165, generate_paired_op
// MajoranaAlgebra.h:127-160): every fully paired monomial of at most K = sc/2 + sc%2 mode pairs over the
// L logical modes, sc = min(schrodinger_cutoff, 2L), by subset size and then in lexicographic order of the
// modes, each holding its reference-state score <b|M|b> (+-1).
mpx_status paired_store(const mpx_config *cfg, const uint64_t *state_mask, std::vector<uint64_t> &keys,
                        std::vector<double> &coefs) {
    const int W = (cfg->num_modes + 31) / 32;
    const int L = cfg->logical_num_modes > 0 ? cfg->logical_num_modes : cfg->num_modes;
    const int sc = std::min(cfg->schrodinger_cutoff, 2 * L);
    const int K = std::min(sc / 2 + sc % 2, L);
    double total = 0.0, binom = 1.0; // sum_{k <= K} C(L, k)
    for (int k = 0; k <= K; ++k) {
        total += binom;
        binom = binom * (L - k) / (k + 1);
    }
    if (total > static_cast<double>(kMaxPairedTerms))
        return fail(nullptr, MPX_ERR_CAPACITY, "schrodinger_cutoff=" + std::to_string(cfg->schrodinger_cutoff) +
                                                   " gives an initial state of " + std::to_string(total) +
                                                   " paired monomials, above the engine's limit of " +
                                                   std::to_string(kMaxPairedTerms));
    keys.reserve(static_cast<size_t>(total) * W);
    coefs.reserve(static_cast<size_t>(total));
    std::vector<int> sel(static_cast<size_t>(std::max(K, 1)));
    for (int k = 0; k <= K; ++k) {
        for (int i = 0; i < k; ++i) sel[i] = i;
        for (;;) {
            uint64_t m[kMaxWords] = {};
            for (int i = 0; i < k; ++i)
                for (int slot = 2 * sel[i]; slot <= 2 * sel[i] + 1; ++slot) {
                    const int bit = 64 * W - 1 - slot;
                    m[bit / 64] |= 1ULL << (bit % 64);
                }
            int na = 0, pop = 0;
            for (int w = 0; w < W; ++w) {
                na += __builtin_popcountll(m[w] & (state_mask != nullptr ? state_mask[w] : 0ULL));
                pop += __builtin_popcountll(m[w]);
            }
            const int odd = cfg->basis == MPX_BASIS_PAULI ? (na & 1) : ((na + pop / 2) & 1);
            keys.insert(keys.end(), m, m + W);
            coefs.push_back(odd ? -1.0 : 1.0);
            int i = k - 1;
            while (i >= 0 && sel[i] == L - k + i) --i;
            if (i < 0) break;
            ++sel[i];
            for (int j = i + 1; j < k; ++j) sel[j] = sel[j - 1] + 1;
        }
    }
    return MPX_OK;
}

mpx_status create_engine(const mpx_config *cfg, const uint64_t *obs_words, const double *obs_coef, uint64_t n_obs,
                         double core, const uint64_t *state_mask, mpx_engine **out, bool shared) {
    if (out == nullptr) return fail(nullptr, MPX_ERR_INVALID, "out is NULL");
    *out = nullptr;
    mpx_status s = validate_cfg(cfg);
    if (s != MPX_OK) return s;
    // The initial store: the observable (Heisenberg), or the paired reference-state monomials with the
    // observable kept apart (Schrodinger).
    std::vector<uint64_t> paired_keys;
    std::vector<double> paired_coef;
    const uint64_t *init_words = obs_words;
    const double *init_coef = obs_coef;
    uint64_t n_init_terms = n_obs;
    if (cfg->has_schrodinger) {
        s = paired_store(cfg, state_mask, paired_keys, paired_coef);
        if (s != MPX_OK) return s;
        init_words = paired_keys.data();
        init_coef = paired_coef.data();
        n_init_terms = paired_coef.size();
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(nullptr, MPX_ERR_NO_DEVICE, "no CUDA device is visible; the engine has no CPU fallback");
    }
    if (cfg->device < 0 || cfg->device >= ndev) return fail(nullptr, MPX_ERR_INVALID, "device ordinal out of range");
    int major = 0, sms = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, cfg->device) != cudaSuccess || major != 10 ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cfg->device) != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, MPX_ERR_NO_DEVICE, "the engine is built for sm_100a (B200) only");
    }
    auto *e = new (std::nothrow) mpx_engine();
    if (e == nullptr) return fail(nullptr, MPX_ERR_NOMEM, "host allocation failed");
    e->cfg = *cfg;
    e->keep_blocks = !shared;
    e->use_pdl = !shared;
    e->W = ((cfg->num_modes + 31) / 32);
    e->tr.cutoff_type = cfg->cutoff_type;
    e->tr.cutoff = cfg->cutoff;
    e->tr.has_lower = cfg->has_lower_atol;
    e->tr.lower = cfg->lower_atol;
    e->tr.has_upper = cfg->has_upper_atol;
    e->tr.upper = cfg->upper_atol;
    e->device = cfg->device;
    e->core = core;
    for (int w = 0; w < e->W; ++w) e->mask.w[w] = state_mask != nullptr ? state_mask[w] : 0ULL;
    // One resident wave of the per-gate kernels (the resolve keeps a prefix per block). Further waves were
    // measured slower on the 100-qubit circuit: 8 blocks per SM 256 ms, 16 333 ms, against 214 ms.
    const int bps = cfg->blocks_per_sm > 0 ? std::min(cfg->blocks_per_sm, kSweepBlocksPerSM) : kSweepBlocksPerSM;
    e->grid = std::min(sms * bps, kMaxGrid);
    e->table_shift = cfg->table_shift > 0 ? std::min(cfg->table_shift, 3) : 1;
    mpx_engine *eng = e;
    auto bail = [&](mpx_status st) {
        g_create_error = e->err;
        mpx_destroy(e);
        return st;
    };
    if (cudaSetDevice(cfg->device) != cudaSuccess || cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
        e->err = "cannot create a CUDA stream";
        return bail(MPX_ERR_CUDA);
    }
    e->pool = engine_pool(cfg->device);
    if (e->pool == nullptr) {
        e->err = "cannot create the device memory pool";
        return bail(MPX_ERR_CUDA);
    }
    // Engine buffers come from the pool, stream-ordered, and pinned host buffers from a cache: creating and
    // destroying an engine waits for no other stream (cudaMalloc / cudaFree would, device-wide).
    cudaError_t ce = dev_alloc(e, reinterpret_cast<void **>(&e->d_cnt), sizeof(Counters));
    if (ce == cudaSuccess) ce = pinned_get(reinterpret_cast<void **>(&e->h_cnt), sizeof(Counters));
    if (ce == cudaSuccess) ce = pinned_get(reinterpret_cast<void **>(&e->h_snap), 2 * sizeof(Counters));
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->ev[0], cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->ev[1], cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&e->sc.blk_q), e->grid * sizeof(uint32_t));
    if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&e->d_partial), e->grid * sizeof(double));
    if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&e->d_out), sizeof(double));
    if (ce == cudaSuccess) ce = pinned_get(reinterpret_cast<void **>(&e->h_out), sizeof(double));
    if (ce == cudaSuccess && n_init_terms > 0) {
        ce = dev_alloc(e, reinterpret_cast<void **>(&e->d_init_keys), n_init_terms * e->W * sizeof(uint64_t));
        if (ce == cudaSuccess)
            ce = dev_alloc(e, reinterpret_cast<void **>(&e->d_init_coef), n_init_terms * sizeof(double));
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(e->d_init_keys, init_words, n_init_terms * e->W * sizeof(uint64_t),
                                 cudaMemcpyHostToDevice, e->stream);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(e->d_init_coef, init_coef, n_init_terms * sizeof(double), cudaMemcpyHostToDevice,
                                 e->stream);
    }
    if (ce == cudaSuccess && cfg->has_schrodinger) {
        // the observable, for <O> = core + observable . state
        e->schr = true;
        e->tr.schr = 1;
        e->tr.occ = e->mask;
        e->n_obs = n_obs;
        const uint64_t k = std::max<uint64_t>(n_obs, 1);
        ce = dev_alloc(e, reinterpret_cast<void **>(&e->d_obs_keys), k * e->W * sizeof(uint64_t));
        if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&e->d_obs_coef), k * sizeof(double));
        if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&e->d_obs_idx), k * sizeof(uint32_t));
        if (ce == cudaSuccess && n_obs > 0)
            ce = cudaMemcpyAsync(e->d_obs_keys, obs_words, n_obs * e->W * sizeof(uint64_t), cudaMemcpyHostToDevice,
                                 e->stream);
        if (ce == cudaSuccess && n_obs > 0)
            ce = cudaMemcpyAsync(e->d_obs_coef, obs_coef, n_obs * sizeof(double), cudaMemcpyHostToDevice, e->stream);
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream); // the caller's arrays may go away
    if (ce != cudaSuccess) {
        e->err = std::string("CUDA setup failed: ") + cudaGetErrorString(ce);
        cudaGetLastError();
        return bail(MPX_ERR_CUDA);
    }
    e->n_init = n_init_terms;
    const uint64_t cap = std::max<uint64_t>({cfg->capacity_hint, 4 * n_init_terms, 4096});
    s = alloc_store(eng, cap, 0);
    if (s != MPX_OK) return bail(s);
    s = load_initial(eng);
    if (s != MPX_OK) return bail(s);
    *out = e;
    return MPX_OK;
}

}  // namespace

extern "C" {

mpx_status mpx_create(const mpx_config *cfg, const uint64_t *obs_words, const double *obs_coef, uint64_t n_obs,
                      double core, const uint64_t *state_mask, mpx_engine **out) {
    return create_engine(cfg, obs_words, obs_coef, n_obs, core, state_mask, out, false);
}

mpx_status mpx_propagate(mpx_engine *e, const uint64_t *gen_words, const double *angles, uint64_t n_layers) {
    if (e == nullptr) return fail(nullptr, MPX_ERR_INVALID, "engine is NULL");
    mpx_engine *eng = e;
    if (n_layers > 0 && (gen_words == nullptr || angles == nullptr))
        return fail(eng, MPX_ERR_INVALID, "gen_words/angles are NULL");
    MPX_CUDA(cudaSetDevice(e->device));
    CircuitDev cd;
    mpx_status s = upload_circuit(e, gen_words, angles, n_layers, cd);
    if (s == MPX_OK) s = run_circuit(e, cd);
    dev_free(e, cd.d_desc);
    cudaStreamSynchronize(e->stream);
    cd.d_desc = nullptr;
    return s;
}

mpx_status mpx_circuit_upload(mpx_engine *e, const uint64_t *gen_words, const double *angles, uint64_t n_layers,
                              mpx_circuit **out) {
    if (e == nullptr || out == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    *out = nullptr;
    if (n_layers > 0 && (gen_words == nullptr || angles == nullptr))
        return fail(eng, MPX_ERR_INVALID, "gen_words/angles are NULL");
    MPX_CUDA(cudaSetDevice(e->device));
    auto *c = new (std::nothrow) mpx_circuit();
    if (c == nullptr) return fail(eng, MPX_ERR_NOMEM, "host allocation failed");
    mpx_status s = upload_circuit(e, gen_words, angles, n_layers, *c);
    c->persistent = true;
    if (s != MPX_OK) {
        mpx_circuit_destroy(c);
        return s;
    }
    *out = c;
    return MPX_OK;
}

mpx_status mpx_circuit_set_angles(mpx_engine *e, mpx_circuit *c, const double *angles) {
    if (e == nullptr || c == nullptr || (c->n > 0 && angles == nullptr)) return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    if (c->W != e->W) return fail(eng, MPX_ERR_INVALID, "circuit was uploaded for a different key width");
    std::vector<GateDesc> h;
    make_descs(e, c->words.data(), angles, c->n, h);
    c->any_cos_zero = false;
    for (const GateDesc &g : h) c->any_cos_zero = c->any_cos_zero || g.cos_zero;
    c->angles.assign(angles, angles + c->n);
    MPX_CUDA(cudaSetDevice(e->device));
    if (c->n > 0) {
        MPX_CUDA(cudaMemcpyAsync(c->d_desc, h.data(), c->n * sizeof(GateDesc), cudaMemcpyHostToDevice, e->stream));
        MPX_CUDA(cudaStreamSynchronize(e->stream));
    }
    return MPX_OK;
}

mpx_status mpx_propagate_circuit(mpx_engine *e, const mpx_circuit *c) {
    if (e == nullptr || c == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    if (c->W != e->W) return fail(eng, MPX_ERR_INVALID, "circuit was uploaded for a different key width");
    MPX_CUDA(cudaSetDevice(e->device));
    return run_circuit(e, *c);
}

void mpx_circuit_destroy(mpx_circuit *c) {
    if (c == nullptr) return;
    if (c->d_desc != nullptr) {
        // pool memory, returned stream-ordered; the circuit may outlive the stream of the engine that made it
        cudaSetDevice(c->device);
        dev_release(c->device, nullptr, c->d_desc);
        cudaStreamSynchronize(nullptr);
    }
    delete c;
}

mpx_status mpx_expectation(mpx_engine *e, double *out) {
    if (e == nullptr || out == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    MPX_CUDA(cudaSetDevice(e->device));
    if (e->schr) {
        // Schrodinger: core + observable . state (MPFunctions.cpp:196-205), each observable term looked up
        uint64_t n_live = 0;
        mpx_status s = mpx_size(e, &n_live);
        if (s != MPX_OK) return s;
        if (e->n_obs > 0) pick_lookup(e->W)(e, e->d_obs_keys, e->n_obs, n_live, e->d_obs_idx);
        k_expect_schr<<<1, kBlock, 0, e->stream>>>(e->d_obs_idx, e->d_obs_coef, e->n_obs, e->st.coef, e->core, e->d_out);
        e->launches += e->n_obs > 0 ? 2 : 1;
    }
    else {
        pick_exp(e->W, e->cfg.basis)(e);
        k_expect_final<<<1, kBlock, 0, e->stream>>>(e->d_partial, static_cast<uint32_t>(e->grid), e->core, e->d_out);
        e->launches += 2;
    }
    MPX_CUDA(cudaGetLastError());
    MPX_CUDA(cudaMemcpyAsync(e->h_out, e->d_out, sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    *out = *e->h_out;
    return MPX_OK;
}

mpx_status mpx_size(mpx_engine *e, uint64_t *out) {
    if (e == nullptr || out == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    MPX_CUDA(cudaSetDevice(e->device));
    MPX_CUDA(cudaMemcpyAsync(e->h_cnt, e->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, e->stream));
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    *out = e->h_cnt->n;
    return MPX_OK;
}

mpx_status mpx_words(mpx_engine *e, uint32_t *out) {
    if (e == nullptr || out == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    *out = static_cast<uint32_t>(e->W);
    return MPX_OK;
}

mpx_status mpx_export(mpx_engine *e, uint64_t *words, double *coefs, uint64_t cap, uint64_t *n_out) {
    if (e == nullptr || n_out == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    uint64_t n = 0;
    mpx_status s = mpx_size(e, &n);
    if (s != MPX_OK) return s;
    *n_out = n;
    const uint64_t k = std::min(n, cap);
    if (k > 0) {
        if (words != nullptr)
            MPX_CUDA(cudaMemcpyAsync(words, e->st.keys, k * e->W * sizeof(uint64_t), cudaMemcpyDeviceToHost, e->stream));
        if (coefs != nullptr)
            MPX_CUDA(cudaMemcpyAsync(coefs, e->st.coef, k * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
        MPX_CUDA(cudaStreamSynchronize(e->stream));
    }
    return MPX_OK;
}

mpx_status mpx_gate_stats(mpx_engine *e, uint64_t *out4, uint64_t max_gates, uint64_t *n_out) {
    if (e == nullptr || n_out == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    const uint64_t L = e->last_gates;
    *n_out = L;
    if (L == 0 || out4 == nullptr) return MPX_OK;
    std::vector<uint64_t> h(4 * L);
    MPX_CUDA(cudaMemcpyAsync(h.data(), e->d_stats, 4 * L * sizeof(uint64_t), cudaMemcpyDeviceToHost, e->stream));
    uint64_t n_final = 0;
    mpx_status s = mpx_size(e, &n_final);
    if (s != MPX_OK) return s;
    for (uint64_t g = 0; g < L; ++g) {
        const uint64_t next = g + 1 < L ? h[4 * (g + 1)] : n_final;
        h[4 * g + 3] = next - h[4 * g];
    }
    const uint64_t k = std::min(L, max_gates);
    std::memcpy(out4, h.data(), 4 * k * sizeof(uint64_t));
    return MPX_OK;
}

mpx_status mpx_reset(mpx_engine *e) {
    if (e == nullptr) return fail(nullptr, MPX_ERR_INVALID, "engine is NULL");
    mpx_engine *eng = e;
    MPX_CUDA(cudaSetDevice(e->device));
    free_adjoint(e);
    clear_start(e);
    return load_initial(e);
}

mpx_status mpx_set_cutoff(mpx_engine *e, uint32_t cutoff) {
    if (e == nullptr) return fail(nullptr, MPX_ERR_INVALID, "engine is NULL");
    clear_graphs(e); // truncation settings are kernel arguments baked into captured graphs
    e->cfg.cutoff = cutoff;
    e->tr.cutoff = cutoff;
    return MPX_OK;
}

mpx_status mpx_set_cutoff_type(mpx_engine *e, int32_t cutoff_type) {
    if (e == nullptr) return fail(nullptr, MPX_ERR_INVALID, "engine is NULL");
    if (cutoff_type != MPX_CUTOFF_LENGTH && cutoff_type != MPX_CUTOFF_SUPPORT)
        return fail(e, MPX_ERR_INVALID, "cutoff_type must be 'length' or 'support'");
    if (e->cfg.basis == MPX_BASIS_PAULI && cutoff_type != MPX_CUTOFF_SUPPORT)
        return fail(e, MPX_ERR_INVALID,
                    "Pauli basis requires cutoff_type == Support (Length has no Pauli-weight meaning under the "
                    "Pauli encoding).");
    clear_graphs(e); // truncation settings are kernel arguments baked into captured graphs
    e->cfg.cutoff_type = cutoff_type;
    e->tr.cutoff_type = cutoff_type;
    return MPX_OK;
}

mpx_status mpx_set_lower_atol(mpx_engine *e, int32_t has_value, double value) {
    if (e == nullptr) return fail(nullptr, MPX_ERR_INVALID, "engine is NULL");
    clear_graphs(e); // truncation settings are kernel arguments baked into captured graphs
    if (has_value && e->tr.has_upper && e->tr.upper < value)
        return fail(e, MPX_ERR_STATE, "upper_atol must be greater than or equal to lower_atol.");
    e->cfg.has_lower_atol = has_value;
    e->cfg.lower_atol = value;
    e->tr.has_lower = has_value;
    e->tr.lower = value;
    return MPX_OK;
}

mpx_status mpx_set_upper_atol(mpx_engine *e, int32_t has_value, double value) {
    if (e == nullptr) return fail(nullptr, MPX_ERR_INVALID, "engine is NULL");
    clear_graphs(e); // truncation settings are kernel arguments baked into captured graphs
    if (has_value && e->tr.has_lower && value < e->tr.lower)
        return fail(e, MPX_ERR_STATE, "upper_atol must be greater than or equal to lower_atol.");
    e->cfg.has_upper_atol = has_value;
    e->cfg.upper_atol = value;
    e->tr.has_upper = has_value;
    e->tr.upper = value;
    return MPX_OK;
}

mpx_status mpx_set_basis_change(mpx_engine *e, const uint64_t *rows, uint32_t n_rows) {
    if (e == nullptr) return fail(nullptr, MPX_ERR_INVALID, "engine is NULL");
    mpx_engine *eng = e;
    if (n_rows == 0) {
        clear_graphs(e);
        e->tr.basis_rows = nullptr;
        return MPX_OK;
    }
    if (e->cfg.basis != 0)
        return fail(e, MPX_ERR_INVALID,
                    "Pauli basis does not accept a basis_change (the encoding is already the Jordan-Wigner image).");
    if (n_rows != 2 * static_cast<uint32_t>(e->cfg.num_modes))
        return fail(e, MPX_ERR_INVALID, "basis_change must have exactly 2*logical_num_modes (" +
                                            std::to_string(2 * e->cfg.num_modes) + ") rows; got " +
                                            std::to_string(n_rows) + ".");
    if (rows == nullptr) return fail(e, MPX_ERR_INVALID, "basis_change rows are NULL");
    MPX_CUDA(cudaSetDevice(e->device));
    const size_t bytes = static_cast<size_t>(64 * e->W) * e->W * sizeof(uint64_t); // 2T rows of W words
    if (e->d_basis == nullptr) MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&e->d_basis), bytes));
    MPX_CUDA(cudaMemsetAsync(e->d_basis, 0, bytes, e->stream));
    MPX_CUDA(cudaMemcpyAsync(e->d_basis, rows, static_cast<size_t>(n_rows) * e->W * sizeof(uint64_t),
                             cudaMemcpyHostToDevice, e->stream));
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    clear_graphs(e);
    e->tr.basis_rows = e->d_basis;
    return MPX_OK;
}

mpx_status mpx_set_only_rotate_len_k(mpx_engine *e, int64_t k) {
    if (e == nullptr) return fail(nullptr, MPX_ERR_INVALID, "engine is NULL");
    const int64_t max_k = 2 * static_cast<int64_t>(e->cfg.num_modes);
    if (k > max_k)
        return fail(e, MPX_ERR_INVALID, "only_rotate_len_k=" + std::to_string(k) +
                                            " is out of range; must be 0 < k <= 2*num_qubits");
    clear_graphs(e);
    e->tr.has_len_k = k > 0;
    e->tr.len_k = k > 0 ? static_cast<uint32_t>(k) : 0;
    return MPX_OK;
}

mpx_status mpx_device_view(mpx_engine *e, const uint64_t **keys, double **coefs, uint64_t *n) {
    if (e == nullptr) return fail(nullptr, MPX_ERR_INVALID, "engine is NULL");
    if (keys) *keys = e->st.keys;
    if (coefs) *coefs = e->st.coef;
    if (n) return mpx_size(e, n);
    return MPX_OK;
}

mpx_status mpx_stream(mpx_engine *e, void **stream) {
    if (e == nullptr || stream == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    *stream = e->stream;
    return MPX_OK;
}

mpx_status mpx_launch_count(mpx_engine *e, uint64_t *out) {
    if (e == nullptr || out == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    *out = e->launches;
    return MPX_OK;
}

mpx_status mpx_adjoint_logged(mpx_engine *e, int32_t *out) {
    if (e == nullptr || out == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    *out = e->adj.log_ok ? 1 : 0;
    return MPX_OK;
}

mpx_status mpx_graph_replay_count(mpx_engine *e, uint64_t *out) {
    if (e == nullptr || out == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    *out = e->graph_replays;
    return MPX_OK;
}

// The Schrodinger picture runs the circuit first to last at negated angles (gate descriptor l is circuit
// layer L-1-l at -angle): the adjoint's derivatives per descriptor, mapped back to circuit layers.
void schr_grad_to_layers(const mpx_engine *e, double *grad, uint64_t L) {
    if (!e->schr || L == 0) return;
    const std::vector<double> g(grad, grad + L);
    for (uint64_t l = 0; l < L; ++l) grad[L - 1 - l] = -g[l];
}

mpx_status mpx_adjoint_forward(mpx_engine *e, const mpx_circuit *c, uint64_t segment_gates, double *expectation) {
    if (e == nullptr || c == nullptr || expectation == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    if (c->W != e->W) return fail(eng, MPX_ERR_INVALID, "circuit was uploaded for a different key width");
    MPX_CUDA(cudaSetDevice(e->device));
    mpx_status s = adjoint_forward(e, *c, segment_gates, true);
    if (s != MPX_OK) return s;
    return mpx_expectation(e, expectation);
}

mpx_status mpx_adjoint_backward(mpx_engine *e, const mpx_circuit *c, double *grad_angles) {
    if (e == nullptr || c == nullptr || (c->n > 0 && grad_angles == nullptr))
        return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    if (e->adj.circuit != c || e->adj.L != c->n)
        return fail(eng, MPX_ERR_STATE, "mpx_adjoint_backward needs a preceding mpx_adjoint_forward of the same circuit "
                                        "with no propagation in between");
    MPX_CUDA(cudaSetDevice(e->device));
    if (c->n == 0) return MPX_OK;
    if (e->adj.log_ok) {
        // the forward pass logged everything: the reverse sweep alone
        const mpx_status s = adjoint_backward_logged(e, *c, grad_angles);
        if (s == MPX_OK) schr_grad_to_layers(e, grad_angles, c->n);
        return s;
    }
    if (!e->adj.rec_ok) {
        // the streaming replay runs with the forward pass's only_rotate_len_k
        const Trunc saved = e->tr;
        e->tr.has_len_k = e->adj.len_k > 0;
        e->tr.len_k = e->adj.len_k;
        const mpx_status s = adjoint_backward(e, *c, grad_angles);
        e->tr = saved;
        if (s == MPX_OK) schr_grad_to_layers(e, grad_angles, c->n);
        return s;
    }
    // The forward pass recorded every gate's pairs: replay the segments with the frozen kernels.
    FrozenGraph view;
    mpx_status s = recorded_view(e, view);
    if (s != MPX_OK) return s;
    s = adjoint_backward(e, *c, grad_angles, &view);
    dev_free(e, view.p_count);
    if (s == MPX_OK) schr_grad_to_layers(e, grad_angles, c->n);
    return s;
}

mpx_status mpx_graph_build(mpx_engine *e, const mpx_circuit *c, uint64_t segment_gates, double *expectation) {
    if (e == nullptr || c == nullptr || expectation == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    if (c->W != e->W) return fail(eng, MPX_ERR_INVALID, "circuit was uploaded for a different key width");
    MPX_CUDA(cudaSetDevice(e->device));
    mpx_status s = graph_build(e, *c, segment_gates);
    if (s != MPX_OK) return s;
    return mpx_expectation(e, expectation);
}

static mpx_status check_graph(mpx_engine *e, const mpx_circuit *c) {
    if (e->fg.L == 0 || e->fg.circuit_id != c->id)
        return fail(e, MPX_ERR_STATE, "no graph built for this circuit (mpx_graph_build)");
    return MPX_OK;
}

mpx_status mpx_graph_expectation(mpx_engine *e, const mpx_circuit *c, double *expectation) {
    if (e == nullptr || c == nullptr || expectation == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    mpx_status s = check_graph(e, c);
    if (s != MPX_OK) return s;
    MPX_CUDA(cudaSetDevice(e->device));
    s = frozen_forward(e, *c, 0);
    if (s != MPX_OK) return s;
    return mpx_expectation(e, expectation);
}

mpx_status mpx_graph_gradient(mpx_engine *e, const mpx_circuit *c, uint64_t segment_gates, double *expectation,
                              double *grad_angles) {
    if (e == nullptr || c == nullptr || expectation == nullptr || (c->n > 0 && grad_angles == nullptr))
        return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    mpx_status s = check_graph(e, c);
    if (s != MPX_OK) return s;
    MPX_CUDA(cudaSetDevice(e->device));
    if (segment_gates == 0 && c->n > 0) {
        // one segment: the reverse sweep's logging replay is the forward pass
        s = frozen_single_segment(e);
        if (s == MPX_OK) s = adjoint_backward(e, *c, grad_angles, &e->fg);
        if (s == MPX_OK) s = mpx_expectation(e, expectation);
    }
    else {
        s = frozen_forward(e, *c, segment_gates == 0 ? std::max<uint64_t>(c->n, 1) : segment_gates);
        if (s == MPX_OK) s = mpx_expectation(e, expectation);
        if (s == MPX_OK && c->n > 0) s = adjoint_backward(e, *c, grad_angles, &e->fg);
    }
    if (s == MPX_OK) schr_grad_to_layers(e, grad_angles, c->n);
    e->adj.w_anti = nullptr; // owned by the graph
    free_adjoint(e);
    return s;
}

mpx_status mpx_graph_pare(mpx_engine *e, const mpx_circuit *c, double threshold) {
    if (e == nullptr || c == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    mpx_status s = check_graph(e, c);
    if (s != MPX_OK) return s;
    MPX_CUDA(cudaSetDevice(e->device));
    return graph_pare(e, threshold);
}

mpx_status mpx_set_pair_log(mpx_engine *e, int64_t capacity) {
    if (e == nullptr) return fail(nullptr, MPX_ERR_INVALID, "engine is NULL");
    e->pair_log = capacity;
    return MPX_OK;
}

mpx_status mpx_set_profiling(mpx_engine *e, int32_t on) {
    if (e == nullptr) return fail(nullptr, MPX_ERR_INVALID, "engine is NULL");
    e->profile = on != 0;
    return MPX_OK;
}

mpx_status mpx_kernel_times(mpx_engine *e, double *sweep_ms, double *resolve_ms, double *columns_ms,
                            uint64_t *n_gates) {
    if (e == nullptr) return fail(nullptr, MPX_ERR_INVALID, "engine is NULL");
    if (!e->profile) return fail(e, MPX_ERR_STATE, "profiling is off (mpx_set_profiling)");
    if (sweep_ms) *sweep_ms = e->t_sweep_ms;
    if (resolve_ms) *resolve_ms = e->t_resolve_ms;
    if (columns_ms) *columns_ms = e->t_columns_ms;
    if (n_gates) *n_gates = e->n_sweep;
    return MPX_OK;
}

mpx_status mpx_trim_device_memory(int32_t device) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return fail(nullptr, MPX_ERR_INVALID, "device ordinal out of range");
    }
    cudaMemPool_t pool = engine_pool(device);
    if (pool == nullptr) return fail(nullptr, MPX_ERR_CUDA, "cannot create the device memory pool");
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    release_kept_blocks(device);
    cudaSetDevice(prev);
    if (cudaMemPoolTrimTo(pool, 0) != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, MPX_ERR_CUDA, "cudaMemPoolTrimTo failed");
    }
    return MPX_OK;
}

mpx_status mpx_update_initial_operator(mpx_engine *e, const uint64_t *words, const double *coefs, uint64_t n,
                                       int32_t has_core, double core, uint64_t *missing) {
    if (e == nullptr || (n > 0 && (words == nullptr || coefs == nullptr))) return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    MPX_CUDA(cudaSetDevice(e->device));
    if (e->schr) {
        // Schrodinger: the observable is dotted into the evolved state, so re-weighting it replaces the
        // observable's terms (a term the state does not hold contributes 0)
        if (n > std::max<uint64_t>(e->n_obs, 1)) {
            dev_free(e, e->d_obs_keys);
            dev_free(e, e->d_obs_coef);
            dev_free(e, e->d_obs_idx);
            e->d_obs_keys = nullptr;
            e->d_obs_coef = nullptr;
            e->d_obs_idx = nullptr;
            MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&e->d_obs_keys), n * e->W * sizeof(uint64_t)));
            MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&e->d_obs_coef), n * sizeof(double)));
            MPX_CUDA(dev_alloc(e, reinterpret_cast<void **>(&e->d_obs_idx), n * sizeof(uint32_t)));
        }
        if (n > 0) {
            MPX_CUDA(cudaMemcpyAsync(e->d_obs_keys, words, n * e->W * sizeof(uint64_t), cudaMemcpyHostToDevice, e->stream));
            MPX_CUDA(cudaMemcpyAsync(e->d_obs_coef, coefs, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
        }
        e->n_obs = n;
        if (has_core) e->core = core;
        e->fg.last_for = -2.0; // a pared graph's keep set came from the old observable
        MPX_CUDA(cudaStreamSynchronize(e->stream));
        return MPX_OK;
    }
    uint64_t n_live = 0;
    mpx_status s = mpx_size(e, &n_live);
    if (s != MPX_OK) return s;
    uint64_t *d_keys = nullptr;
    uint32_t *d_idx = nullptr;
    double *d_val = nullptr;
    std::vector<uint32_t> idx(n);
    cudaError_t ce = dev_alloc(e, reinterpret_cast<void **>(&d_keys), std::max<uint64_t>(n, 1) * e->W * sizeof(uint64_t));
    if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&d_idx), std::max<uint64_t>(n, 1) * sizeof(uint32_t));
    if (ce == cudaSuccess) ce = dev_alloc(e, reinterpret_cast<void **>(&d_val), std::max<uint64_t>(n, 1) * sizeof(double));
    if (ce == cudaSuccess && n > 0) {
        ce = cudaMemcpyAsync(d_keys, words, n * e->W * sizeof(uint64_t), cudaMemcpyHostToDevice, e->stream);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(d_val, coefs, n * sizeof(double), cudaMemcpyHostToDevice, e->stream);
        if (ce == cudaSuccess) {
            pick_lookup(e->W)(e, d_keys, n, n_live, d_idx);
            ce = cudaGetLastError();
        }
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(idx.data(), d_idx, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, e->stream);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(e->h_cnt, e->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, e->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    }
    auto drop = [&]() {
        dev_free(e, d_keys);
        dev_free(e, d_idx);
        dev_free(e, d_val);
    };
    if (ce != cudaSuccess) {
        drop();
        cudaGetLastError();
        return fail(eng, ce == cudaErrorMemoryAllocation ? MPX_ERR_NOMEM : MPX_ERR_CUDA,
                    std::string("initial operator update: ") + cudaGetErrorString(ce));
    }
    if (n > 0 && e->h_cnt->err != 0) {
        drop();
        return fail(eng, MPX_ERR_STATE, "hash table probe limit reached (internal error); the store is invalid");
    }
    for (uint64_t k = 0; k < n; ++k) {
        if (idx[k] == kNoStall) {
            drop();
            if (missing != nullptr) *missing = k;
            return fail(eng, MPX_ERR_STATE, "Operator term not found in the operator.");
        }
    }
    // the current coefficients become the new operator (zero elsewhere); graph evaluations start from it
    if (n_live > 0) MPX_CUDA(cudaMemsetAsync(e->st.coef, 0, n_live * sizeof(double), e->stream));
    if (n > 0)
        k_scatter<<<static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 4096)), 256, 0, e->stream>>>(e->st.coef, d_idx,
                                                                                                       d_val, n);
    e->launches += n > 0 ? 2 : 0;
    MPX_CUDA(cudaGetLastError());
    dev_free(e, d_keys);
    dev_free(e, e->d_start_idx);
    dev_free(e, e->d_start_val);
    e->d_start_idx = d_idx;
    e->d_start_val = d_val;
    e->n_start = n;
    e->start_on = true;
    if (has_core) e->core = core;
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    return MPX_OK;
}

mpx_status mpx_memory(mpx_engine *e, mpx_memory_info *out) {
    if (e == nullptr || out == nullptr) return fail(e, MPX_ERR_INVALID, "NULL argument");
    uint64_t n = 0;
    mpx_status s = mpx_size(e, &n);
    if (s != MPX_OK) return s;
    const uint64_t W = static_cast<uint64_t>(e->W);
    *out = mpx_memory_info{};
    out->terms = n;
    out->capacity = e->st.cap;
    out->words = static_cast<uint32_t>(W);
    out->key_bytes = e->st.cap * W * sizeof(uint64_t);
    out->coef_bytes = e->st.cap * sizeof(double);
    out->table_bytes = (e->st.tmask + 1) * sizeof(unsigned long long);
    out->column_bytes = (64 * W + 1) * e->st.cstride * sizeof(uint32_t);
    out->scratch_bytes = e->sc.q_cap * (sizeof(uint32_t) + sizeof(uint8_t) + sizeof(double)) +
                         e->st.cstride * sizeof(uint32_t) + (e->aux_on ? e->st.cap * sizeof(double) : 0);
    out->initial_bytes = e->n_init * (W * sizeof(uint64_t) + sizeof(double)) +
                         e->n_start * (sizeof(uint32_t) + sizeof(double));
    const FrozenGraph &g = e->fg;
    uint64_t pairs = 0;
    for (uint64_t c : g.count) pairs += c;
    out->graph_layers = g.L;
    out->graph_pairs = pairs;
    out->graph_bytes = g.L == 0 ? 0
                                : pairs * (2 * sizeof(uint32_t) + sizeof(int8_t)) +
                                      g.L * (sizeof(uint64_t) + sizeof(unsigned long long)) +
                                      g.L * static_cast<uint64_t>(e->grid) * kWarps * sizeof(uint32_t) +
                                      ((g.n_final + 31) / 32) * sizeof(uint32_t);
    return MPX_OK;
}

mpx_status mpx_graph_info(mpx_engine *e, uint64_t *layers, uint64_t *pairs, uint64_t *cos_only) {
    if (e == nullptr) return fail(nullptr, MPX_ERR_INVALID, "engine is NULL");
    const FrozenGraph &g = e->fg;
    uint64_t p = 0, c = 0;
    for (uint64_t st = 0; st < g.L; ++st) {
        const uint64_t appended = (st + 1 < g.L ? g.n0[st + 1] : g.n_final) - g.n0[st];
        p += g.count[st];
        // anticommuting terms outside every pair: a pair covers its emitter and, unless the partner was
        // appended by this gate, its partner
        c += g.anti[st] + appended - 2 * g.count[st];
    }
    if (layers) *layers = g.L;
    if (pairs) *pairs = p;
    if (cos_only) *cos_only = c;
    return MPX_OK;
}

namespace {

// Copies e's store, settings, last per-gate counters, re-weighted initial operator and frozen graph into
// the freshly created engine d (same configuration, so the same capacities and strides).
mpx_status clone_into(mpx_engine *e, mpx_engine *d) {
    mpx_engine *eng = d;
    const int W = e->W;
    d->tr = e->tr;
    d->tr.basis_rows = nullptr;
    d->pair_log = e->pair_log;
    d->rec_hint = e->rec_hint;
    d->small_path = e->small_path;
    d->use_graphs = e->use_graphs;
    if (e->d_basis != nullptr) {
        const size_t bytes = static_cast<size_t>(64 * W) * W * sizeof(uint64_t);
        MPX_CUDA(dev_alloc(d, reinterpret_cast<void **>(&d->d_basis), bytes));
        MPX_CUDA(cudaMemcpyAsync(d->d_basis, e->d_basis, bytes, cudaMemcpyDeviceToDevice, d->stream));
        if (e->tr.basis_rows != nullptr) d->tr.basis_rows = d->d_basis;
    }
    d->aux_on = e->aux_on;
    mpx_status s = alloc_store(d, e->st.cap, 0);
    if (s != MPX_OK) return s;
    uint64_t n = 0;
    s = mpx_size(e, &n);
    if (s != MPX_OK) return s;
    if (n > 0) {
        MPX_CUDA(cudaMemcpyAsync(d->st.keys, e->st.keys, n * W * sizeof(uint64_t), cudaMemcpyDeviceToDevice, d->stream));
        MPX_CUDA(cudaMemcpyAsync(d->st.coef, e->st.coef, n * sizeof(double), cudaMemcpyDeviceToDevice, d->stream));
    }
    MPX_CUDA(cudaMemcpyAsync(d->st.cols, e->st.cols, (64 * W + 1) * e->st.cstride * sizeof(uint32_t),
                             cudaMemcpyDeviceToDevice, d->stream));
    MPX_CUDA(cudaMemcpyAsync(d->st.table, e->st.table, (e->st.tmask + 1) * sizeof(unsigned long long),
                             cudaMemcpyDeviceToDevice, d->stream));
    MPX_CUDA(cudaMemcpyAsync(d->d_cnt, e->d_cnt, sizeof(Counters), cudaMemcpyDeviceToDevice, d->stream));
    if (e->last_gates > 0) {
        s = ensure_stats(d, e->last_gates);
        if (s != MPX_OK) return s;
        MPX_CUDA(cudaMemcpyAsync(d->d_stats, e->d_stats, 4 * e->last_gates * sizeof(uint64_t), cudaMemcpyDeviceToDevice,
                                 d->stream));
        d->last_gates = e->last_gates;
    }
    if (e->start_on) {
        const uint64_t k = std::max<uint64_t>(e->n_start, 1);
        MPX_CUDA(dev_alloc(d, reinterpret_cast<void **>(&d->d_start_idx), k * sizeof(uint32_t)));
        MPX_CUDA(dev_alloc(d, reinterpret_cast<void **>(&d->d_start_val), k * sizeof(double)));
        if (e->n_start > 0) {
            MPX_CUDA(cudaMemcpyAsync(d->d_start_idx, e->d_start_idx, e->n_start * sizeof(uint32_t),
                                     cudaMemcpyDeviceToDevice, d->stream));
            MPX_CUDA(cudaMemcpyAsync(d->d_start_val, e->d_start_val, e->n_start * sizeof(double),
                                     cudaMemcpyDeviceToDevice, d->stream));
        }
        d->n_start = e->n_start;
        d->start_on = true;
    }
    const FrozenGraph &g = e->fg;
    if (g.L > 0) {
        FrozenGraph &h = d->fg;
        const uint64_t L = g.L;
        std::vector<uint64_t> begin(L);
        MPX_CUDA(cudaMemcpyAsync(begin.data(), g.p_begin, L * sizeof(uint64_t), cudaMemcpyDeviceToHost, e->stream));
        MPX_CUDA(cudaStreamSynchronize(e->stream));
        uint64_t total = 0;
        for (uint64_t st = 0; st < L; ++st) total = std::max(total, begin[st] + g.count[st]);
        const uint64_t n_warps = static_cast<uint64_t>(d->grid) * kWarps;
        const uint64_t nw = std::max<uint64_t>((g.n_final + 31) / 32, 4);
        MPX_CUDA(dev_alloc(d, reinterpret_cast<void **>(&h.src), std::max<uint64_t>(total, 1) * sizeof(uint32_t)));
        MPX_CUDA(dev_alloc(d, reinterpret_cast<void **>(&h.tgt), std::max<uint64_t>(total, 1) * sizeof(uint32_t)));
        MPX_CUDA(dev_alloc(d, reinterpret_cast<void **>(&h.code), std::max<uint64_t>(total, 1) * sizeof(int8_t)));
        MPX_CUDA(dev_alloc(d, reinterpret_cast<void **>(&h.p_begin), L * sizeof(uint64_t)));
        MPX_CUDA(dev_alloc(d, reinterpret_cast<void **>(&h.p_count), L * sizeof(unsigned long long)));
        MPX_CUDA(dev_alloc(d, reinterpret_cast<void **>(&h.w_anti), L * n_warps * sizeof(uint32_t)));
        MPX_CUDA(dev_alloc(d, reinterpret_cast<void **>(&h.done), nw * sizeof(uint32_t)));
        if (total > 0) {
            MPX_CUDA(cudaMemcpyAsync(h.src, g.src, total * sizeof(uint32_t), cudaMemcpyDeviceToDevice, d->stream));
            MPX_CUDA(cudaMemcpyAsync(h.tgt, g.tgt, total * sizeof(uint32_t), cudaMemcpyDeviceToDevice, d->stream));
            MPX_CUDA(cudaMemcpyAsync(h.code, g.code, total * sizeof(int8_t), cudaMemcpyDeviceToDevice, d->stream));
        }
        MPX_CUDA(cudaMemcpyAsync(h.p_begin, g.p_begin, L * sizeof(uint64_t), cudaMemcpyDeviceToDevice, d->stream));
        MPX_CUDA(cudaMemcpyAsync(h.p_count, g.p_count, L * sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                 d->stream));
        MPX_CUDA(cudaMemcpyAsync(h.w_anti, g.w_anti, L * n_warps * sizeof(uint32_t), cudaMemcpyDeviceToDevice, d->stream));
        MPX_CUDA(cudaMemsetAsync(h.done, 0, nw * sizeof(uint32_t), d->stream));
        h.L = L;
        h.n_final = g.n_final;
        h.n0 = g.n0;
        h.anti = g.anti;
        h.count = g.count;
    }
    MPX_CUDA(cudaStreamSynchronize(d->stream));
    return MPX_OK;
}

}  // namespace

mpx_status mpx_clone(mpx_engine *e, const mpx_circuit *c, mpx_engine **out, mpx_circuit **c_out) {
    if (e == nullptr || out == nullptr || (c != nullptr && c_out == nullptr)) return fail(e, MPX_ERR_INVALID, "NULL argument");
    mpx_engine *eng = e;
    *out = nullptr;
    if (c_out != nullptr) *c_out = nullptr;
    if (c != nullptr && c->W != e->W) return fail(eng, MPX_ERR_INVALID, "circuit was uploaded for a different key width");
    MPX_CUDA(cudaSetDevice(e->device));
    MPX_CUDA(cudaStreamSynchronize(e->stream));
    const int W = e->W;
    // the observable the engine was created with (Schrodinger: kept apart from the store)
    const uint64_t n_o = e->schr ? e->n_obs : e->n_init;
    const uint64_t *d_ok = e->schr ? e->d_obs_keys : e->d_init_keys;
    const double *d_oc = e->schr ? e->d_obs_coef : e->d_init_coef;
    std::vector<uint64_t> ik(std::max<uint64_t>(n_o, 1) * W);
    std::vector<double> ic(std::max<uint64_t>(n_o, 1));
    if (n_o > 0) {
        MPX_CUDA(cudaMemcpy(ik.data(), d_ok, n_o * W * sizeof(uint64_t), cudaMemcpyDeviceToHost));
        MPX_CUDA(cudaMemcpy(ic.data(), d_oc, n_o * sizeof(double), cudaMemcpyDeviceToHost));
    }
    mpx_engine *d = nullptr;
    mpx_status s = create_engine(&e->cfg, n_o > 0 ? ik.data() : nullptr, n_o > 0 ? ic.data() : nullptr, n_o, e->core,
                                 e->mask.w, &d, !e->keep_blocks);
    if (s != MPX_OK) return fail(eng, s, mpx_last_error(nullptr));
    s = clone_into(e, d);
    if (s == MPX_OK && c != nullptr) {
        s = mpx_circuit_upload(d, c->words.data(), c->angles.data(), c->n, c_out);
        if (s == MPX_OK && e->fg.L > 0 && e->fg.circuit_id == c->id) d->fg.circuit_id = (*c_out)->id;
    }
    if (s != MPX_OK) {
        const std::string msg = d->err;
        if (c_out != nullptr && *c_out != nullptr) {
            mpx_circuit_destroy(*c_out);
            *c_out = nullptr;
        }
        mpx_destroy(d);
        return fail(eng, s, "clone failed: " + msg);
    }
    *out = d;
    return MPX_OK;
}

mpx_status mpx_current_device(int32_t *device) {
    if (device == nullptr) return fail(nullptr, MPX_ERR_INVALID, "NULL argument");
    int d = 0;
    const cudaError_t ce = cudaGetDevice(&d);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, MPX_ERR_NO_DEVICE, std::string("no current CUDA device: ") + cudaGetErrorString(ce));
    }
    *device = d;
    return MPX_OK;
}

// Internal (not exported): the batch runner's engines, created as sharing the GPU (see create_engine).
mpx_status mpx_internal_create_shared(const mpx_config *cfg, const uint64_t *obs_words, const double *obs_coef,
                                      uint64_t n_obs, double core, const uint64_t *state_mask, mpx_engine **out) {
    return create_engine(cfg, obs_words, obs_coef, n_obs, core, state_mask, out, true);
}

const char *mpx_last_error(const mpx_engine *e) { return e != nullptr ? e->err.c_str() : g_create_error.c_str(); }

void mpx_destroy(mpx_engine *e) {
    if (e == nullptr) return;
    if (e->stream != nullptr) {
        cudaSetDevice(e->device);
        cudaStreamSynchronize(e->stream);
    }
    free_adjoint(e);
    free_graph(e);
    cudaStreamSynchronize(e->stream);
    clear_graphs(e);
    free_store(e);
    dev_free(e, e->d_cnt);
    pinned_put(e->h_cnt, sizeof(Counters));
    pinned_put(e->h_snap, 2 * sizeof(Counters));
    for (auto &ev : e->ev)
        if (ev != nullptr) cudaEventDestroy(ev);
    for (auto &ev : e->pev) cudaEventDestroy(ev);
    dev_free(e, e->sc.blk_q);
    dev_free(e, e->d_partial);
    dev_free(e, e->d_out);
    pinned_put(e->h_out, sizeof(double));
    dev_free(e, e->d_init_keys);
    dev_free(e, e->d_init_coef);
    dev_free(e, e->d_basis);
    dev_free(e, e->d_stats);
    clear_start(e);
    dev_free(e, e->d_obs_keys);
    dev_free(e, e->d_obs_coef);
    dev_free(e, e->d_obs_idx);
    if (e->stream != nullptr) {
        cudaStreamSynchronize(e->stream); // the pool frees above are stream-ordered
        cudaStreamDestroy(e->stream);
    }
    cudaGetLastError();
    delete e;
}

}  // extern "C"
