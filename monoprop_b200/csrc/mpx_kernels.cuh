// mpx_kernels.cuh -- the per-gate kernels of the B200 propagation engine (sm_100a).
//
// One Heisenberg gate = two launches over the device term store:
//   k_sweep   -- anticommutation test from the generator's bit-columns (|fold| bits per term), fused cos
//                scaling of the anticommuting coefficients, lower_atol / structural-cutoff / upper_atol
//                emit gate, rotation phase, leader/follower class; compacts the emitted sine branches into
//                the query arrays and writes the leader-emitted bitmap.
//   k_resolve -- one thread per emitted branch: open-addressing lookup of the partner M^G, the
//                leader/follower rule, the rotation of the pair, or the unique append of the missing partner.
//              It also ORs the appended terms' bits into the bit-columns.
//   k_columns -- builds the bit-columns of a range of stored terms (construction, reset, after the
//                shared-memory path; a regrown store copies its column words instead).
// The two per-gate kernels are launched with programmatic dependent launch (pdl_trigger / pdl_wait).
// Every coefficient slot is written by exactly one thread per gate (the sine partner map M -> M^G is
// injective), so no coefficient atomics are needed (layer_build/FusedApply.h:54-56).
#pragma once

#include <cstdint>

#include "mpx_adjoint.cuh"
#include "mpx_device.cuh"

namespace mpx {

// Index (0-based) of the r-th set bit of a (r < popc(a)), by popcount bisection.
__device__ __forceinline__ int nth_set_bit(uint32_t a, int r) {
    int pos = 0;
#pragma unroll
    for (int width = 16; width >= 1; width >>= 1) {
        const int c = __popc(a & ((1u << width) - 1u));
        if (r >= c) {
            r -= c;
            a >>= width;
            pos += width;
        }
    }
    return pos;
}

constexpr int kWarps = kBlock / 32;
// Resident blocks per SM the per-gate kernels are compiled for (register budget 65536 / (256 x this)).
#ifndef MPX_SWEEP_BLOCKS
#define MPX_SWEEP_BLOCKS 4
#endif
constexpr int kSweepBlocksPerSM = MPX_SWEEP_BLOCKS;
// Build-time tuning of the sweep (nvcc -D...): anticommuting terms per lane whose coefficient loads are in
// flight together, and chunks per warp whose column scans are issued together. Prefetch measured on the
// 100-qubit circuit with the dense finish of the gated terms: 2 188.0 ms, 4 190.5 ms, 6 177.2 ms,
// 8 179.8 ms per propagation (6x6 Hubbard: 24.4-24.6 ms for all).
#ifndef MPX_SWEEP_PREFETCH
#define MPX_SWEEP_PREFETCH 6
#endif
#ifndef MPX_SWEEP_BATCH
#define MPX_SWEEP_BATCH 8
#endif
// Column words per interleave unit of a chunk (a divisor of 32). Measured on the 100-qubit circuit:
// 32 (whole chunks) 227 ms, 8 215 ms, 4 213.5 ms, 1 242 ms per propagate.
#ifndef MPX_SWEEP_UNIT
#define MPX_SWEEP_UNIT 4
#endif
constexpr int kPrefetch = MPX_SWEEP_PREFETCH;
constexpr int kBatch = MPX_SWEEP_BATCH;
constexpr int kUnitWords = MPX_SWEEP_UNIT;
static_assert(kUnitWords >= 1 && kUnitWords <= 32 && 32 % kUnitWords == 0, "interleave unit must divide 32");

// Geometry shared by the sweep and resolve launches of one gate (both use the engine's fixed grid):
// warp w of block b scans the chunks b + grid * (w + warps * i) of 1024 terms each; block b owns the query
// region [b * warps * stride, (b + 1) * warps * stride), at least as many slots as its warps scan terms.
// Term, word and chunk indices are 32-bit: a term index is below 2^32 (the store's capacity limit), so a
// column word index is below 2^27 and a chunk index below 2^22. Query positions stay 64-bit.
struct SweepGeometry {
    uint32_t nwords, nchunks;
    uint64_t stride;
    uint32_t n_warps;
};

__device__ __forceinline__ SweepGeometry sweep_geometry(uint64_t n0) {
    SweepGeometry g;
    g.nwords = static_cast<uint32_t>((n0 + 31) >> 5);
    g.nchunks = (g.nwords + 31) >> 5;
    g.n_warps = gridDim.x * kWarps;
    g.stride = static_cast<uint64_t>((g.nchunks + g.n_warps - 1) / g.n_warps) * 1024;
    return g;
}

// The column word that lane `lane` of chunk c scans. A chunk is 32 / kUnitWords units of kUnitWords
// consecutive words, and unit u of chunk c is word range [(c + u * nchunks) * kUnitWords, + kUnitWords):
// consecutive units of the store belong to consecutive chunks, hence to consecutive blocks. Anticommuting
// terms cluster in index ranges (one gate's appends tend to anticommute with the next gate); with whole
// 1024-term chunks a cluster loads the few blocks that own it, with 128-term units it spreads over
// eight times as many. (c, lane) -> word is a bijection of [0, nchunks) x [0, 32) onto [0, 32 nchunks).
__device__ __forceinline__ uint32_t chunk_word(uint32_t c, int lane, uint32_t nchunks) {
    return (c + static_cast<uint32_t>(lane / kUnitWords) * nchunks) * kUnitWords +
           static_cast<uint32_t>(lane % kUnitWords);
}

// Fused anticommutation scan + cos sweep + emit (Scan.h:193-396 with the fused sweep of Scan.h:343-358).
// Warps scan chunks of 1024 terms (32 column words). The anticommutation bit of 32 terms at once is the
// XOR of the generator's fold columns (Pauli pair_swap(G), Majorana G, plus the |M|-parity column for
// odd |G|): only |fold| bits per term are read, not the 8W-byte key. The anticommuting terms are then
// shared out over all the block's threads, whichever warp's chunk holds them: anticommuting terms
// cluster in index ranges (the appends of one gate tend to anticommute with the next gate), and a warp
// left alone with a dense chunk would hold its whole block at the end. Each term is cos-scaled, and
// only those that pass the lower_atol gate load their key row to build the partner M^G, run the
// structural cutoff / upper_atol rescue and the rotation phase. Emitted branches go to the block's own
// query region (one shared-counter bump per warp and round). With a tape, each warp's anticommuting
// count is saved per step (forward pass of a gradient) and, in REPLAY mode, every anticommuting term's
// index and pre-gate coefficient go to the undo log at its chunk-owning warp's precomputed offset.
// EXT: bit 0 only_rotate_len_k, bit 1 basis_change (instantiated only where the engine uses them).
template <int W, int BASIS, bool REPLAY = false, int EXT = 0>
__global__ void __launch_bounds__(kBlock, kSweepBlocksPerSM) k_sweep(Store st, Scratch sc, Counters *__restrict__ cnt,
                                                   const GateDesc *__restrict__ gates, uint32_t gate, uint32_t step,
                                                   Trunc tr, Tape tp, uint64_t *__restrict__ stats) {
    __shared__ uint32_t s_anti[kWarps][kBatch * 32];
    __shared__ uint32_t s_foll[kWarps][kBatch * 32];
    __shared__ uint32_t s_pfx[kWarps][kBatch * 32];
    __shared__ uint32_t s_emit[kWarps][kBatch * 32];
    __shared__ uint32_t s_wtot[kWarps];     // anticommuting terms of each warp's current batch
    __shared__ uint32_t s_wpfx[kWarps + 1]; // their exclusive prefix over the block's warps
    __shared__ uint32_t s_nw[kWarps];       // column words of each warp's current batch
    __shared__ unsigned long long s_ubase[kWarps]; // REPLAY: each warp's undo-log position
    __shared__ unsigned long long s_fbase;         // logging forward pass: the batch's first undo record
    __shared__ uint32_t s_qn;               // the block's queries so far
    __shared__ uint32_t s_red[kWarps];
    __shared__ uint32_t s_fold[kMaxFoldCols];
    pdl_trigger();
    // the gate (constant circuit data) before the dependency wait, the counters after it
    const GateDesc &gd = gates[gate];
    const int n_fold = gd.n_fold;
    const uint32_t fcol = threadIdx.x < kMaxFoldCols ? gd.fold_cols[threadIdx.x] : 0u;
    const bool empty = gd.empty != 0, g_odd = gd.g_odd != 0;
    const uint32_t pivot_col = gd.pivot_col;
    pdl_wait();
    const uint32_t stall = cnt->stall;
    const uint64_t n0 = cnt->n;
    if (stall != kNoStall) return;
    if (2 * n0 > st.cap) {
        // Not enough room for the worst case (every term appends its partner): stop here, untouched,
        // and let the host grow the store and re-issue this step.
        if (threadIdx.x == 0) atomicMin(&cnt->stall, step);
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        cnt->n0 = n0;
        if constexpr (!REPLAY) {
            stats[4 * static_cast<uint64_t>(step)] = n0;
            if (tp.r_begin != nullptr) tp.r_begin[step] = cnt->rec_total;
        }
    }
    const SweepGeometry geo = sweep_geometry(n0);
    if (threadIdx.x < kMaxFoldCols) s_fold[threadIdx.x] = static_cast<int>(threadIdx.x) < n_fold ? fcol : 0;
    if (threadIdx.x == 0) s_qn = 0;
    if constexpr (REPLAY) {
        if (threadIdx.x < kWarps)
            s_ubase[threadIdx.x] = tp.u_off[(static_cast<uint64_t>(step) - tp.u_off_step0) * geo.n_warps +
                                            blockIdx.x * kWarps + threadIdx.x];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t anti_count = 0;
    if (!empty && n0 != 0) {
        const double cosv = gd.cosv, sinabs = gd.abs_sin;
        const bool cos_zero = gd.cos_zero != 0;
        const int gpop = gd.gpop;
        const uint32_t *__restrict__ pivot = st.cols + static_cast<uint64_t>(pivot_col) * st.cstride;
        const uint32_t *__restrict__ parity = st.cols + static_cast<uint64_t>(64 * W) * st.cstride;
        const uint32_t tail = (n0 & 31) ? ((1u << (n0 & 31)) - 1u) : 0xFFFFFFFFu;
        const uint64_t qbase = static_cast<uint64_t>(blockIdx.x) * kWarps * geo.stride;
        const uint32_t span = static_cast<uint32_t>(kBatch) * geo.n_warps;

        // Consecutive chunks go to consecutive blocks (warp w of block b takes chunks
        // b + grid * (w + warps * i)), so dense index ranges spread over all blocks. Each warp takes its
        // chunks in batches of kBatch (the column loads of the whole batch in flight together); per block
        // iteration, the anticommuting terms of the block's batches form one list in (warp, chunk, lane,
        // bit) order, dealt out in rounds of kBlock * kPrefetch.
        for (uint32_t it0 = blockIdx.x; it0 < geo.nchunks; it0 += span) { // block-uniform
            const uint32_t c0 = it0 + gridDim.x * static_cast<uint32_t>(warp);
            int nb = 0;
            if (c0 < geo.nchunks) {
                const uint32_t left = (geo.nchunks - c0 + geo.n_warps - 1) / geo.n_warps;
                nb = static_cast<int>(left < static_cast<uint32_t>(kBatch) ? left : kBatch);
            }
            int total = 0;
#pragma unroll 2
            for (int b = 0; b < nb; ++b) {
                const uint32_t j = chunk_word(c0 + static_cast<uint32_t>(b) * geo.n_warps, lane, geo.nchunks);
                uint32_t anti = 0, foll = 0;
                if (j < geo.nwords) {
                    if (n_fold <= kMaxFoldCols) {
                        uint32_t v[kMaxFoldCols];
#pragma unroll
                        for (int f = 0; f < kMaxFoldCols; ++f)
                            v[f] = f < n_fold ? st.cols[static_cast<uint64_t>(s_fold[f]) * st.cstride + j] : 0u;
#pragma unroll
                        for (int f = 0; f < kMaxFoldCols; ++f) anti ^= v[f];
                    }
                    else {
#pragma unroll
                        for (int w = 0; w < W; ++w) {
                            for (uint64_t x = gd.fold[w]; x != 0; x &= x - 1) {
                                const uint64_t c = static_cast<uint64_t>(64 * w + __ffsll(static_cast<long long>(x)) - 1);
                                anti ^= st.cols[c * st.cstride + j];
                            }
                        }
                    }
                    if (g_odd) anti ^= parity[j];
                    if (j == geo.nwords - 1) anti &= tail;
                    foll = anti & pivot[j];
                }
                const int cnt_l = __popc(anti);
                int incl = cnt_l;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                    if (lane >= o) incl += t;
                }
                s_anti[warp][b * 32 + lane] = anti;
                s_foll[warp][b * 32 + lane] = foll;
                s_pfx[warp][b * 32 + lane] = static_cast<uint32_t>(total + incl - cnt_l);
                s_emit[warp][b * 32 + lane] = 0;
                total += __shfl_sync(0xFFFFFFFFu, incl, 31);
            }
            if (lane == 0) {
                s_wtot[warp] = static_cast<uint32_t>(total);
                s_nw[warp] = static_cast<uint32_t>(nb * 32);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                uint32_t acc = 0;
#pragma unroll
                for (int w = 0; w < kWarps; ++w) {
                    s_wpfx[w] = acc;
                    acc += s_wtot[w];
                }
                s_wpfx[kWarps] = acc;
                if constexpr (!REPLAY) {
                    if (tp.f_uidx != nullptr)
                        s_fbase = acc != 0 ? atomicAdd(tp.f_utotal, static_cast<unsigned long long>(acc)) : 0ULL;
                }
            }
            __syncthreads();
            const int btotal = static_cast<int>(s_wpfx[kWarps]);
            // Rounds of up to kBlock * kPrefetch anticommuting terms: every thread first issues the
            // coefficient loads of its kPrefetch terms (independent random accesses in flight together),
            // then processes them one by one. loc = owner * (kBatch * 1024) + (batch word) * 32 + bit.
            for (int k = 0; k < btotal; k += kBlock * kPrefetch) {
                int loc[kPrefetch];
                double vv[kPrefetch];
#pragma unroll
                for (int r = 0; r < kPrefetch; ++r) {
                    const int idx = k + kBlock * r + static_cast<int>(threadIdx.x);
                    loc[r] = -1;
                    vv[r] = 0.0;
                    if (idx < btotal) {
                        int ow = 0;
#pragma unroll
                        for (int w = 1; w < kWarps; ++w) ow += (static_cast<int>(s_wpfx[w]) <= idx) ? 1 : 0;
                        const int li = idx - static_cast<int>(s_wpfx[ow]);
                        int lo = 0, hi = static_cast<int>(s_nw[ow]);
                        while (hi - lo > 1) {
                            const int mid = (lo + hi) >> 1;
                            if (static_cast<int>(s_pfx[ow][mid]) <= li) lo = mid;
                            else hi = mid;
                        }
                        const int l = lo * 32 + nth_set_bit(s_anti[ow][lo], li - static_cast<int>(s_pfx[ow][lo]));
                        loc[r] = ow * (kBatch * 1024) + l;
                        const uint32_t chunk = it0 + gridDim.x * static_cast<uint32_t>(ow) +
                                               static_cast<uint32_t>(lo >> 5) * geo.n_warps;
                        vv[r] = st.coef[chunk_word(chunk, lo & 31, geo.nchunks) * 32 + static_cast<uint32_t>(l & 31)];
                    }
                }
                // Phase 1, every prefetched term: membership, cos scaling, undo log and the lower_atol gate.
                // Terms that pass the gate are marked (bit r of cand) instead of being finished here: they
                // are a few per warp (1-10 % of the anticommuting terms), and finishing them in place would
                // run the key load and the partner, cutoff and phase work once per slot for those few lanes.
                uint32_t cand = 0;
#pragma unroll
                for (int r = 0; r < kPrefetch; ++r) {
                    if (k + kBlock * r + 32 * warp >= btotal) break; // warp-uniform
                    const int L = loc[r];
                    const double v = vv[r];
                    const int ow = L < 0 ? 0 : (L / (kBatch * 1024));
                    const int l = L < 0 ? 0 : (L % (kBatch * 1024));
                    const int word = l >> 5; // batch word: chunk (word >> 5), lane (word & 31)
                    const uint32_t term = chunk_word(it0 + gridDim.x * static_cast<uint32_t>(ow) +
                                                         static_cast<uint32_t>(word >> 5) * geo.n_warps,
                                                     word & 31, geo.nchunks) * 32 +
                                          static_cast<uint32_t>(l & 31);
                    bool member = L >= 0;
                    if ((EXT & 1) && member) {
                        // only_rotate_len_k: a term of more than len_k slots is left alone by this gate
                        // (no cos scaling, no emit); the partner values of the others are kept in `aux`
                        uint64_t mk[W];
                        load_key<W>(st.keys, term, mk);
                        int kp = 0;
#pragma unroll
                        for (int w = 0; w < W; ++w) kp += __popcll(mk[w]);
                        member = kp <= static_cast<int>(tr.len_k);
                        if constexpr (REPLAY) {
                            // its undo slot says "not scaled by this gate" (the backward pass skips it)
                            if (!member) {
                                const uint64_t rr = s_ubase[ow] + static_cast<uint64_t>(k + kBlock * r +
                                                                                         static_cast<int>(threadIdx.x) -
                                                                                         static_cast<int>(s_wpfx[ow]));
                                tp.u_idx[rr] = kNoStall;
                            }
                        }
                        else if (!member && tp.f_uidx != nullptr) {
                            const uint64_t rr = s_fbase + static_cast<uint64_t>(k + kBlock * r + static_cast<int>(threadIdx.x));
                            if (rr < tp.f_ucap) tp.f_uidx[rr] = kNoStall;
                        }
                    }
                    if (member) {
                        st.coef[term] = v * cosv;
                        if (cos_zero || (EXT & 1)) sc.aux[term] = v;
                        if constexpr (REPLAY) {
                            const uint64_t rr = s_ubase[ow] + static_cast<uint64_t>(k + kBlock * r +
                                                                                     static_cast<int>(threadIdx.x) -
                                                                                     static_cast<int>(s_wpfx[ow]));
                            tp.u_idx[rr] = static_cast<uint32_t>(term);
                            tp.u_val[rr] = v;
                        }
                        else if (tp.f_uidx != nullptr) {
                            // logging forward pass: the undo record of this term, in the block's dealing order
                            const uint64_t rr = s_fbase + static_cast<uint64_t>(k + kBlock * r + static_cast<int>(threadIdx.x));
                            if (rr < tp.f_ucap) {
                                tp.f_uidx[rr] = term;
                                tp.f_uval[rr] = v;
                            }
                        }
                        if (!(tr.has_lower && sinabs * fabs(v) <= tr.lower)) cand |= 1u << r;
                    }
                }
                // Phase 2: the warp's marked terms, dense, 32 at a time. Candidate c of the warp is slot r_c of
                // lane src (slots in order, lanes in order within a slot); its location and value come over
                // by shuffle, so every lane does the key load and the partner work for one real candidate.
                uint32_t pb[kPrefetch];
                int pfx[kPrefetch];
                int n_cand = 0;
#pragma unroll
                for (int r = 0; r < kPrefetch; ++r) {
                    pb[r] = __ballot_sync(0xFFFFFFFFu, (cand >> r) & 1u);
                    pfx[r] = n_cand;
                    n_cand += __popc(pb[r]);
                }
                for (int base = 0; base < n_cand; base += 32) { // warp-uniform
                    const int ci = base + lane;
                    int r_c = 0;
#pragma unroll
                    for (int r = 1; r < kPrefetch; ++r) r_c += (pfx[r] <= ci) ? 1 : 0;
                    uint32_t pbr = pb[0];
#pragma unroll
                    for (int r = 1; r < kPrefetch; ++r) pbr = (r == r_c) ? pb[r] : pbr;
                    int pr = pfx[0];
#pragma unroll
                    for (int r = 1; r < kPrefetch; ++r) pr = (r == r_c) ? pfx[r] : pr;
                    const bool has = ci < n_cand;
                    const int src = has ? nth_set_bit(pbr, ci - pr) : lane;
                    int L = -1;
                    double v = 0.0;
#pragma unroll
                    for (int r = 0; r < kPrefetch; ++r) {
                        const int Lr = __shfl_sync(0xFFFFFFFFu, loc[r], src);
                        const double vr = __shfl_sync(0xFFFFFFFFu, vv[r], src);
                        if (r == r_c) {
                            L = Lr;
                            v = vr;
                        }
                    }
                    bool emit = false, follower = false;
                    int phase = 0;
                    int ow = 0, l = 0, word = 0;
                    uint32_t term = 0;
                    if (has) {
                        ow = L / (kBatch * 1024);
                        l = L % (kBatch * 1024);
                        word = l >> 5;
                        term = chunk_word(it0 + gridDim.x * static_cast<uint32_t>(ow) +
                                              static_cast<uint32_t>(word >> 5) * geo.n_warps,
                                          word & 31, geo.nchunks) * 32 +
                               static_cast<uint32_t>(l & 31);
                        follower = (s_foll[ow][word] >> (l & 31)) & 1u;
                        const double av = fabs(v);
                        uint64_t m[W], p[W];
                        load_key<W>(st.keys, term, m);
                        int mpop = 0, ov = 0;
#pragma unroll
                        for (int w = 0; w < W; ++w) {
                            const uint64_t gw = gd.g[w];
                            p[w] = m[w] ^ gw;
                            mpop += __popcll(m[w]);
                            ov += __popcll(m[w] & gw);
                        }
                        const int ppop = mpop + gpop - 2 * ov;
                        bool keep;
                        if constexpr ((EXT & 2) != 0) keep = keep_partner_mapped<W>(p, tr);
                        else keep = keep_partner<W>(p, ppop, tr);
                        if (keep || (tr.has_upper && sinabs * av >= tr.upper)) {
                            emit = true;
                            phase = rotation_phase<W, BASIS>(m, p, gd, mpop, ppop);
                        }
                    }
                    const uint32_t eb = __ballot_sync(0xFFFFFFFFu, emit);
                    uint32_t qb = 0;
                    if (lane == 0 && eb != 0) qb = atomicAdd(&s_qn, static_cast<uint32_t>(__popc(eb)));
                    qb = __shfl_sync(0xFFFFFFFFu, qb, 0);
                    if (emit) {
                        const uint64_t q = qbase + qb + __popc(eb & lt_mask);
                        sc.q_src[q] = term;
                        sc.q_flag[q] = static_cast<uint8_t>((follower ? 1 : 0) | (phase_code(phase) << 1));
                        sc.q_val[q] = v;
                        if (!follower) atomicOr(&s_emit[ow][word], 1u << (l & 31));
                    }
                }
            }
            __syncthreads(); // every round of this batch is done: the emit bitmaps are final
            for (int b = 0; b < nb; ++b) {
                const uint32_t j = chunk_word(c0 + static_cast<uint32_t>(b) * geo.n_warps, lane, geo.nchunks);
                if (j < geo.nwords) sc.emit_bits[j] = s_emit[warp][b * 32 + lane];
            }
            anti_count += static_cast<uint32_t>(total);
            if constexpr (REPLAY) {
                if (lane == 0) s_ubase[warp] += static_cast<unsigned long long>(total);
            }
            __syncwarp();
        }
    }
    if (lane == 0) {
        if (tp.w_anti != nullptr && !REPLAY) tp.w_anti[static_cast<uint64_t>(step) * geo.n_warps + blockIdx.x * kWarps + warp] = anti_count;
        s_red[warp] = anti_count;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) t += s_red[w];
        sc.blk_q[blockIdx.x] = s_qn;
        if constexpr (!REPLAY) {
            // per-gate counters for the host (a_g, e_g; zeroed before the range): integer sums, any order
            auto *ctr = reinterpret_cast<unsigned long long *>(stats + 4 * static_cast<uint64_t>(step));
            if (t != 0) atomicAdd(ctr + 1, static_cast<unsigned long long>(t));
            if (s_qn != 0) atomicAdd(ctr + 2, static_cast<unsigned long long>(s_qn));
        }
    }
}

// The other anticommuting terms of one frozen gate (terms < n0 whose fold-column parity is odd) are
// scaled by cos; pair members (done bits, set by k_frozen_pairs) are skipped and their bits cleared.
// Chunk ownership, batching and the block-wide dealing of the anticommuting terms are the sweep's, so
// each sweep warp's terms are the ones it counted in the forward pass. With LOG every anticommuting
// term's pre-gate value goes to the undo log from its chunk-owning warp's offset; pair members get the
// skip index kNoStall there (their adjoint comes from the pair records: k_adj_step).
// With a pared graph (last != nullptr) a term whose value can no longer reach <0|O|0> after this step
// (last[term] < step) keeps its coefficient unscaled. With a graph built under only_rotate_len_k, longb
// (one bit per term) marks the terms of more than k slots: they are never scaled, and their undo entries
// say so (index kNoStall).
template <int W, bool LOG>
__global__ void __launch_bounds__(kBlock, kSweepBlocksPerSM)
    k_frozen_scan(Store st, const GateDesc *__restrict__ gates, uint32_t gate, uint32_t step, uint64_t n0,
                  uint32_t *__restrict__ done, Tape tp, const int32_t *__restrict__ last,
                  const uint32_t *__restrict__ longb) {
    __shared__ uint32_t s_anti[kWarps][kBatch * 32];
    __shared__ uint32_t s_done[kWarps][kBatch * 32];
    __shared__ uint32_t s_long[kWarps][kBatch * 32];
    __shared__ uint32_t s_pfx[kWarps][kBatch * 32];
    __shared__ uint32_t s_wtot[kWarps];
    __shared__ uint32_t s_wpfx[kWarps + 1];
    __shared__ uint32_t s_nw[kWarps];
    __shared__ unsigned long long s_ubase[kWarps];
    __shared__ uint32_t s_fold[kMaxFoldCols];
    pdl_trigger();
    pdl_wait();
    const GateDesc &gd = gates[gate];
    if (gd.empty || n0 == 0) return;
    const int n_fold = gd.n_fold;
    const SweepGeometry geo = sweep_geometry(n0);
    if (threadIdx.x < kMaxFoldCols) s_fold[threadIdx.x] = threadIdx.x < n_fold ? gd.fold_cols[threadIdx.x] : 0;
    if constexpr (LOG) {
        if (threadIdx.x < kWarps)
            s_ubase[threadIdx.x] = tp.u_off[(static_cast<uint64_t>(step) - tp.u_off_step0) * geo.n_warps +
                                            blockIdx.x * kWarps + threadIdx.x];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double C = gd.cosv;
    const uint32_t *__restrict__ parity = st.cols + static_cast<uint64_t>(64 * W) * st.cstride;
    const uint32_t tail = (n0 & 31) ? ((1u << (n0 & 31)) - 1u) : 0xFFFFFFFFu;
    const uint32_t span = static_cast<uint32_t>(kBatch) * geo.n_warps;
    for (uint32_t it0 = blockIdx.x; it0 < geo.nchunks; it0 += span) { // block-uniform
        const uint32_t c0 = it0 + gridDim.x * static_cast<uint32_t>(warp);
        int nb = 0;
        if (c0 < geo.nchunks) {
            const uint32_t left = (geo.nchunks - c0 + geo.n_warps - 1) / geo.n_warps;
            nb = static_cast<int>(left < static_cast<uint32_t>(kBatch) ? left : kBatch);
        }
        int total = 0;
#pragma unroll 2
        for (int b = 0; b < nb; ++b) {
            const uint32_t j = chunk_word(c0 + static_cast<uint32_t>(b) * geo.n_warps, lane, geo.nchunks);
            uint32_t anti = 0, dn = 0, lg = 0; // lg: terms outside the only_rotate_len_k set
            if (j < geo.nwords) {
                if (n_fold <= kMaxFoldCols) {
                    uint32_t v[kMaxFoldCols];
#pragma unroll
                    for (int f = 0; f < kMaxFoldCols; ++f)
                        v[f] = f < n_fold ? st.cols[static_cast<uint64_t>(s_fold[f]) * st.cstride + j] : 0u;
#pragma unroll
                    for (int f = 0; f < kMaxFoldCols; ++f) anti ^= v[f];
                }
                else {
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        for (uint64_t x = gd.fold[w]; x != 0; x &= x - 1) {
                            const uint64_t c = static_cast<uint64_t>(64 * w + __ffsll(static_cast<long long>(x)) - 1);
                            anti ^= st.cols[c * st.cstride + j];
                        }
                    }
                }
                if (gd.g_odd) anti ^= parity[j];
                if (j == geo.nwords - 1) anti &= tail;
                dn = done[j];
                if (dn) done[j] = 0;
                if (longb != nullptr) lg = longb[j];
            }
            const int cnt_l = __popc(anti);
            int incl = cnt_l;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (lane >= o) incl += t;
            }
            s_anti[warp][b * 32 + lane] = anti;
            s_done[warp][b * 32 + lane] = dn;
            s_long[warp][b * 32 + lane] = lg;
            s_pfx[warp][b * 32 + lane] = static_cast<uint32_t>(total + incl - cnt_l);
            total += __shfl_sync(0xFFFFFFFFu, incl, 31);
        }
        if (lane == 0) {
            s_wtot[warp] = static_cast<uint32_t>(total);
            s_nw[warp] = static_cast<uint32_t>(nb * 32);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t acc = 0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) {
                s_wpfx[w] = acc;
                acc += s_wtot[w];
            }
            s_wpfx[kWarps] = acc;
        }
        __syncthreads();
        const int btotal = static_cast<int>(s_wpfx[kWarps]);
        for (int k = 0; k < btotal; k += kBlock * kPrefetch) {
            uint32_t term[kPrefetch];
            double vv[kPrefetch];
            int own[kPrefetch];
            bool skip[kPrefetch], outside[kPrefetch];
#pragma unroll
            for (int r = 0; r < kPrefetch; ++r) {
                const int idx = k + kBlock * r + static_cast<int>(threadIdx.x);
                own[r] = -1;
                term[r] = 0;
                vv[r] = 0.0;
                skip[r] = true;
                outside[r] = false;
                if (idx < btotal) {
                    int ow = 0;
#pragma unroll
                    for (int w = 1; w < kWarps; ++w) ow += (static_cast<int>(s_wpfx[w]) <= idx) ? 1 : 0;
                    const int li = idx - static_cast<int>(s_wpfx[ow]);
                    int lo = 0, hi = static_cast<int>(s_nw[ow]);
                    while (hi - lo > 1) {
                        const int mid = (lo + hi) >> 1;
                        if (static_cast<int>(s_pfx[ow][mid]) <= li) lo = mid;
                        else hi = mid;
                    }
                    const int bit = nth_set_bit(s_anti[ow][lo], li - static_cast<int>(s_pfx[ow][lo]));
                    const uint32_t chunk = it0 + gridDim.x * static_cast<uint32_t>(ow) +
                                           static_cast<uint32_t>(lo >> 5) * geo.n_warps;
                    own[r] = ow;
                    term[r] = chunk_word(chunk, lo & 31, geo.nchunks) * 32 + bit;
                    outside[r] = (s_long[ow][lo] >> bit) & 1u;
                    skip[r] = ((s_done[ow][lo] >> bit) & 1u) || outside[r];
                    vv[r] = st.coef[term[r]];
                }
            }
#pragma unroll
            for (int r = 0; r < kPrefetch; ++r) {
                if (own[r] < 0) continue;
                if constexpr (LOG) {
                    const int idx = k + kBlock * r + static_cast<int>(threadIdx.x);
                    const uint64_t rr = s_ubase[own[r]] + static_cast<uint64_t>(idx - static_cast<int>(s_wpfx[own[r]]));
                    // pair members (handled by the pair records) and terms outside the len_k set (not
                    // scaled) get the "skip" index, so the reverse step needs no done bits
                    tp.u_idx[rr] = skip[r] ? kNoStall : static_cast<uint32_t>(term[r]);
                    tp.u_val[rr] = vv[r];
                }
                if (!skip[r] && (last == nullptr || last[term[r]] >= static_cast<int32_t>(step)))
                    st.coef[term[r]] = vv[r] * C;
            }
        }
        __syncthreads(); // the lists of this batch are consumed
        if constexpr (LOG) {
            if (lane == 0) s_ubase[warp] += static_cast<unsigned long long>(total);
        }
        __syncwarp();
    }
}

constexpr int kMaxGrid = 1024; // largest per-gate grid (148 SMs x at most 4 blocks per SM, with headroom)

// Partner resolve + rotation apply + append (Engine.h:364-513, FusedApply.h:32-83, MPOperator.h:269-278).
// The sweep leaves the emitted branches of a gate in per-sweep-block query regions of very uneven fill
// (anticommuting terms cluster in index ranges, so a few blocks hold most of them). Every resolve block
// therefore first forms the exclusive prefix of the regions' counts in shared memory and takes an equal
// contiguous share of the gate's queries, whichever regions they lie in; a query's region is found by a
// binary search over the prefix. The block works through its share in block-wide rounds, one query per
// thread; appends take one counter bump per round. In REPLAY mode the keys of this gate's appends
// already exist (indices >= n0, inserted by the forward pass): a partner found there is treated as the
// append it was, nothing is inserted, and every rotated or appended pair goes to the tape's pair log with
// both pre-gate coefficients (one counter bump per round).
template <int W, int BASIS, bool REPLAY = false, bool LENK = false>
__global__ void __launch_bounds__(kBlock, kSweepBlocksPerSM) k_resolve(Store st, Scratch sc, Counters *__restrict__ cnt,
                                                     const GateDesc *__restrict__ gates, uint32_t gate, uint32_t step,
                                                     Trunc tr, Tape tp) {
    __shared__ uint32_t warp_cnt[kWarps];
    __shared__ unsigned long long s_base, s_rbase;
    __shared__ uint32_t s_pfx[kMaxGrid + 1]; // exclusive prefix of the regions' query counts
    __shared__ uint32_t s_wsum[kWarps];
    pdl_trigger();
    // the gate (constant circuit data) before the dependency wait; counters and query counts after it
    const GateDesc &gd = gates[gate];
    const bool empty = gd.empty != 0;
    pdl_wait();
    // Thread t owns regions [t*per, (t+1)*per) of the prefix below. Their query counts are loaded together
    // with the counters (neither depends on the other) and kept in registers for both passes.
    const uint32_t G = gridDim.x;
    const uint32_t per = (G + kBlock - 1) / kBlock;
    constexpr uint32_t kPer = (kMaxGrid + kBlock - 1) / kBlock;
    uint32_t qc[kPer];
#pragma unroll
    for (uint32_t i = 0; i < kPer; ++i) {
        const uint32_t r = threadIdx.x * per + i;
        qc[i] = (i < per && r < G) ? sc.blk_q[r] : 0u;
    }
    const uint32_t stall = cnt->stall;
    const uint64_t n0 = cnt->n0;
    if constexpr (!REPLAY) {
        // logging forward pass: this gate's sweep has reserved all its undo records (a stalled step is
        // re-issued and writes this again)
        if (tp.f_ubegin != nullptr && blockIdx.x == 0 && threadIdx.x == 0) tp.f_ubegin[step + 1] = *tp.f_utotal;
    }
    if (stall != kNoStall) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const SweepGeometry geo = sweep_geometry(n0);
    if (empty || n0 == 0) return;
    // prefix of the per-region counts
    uint32_t mine = 0;
#pragma unroll
    for (uint32_t i = 0; i < kPer; ++i) mine += qc[i];
    uint32_t incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    uint32_t wbase = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) wbase += (w < warp) ? s_wsum[w] : 0u;
    {
        uint32_t acc = wbase + incl - mine;
#pragma unroll
        for (uint32_t i = 0; i < kPer; ++i) {
            const uint32_t r = threadIdx.x * per + i;
            if (i < per && r < G) {
                s_pfx[r] = acc;
                acc += qc[i];
            }
        }
    }
    uint32_t Q = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) Q += s_wsum[w];
    if (threadIdx.x == 0) s_pfx[G] = Q;
    __syncthreads();
    if (Q == 0) return;
    // this block's equal share [lo, hi) of the gate's Q queries
    const uint32_t lo = static_cast<uint32_t>((static_cast<uint64_t>(Q) * blockIdx.x) / G);
    const uint32_t hi = static_cast<uint32_t>((static_cast<uint64_t>(Q) * (blockIdx.x + 1)) / G);
    if (lo == hi) return;
    const uint64_t region_slots = static_cast<uint64_t>(kWarps) * geo.stride;
    uint64_t g[W];
#pragma unroll
    for (int w = 0; w < W; ++w) g[w] = gd.g[w];
    const double sinv = gd.sinv, inv_cos = gd.inv_cos;
    const bool cos_zero = gd.cos_zero != 0;

    for (uint32_t tb = lo; tb < hi; tb += kBlock) { // block-uniform rounds
        const uint32_t k = tb + threadIdx.x;
        bool miss = false, rec = false;
        uint64_t p[W];
        uint64_t pos = 0;
        uint32_t tag = 0, src = 0, tgt = 0;
        int8_t code = 0;
        double v = 0.0, ph = 0.0, vt = 0.0;
        double cs = 0.0, cf = 0.0, ax = 0.0; // source, partner and partner's kept pre-gate value
        uint32_t ebw = 0;                    // the partner's word of the leader-emitted bitmap
        if (k < hi) {
            // region of query k: the last r with s_pfx[r] <= k
            uint32_t a = 0, b = G;
            while (b - a > 1) {
                const uint32_t mid = (a + b) >> 1;
                if (s_pfx[mid] <= k) a = mid;
                else b = mid;
            }
            const uint64_t q = a * region_slots + (k - s_pfx[a]);
            // The source's coefficient (for a rotation) is loaded alongside its key; the candidate's key,
            // coefficient and leader bit are loaded together below (measured: a hash carried in the
            // query record instead, sparing the source-key load, made the sweep's emits dearer and the
            // whole propagate 2% slower).
            src = sc.q_src[q];
            const uint8_t flag = sc.q_flag[q];
            v = sc.q_val[q];
            ph = phase_value(static_cast<uint8_t>(flag >> 1));
            uint64_t m[W];
            load_key<W>(st.keys, src, m); // mostly an L2 hit: the sweep has just read this row
            cs = st.coef[src];
            uint64_t h;
            {
                uint64_t pp[W];
#pragma unroll
                for (int w = 0; w < W; ++w) pp[w] = m[w] ^ g[w];
                h = key_hash<W>(pp);
            }
            tag = static_cast<uint32_t>(h >> 32);
            pos = h & st.tmask;
            uint64_t found = ~0ULL;
            int fpop = 0;
            bool gave_up = false;
            for (uint64_t probes = 0;; ++probes) {
                if (probes > st.tmask) { // a full table cannot happen below load 1/2; never spin
                    atomicOr(&cnt->err, 1u);
                    gave_up = true;
                    break;
                }
                const unsigned long long slot = st.table[pos];
                if (slot == kEmptySlot) {
                    miss = true;
                    break;
                }
                const uint32_t idx = static_cast<uint32_t>(slot);
                if ((REPLAY || idx < n0) && static_cast<uint32_t>(slot >> 32) == tag) {
                    uint64_t o[W];
                    load_key<W>(st.keys, idx, o);
                    // what a hit needs, loaded together with the candidate key (a matching tag is almost
                    // always the partner; the values are dropped otherwise)
                    const double cf_c = st.coef[idx];
                    const uint32_t eb_c = sc.emit_bits[idx >> 5];
                    const double ax_c = (LENK || cos_zero) ? sc.aux[idx] : 0.0;
                    bool eq = true;
#pragma unroll
                    for (int w = 0; w < W; ++w) eq = eq && (o[w] == (m[w] ^ g[w]));
                    if (eq) {
                        found = idx;
                        cf = cf_c;
                        ebw = eb_c;
                        ax = ax_c;
#pragma unroll
                        for (int w = 0; w < W; ++w) fpop += __popcll(o[w]);
                        break;
                    }
                }
                pos = (pos + 1) & st.tmask;
            }
#pragma unroll
            for (int w = 0; w < W; ++w) p[w] = m[w] ^ g[w];
            if constexpr (REPLAY) {
                if (miss) { // the forward pass found or appended every partner of this gate
                    atomicOr(&cnt->err, 8u);
                    miss = false;
                }
                else if (!gave_up && found >= n0) {
                    // the append of the forward pass, redone with the same arithmetic as its miss branch
                    // (vt, the partner's value before the gate, goes to the pair log)
                    vt = 0.0;
                    double c_new = (sinv * ph) * v;
                    if (tr.schr) {
                        vt = state_score<W, BASIS>(p, tr.occ);
                        st.coef[src] = __fma_rn(sinv * -ph, vt, cs);
                        c_new = (!cos_zero && !LENK) ? __fma_rn(gd.cosv, vt, (sinv * ph) * v)
                                                     : __fma_rn(sinv * ph, v, gd.cosv * vt);
                    }
                    st.coef[found] = c_new;
                    rec = true;
                    tgt = static_cast<uint32_t>(found);
                    code = static_cast<int8_t>(0x10 | (static_cast<int>(ph) & 0xF));
                    gave_up = true; // handled
                }
            }
            if (!miss && !gave_up) {
                const bool follower = (flag & 1) != 0;
                const bool leader_took_it = follower && ((ebw >> (found & 31)) & 1u);
                if (!leader_took_it) {
                    // cs and cf are the current values of both slots: each slot of a pair is written by the
                    // one thread that rotates the pair (src != found: G is not the identity)
                    if constexpr (LENK) // pre-gate value: kept by the sweep, or untouched (partner outside the cos set)
                        vt = fpop <= static_cast<int>(tr.len_k) ? ax : cf;
                    else
                        vt = cos_zero ? ax : cf * inv_cos;
                    st.coef[src] = __fma_rn(sinv * -ph, vt, cs);
                    st.coef[found] = __fma_rn(sinv * ph, v, cf);
                    rec = true; // a rotated pair (recorded in replay mode and by a recording forward pass)
                    tgt = static_cast<uint32_t>(found);
                    code = static_cast<int8_t>(static_cast<int>(ph) & 0xF);
                    // 0x20: the partner lies outside the only_rotate_len_k set (no cos factor of its own)
                    if constexpr (LENK)
                        if (fpop > static_cast<int>(tr.len_k)) code = static_cast<int8_t>(code | 0x20);
                }
            }
        }
        // Unique appends (forward) or pair records (replay): one counter bump per round.
        const uint32_t ball = __ballot_sync(0xFFFFFFFFu, REPLAY ? rec : miss);
        if (lane == 0) warp_cnt[warp] = __popc(ball);
        __syncthreads();
        uint32_t off = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t t = warp_cnt[w];
            off += (w < warp) ? t : 0u;
            tot += t;
        }
        if (threadIdx.x == 0 && tot > 0) {
            if constexpr (REPLAY) s_rbase = atomicAdd(&tp.p_cnt[step], static_cast<unsigned long long>(tot));
            else s_base = atomicAdd(&cnt->n, static_cast<unsigned long long>(tot));
        }
        __syncthreads();
        if constexpr (REPLAY) {
            if (rec) {
                const uint64_t r = tp.p_base[step] + s_rbase + off + __popc(ball & lt_mask);
                tp.p_src[r] = src;
                tp.p_tgt[r] = tgt;
                tp.p_code[r] = code;
                tp.p_vs[r] = v;
                tp.p_vt[r] = vt;
            }
        }
        else if (miss) {
            const uint64_t idx = s_base + off + __popc(ball & lt_mask);
            store_key<W>(st.keys, idx, p);
            double c_new = (sinv * ph) * v; // Heisenberg: the new term starts from 0
            if (tr.schr) {
                // Schrodinger (FusedApply.h:39-83): the new slot starts from its reference-state score vt,
                // and the pair rotates as a hit does (the source's cos factor is already applied)
                const double vt0 = state_score<W, BASIS>(p, tr.occ);
                st.coef[src] = __fma_rn(sinv * -ph, vt0, cs);
                c_new = (!cos_zero && !LENK) ? __fma_rn(gd.cosv, vt0, (sinv * ph) * v)
                                             : __fma_rn(sinv * ph, v, gd.cosv * vt0);
                vt = vt0; // the new slot's value before the gate, for a logging forward pass
            }
            st.coef[idx] = c_new;
            const unsigned long long mine = (static_cast<unsigned long long>(tag) << 32) | idx;
            for (uint64_t probes = 0;; ++probes) {
                if (probes > st.tmask) {
                    atomicOr(&cnt->err, 2u);
                    break;
                }
                const unsigned long long old = atomicCAS(&st.table[pos], kEmptySlot, mine);
                if (old == kEmptySlot) break;
                pos = (pos + 1) & st.tmask;
            }
            // Bit-columns of the append (InvertedIndex::append_rows, InvertedIndex.h:178-193): each lane ORs
            // its term's bits (column bits of terms not yet stored are zero). On an append-heavy gate this
            // costs about what a separate ballot transposition does, and nothing extra on sparse ones.
            {
                int pop = 0;
                const uint32_t bit = 1u << (idx & 31);
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    pop += __popcll(p[w]);
                    for (uint64_t x = p[w]; x != 0; x &= x - 1)
                        atomicOr(st.cols + static_cast<uint64_t>(64 * w + __ffsll(static_cast<long long>(x)) - 1) *
                                               st.cstride + (idx >> 5),
                                 bit);
                }
                if (pop & 1) atomicOr(st.cols + static_cast<uint64_t>(64 * W) * st.cstride + (idx >> 5), bit);
            }
        }
        if constexpr (!REPLAY) {
            if (tp.r_src != nullptr) {
                // recording forward pass: this round's rotated pairs and appends, one counter bump per round
                const bool has = rec || miss;
                const uint32_t rb = __ballot_sync(0xFFFFFFFFu, has);
                __syncthreads();
                if (lane == 0) warp_cnt[warp] = __popc(rb);
                __syncthreads();
                uint32_t roff = 0, rtot = 0;
#pragma unroll
                for (int w = 0; w < kWarps; ++w) {
                    const uint32_t t = warp_cnt[w];
                    roff += (w < warp) ? t : 0u;
                    rtot += t;
                }
                if (threadIdx.x == 0 && rtot > 0) s_rbase = atomicAdd(&cnt->rec_total, static_cast<unsigned long long>(rtot));
                __syncthreads();
                if (has) {
                    const uint64_t r = s_rbase + roff + __popc(rb & lt_mask);
                    if (r < tp.r_cap) {
                        tp.r_src[r] = src;
                        tp.r_tgt[r] = miss ? static_cast<uint32_t>(s_base + off + __popc(ball & lt_mask)) : tgt;
                        tp.r_code[r] = miss ? static_cast<int8_t>(0x10 | (static_cast<int>(ph) & 0xF)) : code;
                        if (tp.r_vs != nullptr) { // logging forward pass: both values before the gate
                            tp.r_vs[r] = v;
                            tp.r_vt[r] = vt;
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
}

// Writes the bit-columns of terms [lo, hi). A warp takes 8 consecutive column words (256 terms) at a
// time: for each key word, 64 ballots per 32 terms build the 64 columns' words in shared memory, which
// then go out as whole 32-byte sectors (8 words of one column per 8 lanes) instead of 4-byte pieces of
// 64W + 1 different columns. A word that starts below lo already holds valid bits for the terms below lo
// (and zeros above) and is OR-ed; words outside [lo, hi) are not touched; every other word is assigned
// whole (zeros above hi included). With from_counters the range is the current gate's appends [n0, n).
template <int W>
__global__ void __launch_bounds__(kBlock) k_columns(Store st, const Counters *__restrict__ cnt, uint64_t lo,
                                                     uint64_t hi, int from_counters) {
    __shared__ uint32_t s_col[kWarps][64][8];
    if (from_counters) {
        if (cnt->stall != kNoStall) return;
        lo = cnt->n0;
        hi = cnt->n;
    }
    if (hi <= lo) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t w0 = lo >> 5, w1 = (hi + 31) >> 5;
    const uint64_t g_first = w0 >> 3, g_end = (w1 + 7) >> 3;
    const uint64_t n_warps = static_cast<uint64_t>(gridDim.x) * kWarps;
    for (uint64_t grp = g_first + static_cast<uint64_t>(blockIdx.x) * kWarps + warp; grp < g_end; grp += n_warps) {
        const uint64_t j0 = grp * 8;
        int pop[8];
#pragma unroll
        for (int g = 0; g < 8; ++g) pop[g] = 0;
#pragma unroll 1
        for (int w = 0; w < W; ++w) {
#pragma unroll
            for (int g = 0; g < 8; ++g) {
                const uint64_t i = (j0 + g) * 32 + lane;
                const uint64_t x = (i >= lo && i < hi) ? st.keys[i * W + w] : 0ULL;
                pop[g] += __popcll(x);
                uint32_t lo_b = 0, hi_b = 0;
#pragma unroll
                for (int b = 0; b < 32; ++b) {
                    const uint32_t bl = __ballot_sync(0xFFFFFFFFu, (x >> b) & 1ULL);
                    const uint32_t bh = __ballot_sync(0xFFFFFFFFu, (x >> (b + 32)) & 1ULL);
                    if (lane == b) {
                        lo_b = bl;
                        hi_b = bh;
                    }
                }
                s_col[warp][lane][g] = lo_b;
                s_col[warp][lane + 32][g] = hi_b;
            }
            __syncwarp();
            // 64 columns x 8 words: four columns per instruction, eight lanes per column
#pragma unroll 4
            for (int c4 = 0; c4 < 16; ++c4) {
                const int c = c4 * 4 + (lane >> 3), g = lane & 7;
                const uint64_t j = j0 + g;
                if (j >= w0 && j < w1) {
                    uint32_t *dst = st.cols + static_cast<uint64_t>(64 * w + c) * st.cstride + j;
                    const uint32_t v = s_col[warp][c][g];
                    *dst = (j * 32 < lo) ? (*dst | v) : v;
                }
            }
            __syncwarp();
        }
        uint32_t par = 0;
#pragma unroll
        for (int g = 0; g < 8; ++g) {
            const uint32_t b = __ballot_sync(0xFFFFFFFFu, pop[g] & 1);
            if (lane == g) par = b;
        }
        const uint64_t j = j0 + lane;
        if (lane < 8 && j >= w0 && j < w1) {
            uint32_t *dst = st.cols + static_cast<uint64_t>(64 * W) * st.cstride + j;
            *dst = (j * 32 < lo) ? (*dst | par) : par;
        }
    }
}

// Inserts keys [lo, hi) into an empty-initialised table (construction, growth, reset).
template <int W>
__global__ void k_build_table(Store st, Counters *__restrict__ cnt, uint64_t lo, uint64_t hi) {
    for (uint64_t i = lo + blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < hi;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t m[W];
        load_key<W>(st.keys, i, m);
        const uint64_t h = key_hash<W>(m);
        uint64_t pos = h & st.tmask;
        const unsigned long long mine = (static_cast<unsigned long long>(h >> 32) << 32) | i;
        for (uint64_t probes = 0;; ++probes) {
            if (probes > st.tmask) {
                atomicOr(&cnt->err, 4u);
                break;
            }
            const unsigned long long old = atomicCAS(&st.table[pos], kEmptySlot, mine);
            if (old == kEmptySlot) break;
            pos = (pos + 1) & st.tmask;
        }
    }
}

// Store index of each of n query keys (kNoStall when absent): the open-addressing lookup of the resolve,
// for host requests such as re-weighting the initial operator (MPOperator.h:193-232 finds each term of
// the new operator in the store the same way).
template <int W>
__global__ void k_lookup(Store st, const uint64_t *__restrict__ qkeys, uint64_t nq, uint64_t n_live,
                         uint32_t *__restrict__ out, Counters *__restrict__ cnt) {
    for (uint64_t q = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; q < nq;
         q += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t k[W];
        load_key<W>(qkeys, q, k);
        const uint64_t h = key_hash<W>(k);
        const uint32_t tag = static_cast<uint32_t>(h >> 32);
        uint64_t pos = h & st.tmask;
        uint32_t found = kNoStall;
        for (uint64_t probes = 0;; ++probes) {
            if (probes > st.tmask) {
                atomicOr(&cnt->err, 32u);
                break;
            }
            const unsigned long long slot = st.table[pos];
            if (slot == kEmptySlot) break;
            const uint32_t idx = static_cast<uint32_t>(slot);
            if (idx < n_live && static_cast<uint32_t>(slot >> 32) == tag) {
                uint64_t o[W];
                load_key<W>(st.keys, idx, o);
                bool eq = true;
#pragma unroll
                for (int w = 0; w < W; ++w) eq = eq && (o[w] == k[w]);
                if (eq) {
                    found = idx;
                    break;
                }
            }
            pos = (pos + 1) & st.tmask;
        }
        out[q] = found;
    }
}

// Schrodinger picture: <O> = core + sum_t obs_coef[t] * state[idx[t]], the observable dotted into the evolved
// state (MPFunctions.cpp:196-205); idx[t] = kNoStall for a term the state does not hold (contributes 0).
// One block, fixed summation order.
__global__ void __launch_bounds__(kBlock) k_expect_schr(const uint32_t *__restrict__ idx,
                                                         const double *__restrict__ obs_coef, uint64_t n_obs,
                                                         const double *__restrict__ coef, double core,
                                                         double *__restrict__ out) {
    __shared__ double s_red[kBlock / 32];
    double acc = 0.0;
    for (uint64_t t = threadIdx.x; t < n_obs; t += kBlock) {
        const uint32_t j = idx[t];
        if (j != kNoStall) acc += obs_coef[t] * coef[j];
    }
    const double total = block_sum(acc, s_red);
    if (threadIdx.x == 0) out[0] = core + total;
}

// One bit per term (column-word layout): set when the term has more than len_k set slots, i.e. lies
// outside the only_rotate_len_k set of every gate (Scan.h:146-157).
template <int W>
__global__ void k_long_bits(const uint64_t *__restrict__ keys, uint64_t n, uint32_t len_k, uint32_t *__restrict__ out) {
    const uint64_t words = (n + 31) >> 5;
    for (uint64_t base = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) & ~uint64_t(31);
         base < words * 32; base += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t i = base + (threadIdx.x & 31);
        bool is_long = false;
        if (i < n) {
            uint64_t m[W];
            load_key<W>(keys, i, m);
            int pop = 0;
#pragma unroll
            for (int w = 0; w < W; ++w) pop += __popcll(m[w]);
            is_long = pop > static_cast<int>(len_k);
        }
        const uint32_t b = __ballot_sync(0xFFFFFFFFu, is_long);
        if ((threadIdx.x & 31) == 0) out[base >> 5] = b;
    }
}

// coef[idx[k]] = val[k] (indices distinct).
__global__ void k_scatter(double *__restrict__ coef, const uint32_t *__restrict__ idx, const double *__restrict__ val,
                          uint64_t n, uint32_t lo = 0) {
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        if (idx[k] != kNoStall && idx[k] >= lo) coef[idx[k]] = val[k]; // kNoStall: a term the store does not hold
}

// <0|O|0>: per-block partial sums over contiguous chunks, fixed-order tree (MPOperator.h:235-254,
// PauliAlgebra.h:144-147, MajoranaAlgebra.h:56-60).
template <int W, int BASIS>
__global__ void __launch_bounds__(kBlock) k_expect(Store st, const Counters *__restrict__ cnt, StateMask sm,
                                                    double *__restrict__ partial) {
    __shared__ double s_red[kBlock / 32];
    const uint64_t n = cnt->n;
    const uint64_t T = (n + gridDim.x - 1) / gridDim.x;
    const uint64_t begin = static_cast<uint64_t>(blockIdx.x) * T;
    const uint64_t end = min(begin + T, n);
    double acc = 0.0;
    for (uint64_t i = begin + threadIdx.x; i < end; i += kBlock) {
        uint64_t m[W];
        load_key<W>(st.keys, i, m);
        uint64_t unpaired = 0;
        int na = 0, pop = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            unpaired |= (m[w] & kEven) ^ ((m[w] >> 1) & kEven);
            na += __popcll(m[w] & sm.w[w]);
            pop += __popcll(m[w]);
        }
        if (unpaired == 0) {
            const int odd = BASIS == 1 ? (na & 1) : ((na + pop / 2) & 1);
            const double c = st.coef[i];
            acc += odd ? -c : c;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xFFFFFFFFu, acc, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) t += s_red[w];
        partial[blockIdx.x] = t;
    }
}

// core + the block partials, one block: every thread sums a fixed strided subset, then a fixed-order tree.
__global__ void __launch_bounds__(kBlock) k_expect_final(const double *__restrict__ partial, uint32_t nblocks,
                                                          double core, double *__restrict__ out) {
    __shared__ double s_red[kBlock / 32];
    double t = 0.0;
    for (uint32_t b = threadIdx.x; b < nblocks; b += kBlock) t += partial[b];
    const double total = block_sum(t, s_red);
    if (threadIdx.x == 0) out[0] = core + total;
}

} // namespace mpx
