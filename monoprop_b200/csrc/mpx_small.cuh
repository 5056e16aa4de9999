// mpx_small.cuh -- the whole gate loop of a small store in one thread block (sm_100a).
//
// While the store is small (thousands of terms) a gate is a few microseconds of work, and the two
// launches per gate of the streaming path cost more than the work. Here one 1024-thread block keeps
// the store -- keys, coefficients, a hash table of 16-bit term indices, the query list -- in shared
// memory (up to 227 KB) and applies a whole range of gates with block barriers between the phases of
// each gate. The semantics are the streaming path's (Scan.h:193-396, Engine.h:364-513,
// FusedApply.h:32-83): cos-scale every anticommuting term, emit through the lower_atol gate, structural
// cutoff and upper_atol rescue, resolve leaders before followers, append missing partners.
//
// A gate whose appends could exceed the shared capacity is not started: the block writes the store
// back, records the step as the stall point and returns; the host rebuilds the global hash table and
// bit-columns and continues with the streaming kernels from that gate.
#pragma once

#include <cstdint>

#include "mpx_device.cuh"

namespace mpx {

constexpr int kSmallThreads = 1024;
constexpr uint16_t kSmallEmpty = 0xFFFF;

// Shared-memory bytes for capacity `cap` (a multiple of 32) and a table of 2^tbits slots.
__host__ __device__ inline size_t small_smem_bytes(int W, uint32_t cap, uint32_t tbits) {
    return static_cast<size_t>(cap) * (8 * W + 8)         // keys, coefficients
           + static_cast<size_t>(cap / 2) * (8 + 4)        // query values, query sources
           + (static_cast<size_t>(1) << tbits) * 2         // hash table
           + static_cast<size_t>(cap / 32) * 4;            // leader-emitted bitmap
}

// Inserts term i into the shared table. The capacity keeps the load at or below 1/2, so a full table
// means the store is inconsistent: the error flag is set (as the streaming kernels do) instead of
// dropping the term silently.
template <int W>
__device__ __forceinline__ void small_insert(uint16_t *table, uint32_t tmask, const uint64_t *keys, uint32_t i,
                                             Counters *__restrict__ cnt) {
    uint64_t k[W];
#pragma unroll
    for (int w = 0; w < W; ++w) k[w] = keys[i * W + w];
    uint32_t pos = static_cast<uint32_t>(key_hash<W>(k)) & tmask;
    for (uint32_t probes = 0; probes <= tmask; ++probes) {
        if (atomicCAS(&table[pos], kSmallEmpty, static_cast<uint16_t>(i)) == kSmallEmpty) return;
        pos = (pos + 1) & tmask;
    }
    atomicOr(&cnt->err, 16u);
}

template <int W, int BASIS>
__global__ void __launch_bounds__(kSmallThreads, 1)
    k_small(Store st, Counters *__restrict__ cnt, const GateDesc *__restrict__ gates, uint32_t L, uint32_t lo,
            uint32_t hi, Trunc tr, uint64_t *__restrict__ stats, uint32_t cap, uint32_t tbits) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint64_t *keys = reinterpret_cast<uint64_t *>(smem);
    double *coef = reinterpret_cast<double *>(keys + static_cast<size_t>(cap) * W);
    double *qv = coef + cap;
    uint32_t *qs = reinterpret_cast<uint32_t *>(qv + cap / 2);
    uint16_t *table = reinterpret_cast<uint16_t *>(qs + cap / 2);
    const uint32_t tmask = (1u << tbits) - 1u;
    uint32_t *emitb = reinterpret_cast<uint32_t *>(table + (1u << tbits));
    __shared__ uint32_t s_n, s_q, s_anti, s_stall;
    const uint32_t tid = threadIdx.x;
    const int lane = tid & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;

    if (cnt->stall != kNoStall) return;
    const uint32_t n_in = static_cast<uint32_t>(cnt->n);
    if (tid == 0) {
        s_n = n_in;
        s_stall = kNoStall;
    }
    for (uint32_t i = tid; i < n_in * W; i += kSmallThreads) keys[i] = st.keys[i];
    for (uint32_t i = tid; i < n_in; i += kSmallThreads) coef[i] = st.coef[i];
    for (uint32_t i = tid; i <= tmask; i += kSmallThreads) table[i] = kSmallEmpty;
    __syncthreads();
    for (uint32_t i = tid; i < n_in; i += kSmallThreads) small_insert<W>(table, tmask, keys, i, cnt);
    __syncthreads();

    for (uint32_t step = lo; step < hi; ++step) {
        const GateDesc &gd = gates[L - 1 - step];
        const uint32_t n0 = s_n;
        for (uint32_t j = tid; j < (n0 + 31) / 32; j += kSmallThreads) emitb[j] = 0;
        if (tid == 0) {
            s_q = 0;
            s_anti = 0;
        }
        __syncthreads();
        const double cosv = gd.cosv, sinabs = gd.abs_sin, sinv = gd.sinv, inv_cos = gd.inv_cos;
        // pass 1: anticommutation, emit decisions, query list (coefficients untouched)
        uint32_t my_anti = 0;
        if (!gd.empty) {
            for (uint32_t base = 0; base < n0; base += kSmallThreads) {
                const uint32_t i = base + tid;
                bool emit = false, foll = false;
                int phase = 0;
                double v = 0.0;
                if (i < n0) {
                    uint64_t m[W];
#pragma unroll
                    for (int w = 0; w < W; ++w) m[w] = keys[i * W + w];
                    int mpop = 0;
                    if (anticommutes<W>(m, gd, mpop)) {
                        ++my_anti;
                        foll = (m[gd.pivot_word] & gd.pivot_bit) != 0;
                        v = coef[i];
                        const double av = fabs(v);
                        if (!(tr.has_lower && sinabs * av <= tr.lower)) {
                            uint64_t p[W];
                            int ov = 0;
#pragma unroll
                            for (int w = 0; w < W; ++w) {
                                p[w] = m[w] ^ gd.g[w];
                                ov += __popcll(m[w] & gd.g[w]);
                            }
                            const int ppop = mpop + gd.gpop - 2 * ov;
                            if (keep_partner<W>(p, ppop, tr) || (tr.has_upper && sinabs * av >= tr.upper)) {
                                emit = true;
                                phase = rotation_phase<W, BASIS>(m, p, gd, mpop, ppop);
                            }
                        }
                    }
                }
                const uint32_t eb = __ballot_sync(0xFFFFFFFFu, emit);
                uint32_t qb = 0;
                if (lane == 0 && eb) qb = atomicAdd(&s_q, static_cast<uint32_t>(__popc(eb)));
                qb = __shfl_sync(0xFFFFFFFFu, qb, 0);
                if (emit) {
                    const uint32_t q = qb + __popc(eb & lt_mask);
                    qs[q] = i | (foll ? 0x80000000u : 0u) | (static_cast<uint32_t>(phase_code(phase)) << 29);
                    qv[q] = v;
                    if (!foll) atomicOr(&emitb[i >> 5], 1u << (i & 31));
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) my_anti += __shfl_down_sync(0xFFFFFFFFu, my_anti, o);
        if (lane == 0 && my_anti) atomicAdd(&s_anti, my_anti);
        __syncthreads();
        const uint32_t nq = s_q;
        if (n0 + nq > cap) { // the appends might not fit: stop before touching this gate
            if (tid == 0) s_stall = step;
            break;
        }
        // pass 2: cos-scale every anticommuting term
        if (!gd.empty) {
            for (uint32_t i = tid; i < n0; i += kSmallThreads) {
                uint64_t m[W];
#pragma unroll
                for (int w = 0; w < W; ++w) m[w] = keys[i * W + w];
                int mpop = 0;
                if (anticommutes<W>(m, gd, mpop)) coef[i] = coef[i] * cosv;
            }
        }
        __syncthreads();
        // resolve: partner lookup, leader/follower rule, rotation or append
        for (uint32_t q = tid; q < nq; q += kSmallThreads) {
            const uint32_t code = qs[q];
            const uint32_t src = code & 0x1FFFFFFFu;
            const bool follower = (code & 0x80000000u) != 0;
            const double ph = phase_value(static_cast<uint8_t>((code >> 29) & 3u));
            const double v = qv[q];
            uint64_t p[W];
#pragma unroll
            for (int w = 0; w < W; ++w) p[w] = keys[src * W + w] ^ gd.g[w];
            uint32_t pos = static_cast<uint32_t>(key_hash<W>(p)) & tmask;
            uint32_t found = kNoStall;
            bool ended = false;
            for (uint32_t probes = 0; probes <= tmask; ++probes) {
                const uint16_t t = table[pos];
                if (t == kSmallEmpty) {
                    ended = true;
                    break;
                }
                if (t < n0) {
                    bool eq = true;
#pragma unroll
                    for (int w = 0; w < W; ++w) eq = eq && keys[t * W + w] == p[w];
                    if (eq) {
                        found = t;
                        ended = true;
                        break;
                    }
                }
                pos = (pos + 1) & tmask;
            }
            if (!ended) { // every slot probed without an end: the table is inconsistent
                atomicOr(&cnt->err, 16u);
            }
            else if (found != kNoStall) {
                const bool leader_took_it = follower && ((emitb[found >> 5] >> (found & 31)) & 1u);
                if (!leader_took_it) {
                    const double vt = coef[found] * inv_cos;
                    coef[src] = __fma_rn(sinv * -ph, vt, coef[src]);
                    coef[found] = __fma_rn(sinv * ph, v, coef[found]);
                }
            }
            else {
                const uint32_t idx = atomicAdd(&s_n, 1u);
#pragma unroll
                for (int w = 0; w < W; ++w) keys[idx * W + w] = p[w];
                if (tr.schr) { // Schrodinger: the new slot starts from its reference-state score
                    const double vt0 = state_score<W, BASIS>(p, tr.occ);
                    coef[src] = __fma_rn(sinv * -ph, vt0, coef[src]);
                    coef[idx] = __fma_rn(cosv, vt0, (sinv * ph) * v);
                }
                else {
                    coef[idx] = (sinv * ph) * v;
                }
                small_insert<W>(table, tmask, keys, idx, cnt);
            }
        }
        if (tid == 0) {
            stats[4 * static_cast<uint64_t>(step) + 0] = n0;
            stats[4 * static_cast<uint64_t>(step) + 1] = gd.empty ? 0 : s_anti;
            stats[4 * static_cast<uint64_t>(step) + 2] = nq;
        }
        __syncthreads();
    }
    __syncthreads();
    const uint32_t n = s_n;
    for (uint32_t i = tid; i < n * W; i += kSmallThreads) st.keys[i] = keys[i];
    for (uint32_t i = tid; i < n; i += kSmallThreads) st.coef[i] = coef[i];
    if (tid == 0) {
        cnt->n = n;
        cnt->n0 = n;
        cnt->stall = s_stall;
    }
}

}  // namespace mpx
