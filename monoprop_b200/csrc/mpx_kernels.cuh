// mpx_kernels.cuh -- the per-gate kernels of the B200 propagation engine (sm_100a).
//
// One Heisenberg gate = two launches over the device term store:
//   k_sweep   -- streams every key once (HBM-bound): anticommutation parity, fused cos scaling of the
//                anticommuting coefficients, lower_atol / structural-cutoff / upper_atol emit gate,
//                rotation phase, leader/follower class; compacts the emitted sine branches into per-block
//                query regions (no global atomics) and writes the leader-emitted bitmap.
//   k_resolve -- one thread per emitted branch: open-addressing lookup of the partner M^G, the
//                leader/follower rule, the rotation of the pair, or the unique append of the missing partner.
// Every coefficient slot is written by exactly one thread per gate (the sine partner map M -> M^G is
// injective), so no coefficient atomics are needed (layer_build/FusedApply.h:54-56).
#pragma once

#include <cstdint>

#include "mpx_device.cuh"

namespace mpx {

__device__ __forceinline__ uint64_t region_size(uint64_t n0, uint32_t grid) {
    const uint64_t per = (n0 + grid - 1) / grid;
    return (per + kBlock - 1) / kBlock * kBlock;
}

// Fused scan + cos sweep + emit (Scan.h:193-396 with the fused sweep of Scan.h:343-358).
template <int W, int BASIS>
__global__ void __launch_bounds__(kBlock) k_sweep(Store st, Scratch sc, Counters *__restrict__ cnt,
                                                   const GateDesc *__restrict__ gates, uint32_t gate, uint32_t step,
                                                   Trunc tr) {
    __shared__ uint32_t warp_tot[kBlock / 32];
    __shared__ uint32_t warp_anti[kBlock / 32];
    if (cnt->stall != kNoStall) return;
    const uint64_t n0 = cnt->n;
    if (2 * n0 > st.cap) {
        // Not enough room for the worst case (every term appends its partner): stop here, untouched,
        // and let the host grow the store and re-issue this step.
        if (threadIdx.x == 0) atomicMin(&cnt->stall, step);
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt->n0 = n0;
    const GateDesc &gd = gates[gate];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    if (gd.empty) {
        if (threadIdx.x == 0) {
            sc.q_count[blockIdx.x] = 0;
            sc.blk_anti[blockIdx.x] = 0;
        }
        return;
    }
    uint64_t g[W], fold[W], pmask[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
        g[w] = gd.g[w];
        fold[w] = gd.fold[w];
        pmask[w] = (w == gd.pivot_word) ? gd.pivot_bit : 0ULL;
    }
    const double cosv = gd.cosv, sinabs = gd.abs_sin;
    const bool cos_zero = gd.cos_zero != 0;
    const int gpop = gd.gpop;

    const uint64_t T = region_size(n0, gridDim.x);
    const uint64_t begin = static_cast<uint64_t>(blockIdx.x) * T;
    const uint64_t end = min(begin + T, n0);
    uint32_t count = 0, anti_total = 0;
    for (uint64_t base = begin; base < end; base += kBlock) {
        const uint64_t i = base + threadIdx.x;
        bool anti = false, emit = false, foll = false;
        int phase = 0;
        double v = 0.0;
        if (i < end) {
            uint64_t m[W];
            load_key<W>(st.keys, i, m);
            uint64_t par = 0, pv = 0;
            int mpop = 0;
#pragma unroll
            for (int w = 0; w < W; ++w) {
                par ^= m[w] & fold[w];
                pv |= m[w] & pmask[w];
                mpop += __popcll(m[w]);
            }
            anti = ((__popcll(par) ^ (gd.g_odd & mpop)) & 1) != 0;
            if (anti) {
                foll = pv != 0;
                v = st.coef[i];
                st.coef[i] = v * cosv;
                if (cos_zero) sc.aux[i] = v;
                const double av = fabs(v);
                if (!(tr.has_lower && sinabs * av <= tr.lower)) {
                    uint64_t p[W];
                    int ov = 0;
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        p[w] = m[w] ^ g[w];
                        ov += __popcll(m[w] & g[w]);
                    }
                    const int ppop = mpop + gpop - 2 * ov;
                    if (keep_partner<W>(p, ppop, tr) || (tr.has_upper && sinabs * av >= tr.upper)) {
                        emit = true;
                        phase = rotation_phase<W, BASIS>(m, p, gd, mpop, ppop);
                    }
                }
            }
        }
        const uint32_t lead_ball = __ballot_sync(0xFFFFFFFFu, emit && !foll);
        const uint32_t emit_ball = __ballot_sync(0xFFFFFFFFu, emit);
        const uint32_t anti_ball = __ballot_sync(0xFFFFFFFFu, anti);
        const uint64_t wbase = base + static_cast<uint64_t>(warp) * 32;
        if (lane == 0) {
            if (wbase < end) sc.emit_bits[wbase >> 5] = lead_ball;
            warp_tot[warp] = __popc(emit_ball);
            warp_anti[warp] = __popc(anti_ball);
        }
        __syncthreads();
        uint32_t off = 0, tot = 0, atot = 0;
#pragma unroll
        for (int w = 0; w < kBlock / 32; ++w) {
            const uint32_t t = warp_tot[w];
            off += (w < warp) ? t : 0u;
            tot += t;
            atot += warp_anti[w];
        }
        if (emit) {
            const uint64_t q = begin + count + off + __popc(emit_ball & lt_mask);
            sc.q_src[q] = static_cast<uint32_t>(i);
            sc.q_flag[q] = static_cast<uint8_t>((foll ? 1 : 0) | (phase_code(phase) << 1));
            sc.q_val[q] = v;
        }
        count += tot;
        anti_total += atot;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        sc.q_count[blockIdx.x] = count;
        sc.blk_anti[blockIdx.x] = anti_total;
    }
}

// Exclusive scan of the per-block query counts into s_off[0..grid] (s_off[grid] = total).
__device__ __forceinline__ void scan_counts(const uint32_t *__restrict__ counts, uint32_t grid, uint64_t *s_off,
                                            uint64_t *s_part) {
    const uint32_t per = (grid + kBlock - 1) / kBlock;
    const uint32_t lo = threadIdx.x * per;
    uint64_t sum = 0;
    for (uint32_t k = 0; k < per; ++k) {
        const uint32_t j = lo + k;
        if (j < grid) sum += counts[j];
    }
    s_part[threadIdx.x] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t acc = 0;
        for (int t = 0; t < kBlock; ++t) {
            const uint64_t x = s_part[t];
            s_part[t] = acc;
            acc += x;
        }
        s_off[grid] = acc;
    }
    __syncthreads();
    uint64_t acc = s_part[threadIdx.x];
    for (uint32_t k = 0; k < per; ++k) {
        const uint32_t j = lo + k;
        if (j < grid) {
            s_off[j] = acc;
            acc += counts[j];
        }
    }
    __syncthreads();
}

constexpr int kMaxGrid = 148 * 8;

// Partner resolve + rotation apply + append (Engine.h:364-513, FusedApply.h:32-83, MPOperator.h:269-278).
template <int W, int BASIS>
__global__ void __launch_bounds__(kBlock) k_resolve(Store st, Scratch sc, Counters *__restrict__ cnt,
                                                     const GateDesc *__restrict__ gates, uint32_t gate, uint32_t step,
                                                     uint64_t *__restrict__ stats) {
    __shared__ uint64_t s_off[kMaxGrid + 1];
    __shared__ uint64_t s_part[kBlock];
    __shared__ uint32_t warp_miss[kBlock / 32];
    __shared__ unsigned long long s_base;
    if (cnt->stall != kNoStall) return;
    const uint64_t n0 = cnt->n0;
    const GateDesc &gd = gates[gate];
    const uint32_t grid = gridDim.x;
    scan_counts(sc.q_count, grid, s_off, s_part);
    const uint64_t total = s_off[grid];
    if (blockIdx.x == 0) {
        if (threadIdx.x == 0) {
            uint64_t a = 0;
            for (uint32_t b = 0; b < grid; ++b) a += sc.blk_anti[b];
            stats[4 * static_cast<uint64_t>(step) + 0] = n0;
            stats[4 * static_cast<uint64_t>(step) + 1] = gd.empty ? 0 : a;
            stats[4 * static_cast<uint64_t>(step) + 2] = total;
        }
    }
    if (total == 0) return;
    const uint64_t T = region_size(n0, grid);
    uint64_t g[W];
#pragma unroll
    for (int w = 0; w < W; ++w) g[w] = gd.g[w];
    const double sinv = gd.sinv, inv_cos = gd.inv_cos;
    const bool cos_zero = gd.cos_zero != 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;

    for (uint64_t tb = static_cast<uint64_t>(blockIdx.x) * kBlock; tb < total;
         tb += static_cast<uint64_t>(grid) * kBlock) {
        const uint64_t k = tb + threadIdx.x;
        bool miss = false;
        uint64_t p[W];
        uint64_t pos = 0;
        uint32_t tag = 0;
        double v = 0.0, ph = 0.0;
        if (k < total) {
            // region r holding global query k: the last r with s_off[r] <= k
            uint32_t lo = 0, hi = grid;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (s_off[mid] <= k) lo = mid;
                else hi = mid;
            }
            const uint64_t q = static_cast<uint64_t>(lo) * T + (k - s_off[lo]);
            const uint32_t src = sc.q_src[q];
            const uint8_t flag = sc.q_flag[q];
            v = sc.q_val[q];
            ph = phase_value(static_cast<uint8_t>(flag >> 1));
            uint64_t m[W];
            load_key<W>(st.keys, src, m);
#pragma unroll
            for (int w = 0; w < W; ++w) p[w] = m[w] ^ g[w];
            const uint64_t h = key_hash<W>(p);
            tag = static_cast<uint32_t>(h >> 32);
            pos = h & st.tmask;
            uint64_t found = ~0ULL;
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
                if (idx < n0 && static_cast<uint32_t>(slot >> 32) == tag) {
                    uint64_t o[W];
                    load_key<W>(st.keys, idx, o);
                    bool eq = true;
#pragma unroll
                    for (int w = 0; w < W; ++w) eq = eq && (o[w] == p[w]);
                    if (eq) {
                        found = idx;
                        break;
                    }
                }
                pos = (pos + 1) & st.tmask;
            }
            if (!miss && !gave_up) {
                const bool follower = (flag & 1) != 0;
                const bool leader_took_it = follower && ((sc.emit_bits[found >> 5] >> (found & 31)) & 1u);
                if (!leader_took_it) {
                    const double vt = cos_zero ? sc.aux[found] : st.coef[found] * inv_cos;
                    st.coef[src] = __fma_rn(sinv * -ph, vt, st.coef[src]);
                    st.coef[found] = __fma_rn(sinv * ph, v, st.coef[found]);
                }
            }
        }
        // Unique appends: one counter bump per block iteration.
        const uint32_t miss_ball = __ballot_sync(0xFFFFFFFFu, miss);
        if (lane == 0) warp_miss[warp] = __popc(miss_ball);
        __syncthreads();
        uint32_t off = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < kBlock / 32; ++w) {
            const uint32_t t = warp_miss[w];
            off += (w < warp) ? t : 0u;
            tot += t;
        }
        if (threadIdx.x == 0 && tot > 0) s_base = atomicAdd(&cnt->n, static_cast<unsigned long long>(tot));
        __syncthreads();
        if (miss) {
            const uint64_t idx = s_base + off + __popc(miss_ball & lt_mask);
            store_key<W>(st.keys, idx, p);
            st.coef[idx] = (sinv * ph) * v;
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
        }
        __syncthreads();
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

__global__ void k_expect_final(const double *__restrict__ partial, uint32_t nblocks, double core,
                               double *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double t = 0.0;
        for (uint32_t b = 0; b < nblocks; ++b) t += partial[b];
        out[0] = core + t;
    }
}

} // namespace mpx
