// mpx_adjoint.cuh -- reverse-mode gradient of <0|O|0> with respect to every gate angle (sm_100a).
//
// The gradient is that of the frozen-structure surrogate the reference differentiates (ev_and_grad,
// MPFunctions.cpp:207-246; state_operator_derivative_local, Evolution.cpp:439-469): every truncation
// decision of the forward pass is kept, and each gate is the linear map A_g(angle) on the coefficient
// vector
//     anticommuting term i without a rotation partner:  c_i' = C c_i
//     rotated pair (S emitter, T partner):             c_S' = C c_S - s phi c_T,  c_T' = C c_T + s phi c_S
//     appended partner T (c_T = 0 before the gate):      c_S' = C c_S,               c_T' = s phi c_S
// with C = cos(2 angle), s = sin(2 angle). With lambda the adjoint (dE/dc after the gate),
//     dE/dangle_g = lambda'^T (dA_g/dangle) c_pre,   lambda_pre = A_g^T lambda'.
//
// Instead of inverting the forward maps (the reference un-scales by 1/cos, CosineRecompute.h:201-224),
// the forward pass saves the coefficient array at segment boundaries; each segment is replayed from its
// checkpoint with the forward kernels in replay mode, which log the pre-gate value of every
// anticommuting term (undo log) and every rotated or appended pair with both pre-gate values (pair log).
// The reverse sweep over that segment then needs no coefficients, no hash lookups and no division.
#pragma once

#include <cstdint>

#include "mpx_device.cuh"

namespace mpx {

// Logs written by a replayed segment. A step's records are contiguous (per-step bases are prefix sums
// of the forward pass's a_g and e_g). Undo records are placed without atomics: the forward pass saves
// every sweep warp's anticommuting count per step (w_anti), a prefix scan turns them into per-warp
// offsets (u_off), and the replayed warp writes its records in its own scan order from there.
struct Tape {
    uint32_t *u_idx; // undo log: anticommuting term index
    double *u_val;   //           its coefficient before the gate
    uint32_t *p_src; // pair log: emitter S
    uint32_t *p_tgt; //           partner T
    int8_t *p_code;  //           phase (+1 / -1 / 0) | 0x10 when T was appended by this gate
    double *p_vs;    //           c_S before the gate
    double *p_vt;    //           c_T before the gate (0 for an append)
    const uint64_t *u_base;    // [n_steps] first undo record of each step
    const uint64_t *p_base;    // [n_steps] first pair record of each step
    unsigned long long *u_cnt; // [n_steps] undo records per step (filled by the offset scan)
    unsigned long long *p_cnt; // [n_steps] pair records written per step
    const uint64_t *n_next;    // [n_steps] store size after each step (from the forward pass)
    uint32_t *w_anti;          // forward pass: [n_steps][sweep warps] anticommuting terms per warp
    const uint64_t *u_off;     // replay: [steps of the segment][sweep warps] first undo record per warp
    uint64_t u_off_step0;      // step of u_off's first row
    // forward pass of a gradient: every rotated or appended pair (src, tgt, phase | appended) in step order,
    // r_begin[step] its first record; records past r_cap are counted but not written
    uint32_t *r_src;
    uint32_t *r_tgt;
    int8_t *r_code;
    uint64_t *r_begin;
    uint64_t r_cap;
    // forward pass of a gradient that logs everything the reverse sweep needs (no segment replay): both
    // pre-gate values of every recorded pair, and the undo log (index, pre-gate value of every
    // anticommuting term, pair members included). Each sweep block reserves its batch's records with one
    // bump of f_utotal; the next gate's resolve stores where the step's records end (f_ubegin[step + 1]).
    // Records past f_ucap are counted but not written (the log is then unusable).
    double *r_vs;
    double *r_vt;
    uint32_t *f_uidx;
    double *f_uval;
    unsigned long long *f_utotal;
    uint64_t *f_ubegin;
    uint64_t f_ucap;
};

// Per step of a segment: exclusive prefix over the sweep warps' anticommuting counts -> undo offsets
// (one block per step, fixed order).
__global__ void __launch_bounds__(1024) k_undo_offsets(Tape tp, uint32_t n_warps, uint64_t step_lo,
                                                        uint64_t *__restrict__ u_off) {
    __shared__ uint64_t s_part[1024];
    const uint64_t step = step_lo + blockIdx.x;
    const uint32_t *src = tp.w_anti + step * n_warps;
    const uint32_t per = (n_warps + blockDim.x - 1) / blockDim.x;
    const uint32_t lo = threadIdx.x * per;
    uint64_t sum = 0;
    for (uint32_t k = 0; k < per && lo + k < n_warps; ++k) sum += src[lo + k];
    s_part[threadIdx.x] = sum;
    __syncthreads();
    for (uint32_t o = 1; o < blockDim.x; o <<= 1) {
        const uint64_t t = threadIdx.x >= o ? s_part[threadIdx.x - o] : 0;
        __syncthreads();
        s_part[threadIdx.x] += t;
        __syncthreads();
    }
    uint64_t acc = tp.u_base[step] + (threadIdx.x > 0 ? s_part[threadIdx.x - 1] : 0);
    uint64_t *dst = u_off + static_cast<uint64_t>(blockIdx.x) * n_warps;
    for (uint32_t k = 0; k < per && lo + k < n_warps; ++k) {
        dst[lo + k] = acc;
        acc += src[lo + k];
    }
    if (threadIdx.x == blockDim.x - 1) tp.u_cnt[step] = s_part[threadIdx.x];
}

__device__ __forceinline__ double block_sum(double v, double *s_red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < static_cast<int>(blockDim.x / 32); ++w) t += s_red[w];
    __syncthreads();
    return t;
}

// After a replayed gate: the store size the forward pass reached after this step (appended partners
// were looked up, not re-inserted).
__global__ void k_replay_advance(Counters *__restrict__ cnt, const uint64_t *__restrict__ n_next, uint32_t step) {
    pdl_trigger();
    pdl_wait();
    if (threadIdx.x == 0 && blockIdx.x == 0 && cnt->stall == kNoStall) cnt->n = n_next[step];
}

// lambda_i = d<0|O|0>/dc_i = state phase of a fully paired term, else 0 (MPOperator.h:235-254).
template <int W, int BASIS>
__global__ void __launch_bounds__(kBlock) k_adj_init(const uint64_t *__restrict__ keys, uint64_t n, StateMask sm,
                                                      double *__restrict__ lam) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t m[W];
        load_key<W>(keys, i, m);
        uint64_t unpaired = 0;
        int na = 0, pop = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            unpaired |= (m[w] & kEven) ^ ((m[w] >> 1) & kEven);
            na += __popcll(m[w] & sm.w[w]);
            pop += __popcll(m[w]);
        }
        double l = 0.0;
        if (unpaired == 0) {
            const int odd = BASIS == 1 ? (na & 1) : ((na + pop / 2) & 1);
            l = odd ? -1.0 : 1.0;
        }
        lam[i] = l;
    }
}

// dE/dangle of one gate is summed in a fixed order, so the gradient's bits do not depend on block
// scheduling: every block of the two reverse-step kernels writes its partial sum to its own slot
// (pairs kernel: slots [0, grid), undo kernel: [grid, 2 grid)), and the last undo block to finish (one
// counter bump per block) adds all 2 grid partials in slot order and writes the gate's derivative.
struct GradPartials {
    double *part;           // [2 * grid]
    unsigned int *arrivals; // undo blocks finished for the current gate; reset to 0 by the last one
};

// Reverse step, part 1: the gate's rotated and appended pairs. Writes lambda of both endpoints, marks
// them in `done` (the undo pass skips them) and stores this block's share of dE/dangle.
__global__ void __launch_bounds__(kBlock) k_adj_pairs(Tape tp, const GateDesc *__restrict__ gates, uint32_t gate,
                                                       uint32_t step, double *__restrict__ lam,
                                                       uint32_t *__restrict__ done, GradPartials gp) {
    __shared__ double s_red[kBlock / 32];
    pdl_trigger();
    pdl_wait();
    const uint64_t base = tp.p_base[step];
    const uint64_t cnt = tp.p_cnt[step];
    if (cnt == 0) {
        if (threadIdx.x == 0) gp.part[blockIdx.x] = 0.0;
        return;
    }
    const GateDesc &gd = gates[gate];
    const double C = gd.cosv, S = gd.sinv;
    double acc = 0.0;
    for (uint64_t tb = blockIdx.x * static_cast<uint64_t>(kBlock); tb < cnt; tb += static_cast<uint64_t>(gridDim.x) * kBlock) {
        const uint64_t k = tb + threadIdx.x;
        if (k < cnt) {
            const uint64_t r = base + k;
            const uint32_t s = tp.p_src[r], t = tp.p_tgt[r];
            const int8_t code = tp.p_code[r];
            const bool appended = (code & 0x10) != 0;
            const double phi = static_cast<double>(static_cast<int8_t>(code << 4) >> 4);
            const double vs = tp.p_vs[r], vt = tp.p_vt[r];
            const double ls = lam[s], lt = lam[t];
            if (code & 0x20) {
                // partner outside the only_rotate_len_k set: c_T' = c_T + s phi c_S (no cos factor), so
                // d(c_T')/dangle = 2 C phi v_S and lambda_T = lambda_T' - s phi lambda_S'; T is not in the
                // undo log (it is not scaled by this gate), so it takes no done bit
                acc += ls * (-2.0 * S * vs - 2.0 * C * phi * vt) + lt * (2.0 * C * phi * vs);
                lam[s] = C * ls + S * phi * lt;
                lam[t] = lt - S * phi * ls;
                atomicOr(&done[s >> 5], 1u << (s & 31));
                continue;
            }
            // d(c_S')/dangle = -2 s v_S - 2 C phi v_T;  d(c_T')/dangle = -2 s v_T + 2 C phi v_S
            acc += ls * (-2.0 * S * vs - 2.0 * C * phi * vt) + lt * (-2.0 * S * vt + 2.0 * C * phi * vs);
            lam[s] = C * ls + S * phi * lt;
            atomicOr(&done[s >> 5], 1u << (s & 31));
            if (!appended) {
                lam[t] = C * lt - S * phi * ls;
                atomicOr(&done[t >> 5], 1u << (t & 31));
            }
        }
    }
    const double t = block_sum(acc, s_red);
    if (threadIdx.x == 0) gp.part[blockIdx.x] = t;
}

// Reverse step, part 2: every anticommuting term of the gate. Terms not in a pair were only cos-scaled:
// dE/dangle += lambda' (-2 s c_pre), lambda = C lambda'. Pair members were handled by part 1; their
// done bit is cleared here (each appears once in the undo log), so `done` is all zero between gates.
// The last block to finish writes grad[gate], the fixed-order sum of both kernels' partials.
__global__ void __launch_bounds__(kBlock) k_adj_undo(Tape tp, const GateDesc *__restrict__ gates, uint32_t gate,
                                                      uint32_t step, double *__restrict__ lam,
                                                      uint32_t *__restrict__ done, GradPartials gp,
                                                      double *__restrict__ grad) {
    __shared__ double s_red[kBlock / 32];
    __shared__ bool s_last;
    pdl_trigger();
    pdl_wait();
    const uint64_t base = tp.u_base[step];
    const uint64_t cnt = tp.u_cnt[step];
    const GateDesc &gd = gates[gate];
    const double C = gd.cosv, S = gd.sinv;
    double acc = 0.0;
    for (uint64_t tb = blockIdx.x * static_cast<uint64_t>(kBlock); tb < cnt; tb += static_cast<uint64_t>(gridDim.x) * kBlock) {
        const uint64_t k = tb + threadIdx.x;
        if (k < cnt) {
            const uint64_t r = base + k;
            const uint32_t i = tp.u_idx[r];
            const uint32_t bit = 1u << (i & 31);
            if (i == kNoStall) {
                // an anticommuting term outside the only_rotate_len_k set: untouched by the gate
            }
            else if (done[i >> 5] & bit) {
                atomicAnd(&done[i >> 5], ~bit);
            }
            else {
                const double l = lam[i];
                acc += l * (-2.0 * S * tp.u_val[r]);
                lam[i] = C * l;
            }
        }
    }
    const double t = block_sum(acc, s_red);
    if (threadIdx.x == 0) {
        gp.part[gridDim.x + blockIdx.x] = t;
        __threadfence();
        s_last = atomicAdd(gp.arrivals, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    // every partial of this gate is written and visible (each writer fenced before its arrival)
    __threadfence();
    double v = 0.0;
    for (uint32_t k = threadIdx.x; k < 2 * gridDim.x; k += blockDim.x) v += __ldcg(gp.part + k);
    const double total = block_sum(v, s_red);
    if (threadIdx.x == 0) {
        grad[gate] = total;
        *gp.arrivals = 0u;
    }
}

// One reverse step as a single launch, for segments replayed with the frozen kernels: their undo log marks
// pair members with the skip index, so the pair records and the undo entries touch disjoint adjoint
// entries and need no done bits. The step's work is the pair records followed by the undo entries, dealt
// grid-stride over all blocks; each block's share of dE/dangle goes to its slot, and the last block to
// finish writes grad[gate] as the fixed-order sum of the slots (the same arithmetic per record as
// k_adj_pairs and k_adj_undo).
__global__ void __launch_bounds__(kBlock) k_adj_step(Tape tp, const GateDesc *__restrict__ gates, uint32_t gate,
                                                      uint32_t step, double *__restrict__ lam, GradPartials gp,
                                                      double *__restrict__ grad) {
    __shared__ double s_red[kBlock / 32];
    __shared__ bool s_last;
    pdl_trigger();
    pdl_wait();
    const uint64_t pbase = tp.p_base[step], pcnt = tp.p_cnt[step];
    const uint64_t ubase = tp.u_base[step], ucnt = tp.u_cnt[step];
    const uint64_t total = pcnt + ucnt;
    const GateDesc &gd = gates[gate];
    const double C = gd.cosv, S = gd.sinv;
    double acc = 0.0;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(kBlock) + threadIdx.x; k < total;
         k += static_cast<uint64_t>(gridDim.x) * kBlock) {
        if (k < pcnt) {
            const uint64_t r = pbase + k;
            const uint32_t s = tp.p_src[r], t = tp.p_tgt[r];
            const int8_t code = tp.p_code[r];
            const double phi = static_cast<double>(static_cast<int8_t>(code << 4) >> 4);
            const double vs = tp.p_vs[r], vt = tp.p_vt[r];
            const double ls = lam[s], lt = lam[t];
            if (code & 0x20) { // partner outside the only_rotate_len_k set: c_T' = c_T + s phi c_S
                acc += ls * (-2.0 * S * vs - 2.0 * C * phi * vt) + lt * (2.0 * C * phi * vs);
                lam[s] = C * ls + S * phi * lt;
                lam[t] = lt - S * phi * ls;
            }
            else {
                acc += ls * (-2.0 * S * vs - 2.0 * C * phi * vt) + lt * (-2.0 * S * vt + 2.0 * C * phi * vs);
                lam[s] = C * ls + S * phi * lt;
                if ((code & 0x10) == 0) lam[t] = C * lt - S * phi * ls;
            }
        }
        else {
            const uint64_t r = ubase + (k - pcnt);
            const uint32_t i = tp.u_idx[r];
            if (i != kNoStall) {
                const double l = lam[i];
                acc += l * (-2.0 * S * tp.u_val[r]);
                lam[i] = C * l;
            }
        }
    }
    const double t = block_sum(acc, s_red);
    if (threadIdx.x == 0) {
        gp.part[blockIdx.x] = t;
        __threadfence();
        s_last = atomicAdd(gp.arrivals, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double v = 0.0;
    for (uint32_t k = threadIdx.x; k < gridDim.x; k += blockDim.x) v += __ldcg(gp.part + k);
    const double sum = block_sum(v, s_red);
    if (threadIdx.x == 0) {
        grad[gate] = sum;
        *gp.arrivals = 0u;
    }
}

}  // namespace mpx

namespace mpx {

// ----- frozen structure ("graph") evaluation ------------------------------------------------------------
//
// The reference's variational loop builds a surrogate graph once and replays it at new parameters
// (MonomialPropagator.inl:620-690, Evolution.cpp:471-540): every truncation decision of the build is
// kept. Here the build's rotated and appended pairs of every gate are kept (src, tgt, phase | appended),
// and the anticommuting sets are recomputed from the bit-columns (they depend only on the keys). One
// gate at new angles is then two launches: the pairs (exact 2x2 rotations of their pre-gate values) and
// the cos scaling of every other anticommuting term.
struct Frozen {
    const uint32_t *src;
    const uint32_t *tgt;
    const int8_t *code;                  // phase (+1 / -1 / 0) | 0x10 for an appended partner
    const uint64_t *p_begin;             // [n_steps] first pair of each step
    const unsigned long long *p_count;   // [n_steps] pairs of each step
    // Paring (PareGraph.cpp:103-141): last[i] = the last step after which term i can still reach <0|O|0>
    // (-1: never); a step skips the cos scaling of a term with last < step and the rotation of a pair with
    // both endpoints below it. nullptr: no paring.
    const int32_t *last;
    // only_rotate_len_k of a recorded propagation: one bit per term of more than k slots (never cos-scaled,
    // and a pair's partner among them keeps no cos factor, code 0x20); nullptr: every anticommuting term is
    // scaled and 0x20 is ignored (a built graph, as the reference replays it)
    const uint32_t *longb;
};

// ----- paring ---------------------------------------------------------------------------------------------
//
// The reference pares a graph against the reference state (pare_graph, PareGraph.cpp:103-141, keep set
// state.indices_above(threshold), MonomialPropagator.inl:950-960): walking the layers backward, a term is
// kept while its value can still flow into a kept term, and the cos scaling of every other term is skipped.
// The value of <0|O|0> (and its gradient) is unchanged: only terms that can never reach a scored term lose
// their scaling. Relevance only grows toward earlier steps (a pair with one relevant endpoint makes both
// relevant before the gate; a cos-only term keeps its status), so one int per term says up to which step
// the term matters.

// last[i] = n_steps - 1 where term i's reference-state weight exceeds the threshold (|weight| = 1 on a fully
// paired term, 0 elsewhere: indices_above, MPFunctions.cpp:96-105), else -1.
template <int W>
__global__ void __launch_bounds__(kBlock) k_pare_init(const uint64_t *__restrict__ keys, uint64_t n, int32_t keep_paired,
                                                       int32_t last_step, int32_t *__restrict__ last) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t m[W];
        load_key<W>(keys, i, m);
        uint64_t unpaired = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) unpaired |= (m[w] & kEven) ^ ((m[w] >> 1) & kEven);
        last[i] = (unpaired == 0 && keep_paired) ? last_step : -1;
    }
}

// Schrodinger picture: the kept terms after the last step are the observable's terms whose |coefficient|
// exceeds the threshold (indices_above on the driving vector, MonomialPropagator.inl:960-962); `last` is
// -1 everywhere else. idx[t] = kNoStall for an observable term the store does not hold.
__global__ void k_pare_seed(const uint32_t *__restrict__ idx, const double *__restrict__ val, uint64_t n,
                            double threshold, int32_t last_step, int32_t *__restrict__ last) {
    for (uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; t < n;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        if (idx[t] != kNoStall && fabs(val[t]) > threshold) last[idx[t]] = last_step;
}

// One step, backward: a pair with an endpoint still relevant after the step makes both endpoints relevant
// before it. The pairs of one step are disjoint, so no two threads touch the same term.
__global__ void __launch_bounds__(kBlock) k_pare_step(Frozen fz, uint32_t step, int32_t *__restrict__ last) {
    const uint64_t b = fz.p_begin[step], cnt = fz.p_count[step];
    const int32_t st = static_cast<int32_t>(step);
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < cnt;
         k += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t s = fz.src[b + k], t = fz.tgt[b + k];
        const int32_t ls = last[s], lt = last[t];
        if (ls >= st || lt >= st) {
            if (ls < st - 1) last[s] = st - 1;
            if (lt < st - 1) last[t] = st - 1;
        }
    }
}

// Pairs of one frozen gate; with LOG also their pre-gate values into the tape's pair log (the slot of
// pair k is p_base[step] + k, so no counters are needed).
template <bool LOG>
__global__ void __launch_bounds__(kBlock) k_frozen_pairs(double *__restrict__ coef, Frozen fz,
                                                          const GateDesc *__restrict__ gates, uint32_t gate,
                                                          uint32_t step, uint32_t *__restrict__ done, Tape tp) {
    pdl_trigger();
    pdl_wait();
    const uint64_t b = fz.p_begin[step], cnt = fz.p_count[step];
    const GateDesc &gd = gates[gate];
    const double C = gd.cosv, S = gd.sinv;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < cnt;
         k += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t s = fz.src[b + k], t = fz.tgt[b + k];
        const int8_t code = fz.code[b + k];
        const bool appended = (code & 0x10) != 0;
        const double phi = static_cast<double>(static_cast<int8_t>(code << 4) >> 4);
        // An appended partner's slot still holds the value the replay started it from (no earlier gate
        // reaches a term created later): 0 in the Heisenberg picture, the reference-state score in the
        // Schrodinger picture. The reference's replay scales it by cos like every anticommuting term below
        // the post-insert count and adds the sine term (Evolution.cpp:471-511, Engine.h:628-633).
        const double vs = coef[s], vt = coef[t];
        const bool pared = fz.last != nullptr && fz.last[s] < static_cast<int32_t>(step) &&
                           fz.last[t] < static_cast<int32_t>(step);
        // partner outside the only_rotate_len_k set: unscaled in the adjoint of a propagation (longb given);
        // a built graph scales it as any anticommuting term
        const bool unscaled_t = (code & 0x20) != 0 && fz.longb != nullptr;
        if (!pared) {
            coef[s] = C * vs - S * phi * vt;
            coef[t] = (unscaled_t ? vt : C * vt) + S * phi * vs;
        }
        atomicOr(&done[s >> 5], 1u << (s & 31));
        if (!appended && !unscaled_t) atomicOr(&done[t >> 5], 1u << (t & 31));
        if constexpr (LOG) {
            const uint64_t r = tp.p_base[step] + k;
            tp.p_src[r] = s;
            tp.p_tgt[r] = t;
            tp.p_code[r] = unscaled_t ? code : static_cast<int8_t>(code & ~0x20);
            tp.p_vs[r] = vs;
            tp.p_vt[r] = vt;
        }
    }
}

// k_frozen_scan, the other half of a frozen gate, shares the sweep's chunk dealing (mpx_kernels.cuh).

}  // namespace mpx
