// mpx_device.cuh -- device-side algebra and data layout of the B200 propagation engine.
//
// A term store is a structure of arrays in HBM: keys [cap][W] uint64 (row-major, one 8W-byte row per
// term, so a warp streaming 32 consecutive terms reads one contiguous 256W-byte span), coefficients
// [cap] fp64, and an open-addressing hash table of 64-bit slots (hash tag << 32 | term index).
// Nothing is ever deleted (the reference store is append-only: MPOperator.h:266-278).
#pragma once

#include <cstdint>

namespace mpx {

constexpr int kMaxWords = 8;
constexpr uint64_t kEven = 0x5555555555555555ULL;
constexpr unsigned long long kEmptySlot = ~0ULL;
constexpr uint32_t kNoStall = 0xFFFFFFFFu;
constexpr int kBlock = 256;
constexpr int kMaxFoldCols = 8; // fold columns read with independent loads; wider generators loop

// Per-gate constants, precomputed on the host once per circuit (cos/sin through the host libm, the
// same calls the reference makes: layer_build/Engine.h:555-560, FusedApply.h:45-46).
struct GateDesc {
    uint64_t g[kMaxWords];     // generator key G
    uint64_t fold[kMaxWords];  // anticommutation fold: Pauli pair_swap(G), Majorana G
    uint64_t wmask[kMaxWords]; // Majorana interleave mask: bit c set iff #G bits above c is odd
    double cosv, sinv, abs_sin, inv_cos;
    int32_t gpop, gy, g_odd, pivot_word;
    uint64_t pivot_bit;
    int32_t cos_zero, empty;
    int32_t pivot_col; // physical bit index of the pivot: 64 * pivot_word + ctz(pivot_bit)
    int32_t n_fold;    // number of fold columns (set bits of fold)
    uint16_t fold_cols[kMaxFoldCols]; // their physical bit indices, when n_fold <= kMaxFoldCols
};

struct StateMask {
    uint64_t w[kMaxWords]; // slot 2m set for every occupied mode m of the reference state
};

// Engine-wide truncation settings (CutoffContext.h:20-42, AlgebraCommon.h:229-243).
struct Trunc {
    int32_t cutoff_type; // 0 length, 1 support
    uint32_t cutoff;
    int32_t has_lower, has_upper;
    double lower, upper;
    // only_rotate_len_k: terms with more than len_k set slots take no part in a gate (Scan.h:146-157)
    int32_t has_len_k;
    uint32_t len_k;
    // basis_change (Majorana): [2T][W] device rows by slot; the partner's cutoff is judged on its image
    const uint64_t *basis_rows;
    // Schrodinger picture: an appended partner starts from its reference-state score over `occ`
    // (FusedApply.h:39-83) instead of 0
    int32_t schr;
    StateMask occ;
};

// Programmatic dependent launch (sm_90+): the per-gate kernels let the next kernel of the stream be
// scheduled as soon as they start, and that kernel reads only constant circuit data until it waits for
// the previous grid's completion (and memory) with griddepcontrol.wait. Launched without the attribute,
// the wait returns at once.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Device counters, one set per engine.
struct Counters {
    unsigned long long n; // live term count (grows during the resolve kernel)
    unsigned long long n0; // term count at the start of the current gate
    uint32_t stall;        // kNoStall, or the step index at which capacity ran out
    uint32_t err;          // nonzero: a bounded probe loop gave up (table inconsistent); results invalid
    unsigned long long rec_total; // pair records written by a recording forward pass (may exceed capacity)
};

// The key store is kept twice: as rows (keys, for the per-term work) and as bit-columns (cols, for the
// anticommutation test). Column c (physical key bit c, c < 64W; c = 64W is the parity of |M|) is a
// bitmap over terms: word j holds terms 32j .. 32j+31, bit (i & 31) for term i. The bits of a column
// word beyond the live term count are zero.
struct Store {
    uint64_t *keys;
    double *coef;
    unsigned long long *table;
    uint32_t *cols;   // [64W + 1][cstride]
    uint64_t cstride; // 32-bit words per column
    uint64_t tmask;   // table capacity - 1 (power of two)
    uint64_t cap;     // term capacity
};

// Emitted sine branches of the current gate. Block b of the sweep grid owns the query region
// [b * warps * stride, b * warps * stride + blk_q[b]), stride = (chunks per warp) * 1024, at least the
// terms its warps scan, so blocks never contend for a slot or a counter; the resolve block b takes
// the region of the sweep block b.
struct Scratch {
    uint32_t *q_src;     // source term index
    uint8_t *q_flag;     // bit0 follower, bits1-2 phase code (0:+1, 1:-1, 2:0)
    double *q_val;       // pre-gate source coefficient v_src
    uint32_t *blk_q;     // [grid] queries per sweep block
    uint32_t *emit_bits; // leader-emitted flags, one bit per term (column-word layout)
    double *aux;         // pre-gate coefficients, used only for cos == 0 gates
    uint64_t q_cap;      // size of the query arrays
};

__host__ __device__ inline uint64_t mix64(uint64_t x) {
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebULL;
    x ^= x >> 31;
    return x;
}

template <int W>
__device__ __forceinline__ uint64_t key_hash(const uint64_t (&k)[W]) {
    uint64_t h = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) h ^= mix64(k[w] + static_cast<uint64_t>(w));
    return h;
}

template <int W>
__device__ __forceinline__ void load_key(const uint64_t *__restrict__ keys, uint64_t i, uint64_t (&k)[W]) {
    const uint64_t *p = keys + i * W;
    if constexpr (W % 2 == 0) {
#pragma unroll
        for (int w = 0; w < W; w += 2) {
            const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(p + w);
            k[w] = v.x;
            k[w + 1] = v.y;
        }
    }
    else {
#pragma unroll
        for (int w = 0; w < W; ++w) k[w] = p[w];
    }
}

template <int W>
__device__ __forceinline__ void store_key(uint64_t *__restrict__ keys, uint64_t i, const uint64_t (&k)[W]) {
    uint64_t *p = keys + i * W;
    if constexpr (W % 2 == 0) {
#pragma unroll
        for (int w = 0; w < W; w += 2) *reinterpret_cast<ulonglong2 *>(p + w) = make_ulonglong2(k[w], k[w + 1]);
    }
    else {
#pragma unroll
        for (int w = 0; w < W; ++w) p[w] = k[w];
    }
}

__device__ __forceinline__ int nc2(int n) { return (n * (n - 1)) >> 1; }

// Anticommutation of M with the gate: Pauli parity(M & pair_swap(G)) (PauliAlgebra.h:80-83);
// Majorana parity(M & G) ^ (|G| odd & |M| odd) (Scan.h:221-237).
template <int W>
__device__ __forceinline__ bool anticommutes(const uint64_t (&m)[W], const GateDesc &gd, int &mpop) {
    uint64_t par = 0;
    int pop = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        par ^= m[w] & gd.fold[w];
        pop += __popcll(m[w]);
    }
    mpop = pop;
    int bit = __popcll(par) & 1;
    bit ^= gd.g_odd & pop & 1;
    return bit != 0;
}

// Structural keep test on the partner P (AlgebraCommon.h:131-176, CutoffEvaluator::passes_with_popcount).
template <int W>
__device__ __forceinline__ bool keep_partner(const uint64_t (&p)[W], int ppop, const Trunc &tr) {
    if (ppop <= static_cast<int>(tr.cutoff)) return true;
    int xs = 0, os = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        const uint64_t a = p[w] & kEven, b = (p[w] >> 1) & kEven;
        xs += __popcll(a ^ b);
        os += __popcll(a | b);
    }
    if (xs == 0) return true; // fully paired terms are always kept
    const int measure = tr.cutoff_type == 1 ? os : ppop;
    return measure <= static_cast<int>(tr.cutoff);
}

// Structural keep test under basis_change (MonomialPropagatorCommon.h:44-62, change_basis
// MajoranaAlgebra.h:179-189): the image XOR_{slot s in P} row_s is judged by the cutoff, with no popcount
// shortcut (the reference's evaluator falls through to the stored function, AlgebraCommon.h:229-243).
template <int W>
__device__ __forceinline__ bool keep_partner_mapped(const uint64_t (&p)[W], const Trunc &tr) {
    uint64_t q[W];
#pragma unroll
    for (int w = 0; w < W; ++w) q[w] = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        for (uint64_t x = p[w]; x != 0; x &= x - 1) {
            const int slot = 64 * W - 1 - (64 * w + __ffsll(static_cast<long long>(x)) - 1);
            const uint64_t *row = tr.basis_rows + static_cast<uint64_t>(slot) * W;
#pragma unroll
            for (int v = 0; v < W; ++v) q[v] ^= __ldg(row + v);
        }
    }
    int xs = 0, os = 0, pop = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        const uint64_t a = q[w] & kEven, b = (q[w] >> 1) & kEven;
        xs += __popcll(a ^ b);
        os += __popcll(a | b);
        pop += __popcll(q[w]);
    }
    if (xs == 0) return true;
    return (tr.cutoff_type == 1 ? os : pop) <= static_cast<int>(tr.cutoff);
}

// Rotation phase of the sine branch M -> M^G.
// Pauli: e = y(G) + y(M) - y(P) + 2 popcount(z(M) & x(G)); phase = -1 iff e mod 4 == 1 (PauliAlgebra.h:121-140).
// Majorana: (-1)^parity(M & wmask) * {1,0,-1,0}[(C(|M|,2)+C(|G|,2)-C(|P|,2)+3) mod 4] (MajoranaAlgebra.h:104-122).
template <int W, int BASIS>
__device__ __forceinline__ int rotation_phase(const uint64_t (&m)[W], const uint64_t (&p)[W], const GateDesc &gd, int mpop,
                                              int ppop) {
    if constexpr (BASIS == 1) {
        int e = gd.gy;
        int cross = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const uint64_t vm = m[w] & kEven, um = (m[w] >> 1) & kEven;
            const uint64_t vn = p[w] & kEven, un = (p[w] >> 1) & kEven;
            const uint64_t vg = gd.g[w] & kEven, ug = (gd.g[w] >> 1) & kEven;
            e += __popcll(vm & ~um) - __popcll(vn & ~un);
            cross += __popcll(vm & (ug ^ vg));
        }
        return ((e + 2 * cross) & 3) == 1 ? -1 : 1;
    }
    else {
        uint64_t par = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) par ^= m[w] & gd.wmask[w];
        const int power = (nc2(mpop) + nc2(gd.gpop) - nc2(ppop) + 3) & 3;
        const int real = power == 0 ? 1 : (power == 2 ? -1 : 0);
        return (__popcll(par) & 1) ? -real : real;
    }
}

// Reference-state score <b|M|b> of a key: 0 unless fully paired; then Pauli (-1)^{|M & occ|}, Majorana
// (-1)^{|M & occ| + |M|/2} (MPOperator.h:235-254, PauliAlgebra.h:144-147, MajoranaAlgebra.h:56-60).
template <int W, int BASIS>
__device__ __forceinline__ double state_score(const uint64_t (&m)[W], const StateMask &occ) {
    uint64_t unpaired = 0;
    int na = 0, pop = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        unpaired |= (m[w] & kEven) ^ ((m[w] >> 1) & kEven);
        na += __popcll(m[w] & occ.w[w]);
        pop += __popcll(m[w]);
    }
    if (unpaired != 0) return 0.0;
    const int odd = BASIS == 1 ? (na & 1) : ((na + pop / 2) & 1);
    return odd ? -1.0 : 1.0;
}

__device__ __forceinline__ uint8_t phase_code(int phase) { return phase > 0 ? 0 : (phase < 0 ? 1 : 2); }
__device__ __forceinline__ double phase_value(uint8_t code) { return code == 0 ? 1.0 : (code == 1 ? -1.0 : 0.0); }

} // namespace mpx
