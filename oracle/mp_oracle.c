/*
 * mp_oracle.c -- CPU restatement of the reference's Heisenberg per-gate sweep, used ONLY as test
 * infrastructure: the parity tests, __graft_entry__.smoke() and bench.py's cpu_baseline leg call it as
 * the checker. No product code links or calls it.
 *
 * Parity is pinned: tests/test_oracle.py checks this restatement bit-for-bit (monomial sets) and to
 * the last ulp (coefficients) against the unmodified reference engine built by oracle/build_ref.sh, and
 * against the committed golden fixtures in tests/golden/.
 *
 * Semantics restated (reference file:line, paths inside the monoprop project):
 *   - anticommutation fold: Pauli parity(M & pair_swap(G)) (algebra/PauliAlgebra.h:54-64,80-83);
 *     Majorana parity(M & G) ^ (|G| odd & |M| odd) (layer_build/Scan.h:221-237, algebra/Algebra.h:70-72).
 *   - fused cos sweep + emit gate + structural cutoff + upper_atol rescue (layer_build/Scan.h:272-304,
 *     343-358; CutoffContext.h:20-42; algebra/AlgebraCommon.h:131-176,229-243).
 *   - rotation phase: Pauli (algebra/PauliAlgebra.h:121-140); Majorana interleave mask times the
 *     Hermitian phase (algebra/MajoranaAlgebra.h:104-122, algebra/Algebra.h:52-57).
 *   - leader/follower resolve with the matched set (layer_build/Engine.h:464-513, Common.h:31-48),
 *     append-only inserts in leader-then-follower order (Engine.h:432-444, MPOperator.h:269-278).
 *   - rotation apply with the pre-cos partner value recovered as stored*(1/cos)
 *     (layer_build/FusedApply.h:32-83, Engine.h:209-212,599-614).
 *   - only_rotate_len_k: a term with more than k set slots takes no part in the gate (neither cos-scaled
 *     nor emitted; layer_build/Scan.h:146-157,376-391); the gate then runs the two-pass form, partner
 *     values read unscaled and the cos set (anticommuting terms of at most k slots) scaled before the
 *     adds (FusedApply.h:46-52, Engine.h:553,599-614).
 *   - basis_change: the structural cutoff of a partner is judged on its image under the given basis rows
 *     (algebra/MajoranaAlgebra.h:179-189, detail/monomial_propagator/MonomialPropagatorCommon.h:44-62).
 *   - Schrodinger picture: the store starts as every fully paired monomial up to schrodinger_cutoff,
 *     each holding its reference-state score; gates run first to last at the negated angle, a fresh
 *     partner starts from its own score, and <O> is the observable dotted into the evolved state
 *     (MonomialPropagator.inl:146-179,595-620; FusedApply.h:39-83; MPFunctions.cpp:196-205).
 *   - <0|O|0> = core + sum over fully paired rows of phase*c (MPOperator.h:235-254,
 *     algebra/PauliAlgebra.h:144-147, algebra/MajoranaAlgebra.h:56-60, MPFunctions.cpp:196-205).
 *
 * Bit layout (kept identical to the reference so exported keys compare directly): a monomial over a
 * storage tier of T modes has 2T bits in W = T/32 little-endian uint64 words; slot s is bit 2T-1-s
 * (algebra/AlgebraCommon.h:45-52).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MPO_MAXW 8
#define MPO_SCHRODINGER_MAX_TERMS (1ULL << 28) /* largest initial Schrodinger store the oracle builds */
#define EVEN_MASK 0x5555555555555555ULL
#define EMPTY_SLOT 0xFFFFFFFFu

typedef struct {
    int32_t basis;       /* 0 = majorana, 1 = pauli */
    int32_t cutoff_type; /* 0 = length, 1 = support */
    uint32_t cutoff;
    int32_t has_lower;
    double lower;
    int32_t has_upper;
    double upper;
    int32_t words; /* W, 1..8 */
    int32_t has_len_k; /* only_rotate_len_k given */
    uint32_t len_k;
    /* basis_change: [2T][W] rows indexed by slot (rows of slots >= 2 * logical modes are zero), or NULL */
    const uint64_t *basis_rows;
    /* Schrodinger picture (schrodinger >= 0: its cutoff) over `logical_modes` modes */
    int32_t schrodinger;
    int32_t logical_modes;
} mpo_config;

typedef struct {
    mpo_config cfg;
    size_t n, cap;
    uint64_t *keys; /* [cap][W] */
    double *coef;   /* [cap] */
    uint32_t *table;
    size_t tcap; /* power of two */
    uint32_t *mark;
    uint32_t epoch;
    double core;
    uint64_t state_mask[MPO_MAXW];
    /* Schrodinger picture: the observable, kept apart from the evolved state store */
    size_t n_obs;
    uint64_t *obs_keys;
    double *obs_coef;
} mpo_state;

static inline int popc(uint64_t x) { return __builtin_popcountll(x); }

static uint64_t mix64(uint64_t x) {
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebULL;
    x ^= x >> 31;
    return x;
}

static uint64_t key_hash(const uint64_t *k, int W) {
    uint64_t h = 0;
    for (int w = 0; w < W; ++w) h ^= mix64(k[w] + (uint64_t)w);
    return h;
}

static int key_eq(const uint64_t *a, const uint64_t *b, int W) {
    for (int w = 0; w < W; ++w)
        if (a[w] != b[w]) return 0;
    return 1;
}

/* Returns the index of key k, or SIZE_MAX. */
static size_t find(const mpo_state *s, const uint64_t *k) {
    const int W = s->cfg.words;
    size_t pos = (size_t)key_hash(k, W) & (s->tcap - 1);
    for (;;) {
        uint32_t idx = s->table[pos];
        if (idx == EMPTY_SLOT) return SIZE_MAX;
        if (key_eq(s->keys + (size_t)idx * W, k, W)) return idx;
        pos = (pos + 1) & (s->tcap - 1);
    }
}

static void table_put(mpo_state *s, size_t idx) {
    const int W = s->cfg.words;
    size_t pos = (size_t)key_hash(s->keys + idx * W, W) & (s->tcap - 1);
    while (s->table[pos] != EMPTY_SLOT) pos = (pos + 1) & (s->tcap - 1);
    s->table[pos] = (uint32_t)idx;
}

static int reserve(mpo_state *s, size_t need) {
    const int W = s->cfg.words;
    if (need > s->cap) {
        size_t nc = s->cap ? s->cap : 1024;
        while (nc < need) nc *= 2;
        uint64_t *nk = realloc(s->keys, nc * W * sizeof(uint64_t));
        if (!nk) return -1;
        s->keys = nk;
        double *ncf = realloc(s->coef, nc * sizeof(double));
        if (!ncf) return -1;
        s->coef = ncf;
        uint32_t *nm = realloc(s->mark, nc * sizeof(uint32_t));
        if (!nm) return -1;
        memset(nm + s->cap, 0, (nc - s->cap) * sizeof(uint32_t));
        s->mark = nm;
        s->cap = nc;
    }
    size_t want = 16;
    while (want < 2 * need) want *= 2;
    if (want > s->tcap) {
        free(s->table);
        s->table = malloc(want * sizeof(uint32_t));
        if (!s->table) return -1;
        memset(s->table, 0xFF, want * sizeof(uint32_t));
        s->tcap = want;
        for (size_t i = 0; i < s->n; ++i) table_put(s, i);
    }
    return 0;
}

/* --- algebra ------------------------------------------------------------------------------------ */

static void pair_swap(const uint64_t *g, uint64_t *out, int W) {
    for (int w = 0; w < W; ++w) out[w] = ((g[w] & EVEN_MASK) << 1) | ((g[w] >> 1) & EVEN_MASK);
}

/* Bit c set iff the number of G bits strictly above c is odd. */
static void interleave_mask(const uint64_t *g, uint64_t *out, int W) {
    int above = 0;
    memset(out, 0, sizeof(uint64_t) * W);
    for (int c = 64 * W - 1; c >= 0; --c) {
        if (above & 1) out[c / 64] |= 1ULL << (c % 64);
        above += (int)((g[c / 64] >> (c % 64)) & 1ULL);
    }
}

static int keep_struct(const mpo_state *s, const uint64_t *p_in, int pop) {
    const int W = s->cfg.words;
    const uint64_t *p = p_in;
    uint64_t mapped[MPO_MAXW];
    if (s->cfg.basis_rows != NULL) {
        /* basis_change: the cutoff is judged on the image XOR_{slot s in P} row_s (change_basis,
         * algebra/MajoranaAlgebra.h:179-189; MonomialPropagatorCommon.h:44-62), without the popcount fast
         * path (AlgebraCommon.h:229-243 falls through to the stored function) */
        for (int w = 0; w < W; ++w) mapped[w] = 0;
        const int T2 = 64 * W;
        for (int w = 0; w < W; ++w)
            for (uint64_t x = p_in[w]; x; x &= x - 1) {
                const int bit = 64 * w + __builtin_ctzll(x);
                const int slot = T2 - 1 - bit;
                for (int v = 0; v < W; ++v) mapped[v] ^= s->cfg.basis_rows[(size_t)slot * W + v];
            }
        p = mapped;
        pop = 0;
        for (int w = 0; w < W; ++w) pop += popc(mapped[w]);
    }
    /* passes_with_popcount fast path is equivalent: measure <= popcount. */
    int xs = 0, os = 0;
    for (int w = 0; w < W; ++w) {
        uint64_t a = p[w] & EVEN_MASK, b = (p[w] >> 1) & EVEN_MASK;
        xs += popc(a ^ b);
        os += popc(a | b);
    }
    if (xs == 0) return 1;
    int measure = s->cfg.cutoff_type == 1 ? os : pop;
    return measure <= (int)s->cfg.cutoff;
}

static int is_paired(const uint64_t *p, int W) {
    for (int w = 0; w < W; ++w)
        if (((p[w] & EVEN_MASK) ^ ((p[w] >> 1) & EVEN_MASK)) != 0) return 0;
    return 1;
}

static int nc2(int n) { return n * (n - 1) / 2; }

/* <b|M|b> of the reference product state: the state phase of a fully paired row, else 0
 * (MPOperator.h:235-254; PauliAlgebra.h:144-147; MajoranaAlgebra.h:56-60). */
static double state_score(const mpo_state *s, const uint64_t *m) {
    const int W = s->cfg.words;
    if (!is_paired(m, W)) return 0.0;
    int na = 0, pop = 0;
    for (int w = 0; w < W; ++w) {
        na += popc(m[w] & s->state_mask[w]);
        pop += popc(m[w]);
    }
    const int odd = s->cfg.basis == 1 ? (na & 1) : ((na + pop / 2) & 1);
    return odd ? -1.0 : 1.0;
}

typedef struct {
    uint64_t g[MPO_MAXW], fold[MPO_MAXW], wmask[MPO_MAXW];
    int gpop, gy, g_odd, pivot_word;
    uint64_t pivot_bit;
} gate_ctx;

static void make_ctx(const mpo_state *s, const uint64_t *g, gate_ctx *c) {
    const int W = s->cfg.words;
    memcpy(c->g, g, sizeof(uint64_t) * W);
    c->gpop = 0;
    c->gy = 0;
    for (int w = 0; w < W; ++w) {
        c->gpop += popc(g[w]);
        uint64_t v = g[w] & EVEN_MASK, u = (g[w] >> 1) & EVEN_MASK;
        c->gy += popc(v & ~u);
    }
    if (s->cfg.basis == 1) {
        pair_swap(g, c->fold, W);
        c->g_odd = 0;
    }
    else {
        memcpy(c->fold, g, sizeof(uint64_t) * W);
        c->g_odd = c->gpop & 1;
        interleave_mask(g, c->wmask, W);
    }
    c->pivot_word = -1;
    c->pivot_bit = 0;
    for (int w = 0; w < W; ++w) {
        if (g[w]) {
            c->pivot_word = w;
            c->pivot_bit = g[w] & (~g[w] + 1);
            break;
        }
    }
}

static int phase_of(const mpo_state *s, const gate_ctx *c, const uint64_t *m, const uint64_t *p, int mpop, int ov) {
    const int W = s->cfg.words;
    if (s->cfg.basis == 1) {
        long e = c->gy, cross = 0;
        for (int w = 0; w < W; ++w) {
            uint64_t vm = m[w] & EVEN_MASK, um = (m[w] >> 1) & EVEN_MASK;
            uint64_t vn = p[w] & EVEN_MASK, un = (p[w] >> 1) & EVEN_MASK;
            uint64_t vg = c->g[w] & EVEN_MASK, ug = (c->g[w] >> 1) & EVEN_MASK;
            e += popc(vm & ~um);
            e -= popc(vn & ~un);
            cross += popc(vm & (ug ^ vg));
        }
        long t = e + 2 * cross;
        return (((t % 4) + 4) % 4) == 1 ? -1 : 1;
    }
    int par = 0;
    for (int w = 0; w < W; ++w) par ^= popc(m[w] & c->wmask[w]) & 1;
    static const int REAL[4] = {1, 0, -1, 0};
    int ppop = mpop + c->gpop - 2 * ov;
    /* reduced into [0, 4): the reference evaluates this in unsigned arithmetic, where a negative
     * intermediate wraps by 2^64, a multiple of 4 */
    int power = (((nc2(mpop) + nc2(c->gpop) - nc2(ppop) + 3) % 4) + 4) % 4;
    return (par ? -1 : 1) * REAL[power];
}

/* --- public ABI ----------------------------------------------------------------------------------- */

void mpo_destroy(void *hs);

typedef struct {
    size_t src;
    uint64_t p[MPO_MAXW];
    int phase;
    double v;
} query;

void *mpo_create(const mpo_config *cfg,
                 size_t n_terms,
                 const uint64_t *words,
                 const double *coefs,
                 double core,
                 const uint64_t *state_mask) {
    if (cfg->words < 1 || cfg->words > MPO_MAXW) return NULL;
    mpo_state *s = calloc(1, sizeof(mpo_state));
    if (!s) return NULL;
    s->cfg = *cfg;
    s->core = core;
    memcpy(s->state_mask, state_mask, sizeof(uint64_t) * cfg->words);
    const int W = cfg->words;
    if (cfg->schrodinger >= 0) {
        /* Schrodinger picture (MonomialPropagator.inl:146-179): the store starts as every fully paired
         * monomial of at most K = sc/2 + sc%2 pairs over the logical modes, sc = min(schrodinger_cutoff,
         * 2 * modes) (generate_paired_op, MajoranaAlgebra.h:127-160), each holding its reference-state
         * score; the observable is kept apart for the final dot product. */
        s->n_obs = n_terms;
        s->obs_keys = malloc(sizeof(uint64_t) * W * (n_terms ? n_terms : 1));
        s->obs_coef = malloc(sizeof(double) * (n_terms ? n_terms : 1));
        if (!s->obs_keys || !s->obs_coef) {
            mpo_destroy(s);
            return NULL;
        }
        memcpy(s->obs_keys, words, sizeof(uint64_t) * W * n_terms);
        memcpy(s->obs_coef, coefs, sizeof(double) * n_terms);
        const int L = cfg->logical_modes;
        int sc = cfg->schrodinger;
        if (sc > 2 * L) sc = 2 * L;
        int K = sc / 2 + sc % 2;
        if (K > L) K = L;
        /* the initial store holds sum_{k<=K} C(L, k) monomials: refuse sizes an oracle cannot hold */
        double total = 0.0, binom = 1.0;
        for (int k = 0; k <= K; ++k) {
            total += binom;
            binom = binom * (double)(L - k) / (double)(k + 1);
        }
        if (total > (double)MPO_SCHRODINGER_MAX_TERMS) {
            mpo_destroy(s);
            return NULL;
        }
        int sel[256];
        for (int k = 0; k <= K; ++k) {
            /* subsets of k modes in lexicographic order */
            for (int i = 0; i < k; ++i) sel[i] = i;
            for (;;) {
                if (reserve(s, s->n + 1) != 0) {
                    mpo_destroy(s);
                    return NULL;
                }
                uint64_t *m = s->keys + s->n * W;
                memset(m, 0, sizeof(uint64_t) * W);
                for (int i = 0; i < k; ++i)
                    for (int slot = 2 * sel[i]; slot <= 2 * sel[i] + 1; ++slot) {
                        const int bit = 64 * W - 1 - slot;
                        m[bit / 64] |= 1ULL << (bit % 64);
                    }
                s->coef[s->n] = state_score(s, m);
                table_put(s, s->n);
                s->n++;
                int i = k - 1;
                while (i >= 0 && sel[i] == L - k + i) --i;
                if (i < 0) break;
                ++sel[i];
                for (int j = i + 1; j < k; ++j) sel[j] = sel[j - 1] + 1;
            }
        }
        return s;
    }
    if (reserve(s, n_terms ? n_terms : 1) != 0) {
        mpo_destroy(s);
        return NULL;
    }
    for (size_t i = 0; i < n_terms; ++i) {
        memcpy(s->keys + s->n * W, words + i * W, sizeof(uint64_t) * W);
        s->coef[s->n] = coefs[i];
        table_put(s, s->n);
        s->n++;
    }
    return s;
}

/* Applies gates[n_gates-1] .. gates[0] (Heisenberg order, MonomialPropagator.inl:720-733).
 * gen_words: [n_gates][W]; angles: theta[map]*g per gate, in circuit order.
 * counts (optional): per APPLIED gate (application order) {n_g, a_g, e_g, m_g}. */
int mpo_propagate(void *hs, size_t n_gates, const uint64_t *gen_words, const double *angles, uint64_t *counts) {
    mpo_state *s = hs;
    const int W = s->cfg.words;
    query *qs = NULL;
    size_t qcap = 0;
    size_t *miss = NULL;
    const int schr = s->cfg.schrodinger >= 0;
    for (size_t step = 0; step < n_gates; ++step) {
        /* Heisenberg: last gate first; Schrodinger: first gate first at the negated angle
         * (MonomialPropagator.inl:720-733, map_params with phase -1, MPFunctions.cpp:186-193) */
        const size_t gi = schr ? step : n_gates - 1 - step;
        const uint64_t *g = gen_words + gi * W;
        const double ang = schr ? -angles[gi] : angles[gi];
        const double cosv = cos(2.0 * ang);
        const double sinv = sin(2.0 * ang);
        const double abs_sin = fabs(sinv);
        const int fused = cosv != 0.0 && !s->cfg.has_len_k;
        const double inv_cos = fused ? 1.0 / cosv : 1.0;
        gate_ctx c;
        make_ctx(s, g, &c);
        const size_t n0 = s->n;
        if (qcap < n0 + 1) {
            qcap = 2 * (n0 + 1);
            qs = realloc(qs, qcap * sizeof(query));
            miss = realloc(miss, qcap * sizeof(size_t));
            if (!qs || !miss) return -1;
        }
        size_t n_anti = 0, nl = 0, nf = 0;
        /* queries: leaders in [0, nl), followers stored from the top down: [qcap-nf, qcap) */
        if (c.pivot_word >= 0) {
            for (size_t i = 0; i < n0; ++i) {
                const uint64_t *m = s->keys + i * W;
                int par = 0, mpop = 0;
                for (int w = 0; w < W; ++w) {
                    par ^= popc(m[w] & c.fold[w]) & 1;
                    mpop += popc(m[w]);
                }
                if (c.g_odd) par ^= mpop & 1;
                if (!par) continue;
                ++n_anti;
                if (s->cfg.has_len_k && mpop > (int)s->cfg.len_k) continue;
                const double v = s->coef[i];
                if (fused) s->coef[i] = v * cosv;
                const double av = fabs(v);
                if (s->cfg.has_lower && abs_sin * av <= s->cfg.lower) continue;
                uint64_t p[MPO_MAXW];
                int ov = 0;
                for (int w = 0; w < W; ++w) {
                    p[w] = m[w] ^ g[w];
                    ov += popc(m[w] & g[w]);
                }
                const int ppop = mpop + c.gpop - 2 * ov;
                const int keep = keep_struct(s, p, ppop);
                if (!keep && !(s->cfg.has_upper && abs_sin * av >= s->cfg.upper)) continue;
                const int ph = phase_of(s, &c, m, p, mpop, ov);
                const int follower = (m[c.pivot_word] & c.pivot_bit) != 0;
                query *q = follower ? &qs[qcap - 1 - nf++] : &qs[nl++];
                q->src = i;
                memcpy(q->p, p, sizeof(uint64_t) * W);
                q->phase = ph;
                q->v = v;
            }
        }
        /* resolve: leaders then followers (followers in ascending source order) */
        s->epoch++;
        size_t n_miss = 0;
        double *c_arr = s->coef;
        /* Hits are applied after both passes; record them in place of the query (reuse fields). */
        typedef struct {
            size_t src, tgt;
            int phase;
            double vs, vt;
        } hit;
        hit *hits = malloc((nl + nf + 1) * sizeof(hit));
        size_t nh = 0;
        for (size_t k = 0; k < nl + nf; ++k) {
            const int is_leader = k < nl;
            /* followers were pushed top-down; read them back in ascending source order */
            query *q = is_leader ? &qs[k] : &qs[qcap - 1 - (k - nl)];
            if (!is_leader && s->mark[q->src] == s->epoch) continue;
            size_t j = find(s, q->p);
            if (j != SIZE_MAX && j < n0) {
                if (is_leader) s->mark[j] = s->epoch;
                hit h = {q->src, j, q->phase, q->v, fused ? c_arr[j] * inv_cos : c_arr[j]};
                hits[nh++] = h;
            }
            else {
                miss[n_miss++] = (size_t)(q - qs);
            }
        }
        if (reserve(s, n0 + n_miss) != 0) return -1;
        c_arr = s->coef;
        if (!fused) {
            /* two-pass form (cos == 0, or only_rotate_len_k): the cos set is scaled before the adds */
            for (size_t i = 0; i < n0; ++i) {
                const uint64_t *m = s->keys + i * W;
                int par = 0, mpop = 0;
                for (int w = 0; w < W; ++w) {
                    par ^= popc(m[w] & c.fold[w]) & 1;
                    mpop += popc(m[w]);
                }
                if (c.g_odd) par ^= mpop & 1;
                if (par && !(s->cfg.has_len_k && mpop > (int)s->cfg.len_k)) c_arr[i] = cosv * c_arr[i];
            }
        }
        for (size_t k = 0; k < nh; ++k) {
            const hit *h = &hits[k];
            c_arr[h->src] += sinv * (double)(-h->phase) * h->vt;
            c_arr[h->tgt] += sinv * (double)(h->phase) * h->vs;
        }
        for (size_t k = 0; k < n_miss; ++k) {
            const query *q = &qs[miss[k]];
            const size_t idx = s->n++;
            memcpy(s->keys + idx * W, q->p, sizeof(uint64_t) * W);
            if (schr) {
                /* a fresh slot starts from its reference-state score, and the pair rotates as a hit does
                 * (FusedApply.h:39-83: v_tgt read after the extension; cos folded in for the new slot) */
                const double vt = state_score(s, q->p);
                c_arr[q->src] += sinv * (double)(-q->phase) * vt;
                if (fused) {
                    c_arr[idx] = vt;
                    c_arr[idx] = cosv * c_arr[idx] + sinv * (double)q->phase * q->v;
                }
                else {
                    c_arr[idx] = cosv * vt;
                    c_arr[idx] += sinv * (double)q->phase * q->v;
                }
            }
            else {
                c_arr[idx] = sinv * (double)q->phase * q->v;
            }
            table_put(s, idx);
        }
        free(hits);
        if (counts) {
            counts[4 * step + 0] = n0;
            counts[4 * step + 1] = n_anti;
            counts[4 * step + 2] = nl + nf;
            counts[4 * step + 3] = n_miss;
        }
    }
    free(qs);
    free(miss);
    return 0;
}

size_t mpo_size(void *hs) { return ((mpo_state *)hs)->n; }

void mpo_export(void *hs, uint64_t *words, double *coefs) {
    mpo_state *s = hs;
    memcpy(words, s->keys, s->n * s->cfg.words * sizeof(uint64_t));
    memcpy(coefs, s->coef, s->n * sizeof(double));
}

double mpo_expectation(void *hs) {
    mpo_state *s = hs;
    const int W = s->cfg.words;
    double acc = 0.0;
    if (s->cfg.schrodinger >= 0) {
        /* Schrodinger: core + state . observable over the stored rows (MPFunctions.cpp:196-205) */
        for (size_t t = 0; t < s->n_obs; ++t) {
            const size_t j = find(s, s->obs_keys + t * W);
            if (j != SIZE_MAX) acc += s->obs_coef[t] * s->coef[j];
        }
        return s->core + acc;
    }
    for (size_t i = 0; i < s->n; ++i) {
        const uint64_t *m = s->keys + i * W;
        if (!is_paired(m, W)) continue;
        int na = 0, pop = 0;
        for (int w = 0; w < W; ++w) {
            na += popc(m[w] & s->state_mask[w]);
            pop += popc(m[w]);
        }
        int odd = s->cfg.basis == 1 ? (na & 1) : ((na + pop / 2) & 1);
        acc += (odd ? -1.0 : 1.0) * s->coef[i];
    }
    return s->core + acc;
}

void mpo_destroy(void *hs) {
    mpo_state *s = hs;
    if (!s) return;
    free(s->keys);
    free(s->coef);
    free(s->table);
    free(s->mark);
    free(s->obs_keys);
    free(s->obs_coef);
    free(s);
}
