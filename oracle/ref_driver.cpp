// C-ABI driver over the UNMODIFIED reference engine (monoprop's MonomialPropagator<N>), compiled from
// the reference sources by oracle/build_ref.sh into oracle/_ref/libmpref.so.
//
// Test infrastructure only: the parity tests, the golden-fixture generator and bench.py's
// reference/CPU-baseline arm call it as the checker / the timed CPU baseline. No product code links it.
//
// Entry points mirror the reference's own Python-facing methods (src/monoprop/bindings/binder.h:54-274):
// construct, propagate, build_graph, expectation_value[_and_gradient], size, raw coefficient export.
#include <chrono>
#include <complex>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <optional>
#include <string>
#include <vector>

#include "monoprop/MonomialPropagator.h"

using namespace monoprop;

extern "C" {
struct mpref_config {
    int32_t basis;       // 0 = majorana, 1 = pauli
    int32_t cutoff_type; // 0 = length, 1 = support
    uint32_t cutoff;
    int32_t has_lower;
    double lower;
    int32_t has_upper;
    double upper;
    int32_t partitions;        // >= 1
    int32_t logical_num_modes; // modes (Majorana) or qubits (Pauli)
    int32_t len_k;             // only_rotate_len_k, 0 = not given
    int32_t schrodinger_cutoff; // < 0: Heisenberg picture; >= 0: the Schrodinger picture with this cutoff
};
}

namespace {

struct Gates {
    std::vector<VecZ> monos;
    VecZ mapping;
    VecD gen;
};

Gates read_gates(size_t n_layers, const int64_t *off, const int64_t *slots, const double *gen, const int64_t *map) {
    Gates g;
    g.monos.resize(n_layers);
    g.mapping.resize(n_layers);
    g.gen.assign(gen, gen + n_layers);
    for (size_t l = 0; l < n_layers; ++l) {
        for (int64_t k = off[l]; k < off[l + 1]; ++k) {
            g.monos[l].push_back(static_cast<size_t>(slots[k]));
        }
        g.mapping[l] = static_cast<size_t>(map[l]);
    }
    return g;
}

struct Base {
    virtual ~Base() = default;
    virtual void propagate(const Gates &g, const VecD &params) = 0;
    virtual void build_graph(const Gates &g, const VecD &params) = 0;
    virtual double ev(const VecD &params) = 0;
    virtual std::pair<double, VecD> ev_grad(const VecD &params) = 0;
    virtual size_t size() = 0;
    virtual size_t words() = 0;
    virtual double core() = 0;
    virtual size_t export_terms(uint64_t *words, double *coefs, size_t cap, const VecD &params) = 0;
};

template <size_t N>
struct Impl final : Base {
    std::unique_ptr<MonomialPropagator<N>> p;
    std::optional<size_t> len_k;
    Impl(const mpref_config &c, const OperatorDict &op, const VecZ &state,
         const std::optional<std::vector<VecZ>> &basis_change) {
        if (c.len_k > 0) len_k = static_cast<size_t>(c.len_k);
        std::optional<double> lo = c.has_lower ? std::optional<double>(c.lower) : std::nullopt;
        std::optional<double> hi = c.has_upper ? std::optional<double>(c.upper) : std::nullopt;
        std::optional<unsigned int> sc;
        if (c.schrodinger_cutoff >= 0) sc = static_cast<unsigned int>(c.schrodinger_cutoff);
        p = std::make_unique<MonomialPropagator<N>>(op,
                                                    c.cutoff,
                                                    state,
                                                    sc,
                                                    mpi::Comm{},
                                                    lo,
                                                    hi,
                                                    c.cutoff_type == 1 ? CutoffType::Support : CutoffType::Length,
                                                    basis_change,
                                                    static_cast<size_t>(c.logical_num_modes),
                                                    c.basis == 1 ? Basis::Pauli : Basis::Majorana,
                                                    static_cast<size_t>(c.partitions));
    }
    void propagate(const Gates &g, const VecD &params) override {
        p->propagate(g.monos, g.mapping, g.gen, params, len_k);
    }
    void build_graph(const Gates &g, const VecD &params) override {
        p->build_graph(g.monos, g.mapping, g.gen, std::nullopt, params, len_k);
    }
    double ev(const VecD &params) override { return p->expectation_value(params); }
    std::pair<double, VecD> ev_grad(const VecD &params) override { return p->expectation_value_and_gradient(params); }
    size_t size() override { return p->size(); }
    size_t words() override { return Monomial<N>::num_words(); }
    double core() override { return p->core_term(); }
    // the raw coefficients of the current operator (no parameters), or of the stored graph replayed at
    // `params` (contract_partially(params, false), MonomialPropagator.inl:1053-1097)
    size_t export_terms(uint64_t *words, double *coefs, size_t cap, const VecD &params) override {
        const VecD coeffs = p->contract_partially(params, false);
        size_t n = 0;
        constexpr size_t W = Monomial<N>::num_words();
        p->indexing().for_each([&](const auto &mono, size_t idx) {
            if (n >= cap) {
                return;
            }
            for (size_t w = 0; w < W; ++w) {
                words[n * W + w] = mono.word(w);
            }
            coefs[n] = idx < coeffs.size() ? coeffs[idx] : 0.0;
            ++n;
        });
        return n;
    }
};

void set_err(char *err, size_t len, const char *msg) {
    if (err != nullptr && len > 0) {
        std::strncpy(err, msg, len - 1);
        err[len - 1] = '\0';
    }
}

} // namespace

extern "C" {

void *mpref_create(const mpref_config *cfg,
                   size_t n_obs,
                   const int64_t *obs_off,
                   const int64_t *obs_slots,
                   const double *obs_re,
                   const double *obs_im,
                   size_t n_state,
                   const int64_t *state,
                   size_t n_basis,
                   const int64_t *basis_off,
                   const int64_t *basis_slots,
                   char *err,
                   size_t errlen) {
    try {
        OperatorDict op;
        for (size_t t = 0; t < n_obs; ++t) {
            VecZ key;
            for (int64_t k = obs_off[t]; k < obs_off[t + 1]; ++k) {
                key.push_back(static_cast<size_t>(obs_slots[k]));
            }
            op[key] = std::complex<double>(obs_re[t], obs_im[t]);
        }
        VecZ st;
        for (size_t i = 0; i < n_state; ++i) {
            st.push_back(static_cast<size_t>(state[i]));
        }
        std::optional<std::vector<VecZ>> basis;
        if (n_basis > 0) {
            basis.emplace(n_basis);
            for (size_t r = 0; r < n_basis; ++r)
                for (int64_t k = basis_off[r]; k < basis_off[r + 1]; ++k)
                    (*basis)[r].push_back(static_cast<size_t>(basis_slots[k]));
        }
        const int lm = cfg->logical_num_modes;
        const size_t tier = static_cast<size_t>((lm + 31) / 32) * 32;
        switch (tier) {
        case 32: return new Impl<32>(*cfg, op, st, basis);
        case 64: return new Impl<64>(*cfg, op, st, basis);
        case 96: return new Impl<96>(*cfg, op, st, basis);
        case 128: return new Impl<128>(*cfg, op, st, basis);
        default: set_err(err, errlen, "oracle driver built for at most 128 modes"); return nullptr;
        }
    }
    catch (const std::exception &e) {
        set_err(err, errlen, e.what());
        return nullptr;
    }
}

int mpref_propagate(void *h,
                    size_t n_layers,
                    const int64_t *off,
                    const int64_t *slots,
                    const double *gen,
                    const int64_t *map,
                    size_t n_params,
                    const double *params,
                    int32_t build_graph,
                    double *seconds,
                    char *err,
                    size_t errlen) {
    try {
        const Gates g = read_gates(n_layers, off, slots, gen, map);
        const VecD p(params, params + n_params);
        const auto t0 = std::chrono::steady_clock::now();
        if (build_graph != 0) {
            static_cast<Base *>(h)->build_graph(g, p);
        }
        else {
            static_cast<Base *>(h)->propagate(g, p);
        }
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds != nullptr) {
            *seconds = std::chrono::duration<double>(t1 - t0).count();
        }
        return 0;
    }
    catch (const std::exception &e) {
        set_err(err, errlen, e.what());
        return 1;
    }
}

int mpref_expectation(void *h, size_t n_params, const double *params, double *ev, char *err, size_t errlen) {
    try {
        *ev = static_cast<Base *>(h)->ev(VecD(params, params + n_params));
        return 0;
    }
    catch (const std::exception &e) {
        set_err(err, errlen, e.what());
        return 1;
    }
}

int mpref_expectation_and_gradient(void *h,
                                   size_t n_params,
                                   const double *params,
                                   double *ev,
                                   double *grad,
                                   double *seconds,
                                   char *err,
                                   size_t errlen) {
    try {
        const auto t0 = std::chrono::steady_clock::now();
        auto [e, g] = static_cast<Base *>(h)->ev_grad(VecD(params, params + n_params));
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds != nullptr) {
            *seconds = std::chrono::duration<double>(t1 - t0).count();
        }
        *ev = e;
        for (size_t i = 0; i < g.size() && i < n_params; ++i) {
            grad[i] = g[i];
        }
        return 0;
    }
    catch (const std::exception &e) {
        set_err(err, errlen, e.what());
        return 1;
    }
}

size_t mpref_size(void *h) { return static_cast<Base *>(h)->size(); }
size_t mpref_words(void *h) { return static_cast<Base *>(h)->words(); }
double mpref_core(void *h) { return static_cast<Base *>(h)->core(); }

int64_t mpref_export(void *h, uint64_t *words, double *coefs, size_t cap, char *err, size_t errlen) {
    try {
        return static_cast<int64_t>(static_cast<Base *>(h)->export_terms(words, coefs, cap, VecD{}));
    }
    catch (const std::exception &e) {
        set_err(err, errlen, e.what());
        return -1;
    }
}

int64_t mpref_export_at(void *h, size_t n_params, const double *params, uint64_t *words, double *coefs, size_t cap,
                        char *err, size_t errlen) {
    try {
        return static_cast<int64_t>(
            static_cast<Base *>(h)->export_terms(words, coefs, cap, VecD(params, params + n_params)));
    }
    catch (const std::exception &e) {
        set_err(err, errlen, e.what());
        return -1;
    }
}

void mpref_destroy(void *h) { delete static_cast<Base *>(h); }

} // extern "C"
