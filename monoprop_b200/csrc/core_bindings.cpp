// core_bindings.cpp -- the `_core` Python module: per-tier engine classes MonomialPropagator032 ...
// MonomialPropagator256 with the reference's constructor keywords, method names and error types
// (src/monoprop/bindings/binder.h:54-274, bindings.cpp.in:98-134), implemented in C++ over the engine's C
// ABI (include/mpx.h). This host layer does what the reference's C++ facade does around the per-gate
// kernel: validation before mutation, observable encoding (MonomialPropagator.inl:73-188), parameter
// binding angle_l = theta[map_l] * g_l (MPFunctions.cpp:57-69) and the decoded, filtered, 1e-12-rounded
// export of evolved_operator (MonomialPropagator.inl:1099-1127).
//
// Scope: propagate, build_graph + expectation_value[_and_gradient](parameters) over the engine's frozen
// structure (mpx_graph_*), the reusable functionals (with paring), contract_partially,
// update_initial_operator, the rw parameter_mapping, graph_size, memory accounting and __deepcopy__, with
// basis_change (Majorana) and only_rotate_len_k. MPI communicators raise NotImplementedError.
#include <pybind11/complex.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <complex>
#include <cstdint>
#include <map>
#include <memory>
#include <optional>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "mpx.h"

namespace py = pybind11;

namespace {

using OperatorDict = std::map<std::vector<size_t>, std::complex<double>>;

// Reference error classes (MonomialPropagator.h:59-68, MonomialPropagator.inl:46-71): invalid_argument
// subclasses surface as ValueError, runtime_error subclasses as RuntimeError.
struct CutoffConfigError : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};
struct PropagatorConfigError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct GraphStateConflict : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct NotSupported : std::logic_error {
    using std::logic_error::logic_error;
};
// Validation.cpp:24-36 and MPOperator.h:56-59: runtime_error subclasses (RuntimeError in Python)
struct ValidationError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct StaleFunctionalGraph : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct OperatorTermNotFound : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// The calling thread's current CUDA device (engines are created there, as torch.cuda.set_device chooses).
int32_t current_device() {
    int32_t d = 0;
    return mpx_current_device(&d) == MPX_OK ? d : 0;
}

int cutoff_type_code(const std::string &s) {
    if (s == "length") return MPX_CUTOFF_LENGTH;
    if (s == "support") return MPX_CUTOFF_SUPPORT;
    throw std::invalid_argument("Invalid cutoff_type '" + s + "'. Valid options are: 'length', 'support'");
}

int basis_code(const std::string &s) {
    if (s == "majorana") return MPX_BASIS_MAJORANA;
    if (s == "pauli") return MPX_BASIS_PAULI;
    throw std::invalid_argument("Invalid basis '" + s + "'. Valid options are: 'majorana', 'pauli'");
}

// i^k for k = C(w, 2) mod 4: the Hermitian phase of a weight-w Majorana monomial.
std::complex<double> hermitian_phase(size_t w) {
    switch ((w * (w - 1) / 2) % 4) {
    case 0: return {1.0, 0.0};
    case 1: return {0.0, 1.0};
    case 2: return {-1.0, 0.0};
    default: return {0.0, -1.0};
    }
}

template <size_t Tier>
class Propagator {
public:
    static constexpr size_t kWords = Tier / 32;

    Propagator(const OperatorDict &initial_operator, unsigned int cutoff, const std::vector<size_t> &initial_state,
               py::object comm, std::optional<unsigned int> schrodinger_cutoff, std::optional<double> lower_atol,
               std::optional<double> upper_atol, const std::string &cutoff_type,
               std::optional<std::vector<std::vector<size_t>>> basis_change, size_t logical_num_modes,
               const std::string &basis, size_t partitions)
        : logical_(logical_num_modes), state_(initial_state) {
        // partitions: the reference's count of host-thread partitions of the store (0 = automatic). The
        // engine's store is one device-resident structure with no host partitions, so any value gives the
        // same results; it is accepted for drop-in compatibility and otherwise unused.
        (void)partitions;
        if (!comm.is_none()) throw NotSupported("comm: the B200 engine runs on one GPU and takes no communicator");
        if (logical_ == 0 || logical_ > Tier)
            throw PropagatorConfigError("logical_num_modes (" + std::to_string(logical_) + ") must be in the range [1, " +
                                        std::to_string(Tier) + "].");
        cfg_.basis = basis_code(basis);
        cfg_.cutoff_type = cutoff_type_code(cutoff_type);
        if (cfg_.basis == MPX_BASIS_PAULI && cfg_.cutoff_type != MPX_CUTOFF_SUPPORT)
            throw CutoffConfigError("Pauli basis requires cutoff_type == Support (Length has no Pauli-weight meaning "
                                    "under the Pauli encoding).");
        // validate_cutoff_config_ (MonomialPropagator.inl:460-481)
        if (basis_change.has_value()) {
            if (cfg_.basis == MPX_BASIS_PAULI)
                throw CutoffConfigError("Pauli basis does not accept a basis_change (the encoding is already the "
                                        "Jordan-Wigner image).");
            if (basis_change->size() != 2 * logical_)
                throw CutoffConfigError("basis_change must have exactly 2*logical_num_modes (" +
                                        std::to_string(2 * logical_) + ") rows; got " +
                                        std::to_string(basis_change->size()) + ".");
        }
        if (upper_atol && lower_atol && *upper_atol < *lower_atol)
            throw PropagatorConfigError("upper_atol (" + std::to_string(*upper_atol) +
                                        ") must be greater than or equal to lower_atol (" +
                                        std::to_string(*lower_atol) + ").");
        cfg_.cutoff = cutoff;
        cfg_.has_lower_atol = lower_atol.has_value();
        cfg_.lower_atol = lower_atol.value_or(0.0);
        cfg_.has_upper_atol = upper_atol.has_value();
        cfg_.upper_atol = upper_atol.value_or(0.0);
        // The engine sizes keys by the storage tier of num_modes; pass the tier so W = Tier/32 and keys
        // compare word for word with the reference's Monomial<Tier>.
        cfg_.num_modes = static_cast<int32_t>(Tier);
        cfg_.device = current_device();
        cfg_.capacity_hint = 0;
        // Schrodinger picture (MonomialPropagator.inl:146-179): the engine builds the paired initial state
        // over the logical modes and keeps this operator apart for <O> = core + operator . state
        cfg_.has_schrodinger = schrodinger_cutoff.has_value() ? 1 : 0;
        cfg_.schrodinger_cutoff = static_cast<int32_t>(schrodinger_cutoff.value_or(0));
        cfg_.logical_num_modes = static_cast<int32_t>(logical_);

        std::vector<uint64_t> keys;
        std::vector<double> coefs;
        for (const auto &[indices, c] : initial_operator) {
            std::vector<uint64_t> k(kWords, 0);
            encode(indices, 2 * logical_, k.data());
            const double enc = encode_coeff(indices.size(), c);
            if (indices.empty()) {
                core_ = enc;
                continue;
            }
            keys.insert(keys.end(), k.begin(), k.end());
            coefs.push_back(enc);
        }
        std::vector<uint64_t> mask(kWords, 0);
        std::vector<size_t> occ;
        for (size_t m : initial_state) {
            if (m >= logical_)
                throw std::invalid_argument("initial_state index " + std::to_string(m) + " is out of range; must be "
                                            "less than " + std::to_string(logical_) + ".");
            occ.push_back(2 * m);
        }
        encode(occ, 2 * Tier, mask.data());
        const std::vector<uint64_t> rows = basis_rows(basis_change);
        check(mpx_create(&cfg_, keys.empty() ? nullptr : keys.data(), coefs.empty() ? nullptr : coefs.data(),
                         coefs.size(), core_, mask.data(), &e_),
              nullptr);
        if (!rows.empty()) {
            const mpx_status st = mpx_set_basis_change(e_, rows.data(), static_cast<uint32_t>(2 * Tier));
            if (st != MPX_OK) {
                const std::string msg = mpx_last_error(e_);
                mpx_destroy(e_);
                e_ = nullptr;
                throw std::runtime_error(msg);
            }
            basis_change_ = basis_change;
        }
    }

    // basis_change rows by slot, each slot set once (indices_to_bitset_checked, AlgebraCommon.h:44-63); the
    // rows of the slots above 2 * logical_num_modes stay zero. Empty when there is no basis change.
    std::vector<uint64_t> basis_rows(const std::optional<std::vector<std::vector<size_t>>> &basis_change) const {
        std::vector<uint64_t> rows;
        if (!basis_change.has_value()) return rows;
        rows.assign(2 * Tier * kWords, 0);
        for (size_t r = 0; r < basis_change->size(); ++r)
            for (size_t s : (*basis_change)[r]) {
                if (s >= 2 * logical_)
                    throw std::runtime_error("Majorana/Pauli index " + std::to_string(s) +
                                             " is out of range; must be less than " + std::to_string(2 * logical_) + ".");
                const size_t b = 2 * Tier - 1 - s;
                rows[r * kWords + b / 64] |= 1ULL << (b % 64);
            }
        return rows;
    }

    // basis_change property (binder.h:185-188; update_basis_change validates like the constructor)
    std::optional<std::vector<std::vector<size_t>>> basis_change() const { return basis_change_; }
    void set_basis_change(const std::optional<std::vector<std::vector<size_t>>> &basis_change) {
        if (basis_change.has_value()) {
            if (cfg_.basis == MPX_BASIS_PAULI)
                throw CutoffConfigError("Pauli basis does not accept a basis_change (the encoding is already the "
                                        "Jordan-Wigner image).");
            if (basis_change->size() != 2 * logical_)
                throw CutoffConfigError("basis_change must have exactly 2*logical_num_modes (" +
                                        std::to_string(2 * logical_) + ") rows; got " +
                                        std::to_string(basis_change->size()) + ".");
        }
        const std::vector<uint64_t> rows = basis_rows(basis_change);
        check(mpx_set_basis_change(e_, rows.empty() ? nullptr : rows.data(),
                                   rows.empty() ? 0u : static_cast<uint32_t>(2 * Tier)),
              e_);
        basis_change_ = basis_change;
    }

    ~Propagator() {
        if (circ_ != nullptr) mpx_circuit_destroy(circ_);
        mpx_destroy(e_);
    }
    Propagator(const Propagator &) = delete;
    Propagator &operator=(const Propagator &) = delete;

    // MonomialPropagator<N>::propagate (MonomialPropagator.h:121-125, .inl:692-718).
    void propagate(const std::vector<std::vector<size_t>> &majoranas, const std::vector<size_t> &parameter_mapping,
                   const std::vector<double> &gen_coeffs, const std::vector<double> &parameters,
                   std::optional<unsigned int> only_rotate_len_k) {
        // validate_only_rotate_len_k_ (Validation.cpp:119-128): a runtime_error subclass in the reference
        if (only_rotate_len_k.has_value() && (*only_rotate_len_k == 0 || *only_rotate_len_k > 2 * logical_))
            throw PropagatorConfigError("only_rotate_len_k=" + std::to_string(*only_rotate_len_k) +
                                        " is out of range; must be 0 < k <= 2*num_qubits");
        if (majoranas.empty()) return;
        std::vector<uint64_t> words;
        std::vector<double> angles;
        encode_circuit(majoranas, parameter_mapping, gen_coeffs, parameters, words, angles);
        if (circ_ != nullptr)
            throw GraphStateConflict("Cannot propagate() on top of a non-empty graph of " +
                                     std::to_string(mapping_.size()) +
                                     " layer(s): propagate() evolves and contracts in place and assumes no stored "
                                     "graph. Call contract_partially() to fold the existing graph first, or use "
                                     "build_graph() to extend it.");
        check(mpx_set_only_rotate_len_k(e_, only_rotate_len_k.has_value() ? static_cast<int64_t>(*only_rotate_len_k) : 0),
              e_);
        mpx_status st;
        {
            py::gil_scoped_release nogil;
            st = mpx_propagate(e_, words.data(), angles.data(), majoranas.size());
        }
        mpx_set_only_rotate_len_k(e_, 0);
        check(st, e_);
    }

    // MonomialPropagator<N>::build_graph (MonomialPropagator.inl:620-690): a coefficient-informed build at
    // `parameters` whose truncation structure later evaluations keep.
    void build_graph(const std::vector<std::vector<size_t>> &majoranas, const std::vector<size_t> &parameter_mapping,
                     const std::vector<double> &gen_coeffs, std::optional<std::vector<size_t>> gate_indices,
                     std::optional<std::vector<double>> parameters, std::optional<unsigned int> only_rotate_len_k) {
        if (!parameters.has_value())
            throw NotSupported("build_graph without seed parameters (a purely structural graph) is not implemented");
        // validate_only_rotate_len_k_ (Validation.cpp:119-128), as propagate
        if (only_rotate_len_k.has_value() && (*only_rotate_len_k == 0 || *only_rotate_len_k > 2 * logical_))
            throw PropagatorConfigError("only_rotate_len_k=" + std::to_string(*only_rotate_len_k) +
                                        " is out of range; must be 0 < k <= 2*num_qubits");
        std::vector<uint64_t> words;
        std::vector<double> angles;
        encode_circuit(majoranas, parameter_mapping, gen_coeffs, *parameters, words, angles);
        if (gate_indices.has_value()) validate_gate_indices(*gate_indices, majoranas.size());
        if (circ_ != nullptr) mpx_circuit_destroy(circ_);
        circ_ = nullptr;
        check(mpx_circuit_upload(e_, words.data(), angles.data(), majoranas.size(), &circ_), e_);
        mapping_ = parameter_mapping;
        gen_ = gen_coeffs;
        n_params_ = parameters->size();
        // gate index of every layer (a multi-term gate spans several layers); n_gates = largest + 1
        // (MonomialPropagator.inl, n_gates)
        gate_of_layer_.resize(majoranas.size());
        gates_ = 0;
        for (size_t l = 0; l < majoranas.size(); ++l) {
            gate_of_layer_[l] = gate_indices.has_value() ? (*gate_indices)[l] : l;
            gates_ = std::max(gates_, gate_of_layer_[l] + 1);
        }
        ++graph_epoch_;
        double ev = 0.0;
        mpx_status st = mpx_set_only_rotate_len_k(
            e_, only_rotate_len_k.has_value() ? static_cast<int64_t>(*only_rotate_len_k) : 0);
        if (st == MPX_OK) {
            py::gil_scoped_release nogil;
            st = mpx_graph_build(e_, circ_, 0, &ev); // the graph keeps the k it was built with
        }
        mpx_set_only_rotate_len_k(e_, 0);
        if (st != MPX_OK) { // no graph is kept after a failed build
            const std::string msg = mpx_last_error(e_);
            mpx_circuit_destroy(circ_);
            circ_ = nullptr;
            mapping_.clear();
            gen_.clear();
            gate_of_layer_.clear();
            n_params_ = gates_ = 0;
            if (st == MPX_ERR_INVALID) throw std::invalid_argument(msg);
            throw std::runtime_error(msg);
        }
    }

    // expectation_value_functional / expectation_value_and_gradient_functional (binder.h:137-146,
    // MonomialPropagator.inl:1003-1031, make_functional_ :918-1000): a reusable callable over the stored
    // graph. It snapshots the parameter mapping and generator coefficients; a call checks, like the
    // reference, that the initial operator was not re-weighted since (StaleFunctionalGraph), that the
    // parameter count matches (ValidationError) and that the graph still has the same layers.
    // pare_threshold: the graph pared of pairs whose reference-state weight stays below it (PareGraph.cpp).
    template <bool GRAD>
    py::cpp_function functional(py::object self, std::optional<double> pare_threshold) {
        // without a graph the functional evaluates the current operator and takes no parameters
        if (circ_ != nullptr) check(mpx_graph_pare(e_, circ_, pare_threshold.has_value() ? *pare_threshold : -1.0), e_);
        struct Snapshot {
            py::object owner; // keeps the propagator (and its engine) alive while the callable lives
            Propagator *p;
            uint64_t init_epoch, graph_epoch;
            size_t layers, n_params;
            std::vector<size_t> mapping;
            std::vector<double> gen;
            std::optional<double> pare;
        };
        auto snap = std::make_shared<Snapshot>(Snapshot{self, this, init_epoch_, graph_epoch_, mapping_.size(),
                                                        n_params_, mapping_, gen_, pare_threshold});
        return py::cpp_function([snap](const std::vector<double> &params) -> py::object {
            Propagator &p = *snap->p;
            if (p.init_epoch_ != snap->init_epoch)
                throw StaleFunctionalGraph("MP object has been modified since the functional was created. The initial "
                                           "operator was re-weighted, so the coefficients the functional snapshotted "
                                           "are stale; create a new functional.");
            if (params.size() != snap->n_params)
                throw ValidationError("Invalid functional call. Parameter length " + std::to_string(params.size()) +
                                      " does not match the expected number of parameters " +
                                      std::to_string(snap->n_params) + ".");
            const size_t now = p.circ_ != nullptr ? p.mapping_.size() : 0;
            if (now != snap->layers || p.graph_epoch_ != snap->graph_epoch)
                throw StaleFunctionalGraph("MP object has been modified since the functional was created. Previous "
                                           "number of graph layers was " + std::to_string(snap->layers) +
                                           " and now is " + std::to_string(now) + ".");
            if (snap->layers == 0) { // no graph: the current operator
                double ev = 0.0;
                check(mpx_expectation(p.e_, &ev), p.e_);
                if constexpr (!GRAD) return py::float_(ev);
                else return py::make_tuple(ev, std::vector<double>{});
            }
            std::vector<double> angles(snap->mapping.size());
            for (size_t l = 0; l < angles.size(); ++l) angles[l] = params[snap->mapping[l]] * snap->gen[l];
            check(mpx_circuit_set_angles(p.e_, p.circ_, angles.data()), p.e_);
            check(mpx_graph_pare(p.e_, p.circ_, snap->pare.has_value() ? *snap->pare : -1.0), p.e_);
            double ev = 0.0;
            if constexpr (!GRAD) {
                {
                    py::gil_scoped_release nogil;
                    check(mpx_graph_expectation(p.e_, p.circ_, &ev), p.e_);
                }
                return py::float_(ev);
            }
            else {
                std::vector<double> ga(snap->mapping.size());
                {
                    py::gil_scoped_release nogil;
                    check(mpx_graph_gradient(p.e_, p.circ_, 0, &ev, ga.data()), p.e_);
                }
                std::vector<double> grad(snap->n_params, 0.0);
                for (size_t l = 0; l < ga.size(); ++l) grad[snap->mapping[l]] += snap->gen[l] * ga[l];
                return py::make_tuple(ev, grad);
            }
        });
    }

    // update_initial_operator (binder.h:153-156; MonomialPropagator.inl:352-376, MPOperator.h:193-232): every
    // term must already be in the store (else OperatorTermNotFound); the operator becomes op_dict at those
    // terms and zero elsewhere, the empty monomial replaces the core term, and earlier functionals go stale.
    void update_initial_operator(const OperatorDict &op_dict) {
        std::vector<uint64_t> keys;
        std::vector<double> coefs;
        std::vector<const std::vector<size_t> *> order;
        bool has_core = false;
        double core = core_;
        for (const auto &[indices, c] : op_dict) {
            std::vector<uint64_t> k(kWords, 0);
            encode(indices, 2 * logical_, k.data());
            const double enc = encode_coeff(indices.size(), c);
            if (indices.empty()) {
                has_core = true;
                core = enc;
                continue;
            }
            keys.insert(keys.end(), k.begin(), k.end());
            coefs.push_back(enc);
            order.push_back(&indices);
        }
        uint64_t missing = ~0ULL;
        const mpx_status st = mpx_update_initial_operator(e_, keys.empty() ? nullptr : keys.data(),
                                                          coefs.empty() ? nullptr : coefs.data(), coefs.size(),
                                                          has_core ? 1 : 0, core, &missing);
        if (st == MPX_ERR_STATE && missing < order.size()) {
            std::string repr = "[";
            for (size_t i = 0; i < order[missing]->size(); ++i)
                repr += (i ? ", " : "") + std::to_string((*order[missing])[i]);
            throw OperatorTermNotFound("Operator term " + repr + "] not found in the operator.");
        }
        check(st, e_);
        if (has_core) core_ = core;
        ++init_epoch_;
    }

    // parameter_mapping (binder.h:242-246; MonomialPropagator.inl:810-850): per graph layer in circuit order;
    // assigning accepts one entry per layer or one per gate and re-wires the graph's parameters.
    std::vector<size_t> parameter_mapping() const { return circ_ != nullptr ? mapping_ : std::vector<size_t>{}; }
    void set_parameter_mapping(const std::vector<size_t> &pm) {
        const size_t count = circ_ != nullptr ? mapping_.size() : 0, gates = n_gates();
        if (pm.size() == count) {
            if (count == 0) return;
            mapping_ = pm;
        }
        else if (pm.size() == gates) {
            for (size_t l = 0; l < count; ++l) mapping_[l] = pm[gate_of_layer_[l]];
        }
        else {
            throw GraphStateConflict("parameter_mapping has " + std::to_string(pm.size()) + " entries; expected " +
                                     std::to_string(count) + " (per graph layer) or " + std::to_string(gates) +
                                     " (per gate).");
        }
        n_params_ = 0;
        for (size_t m : mapping_) n_params_ = std::max(n_params_, m + 1);
    }

    // graph_size (binder.h:232-234; MonomialPropagator.h:103-104): (cos-only indices, cycles)
    std::pair<size_t, size_t> graph_size() {
        uint64_t layers = 0, pairs = 0, cos_only = 0;
        check(mpx_graph_info(e_, &layers, &pairs, &cos_only), e_);
        if (circ_ == nullptr) return {0, 0};
        return {cos_only, pairs};
    }

    mpx_memory_info memory() {
        mpx_memory_info m{};
        check(mpx_memory(e_, &m), e_);
        return m;
    }

    // operator_memory_breakdown (binder.h:257-273) with the reference's keys, filled from the device store:
    // operator_terms = keys, op_coeffs = coefficients (both at capacity), indexing = the hash table,
    // inverted_index = the bit-column index, init_operator = the initial operator; the reference-state
    // scores are computed on the fly (state_coeffs 0); d_* are diagnostics outside total_bytes.
    std::map<std::string, size_t> operator_memory_breakdown() {
        const mpx_memory_info m = memory();
        std::map<std::string, size_t> b{{"operator_terms_bytes", m.key_bytes},
                                        {"op_coeffs_bytes", m.coef_bytes},
                                        {"state_coeffs_bytes", 0},
                                        {"indexing_bytes", m.table_bytes},
                                        {"init_operator_bytes", m.initial_bytes},
                                        {"initial_state_bytes", state_.size() * sizeof(size_t)},
                                        {"inverted_index_bytes", m.column_bytes}};
        size_t total = 0;
        for (const auto &[k, v] : b) total += v;
        b["total_bytes"] = total;
        b["d_invidx_dense_bytes"] = m.column_bytes;
        b["d_invidx_sparse_bytes"] = 0;
        b["d_invidx_dense_columns"] = 64 * kWords + 1;
        b["d_terms_slack_bytes"] = (m.capacity - m.terms) * 8 * kWords;
        b["d_state_coeffs_nonzero"] = 0;
        b["d_scratch_bytes"] = m.scratch_bytes;
        return b;
    }
    size_t graph_memory_bytes() { return circ_ != nullptr ? memory().graph_bytes : 0; }

    // __deepcopy__ (binder.h:113-116): a second engine with a copy of the store, settings, re-weighted
    // initial operator and graph (the reference shares the immutable graph cores; here they are copied).
    std::unique_ptr<Propagator> deepcopy() const {
        std::unique_ptr<Propagator> p(new Propagator(*this, 0));
        check(mpx_clone(e_, circ_, &p->e_, circ_ != nullptr ? &p->circ_ : nullptr), e_);
        return p;
    }

    // Expectation: with no parameters the current operator's (MPFunctions.cpp:196-205); with parameters the
    // stored graph replayed at them (.inl:1035-1041).
    double expectation_value(const std::vector<double> &parameters) {
        double ev = 0.0;
        if (parameters.empty()) {
            check(mpx_expectation(e_, &ev), e_);
            return ev;
        }
        set_graph_parameters(parameters);
        py::gil_scoped_release nogil;
        check(mpx_graph_expectation(e_, circ_, &ev), e_);
        return ev;
    }

    // (<O>, d<O>/d theta) of the stored graph at `parameters` (.inl:1044-1050, MPFunctions.cpp:207-246);
    // without a graph, the current operator's <O> and an empty gradient.
    std::pair<double, std::vector<double>> expectation_value_and_gradient(const std::vector<double> &parameters) {
        if (circ_ == nullptr) {
            if (!parameters.empty())
                throw GraphStateConflict("expectation_value_and_gradient(parameters) needs a stored graph (build_graph)");
            return {expectation_value(parameters), {}};
        }
        set_graph_parameters(parameters);
        std::vector<double> ga(mapping_.size());
        double ev = 0.0;
        {
            py::gil_scoped_release nogil;
            check(mpx_graph_gradient(e_, circ_, 0, &ev, ga.data()), e_);
        }
        std::vector<double> grad(n_params_, 0.0);
        for (size_t l = 0; l < mapping_.size(); ++l) grad[mapping_[l]] += gen_[l] * ga[l];
        return {ev, grad};
    }

    // contract_partially (MonomialPropagator.inl:1053-1097): the stored graph replayed at `parameters`, as
    // raw coefficients in store order, core term excluded; with no parameters, the current coefficients.
    // inplace consumes the graph: the engine keeps the replayed operator and a plain propagate may follow.
    std::vector<double> contract_partially(const std::vector<double> &parameters, bool inplace) {
        if (!parameters.empty()) {
            if (circ_ == nullptr)
                throw GraphStateConflict("contract_partially(parameters) needs a stored graph (build_graph)");
            expectation_value(parameters); // the engine now holds the graph replayed at `parameters`
        }
        uint64_t n = 0;
        check(mpx_size(e_, &n), e_);
        std::vector<uint64_t> words(n * kWords);
        std::vector<double> coefs(n);
        uint64_t got = 0;
        check(mpx_export(e_, words.data(), coefs.data(), n, &got), e_);
        if (inplace && circ_ != nullptr) {
            mpx_circuit_destroy(circ_);
            circ_ = nullptr;
            mapping_.clear();
            gen_.clear();
            gate_of_layer_.clear();
            n_params_ = 0;
            gates_ = 0;
            ++graph_epoch_;
        }
        return coefs;
    }

    size_t graph_layers() const { return circ_ != nullptr ? mapping_.size() : 0; }
    size_t n_gates() const { return circ_ != nullptr ? gates_ : 0; }

    // {indices: coefficient} of the evolved operator, |c| >= atol, decoded and rounded to 1e-12, with the
    // core term added (binder.h:200-221, MonomialPropagator.inl:1099-1127).
    py::dict evolved_operator(const std::vector<double> &parameters, double atol) {
        if (!parameters.empty()) {
            if (circ_ == nullptr)
                throw GraphStateConflict("evolved_operator(parameters) needs a stored graph; after propagate() call "
                                         "it with no parameters.");
            expectation_value(parameters); // the engine now holds the graph replayed at `parameters`
        }
        uint64_t n = 0;
        check(mpx_size(e_, &n), e_);
        std::vector<uint64_t> words(n * kWords);
        std::vector<double> coefs(n);
        uint64_t got = 0;
        check(mpx_export(e_, words.data(), coefs.data(), n, &got), e_);
        py::dict out;
        for (uint64_t i = 0; i < n; ++i) {
            if (std::abs(coefs[i]) < atol) continue;
            std::vector<size_t> idx = decode(words.data() + i * kWords);
            std::complex<double> c = cfg_.basis == MPX_BASIS_PAULI ? std::complex<double>(coefs[i], 0.0)
                                                                   : coefs[i] * hermitian_phase(idx.size());
            c = {std::round(c.real() * 1e12) / 1e12, std::round(c.imag() * 1e12) / 1e12};
            py::list key;
            for (size_t s : idx) key.append(s);
            out[py::tuple(key)] = c;
        }
        if (!cfg_.has_schrodinger && std::abs(core_) >= atol) out[py::tuple()] = std::complex<double>(core_, 0.0);
        return out;
    }

    size_t size() {
        uint64_t n = 0;
        check(mpx_size(e_, &n), e_);
        return n;
    }

    unsigned int cutoff() const { return cfg_.cutoff; }
    void set_cutoff(unsigned int c) {
        check(mpx_set_cutoff(e_, c), e_);
        cfg_.cutoff = c;
    }
    std::optional<double> lower_atol() const {
        return cfg_.has_lower_atol ? std::optional<double>(cfg_.lower_atol) : std::nullopt;
    }
    void set_lower_atol(std::optional<double> v) {
        check(mpx_set_lower_atol(e_, v.has_value(), v.value_or(0.0)), e_);
        cfg_.has_lower_atol = v.has_value();
        cfg_.lower_atol = v.value_or(0.0);
    }
    std::optional<double> upper_atol() const {
        return cfg_.has_upper_atol ? std::optional<double>(cfg_.upper_atol) : std::nullopt;
    }
    void set_upper_atol(std::optional<double> v) {
        check(mpx_set_upper_atol(e_, v.has_value(), v.value_or(0.0)), e_);
        cfg_.has_upper_atol = v.has_value();
        cfg_.upper_atol = v.value_or(0.0);
    }
    std::string cutoff_type() const { return cfg_.cutoff_type == MPX_CUTOFF_SUPPORT ? "support" : "length"; }
    // cutoff_type setter (binder.h:176-184, update_cutoff_type): same validation as the constructor
    void set_cutoff_type(const std::string &t) {
        const int code = cutoff_type_code(t);
        if (cfg_.basis == MPX_BASIS_PAULI && code != MPX_CUTOFF_SUPPORT)
            throw CutoffConfigError("Pauli basis requires cutoff_type == Support (Length has no Pauli-weight meaning "
                                    "under the Pauli encoding).");
        check(mpx_set_cutoff_type(e_, code), e_);
        cfg_.cutoff_type = code;
    }
    std::string basis() const { return cfg_.basis == MPX_BASIS_PAULI ? "pauli" : "majorana"; }
    bool schrodinger() const { return cfg_.has_schrodinger != 0; }
    size_t num_modes() const { return logical_; }
    double core_term() const { return core_; }
    size_t operator_memory_bytes() { return operator_memory_breakdown().at("total_bytes"); }
    uintptr_t engine_handle() const { return reinterpret_cast<uintptr_t>(e_); }

private:
    void encode_circuit(const std::vector<std::vector<size_t>> &majoranas, const std::vector<size_t> &parameter_mapping,
                        const std::vector<double> &gen_coeffs, const std::vector<double> &parameters,
                        std::vector<uint64_t> &words, std::vector<double> &angles) const {
        const size_t L = majoranas.size();
        // validate_coefficient_lengths and validate_parameters_length (Validation.cpp:50-90)
        if (parameter_mapping.size() != gen_coeffs.size())
            throw ValidationError("The length of parameter_mapping and gen_coeffs must be the same.");
        if (!parameter_mapping.empty()) {
            const size_t expected = *std::max_element(parameter_mapping.begin(), parameter_mapping.end()) + 1;
            if (parameters.size() != expected)
                throw ValidationError("The length of parameters (" + std::to_string(parameters.size()) +
                                      ") must be the same as max(parameter_mapping)+1 (" + std::to_string(expected) +
                                      ").");
        }
        if (parameter_mapping.size() != L)
            throw std::invalid_argument("majoranas (" + std::to_string(L) + "), parameter_mapping (" +
                                        std::to_string(parameter_mapping.size()) + ") and gen_coeffs (" +
                                        std::to_string(gen_coeffs.size()) + ") must have the same length.");
        words.assign(L * kWords, 0);
        angles.assign(L, 0.0);
        for (size_t l = 0; l < L; ++l) {
            if (parameter_mapping[l] >= parameters.size())
                throw std::invalid_argument("parameter_mapping[" + std::to_string(l) + "] = " +
                                            std::to_string(parameter_mapping[l]) + " is out of range for " +
                                            std::to_string(parameters.size()) + " parameters.");
            encode(majoranas[l], 2 * logical_, words.data() + l * kWords);
            angles[l] = parameters[parameter_mapping[l]] * gen_coeffs[l];
        }
    }

    // The stored graph at `parameters`, unpared (validate_parameters_length, Validation.cpp:75-90).
    void set_graph_parameters(const std::vector<double> &parameters) {
        if (circ_ == nullptr) throw GraphStateConflict("no stored graph: call build_graph first");
        if (parameters.size() != n_params_)
            throw ValidationError("The length of parameters (" + std::to_string(parameters.size()) +
                                  ") must be the same as max(parameter_mapping)+1 (" + std::to_string(n_params_) +
                                  ").");
        std::vector<double> angles(mapping_.size());
        for (size_t l = 0; l < mapping_.size(); ++l) angles[l] = parameters[mapping_[l]] * gen_[l];
        check(mpx_circuit_set_angles(e_, circ_, angles.data()), e_);
        check(mpx_graph_pare(e_, circ_, -1.0), e_);
    }

    // validate_gate_indices (Validation.cpp:56-75): one entry per monomial, contiguous runs from 0.
    static void validate_gate_indices(const std::vector<size_t> &gi, size_t n) {
        if (gi.size() != n)
            throw ValidationError("gate_indices has " + std::to_string(gi.size()) + " entries but there are " +
                                  std::to_string(n) + " monomials.");
        if (gi.empty()) return;
        if (gi.front() != 0) throw ValidationError("gate_indices must start at 0; got " + std::to_string(gi.front()) + ".");
        for (size_t i = 1; i < gi.size(); ++i)
            if (gi[i] != gi[i - 1] && gi[i] != gi[i - 1] + 1)
                throw ValidationError("gate_indices must be contiguous runs from 0 (each entry equal to the previous "
                                      "or previous+1); got a jump from " + std::to_string(gi[i - 1]) + " to " +
                                      std::to_string(gi[i]) + " at position " + std::to_string(i) + ".");
    }

    // MSb0 slot layout: slot s -> bit 2*Tier-1-s (AlgebraCommon.h:45-65); `limit` bounds the slot index.
    static void encode(const std::vector<size_t> &slots, size_t limit, uint64_t *out) {
        for (size_t s : slots) {
            if (s >= limit)
                throw std::invalid_argument("Majorana index " + std::to_string(s) +
                                            " is out of range; must be less than " + std::to_string(limit) + ".");
            const size_t b = 2 * Tier - 1 - s;
            out[b / 64] ^= 1ULL << (b % 64);
        }
    }
    static std::vector<size_t> decode(const uint64_t *k) {
        std::vector<size_t> out;
        for (size_t w = 0; w < kWords; ++w)
            for (uint64_t x = k[w]; x != 0; x &= x - 1) out.push_back(2 * Tier - 1 - (64 * w + __builtin_ctzll(x)));
        std::sort(out.begin(), out.end());
        return out;
    }
    double encode_coeff(size_t weight, std::complex<double> c) const {
        if (cfg_.basis == MPX_BASIS_PAULI) {
            if (std::abs(c.imag()) > 1e-10) throw std::runtime_error("Non-real Pauli coeffs detected");
            return c.real();
        }
        const std::complex<double> e = c / hermitian_phase(weight);
        if (std::abs(e.imag()) > 1e-10) throw std::runtime_error("Non-Hermitian coeffs detected");
        return e.real();
    }
    static void check(mpx_status s, const mpx_engine *e) {
        if (s == MPX_OK) return;
        const std::string msg = mpx_last_error(e);
        if (s == MPX_ERR_INVALID) throw std::invalid_argument(msg);
        throw std::runtime_error(msg);
    }

    mpx_config cfg_{};
    std::optional<std::vector<std::vector<size_t>>> basis_change_;
    size_t logical_;
    std::vector<size_t> state_;
    double core_ = 0.0;
    mpx_engine *e_ = nullptr;
    mpx_circuit *circ_ = nullptr; // the stored graph's circuit (build_graph)
    std::vector<size_t> mapping_;
    std::vector<double> gen_;
    std::vector<size_t> gate_of_layer_;
    size_t n_params_ = 0, gates_ = 0;
    uint64_t init_epoch_ = 0;  // bumped by update_initial_operator (functionals made before go stale)
    uint64_t graph_epoch_ = 0; // bumped by build_graph and contract_partially(inplace=True)

    // For __deepcopy__: the host-side state of `o`; the caller fills e_ (and circ_) with engine copies.
    Propagator(const Propagator &o, int)
        : cfg_(o.cfg_), basis_change_(o.basis_change_), logical_(o.logical_), state_(o.state_), core_(o.core_),
          mapping_(o.mapping_), gen_(o.gen_), gate_of_layer_(o.gate_of_layer_), n_params_(o.n_params_),
          gates_(o.gates_), init_epoch_(o.init_epoch_), graph_epoch_(o.graph_epoch_) {}
};

template <size_t Tier>
void bind(py::module_ &m) {
    using P = Propagator<Tier>;
    char name[32];
    std::snprintf(name, sizeof name, "MonomialPropagator%03zu", Tier);
    py::class_<P>(m, name)
        .def(py::init<const OperatorDict &, unsigned int, const std::vector<size_t> &, py::object,
                      std::optional<unsigned int>, std::optional<double>, std::optional<double>, const std::string &,
                      std::optional<std::vector<std::vector<size_t>>>, size_t, const std::string &, size_t>(),
             py::arg("initial_operator"), py::arg("cutoff"), py::arg("initial_state"), py::arg("comm") = py::none(),
             py::arg("schrodinger_cutoff") = py::none(), py::arg("lower_atol") = py::none(),
             py::arg("upper_atol") = py::none(), py::arg("cutoff_type") = "length",
             py::arg("basis_change") = py::none(), py::arg("logical_num_modes") = Tier, py::arg("basis") = "majorana",
             py::arg("partitions") = 0)
        .def("propagate", &P::propagate, py::arg("majoranas"), py::arg("parameter_mapping"), py::arg("gen_coeffs"),
             py::arg("parameters"), py::arg("only_rotate_len_k") = py::none())
        .def("build_graph", &P::build_graph, py::arg("majoranas"), py::arg("parameter_mapping"), py::arg("gen_coeffs"),
             py::arg("gate_indices") = py::none(), py::arg("parameters") = py::none(),
             py::arg("only_rotate_len_k") = py::none())
        .def("expectation_value", &P::expectation_value, py::arg("parameters"))
        .def("expectation_value_and_gradient", &P::expectation_value_and_gradient, py::arg("parameters"))
        .def("evolved_operator", &P::evolved_operator, py::arg("parameters"), py::arg("atol"))
        .def("size", &P::size)
        .def("contract_partially", &P::contract_partially, py::arg("parameters"), py::arg("inplace"))
        .def("graph_size", &P::graph_size)
        .def("graph_memory_bytes", &P::graph_memory_bytes)
        .def("operator_memory_breakdown", &P::operator_memory_breakdown)
        .def("update_initial_operator", &P::update_initial_operator, py::arg("op_dict"))
        .def(
            "expectation_value_functional",
            [](py::object self, std::optional<double> pare_threshold) {
                return self.cast<P &>().template functional<false>(self, pare_threshold);
            },
            py::arg("pare_threshold") = py::none())
        .def(
            "expectation_value_and_gradient_functional",
            [](py::object self, std::optional<double> pare_threshold) {
                return self.cast<P &>().template functional<true>(self, pare_threshold);
            },
            py::arg("pare_threshold") = py::none())
        .def("__deepcopy__", [](const P &self, py::object) { return self.deepcopy(); }, py::arg("memo") = py::none())
        .def_property("parameter_mapping", &P::parameter_mapping, &P::set_parameter_mapping)
        .def("graph_layers", &P::graph_layers)
        .def("n_gates", &P::n_gates)
        .def("operator_memory_bytes", &P::operator_memory_bytes)
        .def("core_term", &P::core_term)
        .def("_engine_handle", &P::engine_handle)
        .def_property("cutoff", &P::cutoff, &P::set_cutoff)
        .def_property("lower_atol", &P::lower_atol, &P::set_lower_atol)
        .def_property("upper_atol", &P::upper_atol, &P::set_upper_atol)
        .def_property("cutoff_type", &P::cutoff_type, &P::set_cutoff_type)
        .def_property("basis_change", &P::basis_change, &P::set_basis_change)
        .def_property_readonly("basis", &P::basis)
        .def_property_readonly("num_modes", &P::num_modes)
        .def_property_readonly("schrodinger", [](P &p) { return p.schrodinger(); })
        .def_property_readonly_static("storage_num_modes", [](py::object) { return Tier; });
}

}  // namespace

PYBIND11_MODULE(_core, m) {
    m.doc() = "B200 propagation engine: per-tier MonomialPropagatorNNN classes over the mpx C ABI";
    py::register_exception<NotSupported>(m, "NotSupportedError", PyExc_NotImplementedError);
    py::register_exception<GraphStateConflict>(m, "GraphStateConflict", PyExc_RuntimeError);
    py::register_exception<PropagatorConfigError>(m, "PropagatorConfigError", PyExc_RuntimeError);
    py::register_exception<CutoffConfigError>(m, "CutoffConfigError", PyExc_ValueError);
    py::register_exception<ValidationError>(m, "ValidationError", PyExc_RuntimeError);
    py::register_exception<StaleFunctionalGraph>(m, "StaleFunctionalGraph", PyExc_RuntimeError);
    py::register_exception<OperatorTermNotFound>(m, "OperatorTermNotFound", PyExc_RuntimeError);
    bind<32>(m);
    bind<64>(m);
    bind<96>(m);
    bind<128>(m);
    bind<160>(m);
    bind<192>(m);
    bind<224>(m);
    bind<256>(m);
    // Module helpers of the reference (MajoranaAlgebra.h:45-51): a weight-w Majorana monomial is
    // anti-Hermitian iff C(w,2) is odd; the generator correction is i^(C(w,2)+1).
    m.def(
        "is_antihermitian", [](const std::vector<size_t> &idx) { return ((idx.size() * (idx.size() - 1) / 2) & 1) != 0; },
        py::arg("indices"));
    m.def(
        "antihermitian_generator_correction",
        [](const std::vector<size_t> &idx) {
            return hermitian_phase(idx.size()) * std::complex<double>(0.0, 1.0);
        },
        py::arg("indices"));
    m.attr("MAX_NUM_MODES") = 256;
    m.attr("has_mpi") = false;
    m.attr("__build_type__") = "Release";
    m.attr("__variant__") = "b200";
    m.attr("__compiler_flags__") = "nvcc -gencode arch=compute_100a,code=sm_100a -O3";
}
