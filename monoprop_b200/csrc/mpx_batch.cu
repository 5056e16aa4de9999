// mpx_batch.cu -- many independent propagation problems (observables, parameter sets, circuits of uneven
// depth) on one GPU at once.
//
// The reference runs one propagator per process. Here a batch is spread over `workers` host threads,
// each driving its own engine and CUDA stream, so the per-gate kernels of different instances run
// concurrently on the GPU: small or shallow instances, which cannot fill 148 SMs alone, share the
// machine, and the deepest instances start first (longest-processing-time order) so the tail is short.
// Device memory is bounded by planned admission: an instance starts only while the expected footprints of
// the running instances fit the free memory measured at the start (expectations learned from the
// instances already finished, see Admission); an allocation failure that still happens waits until
// another worker finishes and retries; only an instance that cannot fit on an otherwise idle GPU is an
// error.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mpx.h"

// Defined in mpx_engine.cu, not exported: mpx_create for an engine that shares the GPU with other
// engines of a batch (plain pool allocations from its first buffer on, no programmatic dependent launch).
extern "C" mpx_status mpx_internal_create_shared(const mpx_config *cfg, const uint64_t *obs_words,
                                                 const double *obs_coef, uint64_t n_obs, double core,
                                                 const uint64_t *state_mask, mpx_engine **out);

namespace {

// Memory admission. Instances start only while the device memory the running ones are expected to need
// fits a budget (the free memory when the batch starts, less a margin). An instance's expectation comes
// from the instances already finished: the largest measured footprint among those at least as deep
// (instances run deepest first, so this is an upper bound by depth), or, before any has finished, an equal
// share of the budget per worker. An allocation failure still waits for a release and retries.
struct Admission {
    uint64_t budget = 0;                          // bytes; 0 = no planning (free memory unknown)
    uint64_t reserved = 0;                        // expected bytes of the running instances
    std::vector<std::pair<uint64_t, uint64_t>> seen; // (layers, measured bytes) of finished instances
    uint64_t fair_share = 0;

    uint64_t expect(uint64_t layers) const {
        uint64_t best = 0;
        bool any = false;
        for (const auto &[l, b] : seen)
            if (l >= layers) {
                best = std::max(best, b);
                any = true;
            }
        return any ? best : fair_share;
    }
};

struct BatchState {
    std::mutex mu;
    std::condition_variable cv;
    int in_flight = 0;
    uint64_t completions = 0;
    std::atomic<uint64_t> next{0};
    std::atomic<bool> failed{false};
    mpx_status status = MPX_OK;
    std::string error;
    Admission adm;
};

// Device bytes an engine holds at the end of its instance (store, table, columns, scratch, graph), with
// the gradient's checkpoints and tape on top when it ran one.
uint64_t footprint(mpx_engine *e, bool gradient) {
    mpx_memory_info m{};
    if (mpx_memory(e, &m) != MPX_OK) return 0;
    const uint64_t b = m.key_bytes + m.coef_bytes + m.table_bytes + m.column_bytes + m.scratch_bytes + m.initial_bytes +
                       m.graph_bytes;
    return gradient ? 2 * b : b + b / 4;
}

// One instance on a fresh engine (the device memory pool makes engine creation cheap). *bytes: its
// measured footprint.
mpx_status run_one(const mpx_config &cfg, mpx_batch_item &it, const mpx_batch_options &opt, std::string &err,
                   uint64_t *bytes) {
    mpx_engine *e = nullptr;
    mpx_status s = mpx_internal_create_shared(&cfg, it.obs_words, it.obs_coef, it.n_obs, it.core, it.state_mask, &e);
    if (s != MPX_OK) {
        err = mpx_last_error(nullptr);
        return s;
    }
    mpx_circuit *c = nullptr;
    s = mpx_circuit_upload(e, it.gen_words, it.angles, it.n_layers, &c);
    if (s == MPX_OK) {
        if (opt.gradient && it.grad_angles != nullptr) {
            s = mpx_adjoint_forward(e, c, opt.segment_gates, it.expectation);
            if (s == MPX_OK) s = mpx_adjoint_backward(e, c, it.grad_angles);
        }
        else {
            s = mpx_propagate_circuit(e, c);
            if (s == MPX_OK) s = mpx_expectation(e, it.expectation);
        }
        if (s == MPX_OK && it.final_terms != nullptr) s = mpx_size(e, it.final_terms);
        if (s == MPX_OK && it.export_n != nullptr)
            s = mpx_export(e, it.export_words, it.export_coefs, it.export_cap, it.export_n);
    }
    if (s != MPX_OK) err = mpx_last_error(e);
    if (s == MPX_OK && bytes != nullptr) *bytes = footprint(e, opt.gradient && it.grad_angles != nullptr);
    mpx_circuit_destroy(c);
    mpx_destroy(e);
    return s;
}

void worker(const mpx_config &cfg, mpx_batch_item *items, const std::vector<uint64_t> &order,
            const mpx_batch_options &opt, BatchState &bs) {
    if (const cudaError_t ce = cudaSetDevice(cfg.device); ce != cudaSuccess) {
        cudaGetLastError();
        std::lock_guard<std::mutex> lock(bs.mu);
        if (!bs.failed.exchange(true)) {
            bs.status = MPX_ERR_CUDA;
            bs.error = "cannot select device " + std::to_string(cfg.device) + ": " + cudaGetErrorString(ce);
        }
        bs.cv.notify_all();
        return;
    }
    for (;;) {
        if (bs.failed.load()) return;
        const uint64_t k = bs.next.fetch_add(1);
        if (k >= order.size()) return;
        mpx_batch_item &it = items[order[k]];
        for (;;) {
            uint64_t seen, want;
            {
                // admission: wait until the expected footprint fits the budget (or nothing else runs)
                std::unique_lock<std::mutex> lock(bs.mu);
                want = bs.adm.expect(it.n_layers);
                bs.cv.wait(lock, [&] {
                    return bs.adm.budget == 0 || bs.in_flight == 0 || bs.adm.reserved + want <= bs.adm.budget ||
                           bs.failed.load();
                });
                if (bs.failed.load()) return;
                bs.adm.reserved += want;
                ++bs.in_flight;
                seen = bs.completions;
            }
            std::string err;
            uint64_t bytes = 0;
            const mpx_status s = run_one(cfg, it, opt, err, &bytes);
            int others;
            {
                std::lock_guard<std::mutex> lock(bs.mu);
                --bs.in_flight;
                ++bs.completions;
                bs.adm.reserved -= want;
                if (s == MPX_OK && bytes > 0) bs.adm.seen.emplace_back(it.n_layers, bytes);
                others = bs.in_flight;
            }
            bs.cv.notify_all();
            if (s == MPX_OK) break;
            if (s == MPX_ERR_NOMEM && others > 0) {
                // memory admission: retry once some other instance has released its store
                std::unique_lock<std::mutex> lock(bs.mu);
                bs.cv.wait(lock, [&] { return bs.completions > seen + 1 || bs.in_flight == 0 || bs.failed.load(); });
                continue;
            }
            std::lock_guard<std::mutex> lock(bs.mu);
            if (!bs.failed.exchange(true)) {
                bs.status = s;
                bs.error = "instance " + std::to_string(order[k]) + ": " + err;
            }
            bs.cv.notify_all();
            return;
        }
    }
}

}  // namespace

extern "C" {

MPX_API mpx_status mpx_batch_run(const mpx_config *cfg, mpx_batch_item *items, uint64_t n_items,
                                 const mpx_batch_options *opt, char *err, size_t err_len) {
    auto report = [&](mpx_status st, const std::string &msg) {
        if (err != nullptr && err_len > 0) {
            std::strncpy(err, msg.c_str(), err_len - 1);
            err[err_len - 1] = '\0';
        }
        return st;
    };
    if (cfg == nullptr || opt == nullptr || (n_items > 0 && items == nullptr))
        return report(MPX_ERR_INVALID, "NULL argument");
    for (uint64_t i = 0; i < n_items; ++i) {
        const mpx_batch_item &it = items[i];
        if (it.expectation == nullptr || (it.n_layers > 0 && (it.gen_words == nullptr || it.angles == nullptr)) ||
            (it.n_obs > 0 && (it.obs_words == nullptr || it.obs_coef == nullptr)))
            return report(MPX_ERR_INVALID, "batch item " + std::to_string(i) + " has a NULL buffer");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return report(MPX_ERR_NO_DEVICE, "no CUDA device is visible; the engine has no CPU fallback");
    }
    if (cfg->device < 0 || cfg->device >= ndev)
        return report(MPX_ERR_INVALID, "device ordinal " + std::to_string(cfg->device) + " out of range (" +
                                           std::to_string(ndev) + " devices)");
    // deepest first: the longest instances start early, short ones fill in around them
    std::vector<uint64_t> order(n_items);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint64_t a, uint64_t b) { return items[a].n_layers > items[b].n_layers; });
    const int workers = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(opt->workers > 0 ? opt->workers : 8,
                                                                                 std::max<uint64_t>(n_items, 1))));
    BatchState bs;
    {
        // the admission budget: the device's free memory now, less a 10 % margin
        int prev = 0;
        cudaGetDevice(&prev);
        size_t free_b = 0, total_b = 0;
        if (cudaSetDevice(cfg->device) == cudaSuccess && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            bs.adm.budget = free_b - free_b / 10;
            bs.adm.fair_share = bs.adm.budget / static_cast<uint64_t>(workers);
        }
        cudaGetLastError();
        cudaSetDevice(prev);
    }
    std::vector<std::thread> pool;
    pool.reserve(workers);
    for (int w = 0; w < workers; ++w) pool.emplace_back(worker, std::cref(*cfg), items, std::cref(order), std::cref(*opt),
                                                       std::ref(bs));
    for (auto &t : pool) t.join();
    if (bs.failed.load()) return report(bs.status, bs.error);
    return MPX_OK;
}

}  // extern "C"
