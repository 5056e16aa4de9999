// mpx_noalloc.cu -- <0|O|0> over a caller-owned device term store, without any device allocation.
//
// Some callers cannot call cudaMalloc while they run: a host framework that plans and owns every byte
// of device memory up front (an ML or simulation runtime that hands this library pre-sized buffers
// from its own pool) forbids allocations behind its back, and cudaMalloc/cudaFree also synchronise
// the device, stalling the caller's other streams. For them, mpx_expectation_noalloc takes the keys,
// coefficients and output as device pointers and keeps its only scratch -- one fp64 partial sum per
// block -- in the file-scope array below, which lives in the library's device image: every GPU that
// loads libmpx.so holds its 32 KiB until the process exits.
//
// The reduction is the same as the engine's mpx_expectation (MPOperator.h:235-254 scoring,
// PauliAlgebra.h:144-147 / MajoranaAlgebra.h:56-60 phases): core + sum over fully paired keys of
// phase * c. Each block owns a fixed chunk of kNoAllocChunk consecutive terms, so the partial sums and
// the final fixed-order sum do not depend on the device, and n is bounded by
// kNoAllocMaxBlocks * kNoAllocChunk terms.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/mpx.h"
#include "mpx_device.cuh"

namespace {

constexpr uint32_t kNoAllocMaxBlocks = 4096;
constexpr uint64_t kNoAllocChunk = 65536;
constexpr int kMaxDevices = 64;

// The shared scratch. Every call overwrites the partial sum of each block it launches before the final
// kernel reads it, so nothing has to start at zero; calls whose kernels overlap on the GPU (two
// streams, or two host threads) race on this array and must be serialised by the caller.
static __device__ __align__(256) double g_noalloc_partial[kNoAllocMaxBlocks];

// Device address of g_noalloc_partial per device ordinal, looked up once per device (host code cannot
// use the symbol's name as a device pointer: on the host it names a stand-in object).
double *g_partial_addr[kMaxDevices] = {};
std::mutex g_setup_mutex;

template <int W, int BASIS>
__global__ void __launch_bounds__(mpx::kBlock) k_expect_chunked(const uint64_t *__restrict__ keys,
                                                                 const double *__restrict__ coef, uint64_t n,
                                                                 mpx::StateMask sm, double *__restrict__ partial) {
    __shared__ double s_red[mpx::kBlock / 32];
    const uint64_t begin = static_cast<uint64_t>(blockIdx.x) * kNoAllocChunk;
    const uint64_t end = begin + kNoAllocChunk < n ? begin + kNoAllocChunk : n;
    double acc = 0.0;
    for (uint64_t i = begin + threadIdx.x; i < end; i += mpx::kBlock) {
        uint64_t m[W];
        mpx::load_key<W>(keys, i, m);
        uint64_t unpaired = 0;
        int na = 0, pop = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            unpaired |= (m[w] & mpx::kEven) ^ ((m[w] >> 1) & mpx::kEven);
            na += __popcll(m[w] & sm.w[w]);
            pop += __popcll(m[w]);
        }
        if (unpaired == 0) {
            const int odd = BASIS == 1 ? (na & 1) : ((na + pop / 2) & 1);
            const double c = coef[i];
            acc += odd ? -c : c;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xFFFFFFFFu, acc, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < mpx::kBlock / 32; ++w) t += s_red[w];
        partial[blockIdx.x] = t;
    }
}

__global__ void k_expect_chunked_final(const double *__restrict__ partial, uint32_t nblocks, double core,
                                       double *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double t = 0.0;
        for (uint32_t b = 0; b < nblocks; ++b) t += partial[b];
        out[0] = core + t;
    }
}

// Launches through cudaLaunchKernelEx, whose return value is the status of this launch alone: an error
// left pending by the caller's earlier, unrelated work is neither reported as this call's failure nor
// cleared.
template <typename... KArgs, typename... Args>
cudaError_t launch_on(cudaStream_t s, uint32_t blocks, uint32_t threads, void (*kernel)(KArgs...), Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(threads);
    cfg.stream = s;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <int W, int B>
cudaError_t launch(const uint64_t *keys, const double *coef, uint64_t n, const mpx::StateMask &sm, double *partial,
                   uint32_t blocks, cudaStream_t s) {
    return launch_on(s, blocks, mpx::kBlock, &k_expect_chunked<W, B>, keys, coef, n, sm, partial);
}

using LaunchFn = cudaError_t (*)(const uint64_t *, const double *, uint64_t, const mpx::StateMask &, double *,
                                 uint32_t, cudaStream_t);

template <int W>
LaunchFn pick_b(int basis) {
    return basis == MPX_BASIS_PAULI ? &launch<W, 1> : &launch<W, 0>;
}

LaunchFn pick(int W, int basis) {
    switch (W) {
    case 1: return pick_b<1>(basis);
    case 2: return pick_b<2>(basis);
    case 3: return pick_b<3>(basis);
    case 4: return pick_b<4>(basis);
    case 5: return pick_b<5>(basis);
    case 6: return pick_b<6>(basis);
    case 7: return pick_b<7>(basis);
    default: return pick_b<8>(basis);
    }
}

struct ErrBuf {
    char *buf;
    size_t len;
    mpx_status operator()(mpx_status st, const std::string &msg) const {
        if (buf != nullptr && len > 0) {
            std::strncpy(buf, msg.c_str(), len - 1);
            buf[len - 1] = '\0';
        }
        return st;
    }
};

}  // namespace

extern "C" {

MPX_API mpx_status mpx_expectation_noalloc(int32_t basis, uint32_t words, const uint64_t *keys, const double *coefs,
                                           uint64_t n_terms, const uint64_t *state_mask, double core, double *out,
                                           void *stream, char *err, size_t err_len) {
    const ErrBuf nofail{err, err_len};
    if (basis != MPX_BASIS_PAULI && basis != MPX_BASIS_MAJORANA)
        return nofail(MPX_ERR_INVALID, "basis must be MPX_BASIS_PAULI or MPX_BASIS_MAJORANA");
    if (words < 1 || words > static_cast<uint32_t>(mpx::kMaxWords))
        return nofail(MPX_ERR_INVALID, "words must be in [1, 8]");
    if (out == nullptr || (n_terms > 0 && (keys == nullptr || coefs == nullptr)))
        return nofail(MPX_ERR_INVALID, "keys, coefs and out must be device pointers (keys/coefs may be NULL only "
                                       "when n_terms is 0)");
    if (n_terms > static_cast<uint64_t>(kNoAllocMaxBlocks) * kNoAllocChunk)
        return nofail(MPX_ERR_CAPACITY, "n_terms exceeds the allocation-free limit of 268435456 terms "
                                        "(4096 blocks x 65536 terms); use mpx_expectation on an engine instead");
    int dev = -1;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return nofail(MPX_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(ce));
    if (dev < 0 || dev >= kMaxDevices) return nofail(MPX_ERR_INVALID, "device ordinal above 63");
    double *partial = nullptr;
    {
        // First call on this device (which is current here): resolve the scratch array's device address.
        // Callers make this first call before any stream capture on the device begins.
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (g_partial_addr[dev] == nullptr) {
            void *p = nullptr;
            ce = cudaGetSymbolAddress(&p, g_noalloc_partial);
            if (ce != cudaSuccess)
                return nofail(MPX_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce));
            g_partial_addr[dev] = static_cast<double *>(p);
        }
        partial = g_partial_addr[dev];
    }
    mpx::StateMask sm{};
    for (uint32_t w = 0; w < words; ++w) sm.w[w] = state_mask != nullptr ? state_mask[w] : 0ULL;
    const auto s = static_cast<cudaStream_t>(stream);
    const uint32_t blocks = static_cast<uint32_t>((n_terms + kNoAllocChunk - 1) / kNoAllocChunk);
    if (blocks > 0) {
        ce = pick(static_cast<int>(words), basis)(keys, coefs, n_terms, sm, partial, blocks, s);
        if (ce != cudaSuccess)
            return nofail(MPX_ERR_CUDA, std::string("launch of the partial sums: ") + cudaGetErrorString(ce));
    }
    ce = launch_on(s, 1, 32, &k_expect_chunked_final, static_cast<const double *>(partial), blocks, core, out);
    if (ce != cudaSuccess) return nofail(MPX_ERR_CUDA, std::string("launch of the final sum: ") + cudaGetErrorString(ce));
    return MPX_OK;
}

}  // extern "C"
