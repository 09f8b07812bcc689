// MRG32k3a draws for callers that cannot allocate device memory.
//
// casim_b200_debug_rng stages the draws in a buffer it obtains with
// cudaMalloc. Some callers cannot let a library allocate: code running inside
// another framework's memory pool or a fixed-budget real-time host, or a
// process that must not grow its device footprint after start-up. This file
// gives them the same generator with its staging buffer in a fixed device
// array of CB_STATIC_RNG_MAX doubles (2 MiB), which every GPU that loads the
// library holds until the process exits.
#include <cuda_runtime.h>

#include <string>

#include "../../include/casim_b200.h"
#include "mrg32k3a.cuh"

void cb_set_create_error(const std::string& msg);  // capi.cu

namespace {

constexpr int64_t CB_STATIC_RNG_MAX = 262144;  // draws per call (2 MiB of doubles)

// One staging array per device, shared by every call on that device.
__device__ __align__(256) double g_rng_scratch[CB_STATIC_RNG_MAX];

__global__ void k_rng_static(cbrng::State g, long long n, double* out) {
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (long long k = 0; k < n; ++k) out[k] = cbrng::u01d(g);
}

casim_status fail(casim_status s, const std::string& msg) {
    cb_set_create_error(msg);
    return s;
}

}  // namespace

extern "C" casim_status casim_b200_rng_draws_static(const uint32_t seed[6], int64_t n, double* out) {
    if (!seed || !out || n < 0) return fail(CASIM_EINVAL, "rng_draws_static: null pointer or negative count");
    if (n > CB_STATIC_RNG_MAX)
        return fail(CASIM_EINVAL, "rng_draws_static: " + std::to_string(n) + " draws exceed the fixed scratch of " +
                                      std::to_string(CB_STATIC_RNG_MAX));
    {
        // RngStream's CheckSeed rules (CaSim/rngstream.cpp:200-234)
        const uint64_t s6[6] = {seed[0], seed[1], seed[2], seed[3], seed[4], seed[5]};
        if (!cbrng::seed_ok(s6)) return fail(CASIM_EINVAL, "rng_draws_static: not a valid MRG32k3a seed");
    }
    if (n == 0) return CASIM_OK;
    // The host-side name of the array is only a stand-in: its device address is
    // looked up on every call, with the calling thread's current device, so a
    // context that was torn down and rebuilt (cudaDeviceReset) never leaves a
    // stale address behind. The lookup is a host-side table read.
    double* scratch = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&scratch, g_rng_scratch);
    if (e != cudaSuccess) return fail(CASIM_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    cbrng::State g;
    for (int i = 0; i < 6; ++i) g.s[i] = seed[i];
    // every element read back below is written by this launch first, so the
    // contents left by an earlier call need no clearing
    k_rng_static<<<1, 1>>>(g, n, scratch);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(out, scratch, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(CASIM_ECUDA, std::string("rng_draws_static: ") + cudaGetErrorString(e));
    return CASIM_OK;
}
