// Surrogate of the quasi-steady Ca at the RyR mouths: a small MLP
// (n_in -> depth x width, GELU -> n_out) with BF16 weights and activations and
// FP32 accumulation, trained and evaluated on the device by the kernels below.
// It has no counterpart in the reference; the plain RD path of this library
// generates its training snapshots and judges its error.
//
// Every matrix product runs on the 5th-generation tensor cores: one CTA owns a
// 128-row tile of C = A . B^T (A [M x K], B [N x K], both K-major BF16 in HBM),
// stages 128 x 64 and N x 64 slices of A and B in shared memory in the
// canonical no-swizzle K-major layout (8-row x 16-byte core matrices), one
// elected thread issues tcgen05.mma (kind::f16, BF16 inputs, FP32 accumulator
// in TMEM, 128 x N x 16 per instruction) and commits to an mbarrier, and the
// four warps read the accumulator back with tcgen05.ld (lane quarter per warp)
// for a fused epilogue: bias + GELU with BF16 row-major and transposed stores
// (forward), bias only (output layer), GELU' scaling (backward through an
// activation) or a plain FP32 store (weight gradients).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/casim_b200.h"

namespace cbsg {

typedef __nv_bfloat16 bf16;

constexpr int BM = 128;  // rows per CTA (tcgen05 M)
constexpr int BK = 64;   // K slice per pipeline stage (4 instructions of K = 16)
constexpr int THREADS = 128;
constexpr int LBO = 128;               // bytes between K-adjacent core matrices
constexpr int SBO = (BK / 8) * 128;    // bytes between 8-row groups
constexpr int A_STAGE = BM * BK * 2;   // 16 KiB

enum { EPI_HIDDEN = 0, EPI_OUT = 1, EPI_BACK = 2, EPI_PLAIN = 3 };

struct gemm_args {
    const bf16* A;  // [M][K]
    const bf16* B;  // [N][K]
    int M, N, K;
    int BN;         // columns per CTA (grid.y = N / BN)
    int mode;
    const float* bias;  // [N]
    float* C;           // [M][N] FP32 (EPI_OUT, EPI_PLAIN)
    bf16* H;            // [M][N] BF16 (EPI_HIDDEN, EPI_BACK)
    bf16* HT;           // [N][M] BF16, optional
    float* Z;           // [M][N] FP32 pre-activation: written by EPI_HIDDEN (optional), read by EPI_BACK
    int* err;           // set to 1 if an mbarrier wait gave up
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, K-major, no swizzle (version 1 for sm_100)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(LBO >> 4) << 16) | ((uint64_t)(SBO >> 4) << 32) | (1ull << 46);
}

// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// bounded wait for the completion of the phase with the given parity
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (int i = 0; i < (1 << 22); ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}

// one K slice of A (rows m0..m0+127) and B (rows 0..N-1) into a stage, canonical layout
__device__ __forceinline__ void load_stage(const gemm_args& g, int m0, int n0, int k0, uint32_t sa, uint32_t sb) {
    const int tid = threadIdx.x;
    for (int p = tid; p < BM * (BK / 8); p += THREADS) {
        const int r = p >> 3, kk = p & 7;
        cp_async16(sa + (r >> 3) * SBO + kk * LBO + (r & 7) * 16, g.A + (size_t)(m0 + r) * g.K + k0 + kk * 8);
    }
    for (int p = tid; p < g.BN * (BK / 8); p += THREADS) {
        const int r = p >> 3, kk = p & 7;
        cp_async16(sb + (r >> 3) * SBO + kk * LBO + (r & 7) * 16, g.B + (size_t)(n0 + r) * g.K + k0 + kk * 8);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// C = A . B^T with the epilogue g.mode; grid (M / 128, N / BN), BN <= 256 and a multiple
// of 16, K a multiple of 64; dynamic shared memory 2 * (16 KiB + BN * 128 B)
__global__ void __launch_bounds__(THREADS, 1) k_gemm(const __grid_constant__ gemm_args g) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * g.BN;
    const int ncols = g.BN <= 32 ? 32 : g.BN <= 64 ? 64 : g.BN <= 128 ? 128 : 256;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t b_stage = (uint32_t)g.BN * (BK / 8) * 16;
    const uint32_t sa[2] = {sbase, sbase + A_STAGE + b_stage};
    const uint32_t sb[2] = {sbase + A_STAGE, sbase + 2 * A_STAGE + b_stage};

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)), "r"(ncols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = idesc_bf16(g.BN);
    const int kt = g.K / BK;
    bool ok = true;

    load_stage(g, m0, n0, 0, sa[0], sb[0]);
    for (int i = 0; i < kt; ++i) {
        const int s = i & 1;
        asm volatile("cp.async.wait_all;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // make the slice visible to the tensor core
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int j = 0; j < BK / 16; ++j)
                mma_bf16(tmem, sdesc(sa[s] + j * 2 * LBO), sdesc(sb[s] + j * 2 * LBO), idesc, (i > 0 || j > 0) ? 1u : 0u);
            mma_commit(&bars[s]);
        }
        if (i + 1 < kt) {
            const int s2 = (i + 1) & 1;
            if (i >= 1) ok = mbar_wait(&bars[s2], (uint32_t)(((i - 1) >> 1) & 1)) && ok;  // slice i-1 consumed
            load_stage(g, m0, n0, (i + 1) * BK, sa[s2], sb[s2]);
        }
    }
    ok = mbar_wait(&bars[(kt - 1) & 1], (uint32_t)(((kt - 1) >> 1) & 1)) && ok;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok && g.err) atomicExch(g.err, 1);

    // epilogue: warp w reads TMEM lanes 32w..32w+31 = rows m0 + 32w + lane
    const int row = m0 + warp * 32 + lane;
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < g.BN; c0 += 8) {
        uint32_t r[8];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                     : "r"(taddr + c0));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = __uint_as_float(r[j]);
        if (!ok) continue;
        const int cg = n0 + c0;  // global column
        const size_t o = (size_t)row * g.N + cg;
        if (g.mode == EPI_PLAIN) {
#pragma unroll
            for (int j = 0; j < 8; ++j) g.C[o + j] = v[j];
        } else if (g.mode == EPI_OUT) {
#pragma unroll
            for (int j = 0; j < 8; ++j) g.C[o + j] = v[j] + g.bias[cg + j];
        } else {
            __align__(16) bf16 h[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                float y;
                if (g.mode == EPI_HIDDEN) {
                    const float z = v[j] + g.bias[cg + j];
                    if (g.Z) g.Z[o + j] = z;
                    y = gelu(z);
                } else {  // EPI_BACK: gradient w.r.t. the pre-activation
                    y = v[j] * gelu_grad(g.Z[o + j]);
                }
                h[j] = __float2bfloat16_rn(y);
            }
            *(uint4*)(g.H + o) = *(const uint4*)h;
            if (g.HT)
#pragma unroll
                for (int j = 0; j < 8; ++j) g.HT[(size_t)(cg + j) * g.M + row] = h[j];
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

// X FP32 [B][n_in] -> BF16 [B][ld] (zero padded) and its transpose [ld][B]
__global__ void k_cast_in(const float* __restrict__ x, int B, int n_in, int ld, bf16* __restrict__ xb, bf16* __restrict__ xt) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * ld) return;
    const int r = (int)(i / ld), c = (int)(i - (long long)r * ld);
    const bf16 v = __float2bfloat16_rn(c < n_in ? x[(size_t)r * n_in + c] : 0.0f);
    xb[i] = v;
    if (xt) xt[(size_t)c * B + r] = v;
}

// mean-square loss over the first n_out columns; gradient 2 (y - t) / (B n_out) as BF16
// (row-major and transposed); per-block partial sums of the squared error
__global__ void k_mse(const float* __restrict__ y, int ldy, const float* __restrict__ t, int B, int n_out, bf16* __restrict__ dz,
                      bf16* __restrict__ dzt, float* __restrict__ partial) {
    __shared__ float red[256];
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    float se = 0;
    if (i < (long long)B * ldy) {
        const int r = (int)(i / ldy), c = (int)(i - (long long)r * ldy);
        float g = 0;
        if (c < n_out) {
            const float d = y[i] - t[(size_t)r * n_out + c];
            se = d * d;
            g = 2.0f * d / ((float)B * n_out);
        }
        const bf16 gb = __float2bfloat16_rn(g);
        dz[i] = gb;
        dzt[(size_t)c * B + r] = gb;
    }
    red[threadIdx.x] = se;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// fixed-order sum of n partials by one block
__global__ void k_sum(const float* __restrict__ partial, int n, float scale, float* __restrict__ out) {
    __shared__ float red[256];
    float s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0] * scale;
}

// bias gradient: row sums of dZ^T [N][B], one warp per row, fixed order
__global__ void k_rowsum(const bf16* __restrict__ dzt, int N, int B, float* __restrict__ db) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= N) return;
    float s = 0;
    for (int i = lane; i < B; i += 32) s += __bfloat162float(dzt[(size_t)w * B + i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) db[w] = s;
}

// Adam on FP32 master weights [N][K] (+ bias [N]); BF16 copies W [N][K] and W^T [K][N]
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v, const float* __restrict__ g, int N, int K,
                       float lr, float b1, float b2, float eps, float c1, float c2, bf16* __restrict__ wb, bf16* __restrict__ wt) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)N * K) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1 - b1) * gi;
    const float vi = b2 * v[i] + (1 - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) {
        const int r = (int)(i / K), c = (int)(i - (long long)r * K);
        const bf16 b = __float2bfloat16_rn(wi);
        wb[i] = b;
        wt[(size_t)c * N + r] = b;
    }
}

__global__ void k_to_bf16(const float* __restrict__ w, int N, int K, bf16* __restrict__ wb, bf16* __restrict__ wt) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)N * K) return;
    const int r = (int)(i / K), c = (int)(i - (long long)r * K);
    const bf16 b = __float2bfloat16_rn(w[i]);
    wb[i] = b;
    wt[(size_t)c * N + r] = b;
}

}  // namespace cbsg

using namespace cbsg;

struct casim_surrogate_s {
    int n_in = 0, n_out = 0, width = 0, depth = 0;
    int in_pad = 0, out_pad = 0, L = 0, cap = 0;
    std::vector<int> din, dout;
    std::vector<float*> W, b, mW, vW, mb, vb, dW, db;  // FP32
    std::vector<bf16*> Wb, WTb;                          // BF16 copies
    std::vector<float*> Z;                               // [cap][dout] per hidden layer
    std::vector<bf16*> Hb, HTb;                          // [cap][dout], [dout][cap]
    bf16 *Xb = nullptr, *XTb = nullptr;
    float* Y = nullptr;                                  // [cap][out_pad]
    bf16 *DZ[2] = {nullptr, nullptr}, *DZT[2] = {nullptr, nullptr};
    float* partial = nullptr;
    float* loss = nullptr;
    int* err = nullptr;
    long long step = 0;
    long long launches = 0;
    cudaStream_t stream = 0;
    std::string last_error;
    size_t smem_max = 0;
};

namespace {

casim_status fail(casim_sg h, casim_status code, const std::string& msg) {
    if (h) h->last_error = msg;
    return code;
}

template <typename T>
cudaError_t dalloc(T** p, size_t n) {
    return cudaMalloc((void**)p, n * sizeof(T));
}

// two stages of A and B slices; never below 64 KiB so that every descriptor
// walk stays inside the allocation whatever the slice width
size_t gemm_smem(int N) {
    const size_t s = 2 * ((size_t)A_STAGE + (size_t)N * (BK / 8) * 16);
    return s < 65536 ? 65536 : s;
}

// columns per CTA: all of N up to 128, else the widest of 128, 64, 32, 16 dividing N,
// so that small batches still spread over twice the CTAs
int tile_n(int N) {
    if (N <= 128) return N;
    for (int b : {128, 64, 32, 16})
        if (N % b == 0) return b;
    return 16;
}

cudaError_t gemm(casim_sg h, gemm_args g) {
    if (g.M % BM || g.K % BK || g.N % 16 || g.N > 256 || g.N < 16) return cudaErrorInvalidValue;
    g.BN = tile_n(g.N);
    const size_t sm = gemm_smem(g.BN);
    if (sm > h->smem_max) {
        cudaError_t e = cudaFuncSetAttribute(k_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        h->smem_max = sm;
    }
    k_gemm<<<dim3(g.M / BM, g.N / g.BN), THREADS, sm, h->stream>>>(g);
    h->launches++;
    return cudaGetLastError();
}

unsigned long long splitmix(unsigned long long& s) {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

cudaError_t ensure_capacity(casim_sg h, int B) {
    if (B <= h->cap) return cudaSuccess;
    cudaError_t e;
    auto fr = [](void* p) {
        if (p) cudaFree(p);
    };
    for (auto p : h->Z) fr(p);
    for (auto p : h->Hb) fr(p);
    for (auto p : h->HTb) fr(p);
    fr(h->Xb);
    fr(h->XTb);
    fr(h->Y);
    for (int i = 0; i < 2; ++i) {
        fr(h->DZ[i]);
        fr(h->DZT[i]);
    }
    fr(h->partial);
    int maxw = std::max(h->width, h->out_pad);
    h->Z.assign(h->L, nullptr);
    h->Hb.assign(h->L, nullptr);
    h->HTb.assign(h->L, nullptr);
    for (int l = 0; l + 1 < h->L; ++l) {
        if ((e = dalloc(&h->Z[l], (size_t)B * h->dout[l])) != cudaSuccess) return e;
        if ((e = dalloc(&h->Hb[l], (size_t)B * h->dout[l])) != cudaSuccess) return e;
        if ((e = dalloc(&h->HTb[l], (size_t)B * h->dout[l])) != cudaSuccess) return e;
    }
    if ((e = dalloc(&h->Xb, (size_t)B * h->in_pad)) != cudaSuccess) return e;
    if ((e = dalloc(&h->XTb, (size_t)B * h->in_pad)) != cudaSuccess) return e;
    if ((e = dalloc(&h->Y, (size_t)B * h->out_pad)) != cudaSuccess) return e;
    for (int i = 0; i < 2; ++i) {
        if ((e = dalloc(&h->DZ[i], (size_t)B * maxw)) != cudaSuccess) return e;
        if ((e = dalloc(&h->DZT[i], (size_t)B * maxw)) != cudaSuccess) return e;
    }
    if ((e = dalloc(&h->partial, (size_t)B * h->out_pad / 256 + 1)) != cudaSuccess) return e;
    h->cap = B;
    return cudaSuccess;
}

// forward through all layers; training keeps Z and H^T for the backward pass
cudaError_t forward(casim_sg h, const float* x, int B, bool train) {
    cudaError_t e;
    const long long nx = (long long)B * h->in_pad;
    k_cast_in<<<(unsigned)((nx + 255) / 256), 256, 0, h->stream>>>(x, B, h->n_in, h->in_pad, h->Xb, train ? h->XTb : nullptr);
    h->launches++;
    for (int l = 0; l < h->L; ++l) {
        gemm_args g{};
        g.A = l == 0 ? h->Xb : h->Hb[l - 1];
        g.B = h->Wb[l];
        g.M = B;
        g.N = h->dout[l];
        g.K = h->din[l];
        g.bias = h->b[l];
        g.err = h->err;
        if (l + 1 < h->L) {
            g.mode = EPI_HIDDEN;
            g.H = h->Hb[l];
            g.HT = train ? h->HTb[l] : nullptr;
            g.Z = train ? h->Z[l] : nullptr;
        } else {
            g.mode = EPI_OUT;
            g.C = h->Y;
        }
        if ((e = gemm(h, g)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// loss and gradients of all parameters into dW / db
cudaError_t backward(casim_sg h, const float* t, int B) {
    cudaError_t e;
    const long long ny = (long long)B * h->out_pad;
    const int nb = (int)((ny + 255) / 256);
    k_mse<<<nb, 256, 0, h->stream>>>(h->Y, h->out_pad, t, B, h->n_out, h->DZ[0], h->DZT[0], h->partial);
    k_sum<<<1, 256, 0, h->stream>>>(h->partial, nb, 1.0f / ((float)B * h->n_out), h->loss);
    h->launches += 2;
    int cur = 0;
    for (int l = h->L - 1; l >= 0; --l) {
        gemm_args g{};
        g.A = h->DZT[cur];  // [dout][B]
        g.B = l == 0 ? h->XTb : h->HTb[l - 1];  // [din][B]
        g.M = h->dout[l];
        g.N = h->din[l];
        g.K = B;
        g.mode = EPI_PLAIN;
        g.C = h->dW[l];
        g.err = h->err;
        if ((e = gemm(h, g)) != cudaSuccess) return e;
        k_rowsum<<<(h->dout[l] * 32 + 255) / 256, 256, 0, h->stream>>>(h->DZT[cur], h->dout[l], B, h->db[l]);
        h->launches++;
        if (l > 0) {
            gemm_args d{};
            d.A = h->DZ[cur];   // [B][dout]
            d.B = h->WTb[l];    // [din][dout]
            d.M = B;
            d.N = h->din[l];
            d.K = h->dout[l];
            d.mode = EPI_BACK;
            d.Z = h->Z[l - 1];
            d.H = h->DZ[cur ^ 1];
            d.HT = h->DZT[cur ^ 1];
            d.err = h->err;
            if ((e = gemm(h, d)) != cudaSuccess) return e;
            cur ^= 1;
        }
    }
    return cudaSuccess;
}

cudaError_t check_err(casim_sg h) {
    int v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return e;
    return v ? cudaErrorLaunchTimeout : cudaSuccess;
}

}  // namespace

// Library-internal: network output for x [batch][n_in] enqueued on stream st
// without any host synchronisation (capture-safe once cb_sg_net_prepare has
// sized the buffers). The output stays in the handle: *y [batch][*ld].
cudaError_t cb_sg_net_prepare(casim_sg h, int batch) {
    if (!h || batch <= 0 || batch % BM) return cudaErrorInvalidValue;
    return ensure_capacity(h, batch);
}

cudaError_t cb_sg_net_forward(casim_sg h, const float* x, int batch, cudaStream_t st, const float** y, int* ld) {
    if (!h || batch > h->cap) return cudaErrorInvalidValue;
    const cudaStream_t keep = h->stream;
    h->stream = st;
    const cudaError_t e = forward(h, x, batch, false);
    h->stream = keep;
    *y = h->Y;
    *ld = h->out_pad;
    return e;
}

cudaError_t cb_sg_net_error(casim_sg h) { return check_err(h); }

const void* cb_sg_net_output(casim_sg h) { return h ? (const void*)h->Y : nullptr; }

extern "C" {

casim_status casim_b200_sg_create(int n_in, int n_out, int width, int depth, uint64_t seed, casim_sg* out) {
    if (!out) return CASIM_EINVAL;
    *out = nullptr;
    if (n_in < 1 || n_out < 1 || depth < 1 || width < 64 || width > 256 || width % 64) return CASIM_EINVAL;
    casim_sg h = new casim_surrogate_s();
    h->n_in = n_in;
    h->n_out = n_out;
    h->width = width;
    h->depth = depth;
    h->in_pad = (n_in + 63) / 64 * 64;
    h->out_pad = (n_out + 127) / 128 * 128;
    if (h->in_pad > 256 || h->out_pad > 256) {
        delete h;
        return CASIM_EUNSUPPORTED;
    }
    h->L = depth + 1;
    for (int l = 0; l < h->L; ++l) {
        h->din.push_back(l == 0 ? h->in_pad : width);
        h->dout.push_back(l + 1 < h->L ? width : h->out_pad);
    }
    cudaError_t e = cudaSuccess;
    auto al = [&](std::vector<float*>& v) {
        v.assign(h->L, nullptr);
        for (int l = 0; l < h->L && e == cudaSuccess; ++l) e = dalloc(&v[l], (size_t)h->din[l] * h->dout[l]);
    };
    auto alb = [&](std::vector<float*>& v) {
        v.assign(h->L, nullptr);
        for (int l = 0; l < h->L && e == cudaSuccess; ++l) e = dalloc(&v[l], (size_t)h->dout[l]);
    };
    al(h->W);
    al(h->mW);
    al(h->vW);
    al(h->dW);
    alb(h->b);
    alb(h->mb);
    alb(h->vb);
    alb(h->db);
    h->Wb.assign(h->L, nullptr);
    h->WTb.assign(h->L, nullptr);
    for (int l = 0; l < h->L && e == cudaSuccess; ++l) {
        e = dalloc(&h->Wb[l], (size_t)h->din[l] * h->dout[l]);
        if (e == cudaSuccess) e = dalloc(&h->WTb[l], (size_t)h->din[l] * h->dout[l]);
    }
    if (e == cudaSuccess) e = dalloc(&h->err, 1);
    if (e == cudaSuccess) e = dalloc(&h->loss, 1);
    if (e == cudaSuccess) e = cudaMemset(h->err, 0, sizeof(int));
    // He-uniform initialisation from a splitmix64 stream; padded rows and columns are zero
    unsigned long long st = (unsigned long long)seed;
    for (int l = 0; l < h->L && e == cudaSuccess; ++l) {
        const int K = h->din[l], N = h->dout[l];
        const int kin = l == 0 ? n_in : width, nout = l + 1 < h->L ? N : n_out;
        std::vector<float> w((size_t)N * K, 0.0f), z((size_t)N * K, 0.0f), zb(N, 0.0f);
        const double bound = std::sqrt(6.0 / kin);
        for (int r = 0; r < nout; ++r)
            for (int c = 0; c < kin; ++c) w[(size_t)r * K + c] = (float)((2.0 * ((splitmix(st) >> 11) * 0x1.0p-53) - 1.0) * bound);
        e = cudaMemcpy(h->W[l], w.data(), w.size() * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(h->mW[l], z.data(), z.size() * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(h->vW[l], z.data(), z.size() * 4, cudaMemcpyHostToDevice);
        for (float* p : {h->b[l], h->mb[l], h->vb[l]})
            if (e == cudaSuccess) e = cudaMemcpy(p, zb.data(), zb.size() * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            k_to_bf16<<<(N * K + 255) / 256, 256>>>(h->W[l], N, K, h->Wb[l], h->WTb[l]);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        casim_b200_sg_destroy(h);
        return e == cudaErrorMemoryAllocation ? CASIM_ENOMEM : CASIM_ECUDA;
    }
    *out = h;
    return CASIM_OK;
}

casim_status casim_b200_sg_destroy(casim_sg h) {
    if (!h) return CASIM_OK;
    auto fr = [](void* p) {
        if (p) cudaFree(p);
    };
    for (auto* v : {&h->W, &h->b, &h->mW, &h->vW, &h->mb, &h->vb, &h->dW, &h->db, &h->Z})
        for (float* p : *v) fr(p);
    for (auto* v : {&h->Wb, &h->WTb, &h->Hb, &h->HTb})
        for (bf16* p : *v) fr(p);
    fr(h->Xb);
    fr(h->XTb);
    fr(h->Y);
    for (int i = 0; i < 2; ++i) {
        fr(h->DZ[i]);
        fr(h->DZT[i]);
    }
    fr(h->partial);
    fr(h->loss);
    fr(h->err);
    delete h;
    return CASIM_OK;
}

casim_status casim_b200_sg_set_stream(casim_sg h, void* stream) {
    if (!h) return CASIM_EINVAL;
    h->stream = (cudaStream_t)stream;
    return CASIM_OK;
}

casim_status casim_b200_sg_num_params(casim_sg h, int64_t* n) {
    if (!h || !n) return CASIM_EINVAL;
    long long s = 0;
    for (int l = 0; l < h->L; ++l) s += (long long)h->din[l] * h->dout[l] + h->dout[l];
    *n = s;
    return CASIM_OK;
}

// parameters as FP32 in layer order: W_l [dout][din] (padded), then b_l [dout]
static casim_status params_io(casim_sg h, float* host, bool get, bool grads) {
    if (!h || !host) return CASIM_EINVAL;
    cudaError_t e = cudaStreamSynchronize(h->stream);
    size_t off = 0;
    for (int l = 0; l < h->L && e == cudaSuccess; ++l) {
        const size_t nw = (size_t)h->din[l] * h->dout[l], nb = h->dout[l];
        float* w = grads ? h->dW[l] : h->W[l];
        float* b = grads ? h->db[l] : h->b[l];
        if (get) {
            e = cudaMemcpy(host + off, w, nw * 4, cudaMemcpyDeviceToHost);
            if (e == cudaSuccess) e = cudaMemcpy(host + off + nw, b, nb * 4, cudaMemcpyDeviceToHost);
        } else {
            e = cudaMemcpy(w, host + off, nw * 4, cudaMemcpyHostToDevice);
            if (e == cudaSuccess) e = cudaMemcpy(b, host + off + nw, nb * 4, cudaMemcpyHostToDevice);
            if (e == cudaSuccess) {
                k_to_bf16<<<(unsigned)((nw + 255) / 256), 256, 0, h->stream>>>(w, h->dout[l], h->din[l], h->Wb[l], h->WTb[l]);
                e = cudaGetLastError();
            }
        }
        off += nw + nb;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return e == cudaSuccess ? CASIM_OK : fail(h, CASIM_ECUDA, cudaGetErrorString(e));
}

casim_status casim_b200_sg_get_params(casim_sg h, float* host) { return params_io(h, host, true, false); }
casim_status casim_b200_sg_set_params(casim_sg h, const float* host) { return params_io(h, (float*)host, false, false); }

casim_status casim_b200_sg_forward(casim_sg h, const float* x_dev, int batch, float* y_dev) {
    if (!h || !x_dev || !y_dev || batch <= 0 || batch % BM) return CASIM_EINVAL;
    cudaError_t e = ensure_capacity(h, batch);
    if (e == cudaSuccess) e = forward(h, x_dev, batch, false);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(y_dev, (size_t)h->n_out * 4, h->Y, (size_t)h->out_pad * 4, (size_t)h->n_out * 4, batch,
                              cudaMemcpyDeviceToDevice, h->stream);
    if (e == cudaSuccess) e = check_err(h);
    return e == cudaSuccess ? CASIM_OK : fail(h, e == cudaErrorLaunchTimeout ? CASIM_ETIMEOUT : CASIM_ECUDA, cudaGetErrorString(e));
}

casim_status casim_b200_sg_gradients(casim_sg h, const float* x_dev, const float* t_dev, int batch, float* loss, float* grads_host) {
    if (!h || !x_dev || !t_dev || batch <= 0 || batch % BM) return CASIM_EINVAL;
    cudaError_t e = ensure_capacity(h, batch);
    if (e == cudaSuccess) e = forward(h, x_dev, batch, true);
    if (e == cudaSuccess) e = backward(h, t_dev, batch);
    if (e == cudaSuccess) e = check_err(h);
    if (e == cudaSuccess && loss) e = cudaMemcpy(loss, h->loss, 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(h, e == cudaErrorLaunchTimeout ? CASIM_ETIMEOUT : CASIM_ECUDA, cudaGetErrorString(e));
    return grads_host ? params_io(h, grads_host, true, true) : CASIM_OK;
}

casim_status casim_b200_sg_train_step(casim_sg h, const float* x_dev, const float* t_dev, int batch, float lr, float* loss) {
    if (!h || !x_dev || !t_dev || batch <= 0 || batch % BM || !(lr > 0)) return CASIM_EINVAL;
    cudaError_t e = ensure_capacity(h, batch);
    if (e == cudaSuccess) e = forward(h, x_dev, batch, true);
    if (e == cudaSuccess) e = backward(h, t_dev, batch);
    if (e == cudaSuccess) {
        h->step++;
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        const float c1 = 1.0f - (float)std::pow(b1, (double)h->step), c2 = 1.0f - (float)std::pow(b2, (double)h->step);
        for (int l = 0; l < h->L && e == cudaSuccess; ++l) {
            const int N = h->dout[l], K = h->din[l];
            k_adam<<<(N * K + 255) / 256, 256, 0, h->stream>>>(h->W[l], h->mW[l], h->vW[l], h->dW[l], N, K, lr, b1, b2, eps, c1, c2,
                                                             h->Wb[l], h->WTb[l]);
            k_adam<<<(N + 255) / 256, 256, 0, h->stream>>>(h->b[l], h->mb[l], h->vb[l], h->db[l], N, 1, lr, b1, b2, eps, c1, c2,
                                                         nullptr, nullptr);
            h->launches += 2;
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess && loss) {
        e = cudaMemcpyAsync(loss, h->loss, 4, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
    return e == cudaSuccess ? CASIM_OK : fail(h, CASIM_ECUDA, cudaGetErrorString(e));
}

casim_status casim_b200_sg_check(casim_sg h) {
    if (!h) return CASIM_EINVAL;
    cudaError_t e = check_err(h);
    return e == cudaSuccess ? CASIM_OK : fail(h, e == cudaErrorLaunchTimeout ? CASIM_ETIMEOUT : CASIM_ECUDA, cudaGetErrorString(e));
}

casim_status casim_b200_sg_launches(casim_sg h, int64_t* out) {
    if (!h || !out) return CASIM_EINVAL;
    *out = h->launches;
    return CASIM_OK;
}

casim_status casim_b200_sg_last_error(casim_sg h, char* buf, size_t n) {
    if (!h || !buf || n == 0) return CASIM_EINVAL;
    snprintf(buf, n, "%s", h->last_error.c_str());
    return CASIM_OK;
}

// One GEMM C = A . B^T through the tensor-core kernel (FP32 result), device pointers,
// for checking the kernel on its own: A [M][K], B [N][K] BF16 bit patterns.
casim_status casim_b200_sg_gemm(const void* a_dev, const void* b_dev, int M, int N, int K, float* c_dev) {
    if (!a_dev || !b_dev || !c_dev) return CASIM_EINVAL;
    casim_surrogate_s tmp;
    int* err = nullptr;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return CASIM_ENOMEM;
    cudaMemset(err, 0, sizeof(int));
    tmp.err = err;
    gemm_args g{};
    g.A = (const bf16*)a_dev;
    g.B = (const bf16*)b_dev;
    g.M = M;
    g.N = N;
    g.K = K;
    g.mode = EPI_PLAIN;
    g.C = c_dev;
    g.err = err;
    cudaError_t e = gemm(&tmp, g);
    if (e == cudaSuccess) e = check_err(&tmp);
    cudaFree(err);
    if (e == cudaErrorInvalidValue) return CASIM_EINVAL;
    return e == cudaSuccess ? CASIM_OK : e == cudaErrorLaunchTimeout ? CASIM_ETIMEOUT : CASIM_ECUDA;
}

}  // extern "C"
