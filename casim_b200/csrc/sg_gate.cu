// Surrogate-driven gating, one warp per site: n time steps of the cytosol
// pool and jSR ODEs (lane 0), RyR gating with the held mouth values and the
// RyR currents, without the RD step. The gating consumes the site's MRG32k3a
// stream in the reference's order (CaSim/DyadChannels.cpp:97-130: one draw per
// RyR test, one more per transition) with the warp-parallel scheme of the
// resident kernel: a ring of draws generated 16 per lane from jumped-ahead
// states, 32 RyRs resolved per ballot, one re-evaluation per transition.
#include "engine.h"
#include "pools.cuh"
#include "resident_kernel.cuh"

namespace {

using namespace cbres;

constexpr int SG_MAXCH = 256;  // RyRs per site this kernel serves (two draws each fit one refill)
constexpr int SG_WARPS = 4;    // sites per block

struct sg_warp_smem {
    double ring[RING];
    double p[2][SG_MAXCH];  // transition probability per step of each RyR when closed / open
    int state[SG_MAXCH];
    cb_site_scalars q;
};

__global__ void __launch_bounds__(32 * SG_WARPS) k_sg_warp(const __grid_constant__ cb_model m, int S, int NS, long long n,
                                                          const cb_site* __restrict__ sites, cb_site_scalars* __restrict__ sc,
                                                          int* __restrict__ ch_state, const double* __restrict__ mouth,
                                                          const double* __restrict__ spx0, const double* __restrict__ spc0,
                                                          const double* __restrict__ spx1, const double* __restrict__ spc1,
                                                          const unsigned long long* __restrict__ pow2) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * SG_WARPS + warp;
    if (s >= S) return;  // whole warp
    sg_warp_smem& W = ((sg_warp_smem*)smem_raw)[warp];
    const cb_site st = sites[s];
    const int nch = st.n_ch;
    const double dt = m.dt;
    {
        const unsigned int* src = (const unsigned int*)(sc + s);
        unsigned int* dst = (unsigned int*)&W.q;
        for (int k = lane; k < (int)(sizeof(cb_site_scalars) / 4); k += 32) dst[k] = src[k];
    }
    for (int c = lane; c < nch; c += 32) {
        const double* mo = mouth + (size_t)(st.ch_off + c) * NS;
        const double mg = m.mg_idx >= 0 ? mo[m.mg_idx] : 0.0;
        W.state[c] = ch_state[st.ch_off + c];
        W.p[0][c] = cb_rate(m, spx0, spc0, spx1, spc1, 0, mo[m.ca_idx], mg) * dt;
        W.p[1][c] = cb_rate(m, spx0, spc0, spx1, spc1, 1, mo[m.ca_idx], mg) * dt;
    }
    __syncwarp();
    cbrng::State gl;
    for (int i = 0; i < 6; ++i) gl.s[i] = W.q.rng[i];
    rng_jump(pow2, gl, 2ULL * LANE_DRAWS * lane);  // lane l: draw l*LANE_DRAWS of the first refill
    long long D = 0, we = 0;
    for (long long it = 0; it < n; ++it) {
        if (lane == 0) {
            if (m.cyto_type == CB_CYTO_POOL) cb_pool_step(m, W.q, dt);
            cb_jsr_step(m, W.q, dt);
        }
        if (we - D < 2LL * nch) {  // ring refill: at least two draws per RyR available
            const long long base = we + (long long)lane * LANE_DRAWS;
            for (int i = 0; i < LANE_DRAWS; ++i) W.ring[(base + i) & (RING - 1)] = u01d_fast(gl);
            jump_row(pow2, gl, JUMP_ROW);
            we += WINDOW;
        }
        __syncwarp();
        for (int b0 = 0; b0 < nch; b0 += 32) {
            const int c = b0 + lane;
            const int cnt = min(32, nch - b0);
            const bool act = lane < cnt;
            const int stt = act ? W.state[c] : 0;
            const double p = act ? W.p[stt][c] : 0.0;
            int start = 0;
            while (start < cnt) {
                const bool rem = act && lane >= start;
                const double u = rem ? W.ring[(D + (lane - start)) & (RING - 1)] : 2.0;
                const unsigned int t = __ballot_sync(0xffffffffu, rem && (u < p));
                if (t == 0u) {
                    D += cnt - start;
                    break;
                }
                const int f = __ffs(t) - 1;
                if (lane == f) W.state[c] = 1 - stt;
                D += (f - start) + 2;
                start = f + 1;
            }
        }
        __syncwarp();
        // RyR currents from the held mouth values and the jSR coupling
        for (int j = 0; j < m.n_ions; ++j) {
            double part = 0;
            for (int c = lane; c < nch; c += 32)
                part += W.state[c] * (m.g[j] * (W.q.jsr_new[j] - mouth[(size_t)(st.ch_off + c) * NS + j]));
            part = warp_sum(part);
            if (lane == 0) W.q.total[j] = part;
        }
        __syncwarp();
        if (lane == 0 && !m.jsr_const)
            for (int i = 0; i < m.n_ions; ++i) {
                W.q.IjSR[i] = W.q.total[i] * m.V_elem;
                W.q.nsr[i] = m.nsr[i];
                W.q.jsr[i] = W.q.jsr_new[i];
            }
        __syncwarp();
    }
    if (lane == 0) {
        cbrng::State gd;  // stream state at the next unconsumed draw
        for (int i = 0; i < 6; ++i) gd.s[i] = W.q.rng[i];
        rng_jump(pow2, gd, 2ULL * (unsigned long long)D);
        for (int i = 0; i < 6; ++i) W.q.rng[i] = gd.s[i];
        W.q.draws += (unsigned long long)D;
    }
    __syncwarp();
    {
        const unsigned int* src = (const unsigned int*)&W.q;
        unsigned int* dst = (unsigned int*)(sc + s);
        for (int k = lane; k < (int)(sizeof(cb_site_scalars) / 4); k += 32) dst[k] = src[k];
    }
    for (int c = lane; c < nch; c += 32) ch_state[st.ch_off + c] = W.state[c];
}

}  // namespace

// the warp-per-site kernel when every site has at most SG_MAXCH RyRs
cudaError_t cb_sg_steps_warp(cb_dev& d, long long n, cudaStream_t st, bool* used) {
    *used = false;
    if (d.max_ch > SG_MAXCH) return cudaSuccess;
    cudaError_t e = cb_ensure_pow2(d);
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(sg_warp_smem) * SG_WARPS;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if ((e = cudaStreamIsCapturing(st, &cap)) != cudaSuccess) return e;
    if (cap == cudaStreamCaptureStatusNone) {  // set before any capture (the first call runs eagerly)
        e = cudaFuncSetAttribute(k_sg_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_sg_warp<<<(d.S + SG_WARPS - 1) / SG_WARPS, 32 * SG_WARPS, smem, st>>>(d.m, d.S, d.NS, n, d.sites, d.sc, d.ch_state, d.mouth,
                                                                          d.spx[0], d.spc[0], d.spx[1], d.spc[1], d.rs_pow2);
    *used = true;
    return cudaGetLastError();
}
