// Resident path: every site lives in one thread block's shared memory for all
// K time steps of a launch, so HBM is touched once per site per launch.
//
// One persistent launch walks the packed site table through an atomic work
// queue (sites pre-sorted by decreasing cost). Per site:
//   load     fields, RyR table, site scalars, cytosol (pool scalars or RD3D grid)
//   K steps  phase A: warp 0 = control (efflux/current reductions of the last
//                     Update, jSR coupling, cytosol pool ODE, jSR ODE, RyR gating);
//                     warps 1.. = cleft stencil (and RD3D cytosol stencil),
//                     ping-pong between two smem copies of the fields
//            __syncthreads
//            phase B: all warps = Update: Dirichlet rim, mouth gather, RyR
//                     currents, efflux partials (warp shuffles)
//            __syncthreads
//   store    fields, scalars, RyR states, currents, RNG state
//
// The step semantics are the reference loop body (CaSim/ParallelHybridSolver.cpp:532-540)
// followed by Update() (:270-286): cytosol (CaSim/CytosolPool.cpp:217-288), dyad RD
// (CaSim/DyadRD2DCPU.cpp:394-490, CaSim/DyadRDCPU.cpp:404-506), jSR (CaSim/SRPool.cpp:70-89),
// gating (CaSim/DyadChannels.cpp:97-130) and coupling (CaSim/DyadRD2DCPU.cpp:243-392).
//
// RyR gating consumes the site's MRG32k3a stream in exactly the reference's
// order (one draw per channel, a second one per transition) but without the
// reference's serial loop: warp 0 keeps a ring of pre-generated draws (32
// lanes x 16 contiguous draws per refill, lanes jump-ahead by matrix powers)
// and resolves a chunk of 32 channels with one ballot per transition.
#include <algorithm>
#include <vector>

#include "engine.h"
#include "mrg32k3a.cuh"
#include "physics.cuh"

namespace {

constexpr int RING = 1024;                // pre-generated draws held per site
constexpr int LANE_DRAWS = 16;            // contiguous draws per lane per refill
constexpr int WINDOW = 32 * LANE_DRAWS;   // draws per refill
constexpr int MAX_THREADS = 512;

struct rs_args {
    cb_model m;
    const cb_site* sites;
    const int* order;
    int S;
    int* counter;
    void* fields;
    void* curgrid;
    const int* ch_node;
    const int* ch_owner;
    int* ch_state;
    double* mouth;
    int NS;
    cb_site_scalars* sc;
    void* cyto;
    double* cin;
    const int* rim_cnode;
    const int* dep_ptr;
    const int* dep_term;
    int nc;
    const unsigned long long* pow2;  // [64][2][9]: A1^(2^k), A2^(2^k)
    const double* spx0;
    const double* spc0;
    const double* spx1;
    const double* spc1;
    long long nsteps;
    // smem carve (bytes), identical for every site of the launch
    int np;  // padded node capacity per species
    int max_ch, max_terms;
    int off_fb, off_ca, off_cb, off_terms, off_cin, off_mask, off_chn, off_chs, off_cho, off_flux, off_fluxd,
        off_mi, off_ring, off_red, off_sc, smem_bytes;
};

// ---- MRG32k3a jump-ahead on the device ------------------------------------
__device__ __forceinline__ void mat_apply(const unsigned long long* A, unsigned int* v, unsigned long long m) {
    unsigned long long r[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        unsigned long long acc = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) acc = (acc + (A[3 * i + k] * (unsigned long long)v[k]) % m) % m;
        r[i] = acc;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = (unsigned int)r[i];
}

// advance by `steps` recurrence steps (binary powering with the 2^k table)
__device__ void rng_jump(const unsigned long long* pow2, cbrng::State& g, unsigned long long steps) {
    for (int k = 0; steps; ++k, steps >>= 1)
        if (steps & 1ULL) {
            mat_apply(pow2 + 18 * k, g.s, cbrng::M1);
            mat_apply(pow2 + 18 * k + 9, g.s + 3, cbrng::M2);
        }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ bool is_rim(int x, int y, int nx, int ny) { return x == 0 || y == 0 || x == nx - 1 || y == ny - 1; }

template <typename R, int FM>
__global__ void __launch_bounds__(MAX_THREADS, 1) k_resident(const __grid_constant__ rs_args a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_site;
    const cb_model& m = a.m;
    const int F = m.F, NI = m.n_ions;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, W = blockDim.x >> 5;
    const bool rd3d = m.cyto_type == CB_CYTO_RD3D;
    const int mc = m.mc, mc2 = mc * mc, nc = a.nc, CS = m.n_ions + m.c_n_pairs;

    R* fa = (R*)smem;
    R* fb = (R*)(smem + a.off_fb);
    R* ca = (R*)(smem + a.off_ca);
    R* cb = (R*)(smem + a.off_cb);
    double* terms = (double*)(smem + a.off_terms);
    double* cin_s = (double*)(smem + a.off_cin);
    unsigned int* chmask = (unsigned int*)(smem + a.off_mask);
    int* chn = (int*)(smem + a.off_chn);
    int* chs = (int*)(smem + a.off_chs);
    int* cho = (int*)(smem + a.off_cho);
    R* flux = (R*)(smem + a.off_flux);
    double* fluxd = (double*)(smem + a.off_fluxd);
    double* mi = (double*)(smem + a.off_mi);
    double* ring = (double*)(smem + a.off_ring);
    double* red = (double*)(smem + a.off_red);
    cb_site_scalars& q = *(cb_site_scalars*)(smem + a.off_sc);

    const double dt = m.dt;
    const R dtR = (R)dt;

    for (;;) {
        if (tid == 0) s_site = atomicAdd(a.counter, 1);
        __syncthreads();
        if (s_site >= a.S) break;
        const int s = a.order[s_site];
        const cb_site st = a.sites[s];
        const int nx = st.nx, ny = st.ny, nz = st.nz, nxy = nx * ny, N = nxy * nz, np = st.npad;
        const int nch = st.n_ch;
        const int zmax = m.dim == 2 ? 1 : nz - 1;
        const int T = cb_efflux_terms(nx, ny, zmax);
        const int nrim = cb_rim_count(nx, ny);

        // ---------------------------------------------------------- load
        {
            const int4* src = (const int4*)((const R*)a.fields + st.node_base * F);
            int4* dst = (int4*)fa;
            const int n16 = (int)((size_t)F * np * sizeof(R) / 16);
            for (int k = tid; k < n16; k += blockDim.x) dst[k] = src[k];
            for (int k = tid; k < (np + 31) / 32; k += blockDim.x) chmask[k] = 0u;
            const unsigned int* qs = (const unsigned int*)(a.sc + s);
            unsigned int* qd = (unsigned int*)&q;
            for (int k = tid; k < (int)(sizeof(cb_site_scalars) / 4); k += blockDim.x) qd[k] = qs[k];
            if (rd3d) {
                const R* cs = (const R*)a.cyto + (size_t)s * CS * nc;
                for (int k = tid; k < CS * nc; k += blockDim.x) {
                    R v = cs[k];
                    ca[k] = v;
                    cb[k] = v;
                }
                for (int k = tid; k < CS * mc2; k += blockDim.x) cin_s[k] = a.cin[(size_t)s * CS * mc2 + k];
            }
        }
        __syncthreads();
        for (int c = tid; c < nch; c += blockDim.x) {
            int node = a.ch_node[st.ch_off + c];
            chn[c] = node;
            chs[c] = a.ch_state[st.ch_off + c];
            cho[c] = a.ch_owner[st.ch_off + c];
            atomicOr(&chmask[node >> 5], 1u << (node & 31));
            const double* mo = a.mouth + (size_t)(st.ch_off + c) * a.NS;
            for (int j = 0; j < NI; ++j) {
                mi[c * NI + j] = mo[j];
                // current of the last Update: state * g * (jSR - Ca at the node)
                double fl = chs[c] * (m.g[j] * (q.jsr_new[j] - (double)fa[j * np + node]));
                flux[c * NI + j] = (R)fl;
                fluxd[c * NI + j] = fl;
            }
        }

        // RNG (warp 0): lane l holds the stream at draw D0 + l*LANE_DRAWS of the
        // next window; ring slot k % RING holds draw k (counted from entry)
        cbrng::State g0, gl;
        long long D = 0, we = 0;
        if (warp == 0) {
            for (int i = 0; i < 6; ++i) g0.s[i] = q.rng[i];
            gl = g0;
            rng_jump(a.pow2, gl, 2ULL * LANE_DRAWS * lane);
        }
        __syncthreads();

        // ---------------------------------------------------------- steps
        for (long long it = 0; it < a.nsteps; ++it) {
            const bool last = it == a.nsteps - 1;
            if (warp == 0) {
                // ---- control warp
                if (it > 0) {
                    // reductions of the previous Update (fixed order -> deterministic)
                    for (int f = lane; f < F; f += 32) {
                        double e = 0;
                        for (int w = 0; w < W; ++w) e += red[w * FM + f];
                        q.efflux[f] = e;
                    }
                    for (int j = 0; j < NI; ++j) {
                        double t = 0;
                        for (int c = lane; c < nch; c += 32) t += fluxd[c * NI + j];
                        t = warp_sum(t);
                        if (lane == 0) q.total[j] = t;
                    }
                    __syncwarp();
                    if (lane == 0 && !m.jsr_const)
                        for (int i = 0; i < NI; ++i) {
                            q.IjSR[i] = q.total[i] * m.V_elem;
                            q.nsr[i] = m.nsr[i];
                            q.jsr[i] = q.jsr_new[i];
                        }
                    __syncwarp();
                }
                if (lane == 0) {
                    if (!rd3d) {
                        // cytosol pool ODE (CaSim/CytosolPool.cpp:217-288)
                        double evo_i[CB_MAX_IONS], evo_p[CB_MAX_CPAIRS];
                        int ipd = 0, is = 0;
                        for (int j = 0; j < NI; ++j) {
                            double react = 0;
                            for (int p = 0; p < m.c_n_pairs; ++p) {
                                if (m.c_pair_ion[p] != j) continue;
                                double R1 = m.c_koff[p] * q.c_pairs[p] - m.c_kon[p] * q.c_ions[j] * q.c_free[m.c_pair_buf[p]];
                                evo_p[p] = -R1;
                                react += R1;
                                if (m.c_in_dyad[p]) evo_p[p] += q.efflux[NI + ipd++];
                            }
                            evo_i[j] = react + q.efflux[j];
                            if (m.c_serca[j]) {
                                double i2 = q.c_ions[j] * q.c_ions[j];
                                double K2 = m.c_Kup[is] * m.c_Kup[is];
                                double b2 = m.c_bg[is] * m.c_bg[is];
                                evo_i[j] -= m.c_Jmax[is] * (i2 / (i2 + K2) - b2 / (b2 + K2));
                                ++is;
                            }
                        }
                        for (int j = 0; j < NI; ++j) {
                            evo_i[j] -= m.c_onetau_ion[j] * (q.c_ions[j] - m.c_bg[j]);
                            q.c_ions[j] += evo_i[j] * dt;
                        }
                        ipd = 0;
                        for (int p = 0; p < m.c_n_pairs; ++p) {
                            evo_p[p] -= m.c_onetau_pair[p] * (q.c_pairs[p] - m.c_init[p]);
                            q.c_pairs[p] += evo_p[p] * dt;
                            if (m.c_in_dyad[p]) q.c_bnd[ipd++] = q.c_pairs[p];
                        }
                        for (int b = 0; b < m.c_n_buf; ++b) q.c_free[b] = m.c_Ctot[b];
                        for (int p = 0; p < m.c_n_pairs; ++p) q.c_free[m.c_pair_buf[p]] -= q.c_pairs[p];
                    }
                    // jSR ODE (CaSim/SRPool.cpp:70-89) with the site's own beta
                    if (!m.jsr_const) {
                        double beta = 1;
                        for (int j = 0; j < NI; ++j)
                            beta += m.nCQ[j] * m.K_CQ[j] * m.CQ / ((m.K_CQ[j] + q.jsr[j]) * (m.K_CQ[j] + q.jsr[j]));
                        for (int i = 0; i < NI; ++i) {
                            double Iref = 1 / m.tau_refill[i] * (q.nsr[i] - q.jsr[i]);
                            q.jsr_new[i] = q.jsr[i] + dt / beta * (Iref - q.IjSR[i] / m.V_jsr);
                        }
                        if (m.ca_idx >= 0) q.release += q.IjSR[m.ca_idx] * dt;
                    }
                }
                // ---- ring refill: keep at least 2 draws per channel available
                if (we - D < 2LL * nch) {
                    long long base = we + (long long)lane * LANE_DRAWS;
                    for (int i = 0; i < LANE_DRAWS; ++i) ring[(base + i) & (RING - 1)] = cbrng::u01d(gl);
                    // jump from the end of this lane's chunk to its chunk in the next window
                    rng_jump(a.pow2, gl, 2ULL * LANE_DRAWS * 31);
                    we += WINDOW;
                    __syncwarp();
                }
                // ---- gating (CaSim/DyadChannels.cpp:97-130): draw D+i tests channel i
                // until a transition consumes one extra draw; one ballot per transition
                for (int base = 0; base < nch; base += 32) {
                    const int c = base + lane;
                    const int cnt = min(32, nch - base);
                    const bool act = lane < cnt;
                    double p = 0;
                    int stt = 0;
                    if (act) {
                        stt = chs[c];
                        double cam = mi[c * NI + m.ca_idx];
                        double mgm = m.mg_idx >= 0 ? mi[c * NI + m.mg_idx] : 0.0;
                        p = cb_rate(m, a.spx0, a.spc0, a.spx1, a.spc1, stt, cam, mgm) * dt;
                    }
                    int start = 0;
                    while (start < cnt) {
                        const bool rem = act && lane >= start;
                        double u = rem ? ring[(D + (lane - start)) & (RING - 1)] : 2.0;
                        unsigned int t = __ballot_sync(0xffffffffu, rem && (u < p));
                        if (t == 0u) {
                            D += cnt - start;
                            break;
                        }
                        int f = __ffs(t) - 1;
                        if (lane == f) chs[c] = 1 - stt;
                        D += (f - start) + 2;
                        start = f + 1;
                    }
                }
                __syncwarp();
            } else {
                // ---- worker warps: cleft stencil fa -> fb on interior nodes
                const int wt = tid - 32, NW = blockDim.x - 32;
                const R idx2 = (R)m.inv_dx2, idy2 = (R)m.inv_dy2, idz2 = (R)m.inv_dz2;
                const int ix = nx - 2, ncol = ix * (ny - 2);
                for (int i = wt; i < ncol; i += NW) {
                    const int x = 1 + i % ix, y = 1 + i / ix;
                    for (int z = 0; z < nz; ++z) {
                        const int n = x + nx * y + nxy * z;
                        int zl = n, zr = n;
                        if (m.dim == 3) {
                            zl = z == 0 ? n + nxy : n - nxy;
                            zr = z == nz - 1 ? n - nxy : n + nxy;
                        }
                        // ions (j) and ion-buffer pairs (p) kept in separate register
                        // arrays indexed only by unrolled constants
                        R vi[CB_MAX_IONS], ei[CB_MAX_IONS], vp[FM], ep[FM];
#pragma unroll
                        for (int j = 0; j < CB_MAX_IONS; ++j) {
                            vi[j] = 0;
                            ei[j] = 0;
                            if (j < NI) {
                                const R* v = fa + j * np;
                                R cc = v[n];
                                vi[j] = cc;
                                const R D = (R)m.D_ion[j];
                                if (D != (R)0) {
                                    R lap = (v[n + 1] - 2 * cc + v[n - 1]) * idx2 + (v[n + nx] - 2 * cc + v[n - nx]) * idy2;
                                    if (m.dim == 3) lap = lap + (v[zr] - 2 * cc + v[zl]) * idz2;
                                    ei[j] = D * lap;
                                }
                            }
                        }
#pragma unroll
                        for (int p = 0; p < FM; ++p) {
                            vp[p] = 0;
                            ep[p] = 0;
                            if (p < m.n_pairs) {
                                const R* v = fa + (NI + p) * np;
                                R cc = v[n];
                                vp[p] = cc;
                                const R D = (R)m.D_pair[p];
                                if (D != (R)0) {
                                    R lap = (v[n + 1] - 2 * cc + v[n - 1]) * idx2 + (v[n + nx] - 2 * cc + v[n - nx]) * idy2;
                                    if (m.dim == 3) lap = lap + (v[zr] - 2 * cc + v[zl]) * idz2;
                                    ep[p] = D * lap;
                                }
                            }
                        }
                        // reactions: free buffer of each pair's buffer (total minus its
                        // pairs in pair order), R1 = koff*B - kon*ion*free
                        R r1[FM];
#pragma unroll
                        for (int p = 0; p < FM; ++p) {
                            r1[p] = 0;
                            if (p < m.n_pairs) {
                                const int b = m.pair_buf[p];
                                R fr = (R)m.Ctot[b];
#pragma unroll
                                for (int p2 = 0; p2 < FM; ++p2)
                                    if (p2 < m.n_pairs && m.pair_buf[p2] == b) fr -= vp[p2];
                                R ion = 0;
#pragma unroll
                                for (int j = 0; j < CB_MAX_IONS; ++j)
                                    if (j == m.pair_ion[p]) ion = vi[j];
                                r1[p] = (R)m.koff[p] * vp[p] - (R)m.kon[p] * ion * fr;
                                ep[p] += -r1[p];
                            }
                        }
                        const bool has_ch = (chmask[n >> 5] >> (n & 31)) & 1u;
                        int cown = -1;
                        if (has_ch)
                            for (int c = nch - 1; c >= 0; --c)
                                if (chn[c] == n) {
                                    cown = c;
                                    break;
                                }
                        const bool sl_layer = (m.dim == 2) || (z == nz - 1);
#pragma unroll
                        for (int j = 0; j < CB_MAX_IONS; ++j) {
                            if (j < NI) {
                                R Rj = 0;
#pragma unroll
                                for (int p = 0; p < FM; ++p)
                                    if (p < m.n_pairs && m.pair_ion[p] == j) Rj += r1[p];
                                R e = ei[j] + Rj;
                                if (cown >= 0) e += flux[cown * NI + j];
                                if (sl_layer && m.has_sl[j]) {
                                    R s1 = (R)m.K1[j] + vi[j];
                                    R s2 = (R)m.K2[j] + vi[j];
                                    e *= (R)1 / ((R)1 + (R)(m.N1[j] * m.K1[j]) / (s1 * s1) + (R)(m.N2[j] * m.K2[j]) / (s2 * s2));
                                }
                                fb[j * np + n] = vi[j] + e * dtR;
                            }
                        }
#pragma unroll
                        for (int p = 0; p < FM; ++p)
                            if (p < m.n_pairs) fb[(NI + p) * np + n] = vp[p] + ep[p] * dtR;
                    }
                }
                if (rd3d) {
                    // RD3D cytosol stencil ca -> cb (no reference analog; see the oracle)
                    const R ih2 = (R)m.inv_hc2;
                    const int* ptr = a.dep_ptr + (size_t)s * (mc2 + 1);
                    for (int n = wt; n < nc; n += NW) {
                        const int i = n % mc, j = (n / mc) % mc, k = n / mc2;
                        if (i == 0 || i == mc - 1 || j == 0 || j == mc - 1 || k == mc - 1) continue;
                        const int zl = k == 0 ? n + mc2 : n - mc2, zr = n + mc2;
                        R evo[CB_MAX_CSPECIES], u[CB_MAX_CSPECIES];
                        for (int c = 0; c < CS; ++c) {
                            const R* v = ca + c * nc;
                            R D = (R)(c < NI ? m.D_ion[c] : m.c_D_pair[c - NI]);
                            R cc = v[n];
                            u[c] = cc;
                            evo[c] = D * ((v[n + 1] - 2 * cc + v[n - 1]) * ih2 + (v[n + mc] - 2 * cc + v[n - mc]) * ih2 +
                                          (v[zr] - 2 * cc + v[zl]) * ih2);
                        }
                        R fr[CB_MAX_CBUF];
                        for (int b = 0; b < m.c_n_buf; ++b) fr[b] = (R)m.c_Ctot[b];
                        for (int p = 0; p < m.c_n_pairs; ++p) fr[m.c_pair_buf[p]] -= u[NI + p];
                        int is = 0;
                        for (int j2 = 0; j2 < NI; ++j2) {
                            R ion = u[j2];
                            R react = 0;
                            for (int p = 0; p < m.c_n_pairs; ++p) {
                                if (m.c_pair_ion[p] != j2) continue;
                                R R1 = (R)m.c_koff[p] * u[NI + p] - (R)m.c_kon[p] * ion * fr[m.c_pair_buf[p]];
                                evo[NI + p] += -R1;
                                react += R1;
                            }
                            evo[j2] += react;
                            if (m.c_serca[j2]) {
                                R i2 = ion * ion;
                                R K2 = (R)(m.c_Kup[is] * m.c_Kup[is]);
                                R b2 = (R)(m.c_bg[is] * m.c_bg[is]);
                                evo[j2] -= (R)m.c_Jmax[is] * (i2 / (i2 + K2) - b2 / (b2 + K2));
                                ++is;
                            }
                        }
                        for (int c = 0; c < CS; ++c) {
                            R e = evo[c];
                            if (k == 0) {
                                double dep;
                                if (it == 0) {
                                    dep = cin_s[c * mc2 + n];
                                } else {
                                    int f = c < NI ? c : m.c_dyad_pair[c - NI];
                                    if (f >= 0 && c >= NI) f += NI;
                                    dep = 0;
                                    if (f >= 0)
                                        for (int kk = ptr[n]; kk < ptr[n + 1]; ++kk) dep += terms[a.dep_term[st.term_off + kk] * FM + f];
                                }
                                e += (R)dep;
                            }
                            cb[c * nc + n] = u[c] + e * dtR;
                        }
                    }
                }
            }
            __syncthreads();

            // ---------------------------------------------------- phase B: Update
            // Dirichlet rim from the cytosol (CaSim/DyadRD2DCPU.cpp:274-303); the RD3D
            // cytosol is read as it was at the start of the step (ca)
            for (int t = tid; t < nrim * nz; t += blockDim.x) {
                int r = t % nrim, z = t / nrim, x, y;
                cb_rim_xy(r, nx, ny, x, y);
                const int n = x + nx * y + nxy * z;
                if (!rd3d) {
                    for (int j = 0; j < NI; ++j) fb[j * np + n] = (R)q.c_ions[j];
                    for (int p = 0; p < m.n_pairs; ++p) fb[(NI + p) * np + n] = (R)q.c_bnd[p];
                } else {
                    const int cn = a.rim_cnode[st.rim_off + r];
                    for (int j = 0; j < NI; ++j) fb[j * np + n] = ca[j * nc + cn];
                    for (int p = 0; p < m.n_pairs; ++p) {
                        int cq = m.dyad_c_pair[p];
                        fb[(NI + p) * np + n] = cq >= 0 ? ca[(NI + cq) * nc + cn] : (R)m.pair_init[p];
                    }
                }
            }
            // mouth gather and RyR currents (CaSim/DyadRD2DCPU.cpp:243-264, 361-380)
            for (int c = tid; c < nch; c += blockDim.x) {
                const int n = chn[c];
                const int x = n % nx, y = (n / nx) % ny;
                const bool rim = is_rim(x, y, nx, ny);
                const R* src = rim ? fa : fb;  // mouth is gathered before the rim is reset
                const int stc = chs[c];
                for (int j = 0; j < NI; ++j) {
                    double mv = (double)src[j * np + n];
                    mi[c * NI + j] = mv;
                    double cv = mv;
                    if (rim) {
                        if (!rd3d) cv = (double)(R)q.c_ions[j];
                        else cv = (double)ca[j * nc + a.rim_cnode[st.rim_off + cb_rim_index(x, y, nx, ny)]];
                    }
                    double fl = stc * (m.g[j] * (q.jsr_new[j] - cv));
                    flux[c * NI + j] = (R)fl;
                    fluxd[c * NI + j] = fl;
                }
                if (last) {
                    double* mo = a.mouth + (size_t)(st.ch_off + c) * a.NS;
                    double fr[CB_MAX_BUF];
                    for (int b = 0; b < m.n_buf; ++b) fr[b] = m.Ctot[b];
                    for (int f = 0; f < F; ++f) {
                        double v = (double)src[f * np + n];
                        mo[f] = v;
                        if (f >= NI) fr[m.pair_buf[f - NI]] -= v;
                    }
                    for (int b = 0; b < m.n_buf; ++b) mo[F + b] = fr[b];
                }
            }
            // efflux partials (CaSim/DyadRD2DCPU.cpp:305-350); the rim value u0 is
            // the cytosol value just written
            {
                double part[FM];
#pragma unroll
                for (int f = 0; f < FM; ++f) part[f] = 0;
                for (int t = tid; t < T; t += blockDim.x) {
                    int x0, y0, x1, y1, x2, y2, z;
                    int sel = cb_efflux_term(t, nx, ny, zmax, x0, y0, x1, y1, x2, y2, z);
                    const double sf = sel == 0 ? m.sx : m.sy;
                    const int n1 = x1 + nx * y1 + nxy * z, n2 = x2 + nx * y2 + nxy * z;
                    int cn = 0;
                    if (rd3d) cn = a.rim_cnode[st.rim_off + cb_rim_index(x0, y0, nx, ny)];
#pragma unroll
                    for (int f = 0; f < FM; ++f) {
                        if (f >= F) break;
                        double u0;
                        if (!rd3d) {
                            u0 = f < NI ? (double)(R)q.c_ions[f] : (double)(R)q.c_bnd[f - NI];
                        } else {
                            int cq = f < NI ? f : m.dyad_c_pair[f - NI];
                            u0 = f < NI ? (double)ca[f * nc + cn] : cq >= 0 ? (double)ca[(NI + cq) * nc + cn] : (double)(R)m.pair_init[f - NI];
                        }
                        const double D = f < NI ? m.D_ion[f] : m.D_pair[f - NI];
                        const double gr = 2 * (double)fb[f * np + n1] - 1.5 * u0 - 0.5 * (double)fb[f * np + n2];
                        if (!rd3d) {
                            part[f] += D * m.grad_mult * sf * gr;
                        } else {
                            double v = D * sf * gr * m.inv_hc3;
                            part[f] += v;
                            terms[t * FM + f] = v;
                        }
                    }
                }
#pragma unroll
                for (int f = 0; f < FM; ++f) {
                    if (f >= F) break;
                    double v = warp_sum(part[f]);
                    if (lane == 0) red[warp * FM + f] = v;
                }
            }
            __syncthreads();
            { R* t = fa; fa = fb; fb = t; }
            { R* t = ca; ca = cb; cb = t; }
        }

        // ---------------------------------------------------------- store
        if (warp == 0 && a.nsteps > 0) {
            for (int f = lane; f < F; f += 32) {
                double e = 0;
                for (int w = 0; w < W; ++w) e += red[w * FM + f];
                q.efflux[f] = e;
            }
            for (int j = 0; j < NI; ++j) {
                double t = 0;
                for (int c = lane; c < nch; c += 32) t += fluxd[c * NI + j];
                t = warp_sum(t);
                if (lane == 0) q.total[j] = t;
            }
            __syncwarp();
            if (lane == 0) {
                if (!m.jsr_const)
                    for (int i = 0; i < NI; ++i) {
                        q.IjSR[i] = q.total[i] * m.V_elem;
                        q.nsr[i] = m.nsr[i];
                        q.jsr[i] = q.jsr_new[i];
                    }
                // stream state at the next unconsumed draw
                cbrng::State gd = g0;
                rng_jump(a.pow2, gd, 2ULL * (unsigned long long)D);
                for (int i = 0; i < 6; ++i) q.rng[i] = gd.s[i];
                q.draws += (unsigned long long)D;
            }
        }
        __syncthreads();
        {
            int4* dst = (int4*)((R*)a.fields + st.node_base * F);
            const int4* src = (const int4*)fa;
            const int n16 = (int)((size_t)F * np * sizeof(R) / 16);
            for (int k = tid; k < n16; k += blockDim.x) dst[k] = src[k];
            const unsigned int* qs = (const unsigned int*)&q;
            unsigned int* qd = (unsigned int*)(a.sc + s);
            for (int k = tid; k < (int)(sizeof(cb_site_scalars) / 4); k += blockDim.x) qd[k] = qs[k];
            R* cg = (R*)a.curgrid + st.node_base * NI;
            for (int c = tid; c < nch; c += blockDim.x) {
                a.ch_state[st.ch_off + c] = chs[c];
                if (cho[c])
                    for (int j = 0; j < NI; ++j) cg[j * np + chn[c]] = flux[c * NI + j];
            }
            if (rd3d) {
                R* cd = (R*)a.cyto + (size_t)s * CS * nc;
                for (int k = tid; k < CS * nc; k += blockDim.x) cd[k] = ca[k];
                if (a.nsteps > 0) {
                    const int* ptr = a.dep_ptr + (size_t)s * (mc2 + 1);
                    for (int n = tid; n < mc2; n += blockDim.x)
                        for (int c = 0; c < CS; ++c) {
                            int f = c < NI ? c : m.c_dyad_pair[c - NI];
                            if (f >= 0 && c >= NI) f += NI;
                            double dep = 0;
                            if (f >= 0)
                                for (int kk = ptr[n]; kk < ptr[n + 1]; ++kk) dep += terms[a.dep_term[st.term_off + kk] * FM + f];
                            a.cin[((size_t)s * CS + c) * mc2 + n] = dep;
                        }
                }
            }
        }
        __syncthreads();
    }
}

size_t align16(size_t v) { return (v + 15) / 16 * 16; }

// smem carve for the largest site; returns false if it exceeds the block limit
bool plan(const cb_dev& d, rs_args& a, int FM) {
    const cb_model& m = d.m;
    const size_t rs = d.precision == 0 ? 8 : 4;
    const int np = d.max_nodes;
    size_t off = align16((size_t)m.F * np * rs);
    a.np = np;
    a.off_fb = (int)off;
    off = align16(off + (size_t)m.F * np * rs);
    const int CS = m.n_ions + m.c_n_pairs;
    const bool rd3d = m.cyto_type == CB_CYTO_RD3D;
    a.off_ca = (int)off;
    if (rd3d) off = align16(off + (size_t)CS * d.nc * rs);
    a.off_cb = (int)off;
    if (rd3d) off = align16(off + (size_t)CS * d.nc * rs);
    a.off_terms = (int)off;
    if (rd3d) off = align16(off + (size_t)d.max_terms * FM * 8);
    a.off_cin = (int)off;
    if (rd3d) off = align16(off + (size_t)CS * m.mc * m.mc * 8);
    a.off_mask = (int)off;
    off = align16(off + (size_t)(np + 31) / 32 * 4);
    const int mch = std::max(d.max_ch, 1);
    a.off_chn = (int)off;
    off = align16(off + (size_t)mch * 4);
    a.off_chs = (int)off;
    off = align16(off + (size_t)mch * 4);
    a.off_cho = (int)off;
    off = align16(off + (size_t)mch * 4);
    a.off_flux = (int)off;
    off = align16(off + (size_t)mch * m.n_ions * rs);
    a.off_fluxd = (int)off;
    off = align16(off + (size_t)mch * m.n_ions * 8);
    a.off_mi = (int)off;
    off = align16(off + (size_t)mch * m.n_ions * 8);
    a.off_ring = (int)off;
    off = align16(off + (size_t)RING * 8);
    a.off_red = (int)off;
    off = align16(off + (size_t)(MAX_THREADS / 32) * FM * 8);
    a.off_sc = (int)off;
    off = align16(off + sizeof(cb_site_scalars));
    a.smem_bytes = (int)off;
    a.max_ch = d.max_ch;
    a.max_terms = d.max_terms;
    return off <= 227 * 1024 - 1024;
}

int pick_fm(int F) { return F <= 4 ? 4 : F <= 8 ? 8 : 16; }

template <typename R, int FM>
cudaError_t launch(cb_dev& d, rs_args& a, int threads, cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(k_resident<R, FM>, cudaFuncAttributeMaxDynamicSharedMemorySize, a.smem_bytes);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_resident<R, FM>, threads, a.smem_bytes);
    int grid = std::max(1, std::min(d.S, sms * std::max(per_sm, 1)));
    k_resident<R, FM><<<grid, threads, a.smem_bytes, st>>>(a);
    return cudaGetLastError();
}

int pick_threads(const cb_dev& d) {
    // one worker thread per ~8 interior columns, between 4 and 32 warps
    long long cols = 0;
    (void)cols;
    int nodes = d.max_nodes;
    int t = ((nodes / 8 + 31) / 32 + 1) * 32;
    return std::max(128, std::min(MAX_THREADS, t));
}

}  // namespace

bool cb_resident_fits(const cb_dev& d, int* threads, size_t* smem) {
    rs_args a{};
    int FM = pick_fm(d.m.F);
    // one ring refill must cover two draws per RyR (RING >= WINDOW + 2*max_ch)
    bool ok = plan(d, a, FM) && 2 * d.max_ch <= WINDOW;
    if (threads) *threads = pick_threads(d);
    if (smem) *smem = (size_t)a.smem_bytes;
    return ok;
}

cudaError_t cb_resident_step(cb_dev& d, long long n, cudaStream_t st, long long* launches) {
    if (n <= 0) return cudaSuccess;
    cb_dev& rsd = d;
    if (!rsd.rs_order) {
        // work queue order: largest cleft + cytosol first
        std::vector<cb_site> sites(d.S);
        cudaError_t e = cudaMemcpy(sites.data(), d.sites, sizeof(cb_site) * d.S, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return e;
        std::vector<int> order(d.S);
        for (int s = 0; s < d.S; ++s) order[s] = s;
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            return (long long)sites[x].nx * sites[x].ny * sites[x].nz > (long long)sites[y].nx * sites[y].ny * sites[y].nz;
        });
        if ((e = cudaMalloc(&rsd.rs_order, sizeof(int) * d.S)) != cudaSuccess) return e;
        if ((e = cudaMemcpy(rsd.rs_order, order.data(), sizeof(int) * d.S, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&rsd.rs_counter, sizeof(int))) != cudaSuccess) return e;
        // MRG32k3a: A^(2^k) for k < 64, both components
        std::vector<unsigned long long> p2(64 * 18);
        cbrng::Mat3 a1 = cbrng::step_matrix1(), a2 = cbrng::step_matrix2();
        for (int k = 0; k < 64; ++k) {
            for (int i = 0; i < 9; ++i) {
                p2[18 * k + i] = a1.a[i / 3][i % 3];
                p2[18 * k + 9 + i] = a2.a[i / 3][i % 3];
            }
            a1 = cbrng::matmul(a1, a1, cbrng::M1);
            a2 = cbrng::matmul(a2, a2, cbrng::M2);
        }
        if ((e = cudaMalloc(&rsd.rs_pow2, sizeof(unsigned long long) * p2.size())) != cudaSuccess) return e;
        if ((e = cudaMemcpy(rsd.rs_pow2, p2.data(), sizeof(unsigned long long) * p2.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return e;
    }
    rs_args a{};
    const int FM = pick_fm(d.m.F);
    if (!plan(d, a, FM)) return cudaErrorInvalidConfiguration;
    a.m = d.m;
    a.sites = d.sites;
    a.order = rsd.rs_order;
    a.S = d.S;
    a.counter = rsd.rs_counter;
    a.fields = d.fields[d.cur];
    a.curgrid = d.curgrid;
    a.ch_node = d.ch_node;
    a.ch_owner = d.ch_owner;
    a.ch_state = d.ch_state;
    a.mouth = d.mouth;
    a.NS = d.NS;
    a.sc = d.sc;
    a.cyto = d.cyto[d.ccur];
    a.cin = d.cin;
    a.rim_cnode = d.rim_cnode;
    a.dep_ptr = d.dep_ptr;
    a.dep_term = d.dep_term;
    a.nc = d.nc;
    a.pow2 = rsd.rs_pow2;
    a.spx0 = d.spx[0];
    a.spc0 = d.spc[0];
    a.spx1 = d.spx[1];
    a.spc1 = d.spc[1];
    a.nsteps = n;
    cudaError_t e = cudaMemsetAsync(rsd.rs_counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    const int threads = pick_threads(d);
    if (d.precision == 0) {
        if (FM == 4) e = launch<double, 4>(d, a, threads, st);
        else if (FM == 8) e = launch<double, 8>(d, a, threads, st);
        else e = launch<double, 16>(d, a, threads, st);
    } else {
        if (FM == 4) e = launch<float, 4>(d, a, threads, st);
        else if (FM == 8) e = launch<float, 8>(d, a, threads, st);
        else e = launch<float, 16>(d, a, threads, st);
    }
    if (launches) *launches += 1;
    return e;
}
