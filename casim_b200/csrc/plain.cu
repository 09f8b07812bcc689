// Plain path: one time step = one launch sequence over HBM-resident fields.
//
//   k_pre     one thread per site: cytosol pool ODE (CaSim/CytosolPool.cpp:217-268),
//             jSR pool ODE (CaSim/SRPool.cpp:70-89), two-state gating
//             (CaSim/DyadChannels.cpp:97-130) with the site's MRG32k3a stream
//   k_cyto    RD3D cytosol stencil (this project's 3D cytosol; no reference analog)
//   k_rd      cleft RD step of every interior node (CaSim/DyadRD2DCPU.cpp:394-490,
//             CaSim/DyadRDCPU.cpp:404-506), ping-pong buffers
//   k_update  one block per site: mouth gather, Dirichlet edges, efflux,
//             RyR currents, jSR coupling (CaSim/ParallelHybridSolver.cpp:159-175)
//
// This is the straightforward GPU formulation of the reference step and the
// denominator of the resident path's speed-up; it handles any site size.
#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "engine.h"
#include "mrg32k3a.cuh"
#include "mwc.h"
#include "physics.cuh"
#include "pools.cuh"
#include "stream_kernels.cuh"

namespace {

template <typename R>
__global__ void k_reset(cb_model m, const cb_site* __restrict__ sites, R* __restrict__ A, R* __restrict__ B,
                        R* __restrict__ cur, cb_site_scalars* __restrict__ sc, int* __restrict__ ch_state) {
    const int s = blockIdx.y;
    const cb_site st = sites[s];
    const int F = m.F;
    R* a = A + st.node_base * F;
    R* b = B + st.node_base * F;
    R* c = cur + st.node_base * m.n_ions;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < st.npad; n += gridDim.x * blockDim.x) {
        for (int f = 0; f < F; ++f) {
            R v = (R)(f < m.n_ions ? m.Cb[f] : m.pair_init[f - m.n_ions]);
            a[(long long)f * st.npad + n] = v;
            b[(long long)f * st.npad + n] = v;
        }
        for (int j = 0; j < m.n_ions; ++j) c[(long long)j * st.npad + n] = (R)0;
    }
    if (blockIdx.x == 0) {
        for (int k = threadIdx.x; k < st.n_ch; k += blockDim.x) ch_state[st.ch_off + k] = 0;
        if (threadIdx.x == 0) {
            cb_site_scalars& q = sc[s];
            for (int i = 0; i < CB_MAX_IONS; ++i) {
                q.jsr[i] = q.jsr_new[i] = q.jsr0[i];
                q.IjSR[i] = 0;
                q.nsr[i] = q.jsr0[i];
                q.total[i] = 0;
                q.c_ions[i] = i < m.n_ions ? m.c_bg[i] : 0.0;
            }
            for (int k = 0; k < CB_MAX_SPECIES; ++k) q.efflux[k] = 0;
            for (int b2 = 0; b2 < m.c_n_buf; ++b2) q.c_free[b2] = m.c_Ctot[b2];
            for (int p = 0; p < m.c_n_pairs; ++p) {
                q.c_pairs[p] = m.c_init[p];
                q.c_free[m.c_pair_buf[p]] -= m.c_init[p];
            }
            for (int p = 0; p < m.n_pairs; ++p)
                q.c_bnd[p] = m.dyad_c_pair[p] >= 0 ? m.c_init[m.dyad_c_pair[p]] : m.pair_init[p];
            q.release = 0;
        }
    }
}

template <typename R>
__global__ void k_cyto_reset(cb_model m, int nc, R* __restrict__ A, R* __restrict__ B, double* __restrict__ cin) {
    const int s = blockIdx.y;
    const int CS = m.n_ions + m.c_n_pairs;
    const int mc2 = m.mc * m.mc;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nc; n += gridDim.x * blockDim.x)
        for (int k = 0; k < CS; ++k) {
            R v = (R)(k < m.n_ions ? m.c_bg[k] : m.c_init[k - m.n_ions]);
            long long o = ((long long)s * CS + k) * nc + n;
            A[o] = v;
            B[o] = v;
            if (n < mc2) cin[((long long)s * CS + k) * mc2 + n] = 0.0;
        }
}

__global__ void k_init_open(const cb_site* __restrict__ sites, const int* __restrict__ first, int lo, int hi,
                            cb_site_scalars* __restrict__ sc, int* __restrict__ ch_state, int* __restrict__ ch_micro,
                            const cb_mwc_tab* __restrict__ mwc) {
    int s = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= hi) return;
    const cb_site st = sites[s];
    cb_site_scalars& q = sc[s];
    cbrng::State g;
    for (int i = 0; i < 6; ++i) g.s[i] = q.rng[i];
    // CaSim/DyadChannels.cpp:83-95: one draw per channel (SetMacroState(0, .)),
    // then one more for the channel that is opened
    // (SingleSiteMWC: each draw picks the micro-state of the macro state from the
    // stationary distribution, CaSim/QMatrixModel.cpp:38-58)
    for (int c = 0; c < st.n_ch; ++c) {
        const double u = cbrng::u01d_fold(g);
        ch_state[st.ch_off + c] = 0;
        if (mwc) ch_micro[st.ch_off + c] = cb_mwc_pick(*mwc, 0, u, ch_micro[st.ch_off + c]);
    }
    const double u = cbrng::u01d_fold(g);
    int f = first[s - lo];
    if (f >= 0 && f < st.n_ch) {
        ch_state[st.ch_off + f] = 1;
        if (mwc) {
            const int mi = cb_mwc_pick(*mwc, 1, u, ch_micro[st.ch_off + f]);
            ch_micro[st.ch_off + f] = mi;
            ch_state[st.ch_off + f] = mi >= CB_MWC_OPEN;
        }
    }
    q.draws += (unsigned long long)st.n_ch + 1;
    for (int i = 0; i < 6; ++i) q.rng[i] = g.s[i];
}

__global__ void k_pre(cb_model m, int S, int NS, const cb_site* __restrict__ sites, cb_site_scalars* __restrict__ sc,
                      int* __restrict__ ch_state, const double* __restrict__ mouth, const double* __restrict__ spx0,
                      const double* __restrict__ spc0, const double* __restrict__ spx1, const double* __restrict__ spc1,
                      int* __restrict__ ch_micro, const cb_mwc_tab* __restrict__ mwc) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const cb_site st = sites[s];
    cb_site_scalars& q = sc[s];
    const double dt = m.dt;
    if (m.cyto_type == CB_CYTO_POOL) cb_pool_step(m, q, dt);
    cb_jsr_step(m, q, dt);
    cbrng::State g;
    for (int i = 0; i < 6; ++i) g.s[i] = q.rng[i];
    unsigned long long draws = 0;
    for (int c = 0; c < st.n_ch; ++c) {
        const double* mo = mouth + (long long)(st.ch_off + c) * NS;
        double ca = mo[m.ca_idx];
        double mg = m.mg_idx >= 0 ? mo[m.mg_idx] : 0.0;
        if (mwc) {
            // SingleSiteMWC: escape rate of the micro-state, the second draw picks where to
            const int mi = ch_micro[st.ch_off + c];
            const double r = cb_mwc_exit(m.ch_par, *mwc, mi, ca, mg);
            ++draws;
            if (cbrng::u01d_fold(g) < r * dt) {
                const double u2 = cbrng::u01d_fold(g);
                ++draws;
                const int nx = cb_mwc_next(m.ch_par, *mwc, mi, ca, mg, r, u2);
                ch_micro[st.ch_off + c] = nx;
                ch_state[st.ch_off + c] = nx >= CB_MWC_OPEN;
            }
            continue;
        }
        int state = ch_state[st.ch_off + c];
        double r = cb_rate(m, spx0, spc0, spx1, spc1, state, ca, mg);
        ++draws;
        if (cbrng::u01d_fold(g) < r * dt) {
            (void)cbrng::u01d_fold(g);
            ++draws;
            ch_state[st.ch_off + c] = 1 - state;
        }
    }
    q.draws += draws;
    for (int i = 0; i < 6; ++i) q.rng[i] = g.s[i];
}

template <typename R>
__global__ void __launch_bounds__(256) k_cyto(cb_model m, int nc, const R* __restrict__ in, R* __restrict__ out,
                                              const double* __restrict__ cin) {
    const int s = blockIdx.y;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nc) return;
    const int mc = m.mc, mc2 = mc * mc;
    const int i = n % mc, j = (n / mc) % mc, k = n / mc2;
    if (i == 0 || i == mc - 1 || j == 0 || j == mc - 1 || k == mc - 1) return;
    const int CS = m.n_ions + m.c_n_pairs;
    const R* u = in + (long long)s * CS * nc;
    R* o = out + (long long)s * CS * nc;
    const int zl = k == 0 ? n + mc2 : n - mc2, zr = n + mc2;
    const R ih2 = (R)m.inv_hc2;
    R evo[CB_MAX_CSPECIES];
    for (int c = 0; c < CS; ++c) {
        const R* v = u + (long long)c * nc;
        R D = (R)(c < m.n_ions ? m.D_ion[c] : m.c_D_pair[c - m.n_ions]);
        R cc = v[n];
        evo[c] = D * ((v[n + 1] - 2 * cc + v[n - 1]) * ih2 + (v[n + mc] - 2 * cc + v[n - mc]) * ih2 + (v[zr] - 2 * cc + v[zl]) * ih2);
    }
    R fr[CB_MAX_CBUF];
    for (int b = 0; b < m.c_n_buf; ++b) fr[b] = (R)m.c_Ctot[b];
    for (int p = 0; p < m.c_n_pairs; ++p) fr[m.c_pair_buf[p]] -= u[(long long)(m.n_ions + p) * nc + n];
    int is = 0;
    for (int j2 = 0; j2 < m.n_ions; ++j2) {
        R ion = u[(long long)j2 * nc + n];
        R react = 0;
        for (int p = 0; p < m.c_n_pairs; ++p) {
            if (m.c_pair_ion[p] != j2) continue;
            R B = u[(long long)(m.n_ions + p) * nc + n];
            R R1 = (R)m.c_koff[p] * B - (R)m.c_kon[p] * ion * fr[m.c_pair_buf[p]];
            evo[m.n_ions + p] += -R1;
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
    const R dt = (R)m.dt;
    for (int c = 0; c < CS; ++c) {
        R e = evo[c];
        if (k == 0) e += (R)cin[((long long)s * CS + c) * mc2 + n];
        o[(long long)c * nc + n] = u[(long long)c * nc + n] + e * dt;
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_rd(cb_model m, const cb_site* __restrict__ sites, const R* __restrict__ in,
                                            R* __restrict__ out, const R* __restrict__ curg) {
    const int s = blockIdx.y;
    const cb_site st = sites[s];
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int nxy = st.nx * st.ny;
    if (n >= nxy * st.nz) return;
    const int F = m.F;
    const R* u = in + st.node_base * F;
    R* o = out + st.node_base * F;
    const int x = n % st.nx, y = (n / st.nx) % st.ny, z = n / nxy;
    if (x == 0 || x == st.nx - 1 || y == 0 || y == st.ny - 1) {
        for (int f = 0; f < F; ++f) o[(long long)f * st.npad + n] = u[(long long)f * st.npad + n];
        return;
    }
    const R idx2 = (R)m.inv_dx2, idy2 = (R)m.inv_dy2, idz2 = (R)m.inv_dz2;
    int zl = n, zr = n;
    if (m.dim == 3) {
        zl = z == 0 ? n + nxy : n - nxy;
        zr = z == st.nz - 1 ? n - nxy : n + nxy;
    }
    R val[CB_MAX_SPECIES], evo[CB_MAX_SPECIES];
    for (int f = 0; f < F; ++f) {
        const R* v = u + (long long)f * st.npad;
        R c = v[n];
        val[f] = c;
        R D = (R)(f < m.n_ions ? m.D_ion[f] : m.D_pair[f - m.n_ions]);
        if (D != (R)0) {
            R lap = (v[n + 1] - 2 * c + v[n - 1]) * idx2 + (v[n + st.nx] - 2 * c + v[n - st.nx]) * idy2;
            if (m.dim == 3) lap = lap + (v[zr] - 2 * c + v[zl]) * idz2;
            evo[f] = D * lap;
        } else {
            evo[f] = 0;
        }
    }
    R fr[CB_MAX_BUF];
    for (int b = 0; b < m.n_buf; ++b) fr[b] = (R)m.Ctot[b];
    for (int p = 0; p < m.n_pairs; ++p) fr[m.pair_buf[p]] -= val[m.n_ions + p];
    R Rj[CB_MAX_IONS];
    for (int j = 0; j < m.n_ions; ++j) Rj[j] = 0;
    for (int p = 0; p < m.n_pairs; ++p) {
        int j = m.pair_ion[p];
        R R1 = (R)m.koff[p] * val[m.n_ions + p] - (R)m.kon[p] * val[j] * fr[m.pair_buf[p]];
        evo[m.n_ions + p] += -R1;
        Rj[j] += R1;
    }
    const R dt = (R)m.dt;
    const R* cg = curg + st.node_base * m.n_ions;
    const bool sl_layer = (m.dim == 2) || (z == st.nz - 1);
    for (int j = 0; j < m.n_ions; ++j) {
        R e = evo[j] + Rj[j];
        e += cg[(long long)j * st.npad + n];
        if (sl_layer && m.has_sl[j]) {
            R s1 = (R)m.K1[j] + val[j];
            R s2 = (R)m.K2[j] + val[j];
            e *= (R)1 / ((R)1 + (R)(m.N1[j] * m.K1[j]) / (s1 * s1) + (R)(m.N2[j] * m.K2[j]) / (s2 * s2));
        }
        o[(long long)j * st.npad + n] = val[j] + e * dt;
    }
    for (int p = 0; p < m.n_pairs; ++p) o[(long long)(m.n_ions + p) * st.npad + n] = val[m.n_ions + p] + evo[m.n_ions + p] * dt;
}

// Deterministic block sum of `v` (blockDim.x == 256).
__device__ double block_sum(double v, double* red) {
    red[threadIdx.x] = v;
    __syncthreads();
    for (int w = blockDim.x >> 1; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    double r = red[0];
    __syncthreads();
    return r;
}

template <typename R>
__global__ void __launch_bounds__(256) k_update(cb_model m, int NS, const cb_site* __restrict__ sites, R* __restrict__ fld,
                                                R* __restrict__ curg, const int* __restrict__ ch_node,
                                                const int* __restrict__ ch_owner, const int* __restrict__ ch_state,
                                                double* __restrict__ mouth, cb_site_scalars* __restrict__ sc, int nc,
                                                const R* __restrict__ cyto, double* __restrict__ cin,
                                                const int* __restrict__ rim_cnode, const int* __restrict__ dep_ptr,
                                                const int* __restrict__ dep_term) {
    extern __shared__ double smem[];
    double* red = smem;            // 256
    double* terms = smem + 256;    // RD3D: max_terms * F deposit values
    const int s = blockIdx.x;
    const cb_site st = sites[s];
    cb_site_scalars& q = sc[s];
    const int F = m.F;
    R* u = fld + st.node_base * F;
    const int nx = st.nx, ny = st.ny, nz = st.nz, nxy = nx * ny;
    const long long np = st.npad;
    // 1. mouth values: ions, pairs, free buffers (CaSim/DyadRD2DCPU.cpp:361-380)
    for (int c = threadIdx.x; c < st.n_ch; c += blockDim.x) {
        int node = ch_node[st.ch_off + c];
        double* mo = mouth + (long long)(st.ch_off + c) * NS;
        double fr[CB_MAX_BUF];
        for (int b = 0; b < m.n_buf; ++b) fr[b] = m.Ctot[b];
        for (int f = 0; f < F; ++f) {
            double v = (double)u[f * np + node];
            mo[f] = v;
            if (f >= m.n_ions) fr[m.pair_buf[f - m.n_ions]] -= v;
        }
        for (int b = 0; b < m.n_buf; ++b) mo[F + b] = fr[b];
    }
    __syncthreads();
    // 2. Dirichlet edges from the cytosol (CaSim/DyadRD2DCPU.cpp:274-303)
    const int nrim = cb_rim_count(nx, ny);
    const int CS = m.n_ions + m.c_n_pairs;
    const R* cy = cyto ? cyto + (long long)s * CS * nc : nullptr;
    for (int t = threadIdx.x; t < nrim * nz; t += blockDim.x) {
        int r = t % nrim, z = t / nrim, x, y;
        cb_rim_xy(r, nx, ny, x, y);
        int node = x + nx * y + nxy * z;
        if (m.cyto_type == CB_CYTO_POOL) {
            for (int j = 0; j < m.n_ions; ++j) u[j * np + node] = (R)q.c_ions[j];
            for (int p = 0; p < m.n_pairs; ++p) u[(m.n_ions + p) * np + node] = (R)q.c_bnd[p];
        } else {
            int cn = rim_cnode[st.rim_off + r];
            for (int j = 0; j < m.n_ions; ++j) u[j * np + node] = cy[(long long)j * nc + cn];
            for (int p = 0; p < m.n_pairs; ++p) {
                int cq = m.dyad_c_pair[p];
                u[(m.n_ions + p) * np + node] = cq >= 0 ? cy[(long long)(m.n_ions + cq) * nc + cn] : (R)m.pair_init[p];
            }
        }
    }
    __syncthreads();
    // 3. efflux (CaSim/DyadRD2DCPU.cpp:305-350): per-term values, block sums
    const int zmax = m.dim == 2 ? 1 : nz - 1;
    const int T = cb_efflux_terms(nx, ny, zmax);
    double part[CB_MAX_SPECIES];
    for (int f = 0; f < F; ++f) part[f] = 0;
    const bool rd3d = m.cyto_type == CB_CYTO_RD3D;
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        int x0, y0, x1, y1, x2, y2, z;
        int sel = cb_efflux_term(t, nx, ny, zmax, x0, y0, x1, y1, x2, y2, z);
        double sf = sel == 0 ? m.sx : m.sy;
        int n0 = x0 + nx * y0 + nxy * z, n1 = x1 + nx * y1 + nxy * z, n2 = x2 + nx * y2 + nxy * z;
        for (int f = 0; f < F; ++f) {
            double D = f < m.n_ions ? m.D_ion[f] : m.D_pair[f - m.n_ions];
            double g = 2 * (double)u[f * np + n1] - 1.5 * (double)u[f * np + n0] - 0.5 * (double)u[f * np + n2];
            if (!rd3d) {
                part[f] += D * m.grad_mult * sf * g;
            } else {
                double v = D * sf * g * m.inv_hc3;
                part[f] += v;
                terms[(long long)t * F + f] = v;
            }
        }
    }
    for (int f = 0; f < F; ++f) {
        double tot = block_sum(part[f], red);
        if (threadIdx.x == 0) q.efflux[f] = tot;
    }
    // 4. RD3D: deposit into the cytosol layer z = 0 in term order
    if (rd3d) {
        __syncthreads();
        const int mc2 = m.mc * m.mc;
        const int* ptr = dep_ptr + (long long)s * (mc2 + 1);
        for (int cn = threadIdx.x; cn < mc2; cn += blockDim.x) {
            int lo = ptr[cn], hi = ptr[cn + 1];
            for (int c = 0; c < CS; ++c) {
                int f = c < m.n_ions ? c : m.c_dyad_pair[c - m.n_ions];
                if (f >= 0 && c >= m.n_ions) f += m.n_ions;
                double acc = 0;
                if (f >= 0)
                    for (int k = lo; k < hi; ++k) acc += terms[(long long)dep_term[st.term_off + k] * F + f];
                cin[((long long)s * CS + c) * mc2 + cn] = acc;
            }
        }
    }
    // 5. RyR currents (CaSim/DyadRD2DCPU.cpp:243-264, CaSim/PassiveIonChannel.cpp:28-34)
    R* cg = curg + st.node_base * m.n_ions;
    double tot[CB_MAX_IONS];
    for (int j = 0; j < m.n_ions; ++j) tot[j] = 0;
    for (int c = threadIdx.x; c < st.n_ch; c += blockDim.x) {
        int node = ch_node[st.ch_off + c];
        int state = ch_state[st.ch_off + c];
        for (int j = 0; j < m.n_ions; ++j) {
            double flux = state * (m.g[j] * (q.jsr_new[j] - (double)u[j * np + node]));
            if (ch_owner[st.ch_off + c]) cg[j * np + node] = (R)flux;
            tot[j] += flux;
        }
    }
    for (int j = 0; j < m.n_ions; ++j) {
        double t = block_sum(tot[j], red);
        if (threadIdx.x == 0) q.total[j] = t;
    }
    // 6. jSR coupling (CaSim/SRPool.cpp:55-68)
    if (threadIdx.x == 0 && !m.jsr_const)
        for (int i = 0; i < m.n_ions; ++i) {
            q.IjSR[i] = q.total[i] * m.V_elem;
            q.nsr[i] = m.nsr[i];
            q.jsr[i] = q.jsr_new[i];
        }
}

// The specialised stencils (stream_kernels.cuh) serve 1-2 ions with up to 4 pairs
// and a cleft of one layer (2D) or three (3D) at every site; the first step lists
// the cleft blocks (site, first column). Returns the tile count, 0 if not covered.
int stream_tiles(cb_dev& d) {
    if (d.st_nz >= 0) return d.st_nz > 0 ? d.st_ntiles : 0;
    d.st_nz = 0;
    const int np = d.m.n_pairs, ncp = d.m.c_n_pairs;
    if (d.m.n_ions < 1 || d.m.n_ions > 2 || np > 4 || ncp > 4) return 0;
    std::vector<cb_site> hs(d.S);
    if (cudaMemcpy(hs.data(), d.sites, sizeof(cb_site) * d.S, cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
    const int nz = d.m.dim == 2 ? 1 : 3;
    std::vector<int2> tiles;
    for (int s = 0; s < d.S; ++s) {
        if (hs[s].nz != nz) return 0;
        const int cols = hs[s].nx * hs[s].ny;
        for (int c = 0; c < cols; c += stream::RD_THREADS) tiles.push_back(make_int2(s, c));
    }
    if (tiles.empty() || tiles.size() > (size_t)INT32_MAX) return 0;
    if (cudaMalloc(&d.st_tiles, sizeof(int2) * tiles.size()) != cudaSuccess) return 0;
    if (cudaMemcpy(d.st_tiles, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d.st_tiles);
        d.st_tiles = nullptr;
        return 0;
    }
    d.st_ntiles = (int)tiles.size();
    // the columns that hold a RyR: bit (node_base + x + nx*y), one word per 32 nodes
    std::vector<unsigned> bits((size_t)(d.total_nodes + 31) / 32, 0u);
    std::vector<int> chn((size_t)d.total_ch);
    if (d.total_ch && cudaMemcpy(chn.data(), d.ch_node, sizeof(int) * chn.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
    for (int s = 0; s < d.S; ++s)
        for (int c = 0; c < hs[s].n_ch; ++c) {
            const long long b = hs[s].node_base + chn[hs[s].ch_off + c] % (hs[s].nx * hs[s].ny);
            bits[b >> 5] |= 1u << (b & 31);
        }
    if (cudaMalloc(&d.st_chcol, sizeof(unsigned) * bits.size()) != cudaSuccess) return 0;
    if (cudaMemcpy(d.st_chcol, bits.data(), sizeof(unsigned) * bits.size(), cudaMemcpyHostToDevice) != cudaSuccess) return 0;
    d.st_nz = nz;
    return d.st_ntiles;
}

// jump table of k_pre_r: row l < 32 holds A^(2l), both components (row 31, A^62, also
// takes a lane from one chunk of 32 draws to the next)
bool pre_jump(cb_dev& d) {
    if (d.pre_jump) return true;
    std::vector<unsigned long long> t(32 * 18);
    const cbrng::Mat3 a1 = cbrng::step_matrix1(), a2 = cbrng::step_matrix2();
    cbrng::Mat3 p1{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}}, p2 = p1;  // A^(2l)
    for (int l = 0; l < 32; ++l) {
        for (int i = 0; i < 9; ++i) {
            t[18 * l + i] = p1.a[i / 3][i % 3];
            t[18 * l + 9 + i] = p2.a[i / 3][i % 3];
        }
        for (int k = 0; k < 2; ++k) {
            p1 = cbrng::matmul(a1, p1, cbrng::M1);
            p2 = cbrng::matmul(a2, p2, cbrng::M2);
        }
    }
    if (cudaMalloc(&d.pre_jump, sizeof(unsigned long long) * t.size()) != cudaSuccess) {
        d.pre_jump = nullptr;
        return false;
    }
    if (cudaMemcpy(d.pre_jump, t.data(), sizeof(unsigned long long) * t.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d.pre_jump);
        d.pre_jump = nullptr;
        return false;
    }
    return true;
}

template <typename R, int NI, int NP, bool RD3D>
cudaError_t launch_update_s(cb_dev& d, cudaStream_t st, bool after_step) {
    size_t smem = 8 * (NI + NP + NI) * sizeof(double);
    if (RD3D) smem += (size_t)d.max_terms * (NI + NP) * sizeof(double) + sizeof(int) * ((size_t)d.m.mc * d.m.mc + 1 + d.max_terms);
    auto kern = stream::k_update_s<R, NI, NP, RD3D>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<d.S, stream::UP_THREADS, smem, st>>>(d.m, d.NS, d.sites, (R*)d.fields[d.cur], (R*)d.curgrid, d.ch_node, d.ch_owner, d.ch_state,
                                                d.mouth, d.sc, d.nc, (const R*)d.cyto[1 - d.ccur], d.cin, d.rim_cnode, d.dep_ptr,
                                                d.dep_term, after_step ? (const R*)d.fields[1 - d.cur] : nullptr, d.max_terms);
    return cudaGetLastError();
}

template <typename R, int NI, bool RD3D>
cudaError_t launch_update_np(cb_dev& d, cudaStream_t st, bool after_step) {
    switch (d.m.n_pairs) {
    case 0: return launch_update_s<R, NI, 0, RD3D>(d, st, after_step);
    case 1: return launch_update_s<R, NI, 1, RD3D>(d, st, after_step);
    case 2: return launch_update_s<R, NI, 2, RD3D>(d, st, after_step);
    case 3: return launch_update_s<R, NI, 3, RD3D>(d, st, after_step);
    default: return launch_update_s<R, NI, 4, RD3D>(d, st, after_step);
    }
}

// after_step: right after k_rd_s, which set the rim already
template <typename R>
cudaError_t launch_update(cb_dev& d, cudaStream_t st, bool after_step = false) {
    if (stream_tiles(d) > 0) {
        const bool rd3d = d.m.cyto_type == CB_CYTO_RD3D;
        if (d.m.n_ions == 1)
            return rd3d ? launch_update_np<R, 1, true>(d, st, after_step) : launch_update_np<R, 1, false>(d, st, after_step);
        return rd3d ? launch_update_np<R, 2, true>(d, st, after_step) : launch_update_np<R, 2, false>(d, st, after_step);
    }
    size_t smem = 256 * sizeof(double);
    if (d.m.cyto_type == CB_CYTO_RD3D) smem += (size_t)d.max_terms * d.m.F * sizeof(double);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_update<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    // the rim reads the cytosol as it was before its latest step (RD3D coupling)
    k_update<R><<<d.S, 256, smem, st>>>(d.m, d.NS, d.sites, (R*)d.fields[d.cur], (R*)d.curgrid, d.ch_node, d.ch_owner,
                                        d.ch_state, d.mouth, d.sc, d.nc, (const R*)d.cyto[1 - d.ccur], d.cin, d.rim_cnode,
                                        d.dep_ptr, d.dep_term);
    return cudaGetLastError();
}

template <typename R, int NI, int NP>
void launch_rd_s(cb_dev& d, cudaStream_t st) {
    const R* in = (const R*)d.fields[d.cur];
    R* out = (R*)d.fields[1 - d.cur];
    // the cytosol as it was before its latest step (k_cyto flipped ccur already)
    const R* cy = (const R*)d.cyto[1 - d.ccur];
    if (d.st_nz == 1)
        stream::k_rd_s<R, NI, NP, 1><<<d.st_ntiles, stream::RD_THREADS, 0, st>>>(d.m, d.sites, d.st_tiles, in, out, (const R*)d.curgrid,
                                                                                 d.sc, cy, d.st_chcol);
    else
        stream::k_rd_s<R, NI, NP, 3><<<d.st_ntiles, stream::RD_THREADS, 0, st>>>(d.m, d.sites, d.st_tiles, in, out, (const R*)d.curgrid,
                                                                                 d.sc, cy, d.st_chcol);
}

template <typename R, int NI>
void launch_rd_np(cb_dev& d, cudaStream_t st) {
    switch (d.m.n_pairs) {
    case 0: launch_rd_s<R, NI, 0>(d, st); break;
    case 1: launch_rd_s<R, NI, 1>(d, st); break;
    case 2: launch_rd_s<R, NI, 2>(d, st); break;
    case 3: launch_rd_s<R, NI, 3>(d, st); break;
    default: launch_rd_s<R, NI, 4>(d, st); break;
    }
}

template <typename R, int NI, int NCP>
void launch_cyto_s(cb_dev& d, cudaStream_t st) {
    if (d.m.mc == 25) {
        stream::k_cyto_m<R, NI, NCP, 25><<<d.S, 640, 0, st>>>(d.m, (const R*)d.cyto[d.ccur], (R*)d.cyto[1 - d.ccur], d.cin);
        return;
    }
    const int bps = (d.m.mc * d.m.mc + stream::CY_THREADS - 1) / stream::CY_THREADS;
    stream::k_cyto_s<R, NI, NCP><<<bps * d.S, stream::CY_THREADS, 0, st>>>(d.m, d.nc, bps, (const R*)d.cyto[d.ccur],
                                                                           (R*)d.cyto[1 - d.ccur], d.cin);
}

template <typename R, int NI>
void launch_cyto_np(cb_dev& d, cudaStream_t st) {
    switch (d.m.c_n_pairs) {
    case 0: launch_cyto_s<R, NI, 0>(d, st); break;
    case 1: launch_cyto_s<R, NI, 1>(d, st); break;
    case 2: launch_cyto_s<R, NI, 2>(d, st); break;
    case 3: launch_cyto_s<R, NI, 3>(d, st); break;
    default: launch_cyto_s<R, NI, 4>(d, st); break;
    }
}

template <typename R>
// ev (optional, 5 events): recorded before the gating kernel and after each of the
// gating, cytosol, cleft and Update kernels
cudaError_t launch_step(cb_dev& d, cudaStream_t st, cudaEvent_t* ev = nullptr) {
    auto mark = [&](int k) { return ev ? cudaEventRecord(ev[k], st) : cudaSuccess; };
    cudaError_t e0 = mark(0);
    if (e0 != cudaSuccess) return e0;
    const bool fast = stream_tiles(d) > 0;
    if (fast && !d.mwc && pre_jump(d))
        stream::k_pre_r<<<(d.S + stream::PRE_WARPS - 1) / stream::PRE_WARPS, 32 * stream::PRE_WARPS, 0, st>>>(
            d.m, d.S, d.NS, d.sites, d.sc, d.ch_state, d.mouth, d.spx[0], d.spc[0], d.spx[1], d.spc[1], d.pre_jump, d.gates,
            d.site_gate);
    else if (d.site_gate)
        return cudaErrorNotSupported;  // per-site models need k_pre_r
    else
        k_pre<<<(d.S + 127) / 128, 128, 0, st>>>(d.m, d.S, d.NS, d.sites, d.sc, d.ch_state, d.mouth, d.spx[0], d.spc[0],
                                                   d.spx[1], d.spc[1], d.ch_micro, d.mwc);
    if ((e0 = mark(1)) != cudaSuccess) return e0;
    if (d.m.cyto_type == CB_CYTO_RD3D) {
        if (fast) {
            if (d.m.n_ions == 1) launch_cyto_np<R, 1>(d, st);
            else launch_cyto_np<R, 2>(d, st);
        } else {
            dim3 g((d.nc + 255) / 256, d.S);
            k_cyto<R><<<g, 256, 0, st>>>(d.m, d.nc, (const R*)d.cyto[d.ccur], (R*)d.cyto[1 - d.ccur], d.cin);
        }
        d.ccur ^= 1;
    }
    if ((e0 = mark(2)) != cudaSuccess) return e0;
    if (fast) {
        if (d.m.n_ions == 1) launch_rd_np<R, 1>(d, st);
        else launch_rd_np<R, 2>(d, st);
    } else {
        dim3 g((d.max_nodes + 255) / 256, d.S);
        k_rd<R><<<g, 256, 0, st>>>(d.m, d.sites, (const R*)d.fields[d.cur], (R*)d.fields[1 - d.cur], (const R*)d.curgrid);
    }
    d.cur ^= 1;
    if ((e0 = mark(3)) != cudaSuccess) return e0;
    if ((e0 = launch_update<R>(d, st, fast)) != cudaSuccess) return e0;
    return mark(4);
}

// ---- surrogate-driven gating (no RD): the mouth Ca comes from the surrogate network

// features of every site (one thread per site): per RyR slot its open flag and
// grid position scaled to [-1, 1] by the cleft half-widths, then the jSR Ca of
// the first ion / 1000 uM, then each dyad buffer total relative to its config value
__global__ void k_sg_features(int S, int n_buf, int max_ch, int ld, const cb_site* __restrict__ sites, const int* __restrict__ ch_node,
                              const int* __restrict__ ch_state, const cb_site_scalars* __restrict__ sc, float* __restrict__ X) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const cb_site st = sites[s];
    float* row = X + (size_t)s * ld;
    for (int k = 0; k < ld; ++k) row[k] = 0.0f;
    const float hx = 0.5f * (st.nx - 1), hy = 0.5f * (st.ny - 1);
    for (int c = 0; c < st.n_ch && c < max_ch; ++c) {
        const int node = ch_node[st.ch_off + c];
        const int gx = node % st.nx, gy = (node / st.nx) % st.ny;
        row[3 * c] = (float)ch_state[st.ch_off + c];
        row[3 * c + 1] = (gx - hx) / hx;
        row[3 * c + 2] = (gy - hy) / hy;
    }
    row[3 * max_ch] = (float)(sc[s].jsr_new[0] / 1000.0);
    for (int b = 0; b < n_buf; ++b) row[3 * max_ch + 1 + b] = 1.0f;
}

// mouth Ca of every RyR from the network output: ca_ref * 10^y
__global__ void k_sg_mouth(int S, int NS, int ca_idx, double ca_ref, int ld, const cb_site* __restrict__ sites,
                           const float* __restrict__ Y, double* __restrict__ mouth) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const cb_site st = sites[s];
    for (int c = 0; c < st.n_ch && c < ld; ++c)
        mouth[(size_t)(st.ch_off + c) * NS + ca_idx] = ca_ref * exp10((double)Y[(size_t)s * ld + c]);
}

// n time steps of one site without the RD step: cytosol pool and jSR ODEs and
// RyR gating in the order of k_pre, then the part of Update that needs no
// field: RyR currents from the held mouth values and the jSR coupling
__global__ void k_sg_steps(cb_model m, int S, int NS, long long n, const cb_site* __restrict__ sites, cb_site_scalars* __restrict__ sc,
                           int* __restrict__ ch_state, const double* __restrict__ mouth, const double* __restrict__ spx0,
                           const double* __restrict__ spc0, const double* __restrict__ spx1, const double* __restrict__ spc1) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const cb_site st = sites[s];
    cb_site_scalars& q = sc[s];
    const double dt = m.dt;
    cbrng::State g;
    for (int i = 0; i < 6; ++i) g.s[i] = q.rng[i];
    unsigned long long draws = 0;
    // the mouth values are held, so the transition probability of each state is
    // fixed for the whole call: computed once for the first SG_CACHE RyRs
    constexpr int SG_CACHE = 32;
    double pc[2][SG_CACHE];
    const int ncache = st.n_ch < SG_CACHE ? st.n_ch : SG_CACHE;
    for (int c = 0; c < ncache; ++c) {
        const double* mo = mouth + (long long)(st.ch_off + c) * NS;
        const double ca = mo[m.ca_idx];
        const double mg = m.mg_idx >= 0 ? mo[m.mg_idx] : 0.0;
        pc[0][c] = cb_rate(m, spx0, spc0, spx1, spc1, 0, ca, mg) * dt;
        pc[1][c] = cb_rate(m, spx0, spc0, spx1, spc1, 1, ca, mg) * dt;
    }
    for (long long it = 0; it < n; ++it) {
        if (m.cyto_type == CB_CYTO_POOL) cb_pool_step(m, q, dt);
        cb_jsr_step(m, q, dt);
        for (int c = 0; c < st.n_ch; ++c) {
            const int state = ch_state[st.ch_off + c];
            double p;
            if (c < ncache) {
                p = pc[state][c];
            } else {
                const double* mo = mouth + (long long)(st.ch_off + c) * NS;
                const double mg = m.mg_idx >= 0 ? mo[m.mg_idx] : 0.0;
                p = cb_rate(m, spx0, spc0, spx1, spc1, state, mo[m.ca_idx], mg) * dt;
            }
            ++draws;
            if (cbrng::u01d_fold(g) < p) {
                (void)cbrng::u01d_fold(g);
                ++draws;
                ch_state[st.ch_off + c] = 1 - state;
            }
        }
        double tot[CB_MAX_IONS];
        for (int j = 0; j < m.n_ions; ++j) tot[j] = 0;
        for (int c = 0; c < st.n_ch; ++c) {
            const int state = ch_state[st.ch_off + c];
            const double* mo = mouth + (long long)(st.ch_off + c) * NS;
            for (int j = 0; j < m.n_ions; ++j) tot[j] += state * (m.g[j] * (q.jsr_new[j] - mo[j]));
        }
        for (int j = 0; j < m.n_ions; ++j) q.total[j] = tot[j];
        if (!m.jsr_const)
            for (int i = 0; i < m.n_ions; ++i) {
                q.IjSR[i] = q.total[i] * m.V_elem;
                q.nsr[i] = m.nsr[i];
                q.jsr[i] = q.jsr_new[i];
            }
    }
    q.draws += draws;
    for (int i = 0; i < 6; ++i) q.rng[i] = g.s[i];
}

template <typename R>
cudaError_t reset_impl(cb_dev& d, cudaStream_t st) {
    dim3 g(std::max(1, std::min(64, (d.max_nodes + 255) / 256)), d.S);
    k_reset<R><<<g, 256, 0, st>>>(d.m, d.sites, (R*)d.fields[0], (R*)d.fields[1], (R*)d.curgrid, d.sc, d.ch_state);
    d.cur = 0;
    if (d.m.cyto_type == CB_CYTO_RD3D) {
        dim3 gc((d.nc + 255) / 256, d.S);
        k_cyto_reset<R><<<gc, 256, 0, st>>>(d.m, d.nc, (R*)d.cyto[0], (R*)d.cyto[1], d.cin);
        d.ccur = 0;
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t cb_plain_reset(cb_dev& d, cudaStream_t st) {
    return d.precision == 0 ? reset_impl<double>(d, st) : reset_impl<float>(d, st);
}

cudaError_t cb_plain_init_opening(cb_dev& d, const int* d_first, int lo, int hi, cudaStream_t st) {
    int n = hi - lo;
    if (n <= 0) return cudaSuccess;
    k_init_open<<<(n + 127) / 128, 128, 0, st>>>(d.sites, d_first, lo, hi, d.sc, d.ch_state, d.ch_micro, d.mwc);
    return cudaGetLastError();
}

cudaError_t cb_plain_update(cb_dev& d, cudaStream_t st, long long* launches) {
    if (launches) *launches += 1;
    return d.precision == 0 ? launch_update<double>(d, st) : launch_update<float>(d, st);
}

bool cb_plain_streaming(cb_dev& d) { return stream_tiles(d) > 0; }

bool cb_plain_gating_ready(cb_dev& d) { return stream_tiles(d) > 0 && !d.mwc && pre_jump(d); }

cudaError_t cb_plain_step_marked(cb_dev& d, cudaStream_t st, cudaEvent_t* ev) {
    return d.precision == 0 ? launch_step<double>(d, st, ev) : launch_step<float>(d, st, ev);
}

cudaError_t cb_plain_step(cb_dev& d, long long n, cudaStream_t st, long long* launches) {
    const int per = 3 + (d.m.cyto_type == CB_CYTO_RD3D ? 1 : 0);
    for (long long i = 0; i < n; ++i) {
        cudaError_t e = d.precision == 0 ? launch_step<double>(d, st) : launch_step<float>(d, st);
        if (e != cudaSuccess) return e;
        if (launches) *launches += per;
    }
    return cudaSuccess;
}

cudaError_t cb_sg_features(cb_dev& d, int max_ch, int ld, float* X, cudaStream_t st) {
    k_sg_features<<<(d.S + 127) / 128, 128, 0, st>>>(d.S, d.m.n_buf, max_ch, ld, d.sites, d.ch_node, d.ch_state, d.sc, X);
    return cudaGetLastError();
}

cudaError_t cb_sg_mouth(cb_dev& d, const float* Y, int ld, double ca_ref, cudaStream_t st) {
    k_sg_mouth<<<(d.S + 127) / 128, 128, 0, st>>>(d.S, d.NS, d.m.ca_idx, ca_ref, ld, d.sites, Y, d.mouth);
    return cudaGetLastError();
}

namespace {
// per site: the largest relative error of the network's mouth Ca over its open RyRs (the
// mouths whose Ca sets the release flux; a site with none open has error 0); the max over
// sites (non-negative doubles order as their bit patterns) and the failing sites
__global__ void k_sg_residual(int S, int NS, int ca_idx, double ca_ref, int ld, double tol, const cb_site* __restrict__ sites,
                              const int* __restrict__ ch_state, const float* __restrict__ Y, const double* __restrict__ mouth,
                              unsigned long long* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const cb_site st = sites[s];
    double e = 0;
    for (int c = 0; c < st.n_ch && c < ld; ++c) {
        if (!ch_state[st.ch_off + c]) continue;
        const double rd = mouth[(size_t)(st.ch_off + c) * NS + ca_idx];
        const double pr = ca_ref * exp10((double)Y[(size_t)s * ld + c]);
        const double r = fabs(pr - rd) / fabs(rd);
        e = r > e ? r : (r != r ? INFINITY : e);
    }
    atomicMax(out, (unsigned long long)__double_as_longlong(e));
    if (!(e <= tol)) atomicAdd(out + 1, 1ULL);
}
}  // namespace

cudaError_t cb_sg_residual(const cb_dev& d, const float* Y, int ld, double ca_ref, double tol, unsigned long long* scratch,
                           double* worst, double* fail_fraction, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(scratch, 0, 2 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    k_sg_residual<<<(d.S + 127) / 128, 128, 0, st>>>(d.S, d.NS, d.m.ca_idx, ca_ref, ld, tol, d.sites, d.ch_state, Y, d.mouth, scratch);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    unsigned long long h[2];
    if ((e = cudaMemcpyAsync(h, scratch, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    double w;
    std::memcpy(&w, &h[0], sizeof(w));
    *worst = w;
    *fail_fraction = d.S ? (double)h[1] / d.S : 0.0;
    return cudaSuccess;
}

cudaError_t cb_sg_steps(cb_dev& d, long long n, cudaStream_t st) {
    bool used = false;
    cudaError_t e = cb_sg_steps_warp(d, n, st, &used);
    if (e != cudaSuccess || used) return e;
    k_sg_steps<<<(d.S + 127) / 128, 128, 0, st>>>(d.m, d.S, d.NS, n, d.sites, d.sc, d.ch_state, d.mouth, d.spx[0], d.spc[0],
                                                  d.spx[1], d.spc[1]);
    return cudaGetLastError();
}
