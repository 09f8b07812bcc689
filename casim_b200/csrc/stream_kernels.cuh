// Streaming stencils of the plain path, specialised per species layout.
//
// The plain path keeps every field in HBM and sweeps it once per time step, so
// its stencils are bound by HBM bandwidth when they move each stored value once
// in and once out. These kernels fix the species counts at compile time (ions,
// ion-buffer pairs; cleft layers), so that every per-node quantity lives in
// registers, and give each thread one column of nodes (the cleft's z layers, the
// cytosol's planes): the column's own values are loaded once and serve as the
// z neighbours, the x and y neighbours come from the threads beside it (L1).
// Work is listed per block (site, first column) so that sites of uneven size
// leave no idle blocks. Arithmetic and its order per node are those of the
// generic kernels k_rd and k_cyto (the reference's node update,
// CaSim/DyadRD2DCPU.cpp:394-490, CaSim/DyadRDCPU.cpp:404-506), which stay in use
// for layouts these do not cover, except that FP32 fields divide with the approximate
// reciprocal in the sarcolemmal buffer factor and the SERCA term, as the resident path.
#pragma once

namespace stream {

// FP32: the approximate reciprocal (2 ulp), as the resident path; FP64: IEEE division
__device__ __forceinline__ float sdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double sdiv(double a, double b) { return a / b; }

template <typename R, int NI, int NP, int NZ>
__device__ __forceinline__ void interior_column(const cb_model& m, const cb_site& st, int col, const R* __restrict__ u, R* __restrict__ o,
                                                const R* __restrict__ curg);

constexpr int RD_THREADS = 256;
// resident blocks of k_rd_s asked of the compiler: a full SM (32 registers) where the
// column fits them without spilling (FP32, up to 3 species), fewer for wider columns
constexpr int rd_min_blocks(int w, int F) { return w == 4 ? (F <= 3 ? 8 : 4) : (F <= 3 ? 4 : 2); }
constexpr int CY_THREADS = 128;

// Cleft step of the columns [tile.y, tile.y + 256) of site tile.x. The rim columns take
// the Dirichlet values that the Update would set right after this step
// (CaSim/DyadRD2DCPU.cpp:274-303), from the same sources: the cytosol as it was before
// its latest step (cyto, RD3D) or the pool values of this step (sc); the Update then
// leaves the rim alone (k_update_s with prev set).
template <typename R, int NI, int NP, int NZ>
__global__ void __launch_bounds__(RD_THREADS, rd_min_blocks(sizeof(R), NI + NP)) k_rd_s(const __grid_constant__ cb_model m, const cb_site* __restrict__ sites,
                                                     const int2* __restrict__ tiles, const R* __restrict__ in,
                                                     R* __restrict__ out, const R* __restrict__ curg,
                                                     const cb_site_scalars* __restrict__ sc, const R* __restrict__ cyto,
                                                     const unsigned* __restrict__ chcol) {
    constexpr int F = NI + NP;
    const int2 tl = tiles[blockIdx.x];
    const cb_site st = sites[tl.x];
    const int nx = st.nx, ny = st.ny, nxy = nx * ny;
    const int col = tl.y + (int)threadIdx.x;
    if (col >= nxy) return;
    const long long np = st.npad;
    const R* __restrict__ u = in + st.node_base * F;
    R* __restrict__ o = out + st.node_base * F;
    const int y = col / nx, x = col - y * nx;
    // rim columns: their values are loaded first and stored last, so that a warp with rim
    // and interior lanes does not wait for the rim's loads before the interior's work
    const bool rim = x == 0 || x == nx - 1 || y == 0 || y == ny - 1;
    R b[F];
    if (rim) {
        if (m.cyto_type == CB_CYTO_RD3D) {
            const int CS = m.n_ions + m.c_n_pairs, nc = m.mc * m.mc * m.mc;
            const R* cy = cyto + (long long)tl.x * CS * nc;
            const int cn = cb_rim_cnode(x, y, nx, ny, m.dx, m.dy, m.hc, m.mc);
#pragma unroll
            for (int j = 0; j < NI; ++j) b[j] = cy[(long long)j * nc + cn];
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const int cq = m.dyad_c_pair[p];
                b[NI + p] = cq >= 0 ? cy[(long long)(NI + cq) * nc + cn] : (R)m.pair_init[p];
            }
        } else {
            const cb_site_scalars& q = sc[tl.x];
#pragma unroll
            for (int j = 0; j < NI; ++j) b[j] = (R)q.c_ions[j];
#pragma unroll
            for (int p = 0; p < NP; ++p) b[NI + p] = (R)q.c_bnd[p];
        }
    } else {
        // RyR currents exist only in the columns that hold a RyR (bit col of the site's
        // words in chcol); elsewhere the current grid is zero and is not read
        const long long bit = st.node_base + col;
        const bool has_ch = (chcol[bit >> 5] >> (bit & 31)) & 1u;
        interior_column<R, NI, NP, NZ>(m, st, col, u, o, has_ch ? curg : nullptr);
    }
    if (rim) {
#pragma unroll
        for (int f = 0; f < F; ++f)
#pragma unroll
            for (int z = 0; z < NZ; ++z) __stcs(&o[f * np + col + z * nxy], b[f]);
    }
}

// the interior column of k_rd_s; the loop-invariant model terms are read once
template <typename R, int NI, int NP, int NZ>
__device__ __forceinline__ void interior_column(const cb_model& m, const cb_site& st, int col, const R* __restrict__ u, R* __restrict__ o,
                                                const R* __restrict__ curg) {
    constexpr int F = NI + NP;
    const int nx = st.nx, nxy = nx * st.ny;
    const long long np = st.npad;
    R c[F][NZ];
#pragma unroll
    for (int f = 0; f < F; ++f)
#pragma unroll
        for (int z = 0; z < NZ; ++z) c[f][z] = u[f * np + col + z * nxy];
    const R idx2 = (R)m.inv_dx2, idy2 = (R)m.inv_dy2, idz2 = (R)m.inv_dz2;
    const R dt = (R)m.dt;
    // the column's RyR currents (curg null: none in this column)
    R cur[NI][NZ];
#pragma unroll
    for (int j = 0; j < NI; ++j)
#pragma unroll
        for (int z = 0; z < NZ; ++z) cur[j][z] = curg ? curg[st.node_base * NI + j * np + col + z * nxy] : (R)0;
    R D[F];
#pragma unroll
    for (int f = 0; f < F; ++f) D[f] = (R)(f < NI ? m.D_ion[f] : m.D_pair[f - NI]);
    R koff[NP > 0 ? NP : 1], kon[NP > 0 ? NP : 1], ctot[NP > 0 ? NP : 1];
    unsigned same[NP > 0 ? NP : 1];  // bit q: pair q binds pair p's buffer
    int pion[NP > 0 ? NP : 1];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const int b = m.pair_buf[p];
        koff[p] = (R)m.koff[p];
        kon[p] = (R)m.kon[p];
        ctot[p] = (R)m.Ctot[b];
        pion[p] = NI == 1 ? 0 : m.pair_ion[p];
        unsigned bits = 0;
#pragma unroll
        for (int q = 0; q < NP; ++q)
            if (m.pair_buf[q] == b) bits |= 1u << q;
        same[p] = bits;
    }
#pragma unroll
    for (int z = 0; z < NZ; ++z) {
        const int n = col + z * nxy;
        // reflecting z boundaries: z = 0 and z = nz-1 see their inner neighbour twice
        const int zl = z == 0 ? (NZ > 1 ? 1 : 0) : z - 1;
        const int zr = z == NZ - 1 ? (NZ > 1 ? NZ - 2 : 0) : z + 1;
        R val[F], evo[F];
#pragma unroll
        for (int f = 0; f < F; ++f) {
            const R* v = u + f * np;
            const R cc = c[f][z];
            val[f] = cc;
            if (D[f] != (R)0) {
                R lap = (v[n + 1] - 2 * cc + v[n - 1]) * idx2 + (v[n + nx] - 2 * cc + v[n - nx]) * idy2;
                if (NZ > 1) lap = lap + (c[f][zr] - 2 * cc + c[f][zl]) * idz2;
                evo[f] = D[f] * lap;
            } else {
                evo[f] = 0;
            }
        }
        // free buffer of each pair: its total less every pair bound to it, in pair order
        R Rj[NI > 0 ? NI : 1];
#pragma unroll
        for (int j = 0; j < NI; ++j) Rj[j] = 0;
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            R fr = ctot[p];
#pragma unroll
            for (int q = 0; q < NP; ++q)
                if (same[p] >> q & 1u) fr -= val[NI + q];
            R ion = val[0];
#pragma unroll
            for (int i = 1; i < NI; ++i)
                if (pion[p] == i) ion = val[i];
            const R R1 = koff[p] * val[NI + p] - kon[p] * ion * fr;
            evo[NI + p] += -R1;
#pragma unroll
            for (int i = 0; i < NI; ++i)
                if (pion[p] == i) Rj[i] += R1;
        }
        const bool sl_layer = NZ == 1 || z == NZ - 1;
#pragma unroll
        for (int j = 0; j < NI; ++j) {
            R e = evo[j] + Rj[j];
            e += cur[j][z];
            if (sl_layer && m.has_sl[j]) {
                const R s1 = (R)m.K1[j] + val[j];
                const R s2 = (R)m.K2[j] + val[j];
                e *= sdiv((R)1, (R)1 + sdiv((R)(m.N1[j] * m.K1[j]), s1 * s1) + sdiv((R)(m.N2[j] * m.K2[j]), s2 * s2));
            }
            __stcs(&o[j * np + n], val[j] + e * dt);
        }
#pragma unroll
        for (int p = 0; p < NP; ++p) __stcs(&o[(NI + p) * np + n], val[NI + p] + evo[NI + p] * dt);
    }
}

// RD3D cytosol step: block b serves the columns (i, j) [(b % bps) * 128, +128) of site
// b / bps, planes k = 0 .. mc-2 (the top plane is the bath); plane 0 reflects and takes
// the efflux deposits.
template <typename R, int NI, int NCP>
__global__ void __launch_bounds__(CY_THREADS) k_cyto_s(const __grid_constant__ cb_model m, int nc, int bps, const R* __restrict__ in,
                                                       R* __restrict__ out, const double* __restrict__ cin) {
    constexpr int CS = NI + NCP;
    const int s = blockIdx.x / bps;
    const int mc = m.mc, mc2 = mc * mc;
    const int col = (blockIdx.x - s * bps) * CY_THREADS + (int)threadIdx.x;
    if (col >= mc2) return;
    const int j = col / mc, i = col - j * mc;
    if (i == 0 || i == mc - 1 || j == 0 || j == mc - 1) return;
    const R* __restrict__ u = in + (long long)s * CS * nc;
    R* __restrict__ o = out + (long long)s * CS * nc;
    const double* __restrict__ ci = cin + (long long)s * CS * mc2;
    const R ih2 = (R)m.inv_hc2;
    const R dt = (R)m.dt;
    R D[CS];
#pragma unroll
    for (int c = 0; c < CS; ++c) D[c] = (R)(c < NI ? m.D_ion[c] : m.c_D_pair[c - NI]);
    // the column's planes k-1, k, k+1 (plane -1 reflects to plane 1)
    R lo[CS], cu[CS], hi[CS];
#pragma unroll
    for (int c = 0; c < CS; ++c) {
        cu[c] = u[(long long)c * nc + col];
        hi[c] = u[(long long)c * nc + col + mc2];
        lo[c] = hi[c];
    }
    for (int k = 0; k < mc - 1; ++k) {
        const int n = col + k * mc2;
        R evo[CS];
#pragma unroll
        for (int c = 0; c < CS; ++c) {
            const R* v = u + (long long)c * nc;
            const R cc = cu[c];
            evo[c] = D[c] * ((v[n + 1] - 2 * cc + v[n - 1]) * ih2 + (v[n + mc] - 2 * cc + v[n - mc]) * ih2 + (hi[c] - 2 * cc + lo[c]) * ih2);
        }
        int is = 0;
#pragma unroll
        for (int j2 = 0; j2 < NI; ++j2) {
            const R ion = cu[j2];
            R react = 0;
#pragma unroll
            for (int p = 0; p < NCP; ++p) {
                if (m.c_pair_ion[p] != j2) continue;
                const int b = m.c_pair_buf[p];
                R fr = (R)m.c_Ctot[b];
#pragma unroll
                for (int q = 0; q < NCP; ++q)
                    if (m.c_pair_buf[q] == b) fr -= cu[NI + q];
                const R Bq = cu[NI + p];
                const R R1 = (R)m.c_koff[p] * Bq - (R)m.c_kon[p] * ion * fr;
                evo[NI + p] += -R1;
                react += R1;
            }
            evo[j2] += react;
            if (m.c_serca[j2]) {
                const R i2 = ion * ion;
                const R K2 = (R)(m.c_Kup[is] * m.c_Kup[is]);
                const R b2 = (R)(m.c_bg[is] * m.c_bg[is]);
                evo[j2] -= (R)m.c_Jmax[is] * (sdiv(i2, i2 + K2) - b2 / (b2 + K2));
                ++is;
            }
        }
#pragma unroll
        for (int c = 0; c < CS; ++c) {
            R e = evo[c];
            if (k == 0) e += (R)ci[(long long)c * mc2 + col];
            o[(long long)c * nc + n] = cu[c] + e * dt;
        }
        if (k + 2 < mc) {
#pragma unroll
            for (int c = 0; c < CS; ++c) {
                lo[c] = cu[c];
                cu[c] = hi[c];
                hi[c] = u[(long long)c * nc + n + 2 * mc2];
            }
        }
    }
}

// The cytosol step above for a grid of MC^3 nodes fixed at compile time (MC = 25, the
// grid of the shipped configs), one block per site so that every x and y neighbour a
// column reads belongs to the block: the column's MC - 1 planes unrolled, every
// neighbour at a constant offset from the column's base, and the loop-invariant parts
// of the reaction and SERCA terms computed once (by the same expressions).
template <typename R, int NI, int NCP, int MC>
__global__ void __launch_bounds__((MC * MC + 31) / 32 * 32) k_cyto_m(const __grid_constant__ cb_model m, const R* __restrict__ in,
                                                                     R* __restrict__ out, const double* __restrict__ cin) {
    constexpr int CS = NI + NCP, MC2 = MC * MC, NC = MC2 * MC;
    const int s = blockIdx.x;
    const int col = (int)threadIdx.x;
    if (col >= MC2) return;
    const int j = col / MC, i = col - j * MC;
    // the bath columns copy their values plane by plane with the others, so that every
    // memory sector the block writes is written whole (a partly written sector is read
    // back from memory when it leaves L2)
    const bool bath = i == 0 || i == MC - 1 || j == 0 || j == MC - 1;
    const R* __restrict__ u = in + (long long)s * CS * NC + col;
    R* __restrict__ o = out + (long long)s * CS * NC + col;
    const double* __restrict__ ci = cin + (long long)s * CS * MC2 + col;
    const R ih2 = (R)m.inv_hc2;
    const R dt = (R)m.dt;
    R D[CS];
#pragma unroll
    for (int c = 0; c < CS; ++c) D[c] = (R)(c < NI ? m.D_ion[c] : m.c_D_pair[c - NI]);
    R koff[NCP > 0 ? NCP : 1], kon[NCP > 0 ? NCP : 1], ctot[NCP > 0 ? NCP : 1];
    unsigned same[NCP > 0 ? NCP : 1];  // bit q: pair q binds pair p's buffer
    int pion[NCP > 0 ? NCP : 1];
#pragma unroll
    for (int p = 0; p < NCP; ++p) {
        const int b = m.c_pair_buf[p];
        koff[p] = (R)m.c_koff[p];
        kon[p] = (R)m.c_kon[p];
        ctot[p] = (R)m.c_Ctot[b];
        pion[p] = NI == 1 ? 0 : m.c_pair_ion[p];
        unsigned bits = 0;
#pragma unroll
        for (int q = 0; q < NCP; ++q)
            if (m.c_pair_buf[q] == b) bits |= 1u << q;
        same[p] = bits;
    }
    bool serca[NI];
    R jmax[NI], k2[NI], bterm[NI];
    {
        int is = 0;
#pragma unroll
        for (int j2 = 0; j2 < NI; ++j2) {
            serca[j2] = m.c_serca[j2] != 0;
            jmax[j2] = k2[j2] = bterm[j2] = 0;
            if (serca[j2]) {
                k2[j2] = (R)(m.c_Kup[is] * m.c_Kup[is]);
                const R b2 = (R)(m.c_bg[is] * m.c_bg[is]);
                bterm[j2] = b2 / (b2 + k2[j2]);
                jmax[j2] = (R)m.c_Jmax[is];
                ++is;
            }
        }
    }
    // planes k-1, k, k+1 of the column and, loaded ahead, k+2 and k+3 (plane -1
    // reflects to plane 1)
    R lo[CS], cu[CS], hi[CS], p2[CS], p3[CS];
#pragma unroll
    for (int c = 0; c < CS; ++c) {
        cu[c] = u[c * NC];
        hi[c] = u[c * NC + MC2];
        p2[c] = u[c * NC + 2 * MC2];
        p3[c] = u[c * NC + 3 * MC2];
        lo[c] = hi[c];
    }
#pragma unroll
    for (int k = 0; k < MC - 1; ++k) {
        const int n = k * MC2;
        if (bath) {
#pragma unroll
            for (int c = 0; c < CS; ++c) __stcs(&o[c * NC + n], cu[c]);
        } else {
            R evo[CS];
#pragma unroll
            for (int c = 0; c < CS; ++c) {
                const R* v = u + c * NC + n;
                const R cc = cu[c];
                evo[c] = D[c] * ((v[1] - 2 * cc + v[-1]) * ih2 + (v[MC] - 2 * cc + v[-MC]) * ih2 + (hi[c] - 2 * cc + lo[c]) * ih2);
            }
#pragma unroll
            for (int j2 = 0; j2 < NI; ++j2) {
                const R ion = cu[j2];
                R react = 0;
#pragma unroll
                for (int p = 0; p < NCP; ++p) {
                    if (pion[p] != j2) continue;
                    R fr = ctot[p];
#pragma unroll
                    for (int q = 0; q < NCP; ++q)
                        if (same[p] >> q & 1u) fr -= cu[NI + q];
                    const R R1 = koff[p] * cu[NI + p] - kon[p] * ion * fr;
                    evo[NI + p] += -R1;
                    react += R1;
                }
                evo[j2] += react;
                if (serca[j2]) {
                    const R i2 = ion * ion;
                    evo[j2] -= jmax[j2] * (sdiv(i2, i2 + k2[j2]) - bterm[j2]);
                }
            }
#pragma unroll
            for (int c = 0; c < CS; ++c) {
                R e = evo[c];
                if (k == 0) e += (R)ci[c * MC2];
                __stcs(&o[c * NC + n], cu[c] + e * dt);
            }
        }
#pragma unroll
        for (int c = 0; c < CS; ++c) {
            lo[c] = cu[c];
            cu[c] = hi[c];
            hi[c] = p2[c];
            p2[c] = p3[c];
            if (k + 4 < MC) p3[c] = u[c * NC + n + 4 * MC2];
        }
    }
}

}  // namespace stream

namespace stream {

constexpr int UP_THREADS = 256;

// Sum of each of the K per-thread values over the block (UP_THREADS threads) in a fixed
// order: warp butterflies, then the warp partials in warp order; every thread gets the
// sums. red holds (UP_THREADS / 32) * K doubles.
template <int K>
__device__ __forceinline__ void block_sums(double (&v)[K], double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();  // red may still be read from its previous use
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) red[warp * K + k] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = red[k];
#pragma unroll
        for (int w = 1; w < UP_THREADS / 32; ++w) s += red[w * K + k];
        v[k] = s;
    }
}

// The Update of one site per block (CaSim/ParallelHybridSolver.cpp:159-175): mouth
// values, Dirichlet rim from the cytosol, efflux through the rim, the RD3D deposits
// into cytosol layer 0, RyR currents and the jSR coupling; the steps, their order and
// the values they read are those of the generic k_update, the per-node quantities in
// registers and the block sums by warp shuffles.
template <typename R, int NI, int NP, bool RD3D>
__global__ void __launch_bounds__(UP_THREADS) k_update_s(const __grid_constant__ cb_model m, int NS, const cb_site* __restrict__ sites,
                                                         R* __restrict__ fld, R* __restrict__ curg, const int* __restrict__ ch_node,
                                                         const int* __restrict__ ch_owner, const int* __restrict__ ch_state,
                                                         double* __restrict__ mouth, cb_site_scalars* __restrict__ sc, int nc,
                                                         const R* __restrict__ cyto, double* __restrict__ cin,
                                                         const int* __restrict__ rim_cnode, const int* __restrict__ dep_ptr,
                                                         const int* __restrict__ dep_term, const R* __restrict__ prev, int max_terms) {
    constexpr int F = NI + NP;
    constexpr int CSM = NI + 4;  // cytosol species slots (ions + at most 4 pairs)
    const int CS = m.n_ions + m.c_n_pairs;
    extern __shared__ double smem[];
    double* red = smem;                   // (UP_THREADS / 32) * (F + NI)
    double* terms = smem + 8 * (F + NI);  // RD3D: [term][F] efflux values
    const int s = blockIdx.x;
    const cb_site st = sites[s];
    cb_site_scalars& q = sc[s];
    R* u = fld + st.node_base * F;
    const int nx = st.nx, ny = st.ny, nz = st.nz, nxy = nx * ny;
    const long long np = st.npad;
    // RD3D: the site's deposit lists (per layer-0 cytosol node its efflux terms, in term
    // order) staged in shared memory behind the terms, loaded here so that the loads
    // overlap the phases before the deposit sums
    const int zmax0 = nz == 1 ? 1 : nz - 1;
    const int T0 = cb_efflux_terms(nx, ny, zmax0);
    int* s_ptr = (int*)(terms + (size_t)max_terms * F);
    int* s_term = s_ptr + (RD3D ? m.mc * m.mc + 1 : 0);
    if (RD3D) {
        const int mc2 = m.mc * m.mc;
        const int* ptr = dep_ptr + (long long)s * (mc2 + 1);
        for (int k = threadIdx.x; k <= mc2; k += UP_THREADS) s_ptr[k] = ptr[k];
        const int* dtm = dep_term + st.term_off;
        for (int k = threadIdx.x; k < T0; k += UP_THREADS) s_term[k] = dtm[k];
    }
    // 1. mouth values: ions, pairs, free buffers (CaSim/DyadRD2DCPU.cpp:361-380). After
    // k_rd_s (prev set) the rim holds its Dirichlet values already; a RyR on the rim
    // reads the value the step carried over there, which is prev's
    for (int c = threadIdx.x; c < st.n_ch; c += UP_THREADS) {
        const int node = ch_node[st.ch_off + c];
        double* mo = mouth + (long long)(st.ch_off + c) * NS;
        const R* src = u;
        if (prev) {
            const int cx = node % nx, cyy = (node / nx) % ny;
            if (cx == 0 || cx == nx - 1 || cyy == 0 || cyy == ny - 1) src = prev + st.node_base * F;
        }
        double v[F];
#pragma unroll
        for (int f = 0; f < F; ++f) v[f] = (double)src[f * np + node];
#pragma unroll
        for (int f = 0; f < F; ++f) mo[f] = v[f];
        for (int b = 0; b < m.n_buf; ++b) {
            double fr = m.Ctot[b];
#pragma unroll
            for (int p = 0; p < NP; ++p)
                if (m.pair_buf[p] == b) fr -= v[NI + p];
            mo[F + b] = fr;
        }
    }
    __syncthreads();
    // 2. Dirichlet edges from the cytosol (CaSim/DyadRD2DCPU.cpp:274-303), unless k_rd_s
    // set them (prev set)
    const int nrim = prev ? 0 : cb_rim_count(nx, ny);
    const R* cy = RD3D ? cyto + (long long)s * CS * nc : nullptr;
    for (int t = threadIdx.x; t < nrim * nz; t += UP_THREADS) {
        const int z = t / nrim, r = t - z * nrim;
        int x, y;
        cb_rim_xy(r, nx, ny, x, y);
        const int node = x + nx * y + nxy * z;
        if (!RD3D) {
#pragma unroll
            for (int j = 0; j < NI; ++j) u[j * np + node] = (R)q.c_ions[j];
#pragma unroll
            for (int p = 0; p < NP; ++p) u[(NI + p) * np + node] = (R)q.c_bnd[p];
        } else {
            const int cn = rim_cnode[st.rim_off + r];
#pragma unroll
            for (int j = 0; j < NI; ++j) u[j * np + node] = cy[(long long)j * nc + cn];
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const int cq = m.dyad_c_pair[p];
                u[(NI + p) * np + node] = cq >= 0 ? cy[(long long)(NI + cq) * nc + cn] : (R)m.pair_init[p];
            }
        }
    }
    __syncthreads();
    // 3. efflux (CaSim/DyadRD2DCPU.cpp:305-350): per-term values, block sums
    const int zmax = nz == 1 ? 1 : nz - 1;
    const int T = cb_efflux_terms(nx, ny, zmax);
    double part[F];
#pragma unroll
    for (int f = 0; f < F; ++f) part[f] = 0;
    for (int t = threadIdx.x; t < T; t += UP_THREADS) {
        int x0, y0, x1, y1, x2, y2, z;
        const int sel = cb_efflux_term(t, nx, ny, zmax, x0, y0, x1, y1, x2, y2, z);
        const double sf = sel == 0 ? m.sx : m.sy;
        const int n0 = x0 + nx * y0 + nxy * z, n1 = x1 + nx * y1 + nxy * z, n2 = x2 + nx * y2 + nxy * z;
        double a0[F], a1[F], a2[F];
#pragma unroll
        for (int f = 0; f < F; ++f) {
            a0[f] = (double)u[f * np + n0];
            a1[f] = (double)u[f * np + n1];
            a2[f] = (double)u[f * np + n2];
        }
#pragma unroll
        for (int f = 0; f < F; ++f) {
            const double D = f < NI ? m.D_ion[f] : m.D_pair[f - NI];
            const double g = 2 * a1[f] - 1.5 * a0[f] - 0.5 * a2[f];
            if (!RD3D) {
                part[f] += D * m.grad_mult * sf * g;
            } else {
                const double v = D * sf * g * m.inv_hc3;
                part[f] += v;
                terms[(long long)t * F + f] = v;
            }
        }
    }
    block_sums<F>(part, red);  // its barriers also publish the terms
    if (threadIdx.x == 0)
#pragma unroll
        for (int f = 0; f < F; ++f) q.efflux[f] = part[f];
    // 4. RD3D: deposit into the cytosol layer z = 0 in term order
    if (RD3D) {
        const int mc2 = m.mc * m.mc;
        const int* ptr = s_ptr;
        const int* dtm = s_term;
        for (int cn = threadIdx.x; cn < mc2; cn += UP_THREADS) {
            const int lo = ptr[cn], hi = ptr[cn + 1];
            double acc[CSM];
#pragma unroll
            for (int c = 0; c < CSM; ++c) acc[c] = 0;
            for (int k = lo; k < hi; ++k) {
                const int t = dtm[k];
#pragma unroll
                for (int c = 0; c < CSM; ++c) {
                    if (c >= CS) break;
                    int f = c < NI ? c : m.c_dyad_pair[c - NI];
                    if (f >= 0 && c >= NI) f += NI;
                    if (f >= 0) acc[c] += terms[(long long)t * F + f];
                }
            }
#pragma unroll
            for (int c = 0; c < CSM; ++c)
                if (c < CS) cin[((long long)s * CS + c) * mc2 + cn] = acc[c];
        }
    }
    // 5. RyR currents (CaSim/DyadRD2DCPU.cpp:243-264, CaSim/PassiveIonChannel.cpp:28-34)
    R* cg = curg + st.node_base * NI;
    double tot[NI];
#pragma unroll
    for (int j = 0; j < NI; ++j) tot[j] = 0;
    for (int c = threadIdx.x; c < st.n_ch; c += UP_THREADS) {
        const int node = ch_node[st.ch_off + c];
        const int state = ch_state[st.ch_off + c];
        const int own = ch_owner[st.ch_off + c];
#pragma unroll
        for (int j = 0; j < NI; ++j) {
            const double flux = state * (m.g[j] * (q.jsr_new[j] - (double)u[j * np + node]));
            if (own) cg[j * np + node] = (R)flux;
            tot[j] += flux;
        }
    }
    block_sums<NI>(tot, red);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < NI; ++j) q.total[j] = tot[j];
        // 6. jSR coupling (CaSim/SRPool.cpp:55-68)
        if (!m.jsr_const)
#pragma unroll
            for (int i = 0; i < NI; ++i) {
                q.IjSR[i] = q.total[i] * m.V_elem;
                q.nsr[i] = m.nsr[i];
                q.jsr[i] = q.jsr_new[i];
            }
    }
}

// Pools and two-state gating of one site per warp (CaSim/CytosolPool.cpp:217-268,
// CaSim/SRPool.cpp:70-89, CaSim/DyadChannels.cpp:97-130). The site's MRG32k3a stream is
// consumed in the reference's order (one draw per RyR test in RyR order, one more per
// transition) without a serial loop: lane l jumps to draw l of the stream (jump table J,
// row l: A^(2l)), the lanes draw 32 consecutive values at a time (then jump by A^62,
// row 31, to their draw of the next 32), and 32 RyRs are resolved per ballot, one more
// ballot after each transition. The stream state left behind is that at the first
// unused draw, as after the serial loop. With site_gate set, site s gates by
// gates[site_gate[s]] (per-site gating models) instead of the batch's model.
constexpr int PRE_WARPS = 4;
__global__ void __launch_bounds__(32 * PRE_WARPS) k_pre_r(const __grid_constant__ cb_model m, int S, int NS,
                                                          const cb_site* __restrict__ sites, cb_site_scalars* __restrict__ sc,
                                                          int* __restrict__ ch_state, const double* __restrict__ mouth,
                                                          const double* __restrict__ spx0, const double* __restrict__ spc0,
                                                          const double* __restrict__ spx1, const double* __restrict__ spc1,
                                                          const unsigned long long* __restrict__ J, const cb_gate* __restrict__ gates,
                                                          const int* __restrict__ site_gate) {
    __shared__ double s_u[PRE_WARPS][64];  // draws [we - 64, we), slot = draw & 63
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int s = blockIdx.x * PRE_WARPS + w;
    if (s >= S) return;  // whole warp
    const cb_site st = sites[s];
    cb_site_scalars& q = sc[s];
    const double dt = m.dt;
    if (lane == 0) {
        if (m.cyto_type == CB_CYTO_POOL) cb_pool_step(m, q, dt);
        cb_jsr_step(m, q, dt);
    }
    cbrng::State gl;  // this lane's draw we + lane
#pragma unroll
    for (int i = 0; i < 6; ++i) gl.s[i] = q.rng[i];
    cbrng::jump_by(J + 18 * lane, gl);
    cbrng::State gs = gl;  // state at this lane's draw of the latest chunk
    long long D = 0, we = 0;
    const int nch = st.n_ch;
    for (int c0 = 0; c0 < nch; c0 += 32) {
        const int cnt = min(32, nch - c0);
        const int c = c0 + lane;
        const bool act = lane < cnt;
        double p = 0;
        int stt = 0;
        if (act) {
            const double* mo = mouth + (long long)(st.ch_off + c) * NS;
            const double mg = m.mg_idx >= 0 ? mo[m.mg_idx] : 0.0;
            stt = ch_state[st.ch_off + c];
            if (site_gate) {  // the site's own gating model
                const cb_gate& g = gates[site_gate[s]];
                p = cb_rate(g, g.spx[0], g.spc[0], g.spx[1], g.spc[1], stt, mo[m.ca_idx], mg) * dt;
            } else {
                p = cb_rate(m, spx0, spc0, spx1, spc1, stt, mo[m.ca_idx], mg) * dt;
            }
        }
        int start = 0;
        while (start < cnt) {
            // draws D .. D + (cnt - start) - 1 must be in the ring
            while (we < D + (cnt - start)) {
                gs = gl;
                s_u[w][(we + lane) & 63] = cbrng::u01d_fold(gl);
                cbrng::jump_by(J + 18 * 31, gl);
                we += 32;
                __syncwarp();
            }
            const bool rem = act && lane >= start;
            const double u = rem ? s_u[w][(D + (lane - start)) & 63] : 2.0;
            const unsigned int t = __ballot_sync(0xffffffffu, rem && (u < p));
            if (t == 0u) {
                D += cnt - start;
                break;
            }
            const int f = __ffs(t) - 1;
            if (lane == f) ch_state[st.ch_off + c] = 1 - stt;
            D += (f - start) + 2;
            start = f + 1;
        }
        __syncwarp();
    }
    // the state at draw D: lane D - (we - 32) of the latest chunk before its draw, or, past
    // the chunk, lane D - we at its next chunk's draw (D - we is 0 or 1)
    const bool in_chunk = D < we;
    const int k = in_chunk ? (int)(D - (we - 32)) : (int)(D - we);
    unsigned int out[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) out[i] = __shfl_sync(0xffffffffu, in_chunk ? gs.s[i] : gl.s[i], k);
    if (lane == 0) {
        q.draws += (unsigned long long)D;
#pragma unroll
        for (int i = 0; i < 6; ++i) q.rng[i] = out[i];
    }
}

}  // namespace stream
