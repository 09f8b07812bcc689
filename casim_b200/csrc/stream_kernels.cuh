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
// for layouts these do not cover.
#pragma once

namespace stream {

constexpr int RD_THREADS = 256;
constexpr int CY_THREADS = 128;

// Cleft step of the columns [tile.y, tile.y + 256) of site tile.x.
template <typename R, int NI, int NP, int NZ>
__global__ void __launch_bounds__(RD_THREADS) k_rd_s(const __grid_constant__ cb_model m, const cb_site* __restrict__ sites,
                                                     const int2* __restrict__ tiles, const R* __restrict__ in,
                                                     R* __restrict__ out, const R* __restrict__ curg) {
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
    R c[F][NZ];
#pragma unroll
    for (int f = 0; f < F; ++f)
#pragma unroll
        for (int z = 0; z < NZ; ++z) c[f][z] = u[f * np + col + z * nxy];
    if (x == 0 || x == nx - 1 || y == 0 || y == ny - 1) {
        // rim nodes carry over; the Update sets them from the cytosol
#pragma unroll
        for (int f = 0; f < F; ++f)
#pragma unroll
            for (int z = 0; z < NZ; ++z) o[f * np + col + z * nxy] = c[f][z];
        return;
    }
    const R idx2 = (R)m.inv_dx2, idy2 = (R)m.inv_dy2, idz2 = (R)m.inv_dz2;
    const R dt = (R)m.dt;
    const R* __restrict__ cg = curg + st.node_base * NI;
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
            const R D = (R)(f < NI ? m.D_ion[f] : m.D_pair[f - NI]);
            if (D != (R)0) {
                R lap = (v[n + 1] - 2 * cc + v[n - 1]) * idx2 + (v[n + nx] - 2 * cc + v[n - nx]) * idy2;
                if (NZ > 1) lap = lap + (c[f][zr] - 2 * cc + c[f][zl]) * idz2;
                evo[f] = D * lap;
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
            const int b = m.pair_buf[p];
            R fr = (R)m.Ctot[b];
#pragma unroll
            for (int q = 0; q < NP; ++q)
                if (m.pair_buf[q] == b) fr -= val[NI + q];
            const int j = m.pair_ion[p];
            R ion = val[0];
#pragma unroll
            for (int i = 1; i < NI; ++i)
                if (j == i) ion = val[i];
            const R R1 = (R)m.koff[p] * val[NI + p] - (R)m.kon[p] * ion * fr;
            evo[NI + p] += -R1;
#pragma unroll
            for (int i = 0; i < NI; ++i)
                if (j == i) Rj[i] += R1;
        }
        const bool sl_layer = NZ == 1 || z == NZ - 1;
#pragma unroll
        for (int j = 0; j < NI; ++j) {
            R e = evo[j] + Rj[j];
            e += cg[j * np + n];
            if (sl_layer && m.has_sl[j]) {
                const R s1 = (R)m.K1[j] + val[j];
                const R s2 = (R)m.K2[j] + val[j];
                e *= (R)1 / ((R)1 + (R)(m.N1[j] * m.K1[j]) / (s1 * s1) + (R)(m.N2[j] * m.K2[j]) / (s2 * s2));
            }
            o[j * np + n] = val[j] + e * dt;
        }
#pragma unroll
        for (int p = 0; p < NP; ++p) o[(NI + p) * np + n] = val[NI + p] + evo[NI + p] * dt;
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
                evo[j2] -= (R)m.c_Jmax[is] * (i2 / (i2 + K2) - b2 / (b2 + K2));
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

}  // namespace stream
