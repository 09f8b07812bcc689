// Resident path kernel: each site lives in the shared memory of a thread-block
// cluster (1..16 blocks, one per SM) for all K time steps of a launch, so HBM
// is touched once per site per launch. Host logic: resident.cu.
//
// Layout of a site over the C blocks (ranks) of its cluster:
//   cleft   rows y in [lo_r, hi_r) per rank (lo_r = r*ny/C), stored with one halo
//           row on each side, all x and z, every stored species, ping-pong;
//   RD3D    cytosol planes k in [plo_r, phi_r) of the updated range [0, mc-1),
//           stored with one halo plane on each side, ping-pong.
// Per step (the reference loop body CaSim/ParallelHybridSolver.cpp:421-429
// followed by Update(), :270-286):
//   phase A  warp 0: RyR gating (CaSim/DyadChannels.cpp:97-130);
//            warp 1: reductions of the previous Update, jSR coupling, cytosol
//            pool ODE (CaSim/CytosolPool.cpp:217-288), jSR ODE (CaSim/SRPool.cpp:70-89);
//            both run redundantly and bit-identically on every rank;
//            warps 2..: cleft stencil of the rank's rows (CaSim/DyadRD2DCPU.cpp:394-490,
//            CaSim/DyadRDCPU.cpp:404-506), a lane marching down a strip of rows
//            with the previous, current and next row in registers, and the
//            RD3D cytosol planes, marching along z.
//   phase B  Dirichlet rim, mouth gather, RyR currents, efflux
//            (CaSim/DyadRD2DCPU.cpp:243-392) of the rank's rows; halo rows and
//            planes, mouth values, partial sums and RD3D coupling values are
//            stored into the peers' shared memory (DSMEM) in slots double-
//            buffered by step parity.
//   one cluster barrier (release/acquire) per step.
//
// RyR gating consumes the site's MRG32k3a stream in exactly the reference's
// order without its serial loop: warp 0 keeps a ring of pre-generated draws
// (32 lanes x 16 contiguous draws per refill, lanes jumped ahead by matrix
// powers) and resolves 32 channels per ballot, re-evaluating after each
// transition, which consumes one extra draw.
#pragma once
#include <cooperative_groups.h>

#include "engine.h"
#include "mrg32k3a.cuh"
#include "physics.cuh"

namespace cbres {

namespace cg = cooperative_groups;

constexpr int RING = 1024;               // pre-generated draws per site
constexpr int LANE_DRAWS = 16;           // contiguous draws per lane per refill
constexpr int WINDOW = 32 * LANE_DRAWS;  // draws per refill
constexpr int MAX_THREADS = 512;
constexpr int MAX_WARPS = MAX_THREADS / 32;
constexpr int JUMP_ROW = 64;             // pow table row holding A^(2*31*LANE_DRAWS)

// Threads per block a kernel is compiled for. A stencil lane keeps three rows
// of CSM species x NZ layers in registers; FP64 3D layouts with many species
// get 255 registers per thread (256 threads) instead of 128 (512 threads).
// block size bound of a specialisation; clusters of 4 and more blocks stop at 384 threads
// (three warps per SM sub-partition) so that the step loop keeps its values in registers (168
// per thread instead of 128)
__host__ __device__ constexpr int max_threads(int rbytes, int csm, int nz, int C) {
    return 3 * nz * csm * rbytes / 4 > 60 ? 256 : C >= 4 ? 384 : 512;
}
// pair capacity of the kernel specialisation that serves NI ions and NP pairs
__host__ __device__ constexpr int npm_of(int NI, int NP) { return NP <= 2 ? 2 : 4; }

// Stencil constants in the field precision R, so that they are kernel-parameter
// operands of the arithmetic (each value is the (R) cast of the model's double,
// or of the product noted).
template <typename R>
struct rs_const {
    R D_ion[CB_MAX_IONS], K1[CB_MAX_IONS], K2[CB_MAX_IONS];
    R A1[CB_MAX_IONS], A2[CB_MAX_IONS];  // (R)(N1*K1), (R)(N2*K2)
    R D_pair[CB_MAX_PAIRS], kon[CB_MAX_PAIRS], koff[CB_MAX_PAIRS];
    R ctp[CB_MAX_PAIRS];                 // total of the pair's buffer
    int same[CB_MAX_PAIRS];              // bit p2: pair p2 binds the same buffer
    R idx2, idy2, idz2, dt, ih2;
    // RD3D cytosol species c: ions, then cytosol pairs at NI + p
    R cD[CB_MAX_CSPECIES], ckon[CB_MAX_CSPECIES], ckoff[CB_MAX_CSPECIES], cctp[CB_MAX_CSPECIES];
    int csame[CB_MAX_CSPECIES];          // bit c2: species c2 is a pair of the same buffer
    int cdep[CB_MAX_CSPECIES];           // deposit slot feeding species c, or -1
    R Kup2[CB_MAX_IONS], Jmax[CB_MAX_IONS];  // by SERCA index: (R)(Kup^2)
    R serca0[CB_MAX_IONS];                   // (R)(bg^2 / (bg^2 + Kup^2)): SERCA uptake at rest
};

// a field-precision constant of the launch, read straight from the kernel parameter
#define RSK(x) (sizeof(R) == 4 ? (R)a.kf.x : (R)a.kd.x)

// FP32: a * (1/b) with the approximate reciprocal (2 ulp); FP64: IEEE division
__device__ __forceinline__ float div_fast(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double div_fast(double a, double b) { return a / b; }

// division by a per-site constant d >= 1 as a multiply-high and a shift
// (round-up reciprocal m = floor(2^32 (2^s - d) / d) + 1, s = ceil(log2 d));
// exact for 0 <= n < 2^31
struct fastdiv {
    unsigned m, s;
};
__device__ __forceinline__ fastdiv make_fastdiv(unsigned d) {
    unsigned s = 0;
    while ((1u << s) < d) ++s;
    return {(unsigned)(((1ull << 32) * ((1ull << s) - d)) / d + 1), s};
}
__device__ __forceinline__ int fdiv(int n, fastdiv f) { return (int)((__umulhi((unsigned)n, f.m) + (unsigned)n) >> f.s); }

template <bool B>
struct bconst {
    static constexpr bool value = B;
};

struct rs_args {
    // cumulative row weights of the ranks: rank r holds rows [ny*rw[r]/rw[C], ny*rw[r+1]/rw[C])
    unsigned short rw[17];
    cb_model m;
    rs_const<float> kf;
    rs_const<double> kd;
    const cb_site* sites;
    const int* order;  // sites of this launch, largest first
    int S;             // sites in order[]
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
    const unsigned long long* pow2;  // [65][2][9]: A^(2^k) for k < 64, then the refill jump
    const double* spx0;
    const double* spc0;
    const double* spx1;
    const double* spc1;
    long long nsteps;
    // shared-memory carve (bytes, identical for every block of the launch)
    int cap_cleft;  // stored cleft nodes per species per rank
    int cap_cyto;   // stored cytosol nodes per species per rank
    int cps;        // stride of a stored cytosol plane (mc^2 rounded up to 16 bytes)
    int max_ch, max_terms, max_rim, FD;
    int off_fb, off_ca, off_cb, off_chidx, off_chn, off_chs, off_cho, off_chr, off_ftab, off_pg, off_ring, off_redw,
        off_rede, off_redt, off_terms, off_crim, off_ulist, off_rimc, off_slot, off_dptr, off_dterm, off_ltask, off_sc, smem_bytes;
};

using cbrng::fold_mod;
__device__ __forceinline__ double u01d_fast(cbrng::State& g) { return cbrng::u01d_fold(g); }

using cbrng::mat_apply;

__device__ __forceinline__ void jump_row(const unsigned long long* pow2, cbrng::State& g, int k) {
    mat_apply<cbrng::M1>(pow2 + 18 * k, g.s);
    mat_apply<cbrng::M2>(pow2 + 18 * k + 9, g.s + 3);
}

// advance by `steps` recurrence steps (binary powering with the 2^k table)
__device__ __forceinline__ void rng_jump(const unsigned long long* pow2, cbrng::State& g, unsigned long long steps) {
    for (int k = 0; steps; ++k, steps >>= 1)
        if (steps & 1ULL) jump_row(pow2, g, k);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int C>
__device__ __forceinline__ void cluster_barrier() {
    if constexpr (C == 1) __syncthreads();
    else cg::this_cluster().sync();
}

// pointer to `p` (this block's shared memory) in the shared memory of rank r
template <int C, typename T>
__device__ __forceinline__ T* peer(T* p, int r) {
    if constexpr (C == 1) return p;
    else return cg::this_cluster().map_shared_rank(p, r);
}

__host__ __device__ __forceinline__ int row_lo(const unsigned short* rw, int r, int ny, int C) {
    return (int)(((long long)rw[r] * ny) / rw[C]);
}

// deposit slot of dyad species f (its index among species with a cytosol counterpart), or -1
__device__ __forceinline__ int dslot(const cb_model& m, int NI, int f) {
    int k = 0;
    for (int g = 0; g < f; ++g)
        if (g < NI || m.dyad_c_pair[g - NI] >= 0) ++k;
    return (f < NI || m.dyad_c_pair[f - NI] >= 0) ? k : -1;
}

template <typename R, int NI, int NPM, int NZ, int C>
__global__ void __launch_bounds__(max_threads(sizeof(R), NI + NPM, NZ, C), 1) k_resident(const __grid_constant__ rs_args a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_site;
    // RNG of warp 0, kept in shared memory so it holds no registers during the stencils:
    // lane l's stream at draw s_we + l*LANE_DRAWS; s_D draws consumed
    __shared__ unsigned int s_rng[32 * 6];
    __shared__ long long s_D, s_we;
    __shared__ int s_nu;   // RD3D: slots of this rank's rim
    __shared__ int s_nlt;  // Update rim tasks of this rank
    __shared__ int s_nrow[4];  // first and end row of the lower and the upper neighbour rank
    __shared__ int s_nd;  // RD3D, plane-0 rank: layer-0 cytosol nodes that receive efflux deposits
    constexpr int CSM = NI + NPM;  // cytosol species slots
    constexpr int FP = NI + NPM;   // cleft species slots
    const cb_model& m = a.m;
    const int NP = m.n_pairs, F = NI + NP;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, W = blockDim.x >> 5;
    int rank = 0;
    if constexpr (C > 1) rank = (int)cg::this_cluster().block_rank();
    const bool rd3d = m.cyto_type == CB_CYTO_RD3D;
    const int mc = m.mc, mc2 = mc * mc, nc = a.nc, CS = m.n_ions + m.c_n_pairs;
    const int FD = a.FD;

    R* fa = (R*)smem;
    R* fb = (R*)(smem + a.off_fb);
    R* ca = (R*)(smem + a.off_ca);
    R* cb = (R*)(smem + a.off_cb);
    unsigned short* chidx = (unsigned short*)(smem + a.off_chidx);  // 1 + owning RyR at a node, 0 if none
    int* chn = (int*)(smem + a.off_chn);   // local node of own RyRs, -1 otherwise
    int* chs = (int*)(smem + a.off_chs);   // state of every RyR of the site
    int* cho = (int*)(smem + a.off_cho);   // site node (x + nx*(y + ny*z)) | owner flag in bit 30
    int* chr = (int*)(smem + a.off_chr);   // rim index of own RyRs on the rim, -1 otherwise
    R* ftab = (R*)(smem + a.off_ftab);     // [(1 + max_ch)][NI]: RyR currents, slot 0 is zero
    double* pg = (double*)(smem + a.off_pg);      // [2][max_ch] transition probability of each RyR at the next gating
    double* ring = (double*)(smem + a.off_ring);
    double* redw = (double*)(smem + a.off_redw);  // [MAX_WARPS][F + NI]
    double* rede = (double*)(smem + a.off_rede);  // [2][C][F]
    double* redt = (double*)(smem + a.off_redt);  // [2][C][NI]
    R* terms = (R*)(smem + a.off_terms);          // [2][max_terms][FD] RD3D efflux terms (plane-0 rank)
    unsigned short* crim = (unsigned short*)(smem + a.off_crim);    // RD3D: rim index -> slot of its layer-0 cytosol node
    unsigned short* ulist = (unsigned short*)(smem + a.off_ulist);  // RD3D: layer-0 cytosol node of each slot (this rank's rim)
    R* rimc = (R*)(smem + a.off_rimc);                              // RD3D: [CSM][max_rim] their start-of-step values
    unsigned short* slot_of = (unsigned short*)(smem + a.off_slot); // RD3D: [mc^2] slot of a cytosol node, scratch at load;
    unsigned short* dnode = slot_of;                                // then (plane-0 rank) the nodes that receive deposits
    unsigned short* dptr = (unsigned short*)(smem + a.off_dptr);    // RD3D: deposit list offsets per layer-0 node
    // RD3D: stored position of each efflux term; the terms are stored grouped by receiving
    // layer-0 cytosol node (node cn's in [dptr[cn], dptr[cn + 1]), the oracle's order within)
    unsigned short* tpos = (unsigned short*)(smem + a.off_dterm);
    int* ltask = (int*)(smem + a.off_ltask);                        // Update rim tasks: line | first node << 16
    cb_site_scalars& q = *(cb_site_scalars*)(smem + a.off_sc);

    const double dt = m.dt;
    const int FDn = F + NI;

    for (;;) {
        if (rank == 0 && tid == 0) {
            const int v = atomicAdd(a.counter, 1);
            for (int r = 0; r < C; ++r) *peer<C>(&s_site, r) = v;
        }
        cluster_barrier<C>();
        const int qsite = s_site;
        if (qsite >= a.S) break;
        const int s = a.order[qsite];
        const cb_site st = a.sites[s];
        const int nx = st.nx, ny = st.ny, nz = st.nz, nxy = nx * ny, np = st.npad;
        const int nch = st.n_ch;
        const int zmax = NZ == 1 ? 1 : nz - 1;
        const int lo = row_lo(a.rw, rank, ny, C), hi = row_lo(a.rw, rank + 1, ny, C);
        const int slo = lo > 0 ? lo - 1 : 0, shi = hi < ny ? hi + 1 : ny;
        const int nr = shi - slo;
        const int lstride = nx * nr;  // z stride in local storage
        const int nloc = lstride * nz;
        const int nplanes = mc - 1;
        // RD3D: rank r holds plane block (r + C/2) mod C, so that plane 0 (deposits, rim
        // values) sits on rank r0 = C - C/2, away from the first and last row blocks, which
        // carry the long y-edge rim lines
        const int pb = (rank + C / 2) % C, r0 = (C - C / 2) % C;
        const int plo = rd3d ? (int)(((long long)pb * nplanes) / C) : 0;
        const int phi = rd3d ? (int)(((long long)(pb + 1) * nplanes) / C) : 0;
        const int splo = plo > 0 ? plo - 1 : 0, sphi = phi + 1;
        const int cloc = (sphi - splo) * mc2;
        const int cap = a.cap_cleft, ccap = a.cap_cyto, cps = a.cps;

        // ---------------------------------------------------------- load
        {
            const R* g = (const R*)a.fields + st.node_base * F;
            for (int f = 0; f < FP; ++f)
                for (int z = 0; z < nz; ++z) {
                    const R* src = g + (long long)f * np + (long long)nx * (slo + (long long)ny * z);
                    for (int k = tid; k < lstride; k += blockDim.x) {
                        const R v = f < F ? src[k] : (R)0;  // unused species slots hold zeros
                        fa[f * cap + lstride * z + k] = v;
                        fb[f * cap + lstride * z + k] = v;
                    }
                }
            for (int k = tid; k < nloc; k += blockDim.x) chidx[k] = 0;
            const unsigned int* qs = (const unsigned int*)(a.sc + s);
            unsigned int* qd = (unsigned int*)&q;
            for (int k = tid; k < (int)(sizeof(cb_site_scalars) / 4); k += blockDim.x) qd[k] = qs[k];
            for (int k = tid; k < NI; k += blockDim.x) ftab[k] = (R)0;
            if (rd3d) {
                const R* cs = (const R*)a.cyto + (size_t)s * CS * nc;
                for (int c = 0; c < CSM; ++c)
                    for (int k = tid; k < cloc; k += blockDim.x) {
                        const R v = c < CS ? cs[(size_t)c * nc + (size_t)splo * mc2 + k] : (R)0;
                        const int pl = k / mc2, l = pl * cps + (k - pl * mc2);
                        ca[c * ccap + l] = v;
                        cb[c * ccap + l] = v;
                    }
                const int nrim = cb_rim_count(nx, ny);
                for (int k = tid; k < nrim; k += blockDim.x) crim[k] = (unsigned short)a.rim_cnode[st.rim_off + k];
                for (int k = tid; k < mc2; k += blockDim.x) slot_of[k] = 0xFFFF;
                const int* gp = a.dep_ptr + (size_t)s * (mc2 + 1);
                for (int k = tid; k <= mc2; k += blockDim.x) dptr[k] = (unsigned short)gp[k];
                for (int k = tid; k < gp[mc2]; k += blockDim.x) tpos[a.dep_term[st.term_off + k]] = (unsigned short)k;
            }
        }
        __syncthreads();
        if (rd3d && tid == 0) {
            // the distinct layer-0 cytosol nodes under this rank's rim, in rim order: each
            // step they are gathered from the plane-0 rank once (phase A) instead of at every use
            int nu = 0;
            auto add = [&](int ri) {
                const int cn = crim[ri];
                if (slot_of[cn] == 0xFFFF) {
                    slot_of[cn] = (unsigned short)nu;
                    ulist[nu++] = (unsigned short)cn;
                }
                crim[ri] = slot_of[cn];
            };
            for (int y = lo; y < hi; ++y) {
                add(y);
                add(ny + y);
            }
            if (lo == 0)
                for (int i = 0; i < nx - 2; ++i) add(2 * ny + i);
            if (hi == ny)
                for (int i = 0; i < nx - 2; ++i) add(2 * ny + nx - 2 + i);
            s_nu = nu;
            if (rank == r0) {
                // nodes receiving deposits, the longest term lists first (their items go to
                // different threads of warps 0 and 1)
                int nd = 0;
                for (int cn = 0; cn < mc2; ++cn)
                    if (dptr[cn + 1] > dptr[cn]) dnode[nd++] = (unsigned short)cn;
                for (int i = 1; i < nd; ++i) {
                    const unsigned short v = dnode[i];
                    const int lv = dptr[v + 1] - dptr[v];
                    int j = i - 1;
                    while (j >= 0 && dptr[dnode[j] + 1] - dptr[dnode[j]] < lv) {
                        dnode[j + 1] = dnode[j];
                        --j;
                    }
                    dnode[j + 1] = v;
                }
                s_nd = nd;
            }
        }
        if (tid == 33) {
            for (int side = 0; side < 2; ++side) {
                const int nb = side == 0 ? rank - 1 : rank + 1;
                const bool in = nb >= 0 && nb < C;
                s_nrow[2 * side] = in ? row_lo(a.rw, nb, ny, C) : 0;
                s_nrow[2 * side + 1] = in ? row_lo(a.rw, nb + 1, ny, C) : 0;
            }
        }
        if (tid == 32) {
            // Update rim tasks: 32 consecutive nodes of one line, dealt chunk-major so that
            // the long y-edge lines of the first and last rank spread over the warps (one-block
            // sites: whole lines, one task each)
            const int zm = NZ == 1 ? 1 : nz - 1;
            const int nrw = max(min(hi, ny - 1) - max(lo, 1), 0);
            int nt = 0;
            for (int k = 0;; ++k) {
                bool any = false;
                for (int l = 0; l < 4 * (nz + zm); ++l) {
                    const bool eff = l >= 4 * nz;
                    const int e = (eff ? l - 4 * nz : l) & 3;
                    const bool mine = e == 2 ? lo == 0 : hi == ny;
                    const int len = e < 2 ? (eff ? nrw : hi - lo) : mine ? (eff ? nx : nx - 2) : 0;
                    if (32 * k < len) {
                        ltask[nt++] = l | (32 * k) << 16;
                        any = true;
                    }
                }
                if (!any || C == 1) break;
            }
            s_nlt = nt;
        }
        for (int c = tid; c < nch; c += blockDim.x) {
            const int gnode = a.ch_node[st.ch_off + c];
            const int x = gnode % nx, y = (gnode / nx) % ny, z = gnode / nxy;
            chs[c] = a.ch_state[st.ch_off + c];
            const bool owner = a.ch_owner[st.ch_off + c] != 0;
            cho[c] = gnode | (owner ? (1 << 30) : 0);
            const bool own = y >= lo && y < hi;
            const int ln = own ? x + nx * ((y - slo) + nr * z) : -1;
            chn[c] = ln;
            chr[c] = (x == 0 || y == 0 || x == nx - 1 || y == ny - 1) ? cb_rim_index(x, y, nx, ny) : -1;
            const double* mo = a.mouth + (size_t)(st.ch_off + c) * a.NS;
            pg[a.max_ch + c] = cb_rate(m, a.spx0, a.spc0, a.spx1, a.spc1, chs[c], mo[m.ca_idx], m.mg_idx >= 0 ? mo[m.mg_idx] : 0.0) *
                               m.dt;  // parity-1 slot
            if (own) {
                if (owner) chidx[ln] = (unsigned short)(1 + c);
                for (int j = 0; j < NI; ++j) {
                    // current of the last Update: state * g * (jSR - Ca at the node)
                    const double fl = chs[c] * (m.g[j] * (q.jsr_new[j] - (double)fa[j * cap + ln]));
                    ftab[(1 + c) * NI + j] = (R)fl;
                }
            }
        }
        // RNG (warp 0): lane l holds the stream at draw D + l*LANE_DRAWS of the next window
        if (warp == 0) {
            cbrng::State gl;
            for (int i = 0; i < 6; ++i) gl.s[i] = q.rng[i];
            rng_jump(a.pow2, gl, 2ULL * LANE_DRAWS * lane);
            for (int i = 0; i < 6; ++i) s_rng[lane * 6 + i] = gl.s[i];
            if (lane == 0) s_D = s_we = 0;
        }
        // stencil partition of this rank: a lane owns one interior column of a
        // strip of RS rows; (strip, column) pairs are dealt to the worker lanes
        // in order, so a warp may span two strips and no lane idles on a ragged
        // row end. RS minimises the rounds x (rows per strip + 1 row of setup).
        const int ylo = max(lo, 1), yhi = min(hi, ny - 1);
        const int nrows = max(yhi - ylo, 0);
        const int nxi = nx - 2;
        const int NW = W - 2;
        int RS = max(nrows, 1);
        {
            long long best = 1LL << 62;
            for (int rs = 1; rs <= nrows; ++rs) {
                const int tasks = nxi * ((nrows + rs - 1) / rs);
                const long long cost = (long long)((tasks + 32 * NW - 1) / (32 * NW)) * (rs + 1);
                if (cost < best) {
                    best = cost;
                    RS = rs;
                }
            }
        }
        const int nchunk = (nrows + RS - 1) / RS;
        // RD3D partition: (i, j) columns x chunks of PL planes over the worker threads
        const int ni = mc - 2, ncol = ni * ni, npr = phi - plo, NWT = blockDim.x - 64;
        int PC = 1;
        if (rd3d) {
            long long best = 1LL << 62;
            for (int pc = 1; pc <= npr; ++pc) {
                const long long cost = (long long)((ncol * pc + NWT - 1) / NWT) * ((npr + pc - 1) / pc + 1);
                if (cost < best) {
                    best = cost;
                    PC = pc;
                }
            }
        }
        const int PL = npr > 0 ? (npr + PC - 1) / PC : 1;
        const fastdiv fd_nxi = make_fastdiv(max(nxi, 1)), fd_ncol = make_fastdiv(max(ncol, 1)), fd_ni = make_fastdiv(max(ni, 1));
        cluster_barrier<C>();

        // ---------------------------------------------------------- steps
        for (long long it = 0; it < a.nsteps; ++it) {
            const int par = (int)(it & 1), prv = par ^ 1;
            const bool last = it == a.nsteps - 1;
            if (warp == 0) {
                // ---- RyR gating: draw D+i tests channel i until a transition takes one more draw
                long long D = s_D;
                const long long we = s_we;
                if (we - D < 2LL * nch) {  // ring refill: at least two draws per channel available
                    cbrng::State gl;
                    for (int i = 0; i < 6; ++i) gl.s[i] = s_rng[lane * 6 + i];
                    const long long base = we + (long long)lane * LANE_DRAWS;
                    for (int i = 0; i < LANE_DRAWS; ++i) ring[(base + i) & (RING - 1)] = u01d_fast(gl);
                    jump_row(a.pow2, gl, JUMP_ROW);  // to this lane's chunk of the next window
                    for (int i = 0; i < 6; ++i) s_rng[lane * 6 + i] = gl.s[i];
                    __syncwarp();
                    if (lane == 0) s_we = we + WINDOW;
                }
                __syncwarp();
                // probabilities of the previous Update's mouth values, computed in its phase B
                const double* pprev = pg + prv * a.max_ch;
                for (int base = 0; base < nch; base += 32) {
                    const int c = base + lane;
                    const int cnt = min(32, nch - base);
                    const bool act = lane < cnt;
                    double p = 0;
                    int stt = 0;
                    if (act) {
                        stt = chs[c];
                        p = pprev[c];
                    }
                    int start = 0;
                    while (start < cnt) {
                        const bool rem = act && lane >= start;
                        const double u = rem ? ring[(D + (lane - start)) & (RING - 1)] : 2.0;
                        const unsigned int t = __ballot_sync(0xffffffffu, rem && (u < p));
                        if (t == 0u) {
                            D += cnt - start;
                            break;
                        }
                        const int f = __ffs(t) - 1;
                        if (lane == f) chs[c] = 1 - stt;
                        D += (f - start) + 2;
                        start = f + 1;
                    }
                }
                __syncwarp();
                if (lane == 0) s_D = D;
            } else if (warp == 1) {
                // ---- pools: reductions of the previous Update (rank order on every rank)
                if (it > 0) {
                    for (int f = lane; f < F; f += 32) {
                        double e = 0;
                        for (int r = 0; r < C; ++r) e += rede[(prv * C + r) * F + f];
                        q.efflux[f] = e;
                    }
                    for (int j = lane; j < NI; j += 32) {
                        double t = 0;
                        for (int r = 0; r < C; ++r) t += redt[(prv * C + r) * NI + j];
                        q.total[j] = t;
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
                                const double R1 = m.c_koff[p] * q.c_pairs[p] - m.c_kon[p] * q.c_ions[j] * q.c_free[m.c_pair_buf[p]];
                                evo_p[p] = -R1;
                                react += R1;
                                if (m.c_in_dyad[p]) evo_p[p] += q.efflux[NI + ipd++];
                            }
                            evo_i[j] = react + q.efflux[j];
                            if (m.c_serca[j]) {
                                const double i2 = q.c_ions[j] * q.c_ions[j];
                                const double K2 = m.c_Kup[is] * m.c_Kup[is];
                                const double b2 = m.c_bg[is] * m.c_bg[is];
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
                            const double Iref = 1 / m.tau_refill[i] * (q.nsr[i] - q.jsr[i]);
                            q.jsr_new[i] = q.jsr[i] + dt / beta * (Iref - q.IjSR[i] / m.V_jsr);
                        }
                        if (m.ca_idx >= 0) q.release += q.IjSR[m.ca_idx] * dt;
                    }
                }
                if (rd3d) {
                    // rim values of this step: the plane-0 rank's cytosol plane 0 at the start of the
                    // step (its current buffer, untouched until the step ends)
                    const R* c0 = peer<C>(ca, r0);
                    for (int u = lane; u < s_nu; u += 32) {
                        const int cn = ulist[u];
#pragma unroll
                        for (int c = 0; c < CSM; ++c)
                            if (c < CS) rimc[c * a.max_rim + u] = c0[c * ccap + cn];
                    }
                }
                __syncwarp();
            }
            if (warp < 2 && rd3d && rank == r0) {
                // ---- warps 0 and 1, after the gating and the pools: the efflux deposits of the
                // previous Update per receiving layer-0 cytosol node and deposit slot (each sum
                // replaces its node's first term, which is all plane 0 reads); the worker warps
                // meet this at named barrier 1 before their cytosol planes
                if (it > 0) {
                    R* tp = terms + (size_t)prv * a.max_terms * FD;
                    for (int t = tid; t < s_nd * FD; t += 64) {
                        const int k = t / FD, sl = t - k * FD;
                        const int cn = dnode[k];
                        const int q1 = dptr[cn + 1];
                        int q2 = dptr[cn];
                        // four interleaved partial sums: under a cleft wider than the cytosol the
                        // nodes at the cytosol's edge take dozens of terms
                        double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
                        for (; q2 + 4 <= q1; q2 += 4) {
                            const R t0v = tp[q2 * FD + sl], t1v = tp[(q2 + 1) * FD + sl], t2v = tp[(q2 + 2) * FD + sl],
                                    t3v = tp[(q2 + 3) * FD + sl];
                            s0 += (double)t0v;
                            s1 += (double)t1v;
                            s2 += (double)t2v;
                            s3 += (double)t3v;
                        }
                        for (; q2 < q1; ++q2) s0 += (double)tp[q2 * FD + sl];
                        tp[dptr[cn] * FD + sl] = (R)((s0 + s1) + (s2 + s3));
                    }
                }
                asm volatile("bar.arrive 1, %0;" ::"r"(blockDim.x) : "memory");
            }
            if (warp >= 2) {
                // ---- worker warps: cleft stencil, strips of rows with a lane per x.
                // All FP = NI + NPM species slots are stepped (unused slots hold zeros and
                // have zero coefficients), so the loops carry no species-count tests;
                // constants are kernel-parameter operands.
                const int wk = warp - 2;
                for (int t = wk * 32 + lane; t < nxi * nchunk; t += NW * 32) {
                    const int ch = fdiv(t, fd_nxi);
                    const int x = 1 + (t - ch * nxi);
                    const int y0 = ylo + ch * RS, y1 = min(y0 + RS, yhi);
                    // previous / current / next row of every species and layer
                    R vP[FP][NZ], vC[FP][NZ], vN[FP][NZ];
                    int nrow = x + nx * (y0 - slo);
#pragma unroll
                    for (int f = 0; f < FP; ++f)
#pragma unroll
                        for (int z = 0; z < NZ; ++z) {
                            vP[f][z] = fa[f * cap + nrow - nx + lstride * z];
                            vC[f][z] = fa[f * cap + nrow + lstride * z];
                        }
                    for (int y = y0; y < y1; ++y, nrow += nx) {
#pragma unroll
                        for (int f = 0; f < FP; ++f)
#pragma unroll
                            for (int z = 0; z < NZ; ++z) vN[f][z] = fa[f * cap + nrow + nx + lstride * z];
#pragma unroll
                        for (int z = 0; z < NZ; ++z) {
                            const int n = nrow + lstride * z;
                            const int zl = z == 0 ? (NZ > 1 ? 1 : 0) : z - 1;
                            const int zr = z == NZ - 1 ? (NZ > 1 ? NZ - 2 : 0) : z + 1;
                            R ev[FP];
#pragma unroll
                            for (int f = 0; f < FP; ++f) {
                                ev[f] = 0;
                                const R D = f < NI ? RSK(D_ion[f]) : RSK(D_pair[f - NI]);
                                if (f < NI || D != (R)0) {
                                    const R cc = vC[f][z];
                                    R lap = (fa[f * cap + n + 1] - 2 * cc + fa[f * cap + n - 1]) * RSK(idx2) +
                                            (vN[f][z] - 2 * cc + vP[f][z]) * RSK(idy2);
                                    if constexpr (NZ > 1) lap = lap + (vC[f][zr] - 2 * cc + vC[f][zl]) * RSK(idz2);
                                    ev[f] = D * lap;
                                }
                            }
                            // reactions: R1 = koff*B - kon*ion*free, free = total minus the
                            // buffer's pairs in pair order (CaSim/DyadRD2DCPU.cpp:415-456)
                            R Rj[NI];
#pragma unroll
                            for (int j = 0; j < NI; ++j) Rj[j] = 0;
#pragma unroll
                            for (int p = 0; p < NPM; ++p) {
                                R fr = RSK(ctp[p]);
                                R ion = vC[0][z];
                                if constexpr (NI == 1) {
                                    fr -= vC[1 + p][z];  // one ion: every buffer has one pair
                                } else {
#pragma unroll
                                    for (int p2 = 0; p2 < NPM; ++p2)
                                        if ((a.kf.same[p] >> p2) & 1) fr -= vC[NI + p2][z];
#pragma unroll
                                    for (int j = 1; j < NI; ++j)
                                        if (m.pair_ion[p] == j) ion = vC[j][z];
                                }
                                const R r1 = RSK(koff[p]) * vC[NI + p][z] - RSK(kon[p]) * ion * fr;
                                ev[NI + p] += -r1;
                                if constexpr (NI == 1) {
                                    Rj[0] += r1;
                                } else {
#pragma unroll
                                    for (int j = 0; j < NI; ++j)
                                        if (m.pair_ion[p] == j) Rj[j] += r1;
                                }
                            }
                            const int ci = chidx[n];
#pragma unroll
                            for (int j = 0; j < NI; ++j) {
                                R e = ev[j] + Rj[j];
                                e += ftab[ci * NI + j];
                                if ((NZ == 1 || z == NZ - 1) && m.has_sl[j]) {
                                    const R cc = vC[j][z];
                                    const R s1 = RSK(K1[j]) + cc;
                                    const R s2 = RSK(K2[j]) + cc;
                                    e *= div_fast((R)1, (R)1 + div_fast(RSK(A1[j]), s1 * s1) + div_fast(RSK(A2[j]), s2 * s2));
                                }
                                fb[j * cap + n] = vC[j][z] + e * RSK(dt);
                            }
#pragma unroll
                            for (int p = 0; p < NPM; ++p) fb[(NI + p) * cap + n] = vC[NI + p][z] + ev[NI + p] * RSK(dt);
                        }
#pragma unroll
                        for (int f = 0; f < FP; ++f)
#pragma unroll
                            for (int z = 0; z < NZ; ++z) {
                                vP[f][z] = vC[f][z];
                                vC[f][z] = vN[f][z];
                            }
                    }
                }
                if (rd3d && rank == r0) asm volatile("bar.sync 1, %0;" ::"r"(blockDim.x) : "memory");
                if (rd3d) {
                    // RD3D cytosol of this rank (no reference analog; see the oracle):
                    // a thread per (i, j) column marching along z through a chunk of
                    // planes; all CSM species slots are stepped (unused slots are zero)
                    // dealt from the last thread down: the cleft tasks went to the first warps
                    const int wt = blockDim.x - 1 - tid;
                    for (int t = wt; t < ncol * PC; t += NWT) {
                        const int pc = fdiv(t, fd_ncol), col = t - pc * ncol;
                        const int k0 = plo + pc * PL, k1 = min(k0 + PL, phi);
                        if (k0 >= k1) continue;
                        const int jq = fdiv(col, fd_ni);
                        const int jj = 1 + jq, ii = 1 + (col - jq * ni);
                        const int cn = ii + mc * jj;
                        R uP[CSM], uC[CSM], uN[CSM];
#pragma unroll
                        for (int c = 0; c < CSM; ++c) {
                            uC[c] = ca[c * ccap + cn + cps * (k0 - splo)];
                            uP[c] = k0 > 0 ? ca[c * ccap + cn + cps * (k0 - 1 - splo)] : (R)0;
                        }
                        // one plane; P0: plane 0, whose lower face mirrors and which
                        // receives the efflux deposit of the previous Update
                        auto plane = [&](int k, auto p0) {
                            constexpr bool P0 = decltype(p0)::value;
                            const int ln = cn + cps * (k - splo);
#pragma unroll
                            for (int c = 0; c < CSM; ++c) {
                                uN[c] = ca[c * ccap + ln + cps];
                                if constexpr (P0) uP[c] = uN[c];  // no-flux face: mirror
                            }
                            R evo[CSM];
#pragma unroll
                            for (int c = 0; c < CSM; ++c) {
                                const R* v = ca + c * ccap;
                                const R cc = uC[c];
                                evo[c] = RSK(cD[c]) * ((v[ln + 1] - 2 * cc + v[ln - 1]) * RSK(ih2) + (v[ln + mc] - 2 * cc + v[ln - mc]) * RSK(ih2) +
                                                       (uN[c] - 2 * cc + uP[c]) * RSK(ih2));
                            }
                            int is = 0;
#pragma unroll
                            for (int j2 = 0; j2 < NI; ++j2) {
                                const R ion = uC[j2];
                                R react = 0;
#pragma unroll
                                for (int c = NI; c < CSM; ++c) {
                                    if (NI == 1 || m.c_pair_ion[c - NI] == j2) {
                                        R fr = RSK(cctp[c]);
                                        if constexpr (NI == 1) {
                                            fr -= uC[c];
                                        } else {
#pragma unroll
                                            for (int c2 = NI; c2 < CSM; ++c2)
                                                if ((a.kf.csame[c] >> c2) & 1) fr -= uC[c2];
                                        }
                                        const R R1 = RSK(ckoff[c]) * uC[c] - RSK(ckon[c]) * ion * fr;
                                        evo[c] += -R1;
                                        react += R1;
                                    }
                                }
                                evo[j2] += react;
                                if (m.c_serca[j2]) {
                                    const R i2 = ion * ion;
                                    evo[j2] -= RSK(Jmax[is]) * (div_fast(i2, i2 + RSK(Kup2[is])) - RSK(serca0[is]));
                                    ++is;
                                }
                            }
#pragma unroll
                            for (int c = 0; c < CSM; ++c) {
                                R e = evo[c];
                                if constexpr (P0) {
                                    // deposit of the previous Update (its node sum, formed before the stencil)
                                    double dep = 0;
                                    if (it == 0) {
                                        if (c < CS) dep = a.cin[((size_t)s * CS + c) * mc2 + cn];
                                    } else if (a.kf.cdep[c] >= 0 && dptr[cn + 1] > dptr[cn]) {
                                        dep = (double)terms[(prv * a.max_terms + dptr[cn]) * FD + a.kf.cdep[c]];
                                    }
                                    e += (R)dep;
                                }
                                cb[c * ccap + ln] = uC[c] + e * RSK(dt);
                            }
#pragma unroll
                            for (int c = 0; c < CSM; ++c) {
                                uP[c] = uC[c];
                                uC[c] = uN[c];
                            }
                        };
                        int k = k0;
                        if (k == 0) plane(k++, bconst<true>{});
                        for (; k < k1; ++k) plane(k, bconst<false>{});
                    }
                }
            }
            __syncthreads();

            // ---------------------------------------------------- phase B: Update
            // rim values: the cytosol at the start of this step (pool, or the RD3D
            // layer-0 values gathered in phase A)
            auto rim_value = [&](int f, int ri) -> R {
                if (!rd3d) return f < NI ? (R)q.c_ions[f] : (R)q.c_bnd[f - NI];
                const int u = crim[ri];
                if (f < NI) return rimc[f * a.max_rim + u];
                const int cq = m.dyad_c_pair[f - NI];
                return cq >= 0 ? rimc[(NI + cq) * a.max_rim + u] : (R)m.pair_init[f - NI];
            };
            // lines of this rank's rim in tasks of 32 nodes (a warp per task, lanes along the line):
            //   l < 4*nz         Dirichlet rim (CaSim/DyadRD2DCPU.cpp:274-303), edge e = l & 3, layer l >> 2:
            //                    e 0/1 columns x = 0 / nx-1 over y in [lo, hi); e 2/3 rows y = 0 / ny-1
            //                    over x in [1, nx-2] where this rank holds them
            //   l - 4*nz < 4*zmax  efflux terms (CaSim/DyadRD2DCPU.cpp:305-350) in the same edge order:
            //                    e 0/1 over y in [ylo, yhi); e 2/3 over x in [0, nx-1]
            double epart[CSM];
#pragma unroll
            for (int f = 0; f < CSM; ++f) epart[f] = 0;
            {
                R* t0 = peer<C>(terms + (size_t)par * a.max_terms * FD, r0);
                // one-block sites: the last warps hold the channels (and their rate laws), so
                // the tasks go to the others
                const int WL = C == 1 ? max(1, W - (nch + 31) / 32) : W;
                for (int tk = warp; tk < s_nlt && warp < WL; tk += WL) {
                    const int l = ltask[tk] & 0xFFFF, i0 = ltask[tk] >> 16;
                    const bool eff = l >= 4 * nz;
                    const int le = eff ? l - 4 * nz : l;
                    const int z = le >> 2, e = le & 3;
                    if (!eff) {
                        int len, x0, y0, dxs, ri0;
                        if (e < 2) {
                            len = hi - lo;
                            x0 = e ? nx - 1 : 0;
                            y0 = lo;
                            dxs = 0;
                            ri0 = (e ? ny : 0) + lo;
                        } else {
                            len = nx - 2;
                            x0 = 1;
                            y0 = e == 2 ? 0 : ny - 1;
                            dxs = 1;
                            ri0 = 2 * ny + (e == 2 ? 0 : nx - 2);
                        }
                        for (int i = i0 + lane; i < (C == 1 ? len : min(len, i0 + 32)); i += 32) {
                            const int x = x0 + dxs * i, y = y0 + (1 - dxs) * i;
                            const int n = x + nx * ((y - slo) + nr * z);
#pragma unroll
                            for (int f = 0; f < CSM; ++f)
                                if (f < F) fb[f * cap + n] = rim_value(f, ri0 + i);
                        }
                    } else {
                        int len, x0, y0, dxs, dys, gt0;
                        double sf;
                        if (e < 2) {
                            len = nrows;
                            x0 = e ? nx - 1 : 0;
                            y0 = ylo;
                            dxs = e ? -1 : 1;
                            dys = 0;
                            sf = m.sx;
                            gt0 = (e * (ny - 2) + (ylo - 1)) * zmax + z;
                        } else {
                            len = nx;
                            x0 = 0;
                            y0 = e == 2 ? 0 : ny - 1;
                            dxs = 0;
                            dys = e == 2 ? 1 : -1;
                            sf = m.sy;
                            gt0 = (2 * (ny - 2) + (e - 2) * nx) * zmax + z;
                        }
                        for (int i = i0 + lane; i < (C == 1 ? len : min(len, i0 + 32)); i += 32) {
                            // the edge node walks along the line: y for x-edges, x for y-edges
                            const int xe = e < 2 ? x0 : i, ye = e < 2 ? y0 + i : y0;
                            const int ri = e < 2 ? (e ? ny : 0) + ye
                                                 : (xe == 0 ? ye == 0 ? 0 : ny - 1
                                                            : xe == nx - 1 ? ny + ye : 2 * ny + (e == 2 ? 0 : nx - 2) + xe - 1);
                            const int n1 = (xe + dxs) + nx * ((ye + dys - slo) + nr * z);
                            const int n2 = (xe + 2 * dxs) + nx * ((ye + 2 * dys - slo) + nr * z);
                            // a y-edge line's end nodes step along the x = 0 / nx-1 rim column,
                            // whose Dirichlet values another task of this phase writes: use them directly
                            const int rc = (e >= 2 && (xe == 0 || xe == nx - 1)) ? (xe == 0 ? 0 : ny) : -1;
                            const int gterm = gt0 + i * zmax;
#pragma unroll
                            for (int f = 0; f < CSM; ++f) {
                                if (f < F) {
                                    const double u0 = (double)rim_value(f, ri);
                                    const double D = f < NI ? m.D_ion[f] : m.D_pair[f - NI];
                                    const double u1 = rc >= 0 ? (double)rim_value(f, rc + ye + dys) : (double)fb[f * cap + n1];
                                    const double u2 = rc >= 0 ? (double)rim_value(f, rc + ye + 2 * dys) : (double)fb[f * cap + n2];
                                    const double gr = 2 * u1 - 1.5 * u0 - 0.5 * u2;
                                    if (!rd3d) {
                                        epart[f] += D * m.grad_mult * sf * gr;
                                    } else {
                                        const double v = D * sf * gr * m.inv_hc3;
                                        epart[f] += v;
                                        const int sl = dslot(m, NI, f);
                                        if (sl >= 0) t0[tpos[gterm] * FD + sl] = (R)v;
                                    }
                                }
                            }
                        }
                    }
                }
            }
            // mouth gather and RyR currents of own channels (CaSim/DyadRD2DCPU.cpp:243-264, 361-380),
            // channels from the last thread down so they meet the warps with fewer rim lines; the
            // transition probability of the next gating (CaSim/DyadChannels.cpp:97-130: rate of the
            // current state at the mouth values x dt) is computed here, off the gating warp
            double tpart[NI];
#pragma unroll
            for (int j = 0; j < NI; ++j) tpart[j] = 0;
            const int ct = blockDim.x - 1 - tid;
            double* pcur = pg + par * a.max_ch;
            for (int c = ct; c < nch; c += blockDim.x) {
                const int n = chn[c];
                if (n < 0) continue;
                const int ri = chr[c];
                const R* src = ri >= 0 ? fa : fb;  // the mouth is gathered before the rim is reset
                const int stc = chs[c];
                {
                    const double cam = (double)src[m.ca_idx * cap + n];
                    const double mgm = m.mg_idx >= 0 ? (double)src[m.mg_idx * cap + n] : 0.0;
                    const double p = cb_rate(m, a.spx0, a.spc0, a.spx1, a.spc1, stc, cam, mgm) * dt;
#pragma unroll 1
                    for (int r = 0; r < C; ++r) peer<C>(pcur, r)[c] = p;
                }
#pragma unroll
                for (int j = 0; j < NI; ++j) {
                    const double mv = (double)src[j * cap + n];
                    const double cv = ri >= 0 ? (double)rim_value(j, ri) : mv;
                    const double fl = stc * (m.g[j] * (q.jsr_new[j] - cv));
                    ftab[(1 + c) * NI + j] = (R)fl;
                    tpart[j] += fl;
                }
                if (last) {
                    double* mo = a.mouth + (size_t)(st.ch_off + c) * a.NS;
                    double fr[CB_MAX_BUF];
                    for (int b = 0; b < m.n_buf; ++b) fr[b] = m.Ctot[b];
                    for (int f = 0; f < F; ++f) {
                        const double v = (double)src[f * cap + n];
                        mo[f] = v;
                        if (f >= NI) fr[m.pair_buf[f - NI]] -= v;
                    }
                    for (int b = 0; b < m.n_buf; ++b) mo[F + b] = fr[b];
                }
            }
            // warp partials (warps without terms or channels contribute exact zeros): the
            // butterflies of all values run round by round, so their shuffles overlap
            {
                double wv[CSM + NI];
#pragma unroll
                for (int f = 0; f < CSM; ++f) wv[f] = epart[f];
#pragma unroll
                for (int j = 0; j < NI; ++j) wv[CSM + j] = tpart[j];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                    for (int k = 0; k < CSM + NI; ++k) wv[k] += __shfl_xor_sync(0xffffffffu, wv[k], o);
                if (lane == 0) {
#pragma unroll
                    for (int f = 0; f < CSM; ++f)
                        if (f < F) redw[warp * FDn + f] = wv[f];
#pragma unroll
                    for (int j = 0; j < NI; ++j) redw[warp * FDn + F + j] = wv[CSM + j];
                }
            }
            __syncthreads();
            // rank partials (fixed warp order) into every rank's slot
            if (warp == 0) {
                double v = 0;
                if (lane < FDn) {
                    // four interleaved sums over the warps (a fixed order: every run and every
                    // rank forms the same total)
                    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
                    for (int w = 0; w < W; w += 4) {
                        s0 += redw[w * FDn + lane];
                        if (w + 1 < W) s1 += redw[(w + 1) * FDn + lane];
                        if (w + 2 < W) s2 += redw[(w + 2) * FDn + lane];
                        if (w + 3 < W) s3 += redw[(w + 3) * FDn + lane];
                    }
                    v = (s0 + s1) + (s2 + s3);
                }
                // FDn (at most 20) values x C ranks: one store per lane
                for (int b0 = 0; b0 < FDn * C; b0 += 32) {
                    const int idx = b0 + lane;
                    const int k = idx / C, r = idx - k * C;
                    const double vk = __shfl_sync(0xffffffffu, v, k < FDn ? k : 0);
                    if (idx < FDn * C) {
                        if (k < F) peer<C>(rede, r)[(par * C + rank) * F + k] = vk;
                        else peer<C>(redt, r)[(par * C + rank) * NI + (k - F)] = vk;
                    }
                }
            }
            if constexpr (C > 1) {
                // halo rows into the neighbours' write buffers, a warp per (species, layer) row
                for (int side = 0; side < 2; ++side) {
                    const int nb = side == 0 ? rank - 1 : rank + 1;
                    if (nb < 0 || nb >= C) continue;
                    const int y = side == 0 ? lo : hi - 1;
                    const int nlo = s_nrow[2 * side], nhi = s_nrow[2 * side + 1];
                    const int nslo = nlo > 0 ? nlo - 1 : 0;
                    const int nnr = (nhi < ny ? nhi + 1 : ny) - nslo;
                    R* dst = peer<C>(fb, nb);
                    for (int l = warp; l < F * NZ; l += W) {
                        const int f = l / NZ, z = l - f * NZ;
                        const R* src = fb + f * cap + nx * ((y - slo) + nr * z);
                        R* d = dst + f * cap + nx * ((y - nslo) + nnr * z);
                        for (int x = lane; x < nx; x += 32) d[x] = src[x];
                    }
                }
                if (rd3d && phi > plo) {
                    // cytosol halo planes
                    for (int side = 0; side < 2; ++side) {
                        const int nbb = side == 0 ? pb - 1 : pb + 1;  // neighbour plane block
                        if (nbb < 0 || nbb >= C) continue;
                        const int nb = (nbb + C - C / 2) % C;
                        const int k = side == 0 ? plo : phi - 1;
                        const int nplo = (int)(((long long)nbb * nplanes) / C);
                        const int nsplo = nplo > 0 ? nplo - 1 : 0;
                        R* dst = peer<C>(cb, nb);
                        // whole 16-byte words of the padded plane (the padding goes along)
                        const int nv = cps * (int)sizeof(R) / 16;
                        for (int t = tid; t < CS * nv; t += blockDim.x) {
                            const int c = t / nv, e = t - c * nv;
                            ((uint4*)(dst + c * ccap + (k - nsplo) * cps))[e] = ((const uint4*)(cb + c * ccap + (k - splo) * cps))[e];
                        }
                    }
                }
            }
            cluster_barrier<C>();
            {
                R* t = fa;
                fa = fb;
                fb = t;
            }
            {
                R* t = ca;
                ca = cb;
                cb = t;
            }
        }

        // ---------------------------------------------------------- store
        if (warp == 0 && a.nsteps > 0) {
            const int pl = (int)((a.nsteps - 1) & 1);
            for (int f = lane; f < F; f += 32) {
                double e = 0;
                for (int r = 0; r < C; ++r) e += rede[(pl * C + r) * F + f];
                q.efflux[f] = e;
            }
            for (int j = lane; j < NI; j += 32) {
                double t = 0;
                for (int r = 0; r < C; ++r) t += redt[(pl * C + r) * NI + j];
                q.total[j] = t;
            }
            __syncwarp();
            if (lane == 0) {
                if (!m.jsr_const)
                    for (int i = 0; i < NI; ++i) {
                        q.IjSR[i] = q.total[i] * m.V_elem;
                        q.nsr[i] = m.nsr[i];
                        q.jsr[i] = q.jsr_new[i];
                    }
                cbrng::State gd;  // stream state at the next unconsumed draw
                for (int i = 0; i < 6; ++i) gd.s[i] = q.rng[i];
                const long long D = s_D;
                rng_jump(a.pow2, gd, 2ULL * (unsigned long long)D);
                for (int i = 0; i < 6; ++i) q.rng[i] = gd.s[i];
                q.draws += (unsigned long long)D;
            }
        }
        __syncthreads();
        {
            R* g = (R*)a.fields + st.node_base * F;
            for (int f = 0; f < F; ++f)
                for (int z = 0; z < nz; ++z) {
                    R* dst = g + (long long)f * np + (long long)nx * (lo + (long long)ny * z);
                    const R* src = fa + f * cap + lstride * z + nx * (lo - slo);
                    for (int k = tid; k < nx * (hi - lo); k += blockDim.x) dst[k] = src[k];
                }
            if (rank == 0) {
                const unsigned int* qs = (const unsigned int*)&q;
                unsigned int* qd = (unsigned int*)(a.sc + s);
                for (int k = tid; k < (int)(sizeof(cb_site_scalars) / 4); k += blockDim.x) qd[k] = qs[k];
                for (int c = tid; c < nch; c += blockDim.x) a.ch_state[st.ch_off + c] = chs[c];
            }
            R* cg_ = (R*)a.curgrid + st.node_base * NI;
            for (int c = tid; c < nch; c += blockDim.x)
                if (chn[c] >= 0 && ((cho[c] >> 30) & 1))
                    for (int j = 0; j < NI; ++j) cg_[(size_t)j * np + (cho[c] & ((1 << 30) - 1))] = ftab[(1 + c) * NI + j];
            if (rd3d) {
                R* cd = (R*)a.cyto + (size_t)s * CS * nc;
                for (int c = 0; c < CS; ++c)
                    for (int k = tid; k < (phi - plo) * mc2; k += blockDim.x) {
                        const int pl = k / mc2;
                        cd[(size_t)c * nc + (size_t)plo * mc2 + k] = ca[c * ccap + (plo - splo + pl) * cps + (k - pl * mc2)];
                    }
                if (rank == r0 && a.nsteps > 0) {
                    // deposit of the final Update, for the next launch
                    const int pl = (int)((a.nsteps - 1) & 1);
                    for (int cn = tid; cn < mc2; cn += blockDim.x)
                        for (int c = 0; c < CS; ++c) {
                            const int sl = a.kf.cdep[c];
                            double dep = 0;
                            if (sl >= 0)
                                for (int q2 = dptr[cn]; q2 < dptr[cn + 1]; ++q2)
                                    dep += (double)terms[(pl * a.max_terms + q2) * FD + sl];
                            a.cin[((size_t)s * CS + c) * mc2 + cn] = dep;
                        }
                }
            }
        }
        cluster_barrier<C>();
    }
}

// dry: only report how many clusters of this shape can be resident;
// known > 0: that count, from an earlier dry call
template <typename R, int NI, int NPM, int NZ, int C>
cudaError_t launch_one(const rs_args& a, int threads, cudaStream_t st, int n_sites, int* dry, int known) {
    auto kern = k_resident<R, NI, NPM, NZ, C>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, a.smem_bytes);
    if (e != cudaSuccess) return e;
    if (C > 8) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = a.smem_bytes;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(C);
    int clusters = known;
    if (clusters <= 0) {
        e = cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg);
        if (e != cudaSuccess) return e;
    }
    if (dry) {
        *dry = clusters;
        return cudaSuccess;
    }
    if (clusters < 1) return cudaErrorInvalidConfiguration;
    clusters = clusters < n_sites ? clusters : n_sites;
    cfg.gridDim = dim3(clusters * C);
    return cudaLaunchKernelEx(&cfg, kern, a);
}

template <typename R, int NI, int NPM, int NZ>
cudaError_t launch_c(const rs_args& a, int C, int threads, cudaStream_t st, int n, int* dry, int known) {
    switch (C) {
    case 1: return launch_one<R, NI, NPM, NZ, 1>(a, threads, st, n, dry, known);
    case 2: return launch_one<R, NI, NPM, NZ, 2>(a, threads, st, n, dry, known);
    case 4: return launch_one<R, NI, NPM, NZ, 4>(a, threads, st, n, dry, known);
    case 8: return launch_one<R, NI, NPM, NZ, 8>(a, threads, st, n, dry, known);
    case 16: return launch_one<R, NI, NPM, NZ, 16>(a, threads, st, n, dry, known);
    default: return cudaErrorInvalidConfiguration;
    }
}

// NP: the larger of the cleft's ion-buffer pairs and (RD3D) the cytosol's
template <typename R, int NZ>
cudaError_t dispatch(const rs_args& a, int NI, int NP, int C, int threads, cudaStream_t st, int n, int* dry, int known) {
    if (threads > max_threads(sizeof(R), NI + npm_of(NI, NP), NZ, C)) return cudaErrorInvalidConfiguration;
    if (NI == 1 && NP <= 2) return launch_c<R, 1, 2, NZ>(a, C, threads, st, n, dry, known);
    if (NI == 1 && NP <= 4) return launch_c<R, 1, 4, NZ>(a, C, threads, st, n, dry, known);
    if (NI == 2 && NP <= 2) return launch_c<R, 2, 2, NZ>(a, C, threads, st, n, dry, known);
    if (NI == 2 && NP <= 4) return launch_c<R, 2, 4, NZ>(a, C, threads, st, n, dry, known);
    return cudaErrorInvalidConfiguration;
}

}  // namespace cbres

// per (precision, layers) launchers, each compiled in its own translation unit
cudaError_t cb_res_f32_z1(const cbres::rs_args&, int, int, int, int, cudaStream_t, int, int*, int);
cudaError_t cb_res_f32_z3(const cbres::rs_args&, int, int, int, int, cudaStream_t, int, int*, int);
cudaError_t cb_res_f64_z1(const cbres::rs_args&, int, int, int, int, cudaStream_t, int, int*, int);
cudaError_t cb_res_f64_z3(const cbres::rs_args&, int, int, int, int, cudaStream_t, int, int*, int);
