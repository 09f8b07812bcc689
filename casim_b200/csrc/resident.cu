// Resident path, host side: shared-memory plans, size classes of thread-block
// clusters, the MRG32k3a jump table and the per-class launches. The kernel and
// its launch helpers are in resident_kernel.cuh; the specialisations are
// compiled in resident_f32_z1.cu, resident_f32_z3.cu, resident_f64_z1.cu and
// resident_f64_z3.cu.
#include <algorithm>
#include <string>
#include <vector>

#include "resident_kernel.cuh"

using namespace cbres;

namespace {

size_t align16(size_t v) { return (v + 15) / 16 * 16; }

// pair slots the kernel must hold: the cleft's ion-buffer pairs and (RD3D) the cytosol's
int pairs_of(const cb_model& m) { return std::max(m.n_pairs, m.cyto_type == CB_CYTO_RD3D ? m.c_n_pairs : 0); }

template <typename R>
void fill_const(const cb_model& m, rs_const<R>& k) {
    k = rs_const<R>{};
    const int NI = m.n_ions;
    for (int j = 0; j < NI; ++j) {
        k.D_ion[j] = (R)m.D_ion[j];
        k.K1[j] = (R)m.K1[j];
        k.K2[j] = (R)m.K2[j];
        k.A1[j] = (R)(m.N1[j] * m.K1[j]);
        k.A2[j] = (R)(m.N2[j] * m.K2[j]);
        k.Kup2[j] = (R)(m.c_Kup[j] * m.c_Kup[j]);
        {
            const double b2 = m.c_bg[j] * m.c_bg[j], K2 = m.c_Kup[j] * m.c_Kup[j];
            k.serca0[j] = (R)(b2 / (b2 + K2));
        }
        k.Jmax[j] = (R)m.c_Jmax[j];
    }
    for (int p = 0; p < m.n_pairs; ++p) {
        k.D_pair[p] = (R)m.D_pair[p];
        k.kon[p] = (R)m.kon[p];
        k.koff[p] = (R)m.koff[p];
        k.ctp[p] = (R)m.Ctot[m.pair_buf[p]];
        for (int p2 = 0; p2 < m.n_pairs; ++p2)
            if (m.pair_buf[p2] == m.pair_buf[p]) k.same[p] |= 1 << p2;
    }
    k.idx2 = (R)m.inv_dx2;
    k.idy2 = (R)m.inv_dy2;
    k.idz2 = (R)m.inv_dz2;
    k.dt = (R)m.dt;
    k.ih2 = (R)m.inv_hc2;
    // deposit slot of dyad species f: its index among species with a cytosol counterpart
    auto slot = [&](int f) {
        int n = 0;
        for (int g = 0; g < f; ++g)
            if (g < NI || m.dyad_c_pair[g - NI] >= 0) ++n;
        return (f < NI || m.dyad_c_pair[f - NI] >= 0) ? n : -1;
    };
    for (int c = 0; c < CB_MAX_CSPECIES; ++c) k.cdep[c] = -1;
    for (int c = 0; c < NI + m.c_n_pairs && c < CB_MAX_CSPECIES; ++c) {
        if (c < NI) {
            k.cD[c] = (R)m.D_ion[c];
            k.cdep[c] = slot(c);
            continue;
        }
        const int p = c - NI;
        k.cD[c] = (R)m.c_D_pair[p];
        k.ckon[c] = (R)m.c_kon[p];
        k.ckoff[c] = (R)m.c_koff[p];
        k.cctp[c] = (R)m.c_Ctot[m.c_pair_buf[p]];
        for (int p2 = 0; p2 < m.c_n_pairs; ++p2)
            if (m.c_pair_buf[p2] == m.c_pair_buf[p]) k.csame[c] |= 1 << (NI + p2);
        if (m.c_dyad_pair[p] >= 0) k.cdep[c] = slot(NI + m.c_dyad_pair[p]);
    }
}

// shared-memory carve for the sites `idx` with cluster size C
// row weights of the C ranks: even, or (light) 2 shares for the first and last row blocks
// (long y-edge rim lines) and the plane-0 rank (efflux deposits) and 3 for the others
void row_weights(rs_args& a, int C, bool light) {
    const int r0 = (C - C / 2) % C;
    a.rw[0] = 0;
    for (int r = 0; r < 16; ++r)
        a.rw[r + 1] = (unsigned short)(a.rw[r] + (light && C >= 4 && r < C ? (r == 0 || r == C - 1 || r == r0 ? 2 : 3) : 1));
}

bool plan(const cb_dev& d, const std::vector<cb_site>& sites, const std::vector<int>& idx, int C, rs_args& a) {
    const cb_model& m = d.m;
    const size_t rs = d.precision == 0 ? 8 : 4;
    const bool rd3d = m.cyto_type == CB_CYTO_RD3D;
    // channel and efflux-term capacities are the batch maxima, so the plan of a
    // class fits whenever the plan of its largest site does
    int cap = 0, ccap = 0, maxrim = 1, maxlt = 1;
    const int maxch = std::max(d.max_ch, 1), maxt = std::max(d.max_terms, 1);
    for (const cb_site& st : sites) maxrim = std::max(maxrim, cb_rim_count(st.nx, st.ny));
    for (int s : idx) {
        const cb_site& st = sites[s];
        if (st.ny < 3 * C) return false;  // every rank needs three rows (y-edge efflux)
        const int zmax = st.nz == 1 ? 1 : st.nz - 1;
        maxlt = std::max(maxlt, 4 * (st.nz + zmax) * ((std::max(st.nx, st.ny) + 31) / 32));
        for (int r = 0; r < C; ++r) {
            const int lo = row_lo(a.rw, r, st.ny, C), hi = row_lo(a.rw, r + 1, st.ny, C);
            if (hi - lo < 3) return false;
            int slo = lo > 0 ? lo - 1 : 0, shi = hi < st.ny ? hi + 1 : st.ny;
            cap = std::max(cap, (shi - slo) * st.nx * st.nz);
        }
    }
    cap = (cap + 3) / 4 * 4;
    const int CS = m.n_ions + m.c_n_pairs;
    const int mc = m.mc, mc2 = mc * mc;
    // cytosol planes start on 16-byte boundaries in shared memory (vector halo copies)
    const int vr = (int)(16 / rs), cps = (mc2 + vr - 1) / vr * vr;
    if (rd3d) {
        if (mc - 1 < C) return false;
        for (int r = 0; r < C; ++r) {
            int plo = (int)((long long)r * (mc - 1) / C), phi = (int)((long long)(r + 1) * (mc - 1) / C);
            int splo = plo > 0 ? plo - 1 : 0;
            ccap = std::max(ccap, (phi + 1 - splo) * cps);
        }
        ccap = (ccap + 3) / 4 * 4;
    }
    a.cps = cps;
    int FD = 0;
    for (int f = 0; f < m.F; ++f)
        if (f < m.n_ions || m.dyad_c_pair[f - m.n_ions] >= 0) ++FD;
    const int F = m.F, NI = m.n_ions;
    // species slots of the kernel specialisation (the stencils step all of them)
    const int FP = NI + npm_of(NI, pairs_of(m)), CSP = rd3d ? FP : 0;
    size_t off = align16((size_t)FP * cap * rs);
    a.off_fb = (int)off;
    off = align16(off + (size_t)FP * cap * rs);
    a.off_ca = (int)off;
    off = align16(off + (size_t)CSP * ccap * rs);
    a.off_cb = (int)off;
    off = align16(off + (size_t)CSP * ccap * rs);
    a.off_chidx = (int)off;
    off = align16(off + (size_t)cap * 2);
    a.off_chn = (int)off;
    off = align16(off + (size_t)maxch * 4);
    a.off_chs = (int)off;
    off = align16(off + (size_t)maxch * 4);
    a.off_cho = (int)off;
    off = align16(off + (size_t)maxch * 4);
    a.off_chr = (int)off;
    off = align16(off + (size_t)maxch * 4);
    a.off_ftab = (int)off;
    off = align16(off + (size_t)(maxch + 1) * NI * rs);
    a.off_pg = (int)off;
    off = align16(off + (size_t)2 * maxch * 8);
    a.off_ring = (int)off;
    off = align16(off + (size_t)RING * 8);
    a.off_redw = (int)off;
    off = align16(off + (size_t)MAX_WARPS * (F + NI) * 8);
    a.off_rede = (int)off;
    off = align16(off + (size_t)2 * C * F * 8);
    a.off_redt = (int)off;
    off = align16(off + (size_t)2 * C * NI * 8);
    a.off_terms = (int)off;
    if (rd3d) off = align16(off + (size_t)2 * maxt * FD * rs);
    a.off_crim = (int)off;
    if (rd3d) off = align16(off + (size_t)maxrim * 2);
    a.off_ulist = (int)off;
    if (rd3d) off = align16(off + (size_t)maxrim * 2);
    a.off_rimc = (int)off;
    if (rd3d) off = align16(off + (size_t)CSP * maxrim * rs);
    a.off_slot = (int)off;
    if (rd3d) off = align16(off + (size_t)mc2 * 2);
    a.off_dptr = (int)off;
    if (rd3d) off = align16(off + (size_t)(mc2 + 1) * 2);
    a.off_dterm = (int)off;
    if (rd3d) off = align16(off + (size_t)maxt * 2);
    a.off_ltask = (int)off;
    off = align16(off + (size_t)maxlt * 4);
    a.off_sc = (int)off;
    off = align16(off + sizeof(cb_site_scalars));
    a.smem_bytes = (int)off;
    a.cap_cleft = cap;
    a.cap_cyto = ccap;
    a.max_ch = maxch;
    a.max_terms = maxt;
    a.max_rim = maxrim;
    a.FD = FD;
    if (rd3d && (maxt > 65535 || mc2 + 1 > 65535)) return false;  // u16 deposit tables
    return off <= (size_t)(227 * 1024 - 1024);
}

// warps 0 and 1 run gating and the pools; the rest run the stencils
int pick_threads(const cb_dev& d, const std::vector<cb_site>& sites, const std::vector<int>& idx, int C, int cap) {
    long long mx = 0;
    for (int s : idx) mx = std::max(mx, (long long)sites[s].nx * sites[s].ny * sites[s].nz / C);
    // RD3D: the rank's share of the cytosol, a column task per (column, plane chunk)
    if (d.m.cyto_type == CB_CYTO_RD3D) mx += 2LL * (d.m.mc - 2) * (d.m.mc - 2) * (d.m.mc - 1) / C;
    long long t = ((mx / 8 + 31) / 32 + 2) * 32;
    return (int)std::max(128LL, std::min((long long)cap, t));
}

// cleft layers of the specialisation serving the model (0: none)
int layers_of(const cb_model& m, const std::vector<cb_site>& sites) {
    const int nz = m.dim == 2 ? 1 : 3;
    for (const cb_site& s : sites)
        if (s.nz != nz) return 0;
    return nz;
}


int thread_cap(const cb_dev& d, int nz, int C) {
    return max_threads(d.precision == 0 ? 8 : 4, d.m.n_ions + npm_of(d.m.n_ions, pairs_of(d.m)), nz, C);
}

cudaError_t launch_t(const cb_dev& d, const rs_args& a, int nz, int C, int threads, cudaStream_t st, int n, int* dry = nullptr,
                     int known = 0) {
    const int NI = d.m.n_ions, NP = pairs_of(d.m);
    if (d.precision == 0)
        return nz == 1 ? cb_res_f64_z1(a, NI, NP, C, threads, st, n, dry, known) : cb_res_f64_z3(a, NI, NP, C, threads, st, n, dry, known);
    return nz == 1 ? cb_res_f32_z1(a, NI, NP, C, threads, st, n, dry, known) : cb_res_f32_z3(a, NI, NP, C, threads, st, n, dry, known);
}

bool species_supported(const cb_model& m) {
    const int np = pairs_of(m);
    return (m.n_ions == 1 && np <= 4) || (m.n_ions == 2 && np <= 4);
}

// Size classes: each site goes to the smallest cluster size that holds it;
// one launch per class, largest sites first within a class.
bool classify(const cb_dev& d, const std::vector<cb_site>& sites, std::vector<std::vector<int>>& classes, std::vector<int>& cs) {
    static const int sizes[5] = {1, 2, 4, 8, 16};
    std::vector<std::vector<int>> by(5);
    for (int s = 0; s < d.S; ++s) {
        int k = 0;
        while (k < 5 && sizes[k] < d.min_cluster) ++k;
        for (; k < 5; ++k) {
            rs_args a{};
            for (int r = 0; r <= 16; ++r) a.rw[r] = (unsigned short)r;
            std::vector<int> one{s};
            if (plan(d, sites, one, sizes[k], a)) break;
        }
        if (k == 5) return false;
        by[k].push_back(s);
    }
    classes.clear();
    cs.clear();
    for (int k = 0; k < 5; ++k)
        if (!by[k].empty()) {
            std::stable_sort(by[k].begin(), by[k].end(), [&](int x, int y) {
                return (long long)sites[x].nx * sites[x].ny * sites[x].nz > (long long)sites[y].nx * sites[y].ny * sites[y].nz;
            });
            classes.push_back(by[k]);
            cs.push_back(sizes[k]);
        }
    return true;
}

}  // namespace

bool cb_resident_fits(const cb_dev& d, int* threads, size_t* smem, std::string* why) {
    auto no = [&](const std::string& w) {
        if (why) *why = w;
        return false;
    };
    if (!species_supported(d.m)) return no("species layout not specialised (1-2 ions, at most 4 ion-buffer pairs)");
    if (d.m.ch_model == CB_SINGLE_SITE_MWC) return no("60-state RyR gating runs on the plain path");
    if (2 * d.max_ch > WINDOW) return no("more than 256 RyRs in a site");
    std::vector<cb_site> sites(d.S);
    if (cudaMemcpy(sites.data(), d.sites, sizeof(cb_site) * d.S, cudaMemcpyDeviceToHost) != cudaSuccess) return no("cudaMemcpy");
    const int nz = layers_of(d.m, sites);
    if (nz == 0) return no("the resident path is specialised for 3D clefts of 3 layers");
    std::vector<std::vector<int>> classes;
    std::vector<int> cs;
    if (!classify(d, sites, classes, cs)) return no("a site does not fit the shared memory of a 16-block cluster");
    // every class must be schedulable (a 16-block cluster needs 16 SMs of one GPC)
    for (size_t k = 0; k < classes.size(); ++k) {
        rs_args a{};
        for (int r = 0; r <= 16; ++r) a.rw[r] = (unsigned short)r;
        if (!plan(d, sites, classes[k], cs[k], a)) return no("the shared-memory plan of a cluster class does not fit");
        a.m = d.m;
        fill_const(d.m, a.kf);
        fill_const(d.m, a.kd);
        int clusters = 0;
        const int thr = pick_threads(d, sites, classes[k], cs[k], thread_cap(d, nz, cs[k]));
        cudaError_t e = launch_t(d, a, nz, cs[k], thr, 0, 0, &clusters);
        if (e != cudaSuccess || clusters < 1) {
            cudaGetLastError();
            return no("clusters of " + std::to_string(cs[k]) + " blocks with " + std::to_string(a.smem_bytes) +
                      " B of shared memory each cannot be resident (" + std::string(cudaGetErrorString(e)) + ", " +
                      std::to_string(clusters) + " clusters)");
        }
        if (k == 0) {
            if (threads) *threads = thr;
            if (smem) *smem = (size_t)a.smem_bytes;
        }
        if (why) {
            *why += (k ? ", " : "resident: ") + std::to_string(classes[k].size()) + " sites on clusters of " +
                    std::to_string(cs[k]) + " (" + std::to_string(a.smem_bytes / 1024) + " KiB, " + std::to_string(thr) +
                    " threads, " + std::to_string(clusters) + " resident)";
        }
    }
    return true;
}

// MRG32k3a jump table of the batch (resident gating and surrogate gating)
cudaError_t cb_ensure_pow2(cb_dev& d) {
    if (d.rs_pow2) return cudaSuccess;
    cudaError_t e;
    // MRG32k3a: A^(2^k) for k < 64 (both components), then the refill jump A^(2*31*LANE_DRAWS)
    std::vector<unsigned long long> p2(65 * 18);
    cbrng::Mat3 a1 = cbrng::step_matrix1(), a2 = cbrng::step_matrix2();
    for (int k = 0; k < 64; ++k) {
        for (int i = 0; i < 9; ++i) {
            p2[18 * k + i] = a1.a[i / 3][i % 3];
            p2[18 * k + 9 + i] = a2.a[i / 3][i % 3];
        }
        a1 = cbrng::matmul(a1, a1, cbrng::M1);
        a2 = cbrng::matmul(a2, a2, cbrng::M2);
    }
    cbrng::Mat3 j1{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}}, j2 = j1;
    unsigned long long steps = 2ULL * 31 * LANE_DRAWS;
    for (int k = 0; steps; ++k, steps >>= 1)
        if (steps & 1ULL) {
            cbrng::Mat3 b1, b2;
            for (int i = 0; i < 9; ++i) {
                b1.a[i / 3][i % 3] = p2[18 * k + i];
                b2.a[i / 3][i % 3] = p2[18 * k + 9 + i];
            }
            j1 = cbrng::matmul(b1, j1, cbrng::M1);
            j2 = cbrng::matmul(b2, j2, cbrng::M2);
        }
    for (int i = 0; i < 9; ++i) {
        p2[18 * JUMP_ROW + i] = j1.a[i / 3][i % 3];
        p2[18 * JUMP_ROW + 9 + i] = j2.a[i / 3][i % 3];
    }
    if ((e = cudaMalloc(&d.rs_pow2, sizeof(unsigned long long) * p2.size())) != cudaSuccess) return e;
    if ((e = cudaMemcpy(d.rs_pow2, p2.data(), sizeof(unsigned long long) * p2.size(), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    return cudaSuccess;
}

// launch plan of a batch, built on the first step and reused: one entry per
// cluster-size class with its static arguments, block size and resident clusters
struct cb_rs_plan {
    int nz = 0;
    std::vector<rs_args> args;
    std::vector<int> cs, threads, clusters;
    // several classes run side by side, one stream each (forked from and joined to the
    // caller's stream), so the clusters of one fill the SMs the others leave free
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> done;
    cudaEvent_t fork = nullptr;
};

void cb_resident_free(cb_dev& d) {
    if (d.rs_plan) {
        for (cudaStream_t s : d.rs_plan->streams) cudaStreamDestroy(s);
        for (cudaEvent_t e : d.rs_plan->done) cudaEventDestroy(e);
        if (d.rs_plan->fork) cudaEventDestroy(d.rs_plan->fork);
    }
    delete d.rs_plan;
    d.rs_plan = nullptr;
}

namespace {

cudaError_t build_plan(cb_dev& d) {
    std::vector<cb_site> sites(d.S);
    cudaError_t e = cudaMemcpy(sites.data(), d.sites, sizeof(cb_site) * d.S, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
    std::vector<std::vector<int>> classes;
    std::vector<int> cs;
    if (!classify(d, sites, classes, cs)) return cudaErrorInvalidConfiguration;
    if (classes.size() > 8) return cudaErrorInvalidConfiguration;
    const int nz = layers_of(d.m, sites);
    if (nz == 0) return cudaErrorInvalidConfiguration;
    std::vector<int> order;
    for (auto& c : classes) order.insert(order.end(), c.begin(), c.end());
    // a failed build leaves no device buffers behind, so that the next call starts clean
    auto undo = [&](cudaError_t err) {
        cudaFree(d.rs_order);
        cudaFree(d.rs_counter);
        d.rs_order = nullptr;
        d.rs_counter = nullptr;
        return err;
    };
    if ((e = cudaMalloc(&d.rs_order, sizeof(int) * d.S)) != cudaSuccess) return undo(e);
    if ((e = cudaMemcpy(d.rs_order, order.data(), sizeof(int) * d.S, cudaMemcpyHostToDevice)) != cudaSuccess) return undo(e);
    if ((e = cudaMalloc(&d.rs_counter, sizeof(int) * 8)) != cudaSuccess) return undo(e);
    if ((e = cb_ensure_pow2(d)) != cudaSuccess) return undo(e);
    cb_rs_plan* P = new cb_rs_plan();
    P->nz = nz;
    int offset = 0;
    for (size_t k = 0; k < classes.size(); ++k) {
        rs_args a{};
        row_weights(a, cs[k], d.light_rows != 0);
        if (d.light_rows && !plan(d, sites, classes[k], cs[k], a)) row_weights(a, cs[k], false);
        if (!plan(d, sites, classes[k], cs[k], a)) {
            delete P;
            return undo(cudaErrorInvalidConfiguration);
        }
        a.m = d.m;
        fill_const(d.m, a.kf);
        fill_const(d.m, a.kd);
        a.sites = d.sites;
        a.order = d.rs_order + offset;
        a.S = (int)classes[k].size();
        a.counter = d.rs_counter + k;
        a.curgrid = d.curgrid;
        a.ch_node = d.ch_node;
        a.ch_owner = d.ch_owner;
        a.ch_state = d.ch_state;
        a.mouth = d.mouth;
        a.NS = d.NS;
        a.sc = d.sc;
        a.cin = d.cin;
        a.rim_cnode = d.rim_cnode;
        a.dep_ptr = d.dep_ptr;
        a.dep_term = d.dep_term;
        a.nc = d.nc;
        a.pow2 = d.rs_pow2;
        a.spx0 = d.spx[0];
        a.spc0 = d.spc[0];
        a.spx1 = d.spx[1];
        a.spc1 = d.spc[1];
        const int threads = pick_threads(d, sites, classes[k], cs[k], thread_cap(d, nz, cs[k]));
        int clusters = 0;
        e = launch_t(d, a, nz, cs[k], threads, 0, a.S, &clusters);
        if (e != cudaSuccess || clusters < 1) {
            delete P;
            return undo(e != cudaSuccess ? e : cudaErrorInvalidConfiguration);
        }
        P->args.push_back(a);
        P->cs.push_back(cs[k]);
        P->threads.push_back(threads);
        P->clusters.push_back(clusters);
        offset += a.S;
    }
    if (P->args.size() > 1) {
        if ((e = cudaEventCreateWithFlags(&P->fork, cudaEventDisableTiming)) != cudaSuccess) {
            delete P;
            return undo(e);
        }
        for (size_t k = 0; k < P->args.size(); ++k) {
            cudaStream_t s = nullptr;
            cudaEvent_t ev = nullptr;
            if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) == cudaSuccess) P->streams.push_back(s);
            if (e == cudaSuccess && (e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) == cudaSuccess) P->done.push_back(ev);
            if (e != cudaSuccess) {
                d.rs_plan = P;
                cb_resident_free(d);
                return undo(e);
            }
        }
    }
    d.rs_plan = P;
    return cudaSuccess;
}

}  // namespace

cudaError_t cb_resident_step(cb_dev& d, long long n, cudaStream_t st, long long* launches) {
    if (n <= 0) return cudaSuccess;
    cudaError_t e;
    if (!d.rs_plan && (e = build_plan(d)) != cudaSuccess) return e;
    const cb_rs_plan& P = *d.rs_plan;
    if ((e = cudaMemsetAsync(d.rs_counter, 0, sizeof(int) * 8, st)) != cudaSuccess) return e;
    const bool side = !P.streams.empty();
    if (side && (e = cudaEventRecord(P.fork, st)) != cudaSuccess) return e;
    // largest clusters first: the smaller ones then fill the SMs they leave and the tail
    for (size_t j = P.args.size(); j-- > 0;) {
        rs_args a = P.args[j];
        a.fields = d.fields[d.cur];
        a.cyto = d.cyto[d.ccur];
        a.nsteps = n;
        cudaStream_t sj = side ? P.streams[j] : st;
        if (side && (e = cudaStreamWaitEvent(sj, P.fork, 0)) != cudaSuccess) return e;
        e = launch_t(d, a, P.nz, P.cs[j], P.threads[j], sj, a.S, nullptr, P.clusters[j]);
        if (e != cudaSuccess) return e;
        if (launches) *launches += 1;
        if (side) {
            if ((e = cudaEventRecord(P.done[j], sj)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(st, P.done[j], 0)) != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

// ---------------------------------------------------------------- autotuning
namespace {

// the device state a resident launch reads and writes, copied aside and put back
struct state_copy {
    std::vector<std::pair<void*, size_t>> bufs;  // (live buffer, bytes)
    std::vector<void*> saved;
    cudaError_t take(const cb_dev& d) {
        const size_t rs = d.precision == 0 ? 8 : 4;
        bufs = {{d.fields[d.cur], (size_t)d.total_nodes * d.m.F * rs},
                {d.curgrid, (size_t)d.total_nodes * d.m.n_ions * rs},
                {d.ch_state, (size_t)d.total_ch * sizeof(int)},
                {d.mouth, (size_t)d.total_ch * d.NS * sizeof(double)},
                {d.sc, (size_t)d.S * sizeof(cb_site_scalars)}};
        if (d.nc > 0) {
            bufs.push_back({d.cyto[d.ccur], (size_t)d.S * d.CS * d.nc * rs});
            bufs.push_back({d.cin, (size_t)d.S * d.CS * d.m.mc * d.m.mc * sizeof(double)});
        }
        for (auto& b : bufs) {
            void* p = nullptr;
            cudaError_t e = cudaMalloc(&p, b.second);
            if (e != cudaSuccess) return e;
            saved.push_back(p);
            if ((e = cudaMemcpy(p, b.first, b.second, cudaMemcpyDeviceToDevice)) != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    cudaError_t put_back(cudaStream_t st) {
        for (size_t k = 0; k < bufs.size(); ++k) {
            cudaError_t e = cudaMemcpyAsync(bufs[k].first, saved[k], bufs[k].second, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return e;
        }
        return cudaStreamSynchronize(st);
    }
    ~state_copy() {
        for (void* p : saved) cudaFree(p);
    }
};

}  // namespace

// Block size and cluster size of every class chosen by measurement: each candidate runs
// `steps` time steps of its class alone (the other classes idle) from the same state,
// which is put back after every trial and at the end. Candidates: 256 to the
// specialisation's bound in steps of 64 threads, at the class's cluster size and, where
// the class's sites fit it, at twice that size; from 4 blocks on, with even rows and with
// fewer rows on the ranks that carry the y-edge rim lines and the plane-0 deposits.
cudaError_t cb_resident_autotune(cb_dev& d, long long steps, cudaStream_t st, std::string* report) {
    cudaError_t e;
    if (!d.rs_plan && (e = build_plan(d)) != cudaSuccess) return e;
    cb_rs_plan& P = *d.rs_plan;
    if (steps < 1) return cudaErrorInvalidValue;
    std::vector<cb_site> sites(d.S);
    if ((e = cudaMemcpy(sites.data(), d.sites, sizeof(cb_site) * d.S, cudaMemcpyDeviceToHost)) != cudaSuccess) return e;
    std::vector<std::vector<int>> classes;
    std::vector<int> cs;
    if (!classify(d, sites, classes, cs) || classes.size() != P.args.size()) return cudaErrorInvalidConfiguration;
    state_copy snap;
    if ((e = snap.take(d)) != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::string rep;
    for (size_t k = 0; k < P.args.size(); ++k) {
        struct cand {
            int C, threads, clusters, light;
            rs_args a;
            float ms;
        };
        std::vector<cand> cands;
        for (int C : {cs[k], 2 * cs[k]}) {
            if (C > 16) continue;
            for (int light = 0; light < (C >= 4 ? 2 : 1); ++light) {
                // light: the first and last row blocks (long y-edge rim lines) and the rank of
                // plane 0 (efflux deposits) take 2 shares of the rows, the others 3
                rs_args a = P.args[k];  // plan() rewrites only the shared-memory layout
                row_weights(a, C, light != 0);
                if (!plan(d, sites, classes[k], C, a)) continue;
                const int cap = thread_cap(d, P.nz, C);
                for (int t = 256; t <= cap; t += 64) {
                    int clusters = 0;
                    if (launch_t(d, a, P.nz, C, t, 0, a.S, &clusters) != cudaSuccess || clusters < 1) {
                        cudaGetLastError();
                        continue;
                    }
                    cands.push_back({C, t, clusters, light, a, 0.f});
                }
            }
        }
        for (auto& c : cands) {
            float best = 1e30f;
            for (int rep_i = 0; rep_i < 2; ++rep_i) {  // the first run also loads the specialisation
                rs_args a = c.a;
                a.fields = d.fields[d.cur];
                a.cyto = d.cyto[d.ccur];
                a.nsteps = steps;
                if ((e = cudaMemsetAsync(a.counter, 0, sizeof(int), st)) != cudaSuccess) return e;
                cudaEventRecord(e0, st);
                if ((e = launch_t(d, a, P.nz, c.C, c.threads, st, a.S, nullptr, c.clusters)) != cudaSuccess) return e;
                cudaEventRecord(e1, st);
                if ((e = cudaEventSynchronize(e1)) != cudaSuccess) return e;
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                best = std::min(best, ms);
                if ((e = snap.put_back(st)) != cudaSuccess) return e;
            }
            c.ms = best;
        }
        if (cands.empty()) continue;
        const cand* b = &cands[0];
        for (auto& c : cands)
            if (c.ms < b->ms) b = &c;
        float cur_ms = -1;
        for (auto& c : cands)
            if (c.C == P.cs[k] && c.threads == P.threads[k] && !c.light) cur_ms = c.ms;
        rep += (k ? "; " : "") + std::to_string(classes[k].size()) + " sites: clusters of " + std::to_string(P.cs[k]) + " x " +
               std::to_string(P.threads[k]) + " threads (" + std::to_string(cur_ms) + " ms) -> " + std::to_string(b->C) + " x " +
               std::to_string(b->threads) + (b->light ? " light edge rows" : "") + " (" + std::to_string(b->ms) + " ms)";
        P.cs[k] = b->C;
        P.threads[k] = b->threads;
        P.clusters[k] = b->clusters;
        P.args[k] = b->a;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (report) *report = rep;
    return snap.put_back(st);
}
