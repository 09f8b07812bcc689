// C ABI of libcasim_b200.so (declared in include/casim_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/casim_b200.h"
#include "engine.h"
#include "mwc.h"
#include "parse.h"
#include "mrg32k3a.cuh"
#include "physics.cuh"

struct casim_b200_sim {
    cb_config cfg;
    cb_dev d;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    int path = CASIM_PATH_PLAIN;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timed = false;  // both events recorded by a step
    double last_ms = 0;
    long long last_launches = 0;
    std::vector<void*> allocs;
    std::string resident_why;  // how the resident path splits the batch, or why it was not chosen
    // surrogate-driven gating: feature buffer and one captured window
    float* sg_x = nullptr;
    int sg_rows = 0, sg_ld = 0, sg_maxch = 0, sg_window = 0;
    void* sg_net = nullptr;
    const void* sg_out = nullptr;  // the network's output buffer when the window was captured
    cudaGraphExec_t sg_exec = nullptr;
    unsigned long long* sg_res = nullptr;  // residual check: max error bits, failing sites
    // open-RyR traces: [site][tr_max] u16, a sample every tr_every steps of casim_b200_step
    uint16_t* tr = nullptr;
    long long tr_every = 0, tr_max = 0, tr_n = 0, tr_phase = 0;
};

namespace {

thread_local std::string g_create_err;

struct cuda_fail : std::runtime_error {
    cudaError_t code;
    cuda_fail(cudaError_t c, const std::string& w) : std::runtime_error(w + ": " + cudaGetErrorString(c)), code(c) {}
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw cuda_fail(e, what);
}

// a request outside what this build serves (CASIM_EUNSUPPORTED)
struct unsupported : std::runtime_error {
    using std::runtime_error::runtime_error;
};

template <typename T>
T* dalloc(casim_b200_sim* h, size_t n) {
    void* p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) throw cuda_fail(e, "cudaMalloc");
    h->allocs.push_back(p);
    return (T*)p;
}

template <typename T>
T* dupload(casim_b200_sim* h, const std::vector<T>& v) {
    T* p = dalloc<T>(h, v.size());
    if (!v.empty()) ck(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
    return p;
}

casim_status set_err(casim_b200_sim* h, casim_status s, const std::string& msg) {
    if (h) h->err = msg;
    else g_create_err = msg;
    return s;
}

#define GUARD(h)                                                            \
    if (!(h)) return CASIM_EINVAL;                                          \
    try {
#define END_GUARD(h)                                                        \
    }                                                                       \
    catch (const cuda_fail& e) {                                            \
        return set_err(h, e.code == cudaErrorMemoryAllocation ? CASIM_ENOMEM : CASIM_ECUDA, e.what()); \
    }                                                                       \
    catch (const unsupported& e) {                                          \
        return set_err(h, CASIM_EUNSUPPORTED, e.what());                    \
    }                                                                       \
    catch (const std::exception& e) {                                       \
        return set_err(h, CASIM_EINVAL, e.what());                          \
    }

void check_site(casim_b200_sim* h, int site) {
    if (site < 0 || site >= h->d.S) throw std::runtime_error("site index " + std::to_string(site) + " out of range");
}

// node index in the reference order for (x, y, z)
inline long long ref_index(const cb_site& s, int dim, int x, int y, int z) {
    return dim == 2 ? (long long)y + (long long)s.ny * x : (long long)z + (long long)s.nz * ((long long)y + (long long)s.ny * x);
}

void build_device(casim_b200_sim* h, int precision) {
    const cb_config& cfg = h->cfg;
    cb_dev& d = h->d;
    d.m = cfg.m;
    d.S = (int)cfg.sites.size();
    d.precision = precision;
    d.min_cluster = cfg.min_cluster;
    d.light_rows = cfg.light_rows;
    if (cfg.generic_kernels) d.st_nz = 0;  // the specialised streaming kernels stay off
    d.NS = cfg.m.F + cfg.m.n_buf;
    const size_t rs = precision == 0 ? sizeof(double) : sizeof(float);
    std::vector<cb_site> sites(d.S);
    std::vector<int> ch_node, ch_owner;
    std::vector<cb_site_scalars> sc(d.S);
    std::vector<int> rim_cnode, dep_ptr, dep_term;
    long long nb = 0;
    int choff = 0, rimoff = 0, termoff = 0;
    const int mc = cfg.m.mc;
    const bool rd3d = cfg.m.cyto_type == CB_CYTO_RD3D;
    for (int s = 0; s < d.S; ++s) {
        const cb_site_host& sh = cfg.sites[s];
        cb_site& st = sites[s];
        st.nx = sh.nx;
        st.ny = sh.ny;
        st.nz = cfg.m.dim == 3 ? sh.nz : 1;
        int N = st.nx * st.ny * st.nz;
        st.npad = (N + 31) / 32 * 32;
        st.node_base = nb;
        nb += st.npad;
        st.n_ch = (int)sh.ch_node_xyz.size() / 3;
        st.ch_off = choff;
        choff += st.n_ch;
        d.max_nodes = std::max(d.max_nodes, st.npad);
        d.max_ch = std::max(d.max_ch, st.n_ch);
        int zmax = cfg.m.dim == 2 ? 1 : st.nz - 1;
        int T = cb_efflux_terms(st.nx, st.ny, zmax);
        d.max_terms = std::max(d.max_terms, T);
        std::map<int, int> last_at;
        for (int c = 0; c < st.n_ch; ++c) {
            int x = sh.ch_node_xyz[3 * c], y = sh.ch_node_xyz[3 * c + 1], z = sh.ch_node_xyz[3 * c + 2];
            int node = x + st.nx * (y + st.ny * z);
            ch_node.push_back(node);
            last_at[node] = c;
        }
        for (int c = 0; c < st.n_ch; ++c) ch_owner.push_back(last_at[ch_node[st.ch_off + c]] == c ? 1 : 0);
        std::memset(&sc[s], 0, sizeof(cb_site_scalars));
        for (int i = 0; i < CB_MAX_IONS; ++i) sc[s].jsr0[i] = sh.jsr0[i];
        for (int i = 0; i < 6; ++i) sc[s].rng[i] = sh.seed[i];
        if (rd3d) {
            // rim -> nearest layer-0 cytosol node, clamped to the updated range
            int nrim = cb_rim_count(st.nx, st.ny);
            st.rim_off = rimoff;
            for (int r = 0; r < nrim; ++r) {
                int x, y;
                cb_rim_xy(r, st.nx, st.ny, x, y);
                rim_cnode.push_back(cb_rim_cnode(x, y, st.nx, st.ny, cfg.m.dx, cfg.m.dy, cfg.m.hc, mc));
            }
            rimoff += nrim;
            // deposit lists: efflux terms grouped by receiving cytosol node, term order kept
            std::vector<std::vector<int>> lists(mc * mc);
            for (int t = 0; t < T; ++t) {
                int x0, y0, x1, y1, x2, y2, z;
                cb_efflux_term(t, st.nx, st.ny, zmax, x0, y0, x1, y1, x2, y2, z);
                int r = cb_rim_index(x0, y0, st.nx, st.ny);
                lists[rim_cnode[st.rim_off + r]].push_back(t);
            }
            st.term_off = termoff;
            int acc = 0;
            for (int cn = 0; cn < mc * mc; ++cn) {
                dep_ptr.push_back(acc);
                for (int t : lists[cn]) dep_term.push_back(t);
                acc += (int)lists[cn].size();
            }
            dep_ptr.push_back(acc);
            termoff += acc;
        }
    }
    d.total_nodes = nb;
    d.total_ch = choff;
    d.sites = dupload(h, sites);
    d.sc = dupload(h, sc);
    d.ch_node = dupload(h, ch_node);
    d.ch_owner = dupload(h, ch_owner);
    d.ch_state = dalloc<int>(h, (size_t)choff);
    ck(cudaMemset(d.ch_state, 0, sizeof(int) * (size_t)std::max(choff, 1)), "cudaMemset");
    if (cfg.m.ch_model == CB_SINGLE_SITE_MWC) {
        // initial distribution at the initial mouth values: the ions' concentrations
        // (the map InitOpening reads before any gating, CaSim/DyadChannels.h:25-58)
        cb_mwc_tab tab;
        cb_mwc_build(cfg.m.ch_par, cfg.m.Cb[cfg.m.ca_idx], cfg.m.Cb[cfg.m.mg_idx], tab);
        cb_mwc_tab* dt = dalloc<cb_mwc_tab>(h, 1);
        ck(cudaMemcpy(dt, &tab, sizeof(tab), cudaMemcpyHostToDevice), "cudaMemcpy");
        d.mwc = dt;
        d.ch_micro = dalloc<int>(h, (size_t)choff);
        ck(cudaMemset(d.ch_micro, 0, sizeof(int) * (size_t)std::max(choff, 1)), "cudaMemset");
    }
    d.mouth = dalloc<double>(h, (size_t)choff * d.NS);
    ck(cudaMemset(d.mouth, 0, sizeof(double) * (size_t)std::max(choff * d.NS, 1)), "cudaMemset");
    for (int k = 0; k < 2; ++k) d.fields[k] = dalloc<char>(h, (size_t)nb * cfg.m.F * rs);
    d.curgrid = dalloc<char>(h, (size_t)nb * cfg.m.n_ions * rs);
    if (rd3d) {
        d.nc = mc * mc * mc;
        d.CS = cfg.m.n_ions + cfg.m.c_n_pairs;
        for (int k = 0; k < 2; ++k) d.cyto[k] = dalloc<char>(h, (size_t)d.S * d.CS * d.nc * rs);
        d.cin = dalloc<double>(h, (size_t)d.S * d.CS * mc * mc);
        d.rim_cnode = dupload(h, rim_cnode);
        d.dep_ptr = dupload(h, dep_ptr);
        d.dep_term = dupload(h, dep_term);
    }
    for (int w = 0; w < 2; ++w)
        if (!cfg.sp_x[w].empty()) {
            d.spx[w] = dupload(h, cfg.sp_x[w]);
            d.spc[w] = dupload(h, cfg.sp_c[w]);
        }
    d.err_flag = dalloc<int>(h, 4);
    ck(cudaMemset(d.err_flag, 0, 4 * sizeof(int)), "cudaMemset");
}

}  // namespace

// error text for calls that have no handle (read back through casim_b200_last_error(NULL, ...))
void cb_set_create_error(const std::string& msg) { g_create_err = msg; }

extern "C" {

casim_status casim_b200_create(const char* json_text, const char* base_dir, casim_precision precision, casim_path path,
                               const casim_site_table* sites, casim_h* out) {
    if (!json_text || !out) return set_err(nullptr, CASIM_EINVAL, "null argument");
    *out = nullptr;
    if (precision != CASIM_FP64 && precision != CASIM_FP32) return set_err(nullptr, CASIM_EINVAL, "bad precision");
    casim_b200_sim* h = new casim_b200_sim();
    try {
        h->cfg = cb_parse_config(json_text, base_dir ? base_dir : "", sites);
        double cfl = cb_cfl_number(h->cfg.m);
        if (!(cfl <= 1.0)) {
            std::string msg = "explicit step unstable: dt*D*sum(2/h^2) = " + std::to_string(cfl) + " > 1";
            delete h;
            return set_err(nullptr, CASIM_EUNSTABLE, msg);
        }
        int dev = 0;
        ck(cudaGetDevice(&dev), "cudaGetDevice");
        ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        h->own_stream = true;
        ck(cudaEventCreate(&h->ev0), "cudaEventCreate");
        ck(cudaEventCreate(&h->ev1), "cudaEventCreate");
        build_device(h, precision == CASIM_FP64 ? 0 : 1);
        int thr = 0;
        size_t smem = 0;
        std::string why;
        bool fits = cb_resident_fits(h->d, &thr, &smem, &why);
        h->resident_why = why;
        if (path == CASIM_PATH_RESIDENT && !fits) {
            std::string msg = "resident path unavailable: " + why;
            casim_b200_destroy(h);
            return set_err(nullptr, CASIM_EUNSUPPORTED, msg);
        }
        h->path = (path == CASIM_PATH_PLAIN || !fits) ? CASIM_PATH_PLAIN : CASIM_PATH_RESIDENT;
        if (path == CASIM_PATH_AUTO && fits) {
            // large 3D batches stream faster than they run resident (measured on the
            // 4096-dyad RD3D workload: 146 against 85 site-ms/s; 2D batches of 100 and
            // 1024 sites: resident 5.5x and 2.7x the streaming path)
            const bool rd3d = h->d.m.cyto_type == CB_CYTO_RD3D;
            const size_t w = precision == CASIM_FP64 ? 8 : 4;
            const size_t state = (size_t)h->d.total_nodes * h->d.m.F * w + (rd3d ? (size_t)h->d.S * h->d.CS * h->d.nc * w : 0);
            int dev = 0, l2 = 0;
            ck(cudaGetDevice(&dev), "cudaGetDevice");
            ck(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev), "cudaDeviceGetAttribute");
            if ((rd3d || h->d.m.dim == 3) && state > (size_t)l2 && cb_plain_streaming(h->d)) {
                h->path = CASIM_PATH_PLAIN;
                h->resident_why = "streaming: state of " + std::to_string(state >> 20) + " MiB exceeds the " +
                                  std::to_string(l2 >> 20) + " MiB L2 (resident would be: " + why + ")";
            }
        }
        ck(cb_plain_reset(h->d, h->stream), "reset");
        ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    } catch (const cuda_fail& e) {
        std::string msg = e.what();
        casim_status s = e.code == cudaErrorMemoryAllocation ? CASIM_ENOMEM : CASIM_ECUDA;
        casim_b200_destroy(h);
        return set_err(nullptr, s, msg);
    } catch (const std::exception& e) {
        std::string msg = e.what();
        casim_b200_destroy(h);
        return set_err(nullptr, CASIM_EINVAL, msg);
    }
    *out = h;
    return CASIM_OK;
}

casim_status casim_b200_destroy(casim_h h) {
    if (!h) return CASIM_EINVAL;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void* p : h->allocs) cudaFree(p);
    if (h->d.rs_order) cudaFree(h->d.rs_order);
    if (h->d.rs_counter) cudaFree(h->d.rs_counter);
    if (h->d.rs_pow2) cudaFree(h->d.rs_pow2);
    if (h->d.st_tiles) cudaFree(h->d.st_tiles);
    if (h->d.st_chcol) cudaFree(h->d.st_chcol);
    if (h->d.pre_jump) cudaFree(h->d.pre_jump);
    cb_resident_free(h->d);
    if (h->sg_exec) cudaGraphExecDestroy(h->sg_exec);
    if (h->tr) cudaFree(h->tr);
    if (h->sg_res) cudaFree(h->sg_res);
    if (h->sg_x) cudaFree(h->sg_x);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return CASIM_OK;
}

casim_status casim_b200_last_error(casim_h h, char* buf, size_t n) {
    const std::string& e = h ? h->err : g_create_err;
    if (buf && n) {
        size_t k = std::min(n - 1, e.size());
        std::memcpy(buf, e.data(), k);
        buf[k] = 0;
    }
    return CASIM_OK;
}

casim_status casim_b200_info(casim_h h, casim_info* o) {
    if (!h || !o) return CASIM_EINVAL;
    o->n_sites = h->d.S;
    o->dim = h->d.m.dim;
    o->n_ions = h->d.m.n_ions;
    o->n_pairs = h->d.m.n_pairs;
    o->n_buffers = h->d.m.n_buf;
    o->n_cyto_species = h->d.m.n_ions + h->d.m.c_n_pairs;
    o->cyto_nodes = h->d.nc;
    o->precision = h->d.precision;
    o->path = h->path;
    o->max_channels = h->d.max_ch;
    long long tn = 0;
    for (auto& s : h->cfg.sites) tn += (long long)s.nx * s.ny * (h->d.m.dim == 3 ? s.nz : 1);
    o->total_nodes = tn;
    o->dt_ms = h->d.m.dt;
    o->element_volume = h->d.m.V_elem;
    return CASIM_OK;
}

casim_status casim_b200_species_name(casim_h h, int32_t index, char* buf, size_t n) {
    if (!h || !buf || !n) return CASIM_EINVAL;
    std::string name;
    const cb_config& c = h->cfg;
    int ni = (int)c.ion_names.size(), np = (int)c.pair_names.size(), nb = (int)c.buf_names.size();
    if (index < 0 || index >= ni + np + nb) return set_err(h, CASIM_EINVAL, "species index out of range");
    name = index < ni ? c.ion_names[index] : index < ni + np ? c.pair_names[index - ni] : c.buf_names[index - ni - np];
    size_t k = std::min(n - 1, name.size());
    std::memcpy(buf, name.data(), k);
    buf[k] = 0;
    return CASIM_OK;
}

casim_status casim_b200_cyto_species_name(casim_h h, int32_t index, char* buf, size_t n) {
    if (!h || !buf || !n) return CASIM_EINVAL;
    const cb_config& c = h->cfg;
    int ni = (int)c.ion_names.size(), np = (int)c.cyto_pair_names.size();
    if (index < 0 || index >= ni + np) return set_err(h, CASIM_EINVAL, "cytosol species index out of range");
    const std::string& name = index < ni ? c.ion_names[index] : c.cyto_pair_names[index - ni];
    size_t k = std::min(n - 1, name.size());
    std::memcpy(buf, name.data(), k);
    buf[k] = 0;
    return CASIM_OK;
}

casim_status casim_b200_set_stream(casim_h h, void* s) {
    if (!h) return CASIM_EINVAL;
    cudaStreamSynchronize(h->stream);
    if (s) {
        if (h->own_stream) cudaStreamDestroy(h->stream);
        h->stream = (cudaStream_t)s;
        h->own_stream = false;
    }
    return CASIM_OK;
}

casim_status casim_b200_reset(casim_h h) {
    GUARD(h)
    ck(cb_plain_reset(h->d, h->stream), "reset");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_init_opening(casim_h h, int32_t site, int32_t channel) {
    GUARD(h)
    check_site(h, site);
    int* dfirst = nullptr;
    ck(cudaMallocAsync(&dfirst, sizeof(int), h->stream), "cudaMallocAsync");
    ck(cudaMemcpyAsync(dfirst, &channel, sizeof(int), cudaMemcpyHostToDevice, h->stream), "cudaMemcpyAsync");
    ck(cb_plain_init_opening(h->d, dfirst, site, site + 1, h->stream), "init_opening");
    ck(cudaFreeAsync(dfirst, h->stream), "cudaFreeAsync");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_update(casim_h h) {
    GUARD(h)
    long long l = 0;
    ck(cb_plain_update(h->d, h->stream, &l), "update");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_start(casim_h h, const int32_t* first_channel) {
    GUARD(h)
    if (!first_channel) throw std::runtime_error("first_channel is null");
    ck(cb_plain_reset(h->d, h->stream), "reset");
    int* dfirst = dalloc<int>(h, (size_t)h->d.S);
    ck(cudaMemcpyAsync(dfirst, first_channel, sizeof(int) * h->d.S, cudaMemcpyHostToDevice, h->stream), "cudaMemcpyAsync");
    ck(cb_plain_init_opening(h->d, dfirst, 0, h->d.S, h->stream), "init_opening");
    long long l = 0;
    ck(cb_plain_update(h->d, h->stream, &l), "update");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    cudaFree(dfirst);
    h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)dfirst), h->allocs.end());
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_set_site_jsr(casim_h h, const double* jsr) {
    GUARD(h)
    if (!jsr) throw std::runtime_error("jsr_init is null");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    std::vector<cb_site_scalars> sc(h->d.S);
    ck(cudaMemcpy(sc.data(), h->d.sc, sizeof(cb_site_scalars) * h->d.S, cudaMemcpyDeviceToHost), "cudaMemcpy");
    for (int s = 0; s < h->d.S; ++s)
        for (int i = 0; i < h->d.m.n_ions; ++i) sc[s].jsr0[i] = jsr[(size_t)s * h->d.m.n_ions + i];
    ck(cudaMemcpy(h->d.sc, sc.data(), sizeof(cb_site_scalars) * h->d.S, cudaMemcpyHostToDevice), "cudaMemcpy");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_step(casim_h h, int64_t n) {
    GUARD(h)
    if (n < 0) throw std::runtime_error("negative step count");
    long long launches = 0;
    ck(cudaEventRecord(h->ev0, h->stream), "cudaEventRecord");
    auto run = [&](long long k) {
        if (h->path == CASIM_PATH_RESIDENT) ck(cb_resident_step(h->d, k, h->stream, &launches), "resident step");
        else ck(cb_plain_step(h->d, k, h->stream, &launches), "plain step");
    };
    if (h->tr && h->tr_n < h->tr_max) {
        // stop at every sample time of the open-RyR trace
        long long left = n;
        while (left > 0 && h->tr_n < h->tr_max) {
            const long long k = std::min(left, h->tr_every - h->tr_phase);
            run(k);
            left -= k;
            h->tr_phase += k;
            if (h->tr_phase == h->tr_every) {
                ck(cb_trace_record(h->d, h->tr, h->tr_max, h->tr_n++, h->stream), "trace record");
                ++launches;
                h->tr_phase = 0;
            }
        }
        if (left > 0) run(left);
    } else {
        run(n);
    }
    ck(cudaEventRecord(h->ev1, h->stream), "cudaEventRecord");
    h->timed = true;
    h->last_launches = launches;
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_profile_step(casim_h h, double* ms, int32_t n, int32_t* count) {
    GUARD(h)
    if (!ms || n < 1 || !count) throw std::runtime_error("profile_step: bad argument");
    if (h->tr) throw std::runtime_error("profile_step: not with an open-RyR trace enabled");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    if (h->path == CASIM_PATH_RESIDENT) {
        long long launches = 0;
        ck(cudaEventRecord(h->ev0, h->stream), "cudaEventRecord");
        ck(cb_resident_step(h->d, 1, h->stream, &launches), "resident step");
        ck(cudaEventRecord(h->ev1, h->stream), "cudaEventRecord");
        ck(cudaEventSynchronize(h->ev1), "cudaEventSynchronize");
        float t = 0;
        ck(cudaEventElapsedTime(&t, h->ev0, h->ev1), "cudaEventElapsedTime");
        ms[0] = t;
        *count = 1;
    } else {
        cudaEvent_t ev[5] = {};
        for (int k = 0; k < 5; ++k) ck(cudaEventCreate(&ev[k]), "cudaEventCreate");
        cudaError_t e = cb_plain_step_marked(h->d, h->stream, ev);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[4]);
        float t[4] = {};
        for (int k = 0; k < 4 && e == cudaSuccess; ++k) e = cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]);
        for (int k = 0; k < 5; ++k) cudaEventDestroy(ev[k]);
        ck(e, "profile_step");
        for (int k = 0; k < 4 && k < n; ++k) ms[k] = t[k];
        *count = n < 4 ? n : 4;
    }
    h->timed = false;
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_set_site_gating(casim_h h, const char* json_text, const char* base_dir, const int32_t* sites, int32_t n) {
    GUARD(h)
    if (!json_text || !sites || n < 1) throw std::runtime_error("set_site_gating: bad argument");
    if (h->path != CASIM_PATH_PLAIN) throw unsupported("per-site gating models run on the plain path (create the handle with it)");
    if (h->d.mwc || h->d.m.ch_model == CB_SINGLE_SITE_MWC) throw unsupported("per-site gating models are two-state models");
    if (!cb_plain_gating_ready(h->d)) throw unsupported("per-site gating models need the specialised streaming kernels");
    for (int k = 0; k < n; ++k) check_site(h, sites[k]);
    // parse the JSON against a one-site table shaped like site 0 (no coordinates file is
    // read: only the gating model is taken from it)
    cb_site s0{};
    ck(cudaMemcpy(&s0, h->d.sites, sizeof(cb_site), cudaMemcpyDeviceToHost), "cudaMemcpy");
    int32_t tnx = s0.nx, tny = s0.ny, tnz = s0.nz, tnch = 1;
    double tx = 0.5 * (s0.nx - 1) * h->d.m.dx, ty = 0.5 * (s0.ny - 1) * h->d.m.dy;
    uint32_t tseed[6] = {12345, 12345, 12345, 12345, 12345, 12345};
    casim_site_table tab{};
    tab.n_sites = 1;
    tab.nx = &tnx;
    tab.ny = &tny;
    tab.nz = &tnz;
    tab.n_channels = &tnch;
    tab.ch_x = &tx;
    tab.ch_y = &ty;
    tab.seeds = tseed;
    const cb_config cfg = cb_parse_config(json_text, base_dir ? base_dir : "", &tab);
    if (cfg.m.ch_model == CB_SINGLE_SITE_MWC) throw unsupported("per-site gating models are two-state models");
    if (cfg.m.n_ions != h->d.m.n_ions || cfg.m.ca_idx != h->d.m.ca_idx || cfg.m.mg_idx != h->d.m.mg_idx)
        throw std::runtime_error("the gating model's JSON names other ions than the handle's");
    std::vector<cb_gate> gates(CB_MAX_GATES);
    int n_gates = h->d.n_gates;
    if (n_gates == 0) {  // gate 0: the handle's own model, every site on it
        cb_gate& g = gates[0];
        g.ch_model = h->d.m.ch_model;
        for (int i = 0; i < CB_MAX_CHPAR; ++i) g.ch_par[i] = h->d.m.ch_par[i];
        for (int w = 0; w < 2; ++w) {
            g.sp_n[w] = h->d.m.sp_n[w];
            g.spx[w] = h->d.spx[w];
            g.spc[w] = h->d.spc[w];
        }
        h->d.gates = dalloc<cb_gate>(h, CB_MAX_GATES);
        h->d.site_gate = dalloc<int>(h, (size_t)h->d.S);
        ck(cudaMemsetAsync(h->d.site_gate, 0, sizeof(int) * (size_t)h->d.S, h->stream), "cudaMemset");
        n_gates = 1;
    } else {
        ck(cudaMemcpy(gates.data(), h->d.gates, sizeof(cb_gate) * CB_MAX_GATES, cudaMemcpyDeviceToHost), "cudaMemcpy");
    }
    if (n_gates >= CB_MAX_GATES) throw unsupported("at most " + std::to_string(CB_MAX_GATES - 1) + " extra gating models per handle");
    cb_gate& g = gates[n_gates];
    g.ch_model = cfg.m.ch_model;
    for (int i = 0; i < CB_MAX_CHPAR; ++i) g.ch_par[i] = cfg.m.ch_par[i];
    for (int w = 0; w < 2; ++w) {
        g.sp_n[w] = cfg.m.sp_n[w];
        g.spx[w] = cfg.sp_x[w].empty() ? nullptr : dupload(h, cfg.sp_x[w]);
        g.spc[w] = cfg.sp_c[w].empty() ? nullptr : dupload(h, cfg.sp_c[w]);
    }
    ck(cudaMemcpy(h->d.gates, gates.data(), sizeof(cb_gate) * CB_MAX_GATES, cudaMemcpyHostToDevice), "cudaMemcpy");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    std::vector<int> idx(n);
    for (int k = 0; k < n; ++k) idx[k] = n_gates;
    for (int k = 0; k < n; ++k) ck(cudaMemcpy(h->d.site_gate + sites[k], &idx[k], sizeof(int), cudaMemcpyHostToDevice), "cudaMemcpy");
    h->d.n_gates = n_gates + 1;
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_trace_enable(casim_h h, int64_t every_steps, int64_t max_samples) {
    GUARD(h)
    if (every_steps < 1 || max_samples < 1) throw std::runtime_error("trace needs every_steps >= 1 and max_samples >= 1");
    if ((double)max_samples * h->d.S * sizeof(uint16_t) > 16e9) throw std::runtime_error("trace larger than 16 GB");
    if (h->tr) {
        ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
        ck(cudaFree(h->tr), "cudaFree");
        h->tr = nullptr;
    }
    void* p = nullptr;
    ck(cudaMalloc(&p, (size_t)max_samples * h->d.S * sizeof(uint16_t)), "cudaMalloc");
    h->tr = (uint16_t*)p;
    h->tr_every = every_steps;
    h->tr_max = max_samples;
    h->tr_n = 0;
    h->tr_phase = 0;
    ck(cb_trace_record(h->d, h->tr, h->tr_max, h->tr_n++, h->stream), "trace record");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_trace_count(casim_h h, int64_t* n_samples) {
    if (!h || !n_samples) return CASIM_EINVAL;
    *n_samples = h->tr ? h->tr_n : 0;
    return CASIM_OK;
}

casim_status casim_b200_get_open_traces(casim_h h, uint16_t* out) {
    GUARD(h)
    if (!out) throw std::runtime_error("null output");
    if (!h->tr) throw std::runtime_error("no trace: call casim_b200_trace_enable first");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    ck(cudaMemcpy2D(out, (size_t)h->tr_n * sizeof(uint16_t), h->tr, (size_t)h->tr_max * sizeof(uint16_t),
                    (size_t)h->tr_n * sizeof(uint16_t), (size_t)h->d.S, cudaMemcpyDeviceToHost),
       "cudaMemcpy2D");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_release_analysis(casim_h h, double hist_dt_ms, double max_time_ms, int32_t nadir, double* per_site,
                                         int32_t* hist_all, int32_t* hist_quark, int32_t* hist_blip, int32_t* hist_spark,
                                         int32_t* class_counts) {
    GUARD(h)
    if (!h->tr || h->tr_n < 1) throw std::runtime_error("no trace: call casim_b200_trace_enable first");
    if (!(hist_dt_ms > 0) || !(max_time_ms >= 0) || nadir < 0) throw std::runtime_error("bad histogram arguments");
    if (!per_site || !hist_all || !hist_quark || !hist_blip || !hist_spark || !class_counts) throw std::runtime_error("null output");
    const double ts = (double)h->tr_every * h->d.m.dt;  // ms between samples
    const long long nh = (long long)(max_time_ms / hist_dt_ms);  // CaSim/IndChannelCREAnalyzer.cpp:58
    if (nh > 100000000LL) throw std::runtime_error("histogram longer than 1e8 bins");
    const int mch = h->d.max_ch, S = h->d.S;
    const size_t na = (size_t)(nh + 1) * (mch + 1), nq = (size_t)(nh + 1) * 2, nb = (size_t)(nh + 1) * (nadir + 1);
    void* buf = nullptr;
    const size_t bytes = (size_t)S * 5 * sizeof(double) + (S + 3 + 2 * na + nq + nb) * sizeof(int);
    ck(cudaMalloc(&buf, bytes), "cudaMalloc");
    double* d_ps = (double*)buf;
    int* d_cls = (int*)(d_ps + (size_t)S * 5);
    int* d_cnt = d_cls + S;
    int* d_all = d_cnt + 3;
    int* d_q = d_all + na;
    int* d_b = d_q + nq;
    int* d_s = d_b + nb;
    cudaError_t e = cb_cre_analysis(h->d, h->tr, h->tr_max, h->tr_n, ts, hist_dt_ms, nh, nadir, d_ps, d_cls, d_all, d_q, d_b, d_s,
                                    d_cnt, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) e = cudaMemcpy(per_site, d_ps, (size_t)S * 5 * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(class_counts, d_cnt, 3 * sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(hist_all, d_all, na * sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(hist_quark, d_q, nq * sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(hist_blip, d_b, nb * sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(hist_spark, d_s, na * sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(buf);
    ck(e, "release analysis");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_autotune(casim_h h, int64_t steps_per_trial, char* report, size_t n) {
    GUARD(h)
    if (steps_per_trial < 1) throw std::runtime_error("steps_per_trial must be >= 1");
    std::string rep = "plain path: nothing to tune";
    if (h->path == CASIM_PATH_RESIDENT) {
        ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
        ck(cb_resident_autotune(h->d, steps_per_trial, h->stream, &rep), "autotune");
    }
    if (report && n) {
        const size_t k = std::min(n - 1, rep.size());
        std::memcpy(report, rep.data(), k);
        report[k] = 0;
    }
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_synchronize(casim_h h) {
    GUARD(h)
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    float ms = 0;
    // only after a step recorded both events; a failed query must not leave
    // its error behind for the next cudaGetLastError of another library
    if (h->timed) {
        if (cudaEventElapsedTime(&ms, h->ev0, h->ev1) == cudaSuccess) h->last_ms = ms;
        else cudaGetLastError();
    }
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_path_note(casim_h h, char* buf, size_t n) {
    if (!h || !buf || !n) return CASIM_EINVAL;
    size_t k = std::min(n - 1, h->resident_why.size());
    std::memcpy(buf, h->resident_why.data(), k);
    buf[k] = 0;
    return CASIM_OK;
}

casim_status casim_b200_last_step_ms(casim_h h, double* out) {
    if (!h || !out) return CASIM_EINVAL;
    *out = h->last_ms;
    return CASIM_OK;
}

casim_status casim_b200_last_step_launches(casim_h h, int64_t* out) {
    if (!h || !out) return CASIM_EINVAL;
    *out = h->last_launches;
    return CASIM_OK;
}

casim_status casim_b200_get_field(casim_h h, int32_t site, int32_t species, double* out) {
    GUARD(h)
    check_site(h, site);
    const cb_model& m = h->d.m;
    if (species < 0 || species >= m.F + m.n_buf) throw std::runtime_error("species out of range");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    cb_site st;
    ck(cudaMemcpy(&st, h->d.sites + site, sizeof(cb_site), cudaMemcpyDeviceToHost), "cudaMemcpy");
    std::vector<double> blk((size_t)m.F * st.npad);
    size_t rs = h->d.precision == 0 ? 8 : 4;
    std::vector<char> raw(blk.size() * rs);
    const char* base = (const char*)h->d.fields[h->d.cur] + (size_t)st.node_base * m.F * rs;
    ck(cudaMemcpy(raw.data(), base, raw.size(), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
    for (size_t k = 0; k < blk.size(); ++k)
        blk[k] = rs == 8 ? ((const double*)raw.data())[k] : (double)((const float*)raw.data())[k];
    for (int z = 0; z < st.nz; ++z)
        for (int y = 0; y < st.ny; ++y)
            for (int x = 0; x < st.nx; ++x) {
                int n = x + st.nx * (y + st.ny * z);
                double v;
                if (species < m.F) {
                    v = blk[(size_t)species * st.npad + n];
                } else {
                    int b = species - m.F;
                    v = m.Ctot[b];
                    for (int p = 0; p < m.n_pairs; ++p)
                        if (m.pair_buf[p] == b) v -= blk[(size_t)(m.n_ions + p) * st.npad + n];
                }
                out[ref_index(st, m.dim, x, y, z)] = v;
            }
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_set_field(casim_h h, int32_t site, int32_t species, const double* in) {
    GUARD(h)
    check_site(h, site);
    const cb_model& m = h->d.m;
    if (species < 0 || species >= m.F) throw std::runtime_error("species out of range (stored species only)");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    cb_site st;
    ck(cudaMemcpy(&st, h->d.sites + site, sizeof(cb_site), cudaMemcpyDeviceToHost), "cudaMemcpy");
    size_t rs = h->d.precision == 0 ? 8 : 4;
    std::vector<char> raw((size_t)st.npad * rs, 0);
    for (int z = 0; z < st.nz; ++z)
        for (int y = 0; y < st.ny; ++y)
            for (int x = 0; x < st.nx; ++x) {
                int n = x + st.nx * (y + st.ny * z);
                double v = in[ref_index(st, m.dim, x, y, z)];
                if (rs == 8) ((double*)raw.data())[n] = v;
                else ((float*)raw.data())[n] = (float)v;
            }
    char* base = (char*)h->d.fields[h->d.cur] + ((size_t)st.node_base * m.F + (size_t)species * st.npad) * rs;
    ck(cudaMemcpy(base, raw.data(), raw.size(), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
    return CASIM_OK;
    END_GUARD(h)
}

static casim_status get_scalars(casim_h h, int32_t site, cb_site_scalars& q) {
    check_site(h, site);
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    ck(cudaMemcpy(&q, h->d.sc + site, sizeof(cb_site_scalars), cudaMemcpyDeviceToHost), "cudaMemcpy");
    return CASIM_OK;
}

casim_status casim_b200_get_mouth(casim_h h, int32_t site, int32_t species, double* out) {
    GUARD(h)
    check_site(h, site);
    if (species < 0 || species >= h->d.NS) throw std::runtime_error("species out of range");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    const cb_site_host& sh = h->cfg.sites[site];
    int nch = (int)sh.ch_node_xyz.size() / 3;
    cb_site st;
    ck(cudaMemcpy(&st, h->d.sites + site, sizeof(cb_site), cudaMemcpyDeviceToHost), "cudaMemcpy");
    std::vector<double> mo((size_t)nch * h->d.NS);
    ck(cudaMemcpy(mo.data(), h->d.mouth + (size_t)st.ch_off * h->d.NS, mo.size() * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    for (int c = 0; c < nch; ++c) out[c] = mo[(size_t)c * h->d.NS + species];
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_get_states(casim_h h, int32_t site, int32_t* out) {
    GUARD(h)
    check_site(h, site);
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    cb_site st;
    ck(cudaMemcpy(&st, h->d.sites + site, sizeof(cb_site), cudaMemcpyDeviceToHost), "cudaMemcpy");
    ck(cudaMemcpy(out, h->d.ch_state + st.ch_off, sizeof(int) * st.n_ch, cudaMemcpyDeviceToHost), "cudaMemcpy");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_get_micro_states(casim_h h, int32_t site, int32_t* out) {
    GUARD(h)
    check_site(h, site);
    if (!out) throw std::runtime_error("null output");
    if (!h->d.ch_micro) throw std::runtime_error("the RyR model has no micro-states (two-state gating)");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    cb_site st;
    ck(cudaMemcpy(&st, h->d.sites + site, sizeof(st), cudaMemcpyDeviceToHost), "cudaMemcpy");
    ck(cudaMemcpy(out, h->d.ch_micro + st.ch_off, sizeof(int) * st.n_ch, cudaMemcpyDeviceToHost), "cudaMemcpy");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_sg_features(casim_h h, int32_t max_channels, int32_t ld, float* x_dev) {
    GUARD(h)
    if (!x_dev || max_channels < 1 || ld < 3 * max_channels + 1 + h->d.m.n_buf) throw std::runtime_error("bad feature layout");
    ck(cb_sg_features(h->d, max_channels, ld, x_dev, h->stream), "surrogate features");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_sg_set_mouth(casim_h h, const float* y_dev, int32_t ld, double ca_ref) {
    GUARD(h)
    if (!y_dev || ld < 1 || !(ca_ref > 0)) throw std::runtime_error("bad network output layout");
    ck(cb_sg_mouth(h->d, y_dev, ld, ca_ref, h->stream), "surrogate mouth");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_sg_gate_steps(casim_h h, int64_t n) {
    GUARD(h)
    if (n < 0) throw std::runtime_error("negative step count");
    if (h->d.m.cyto_type != CB_CYTO_POOL) throw std::runtime_error("surrogate gating needs the pool cytosol");
    if (h->d.m.ch_model == CB_SINGLE_SITE_MWC) throw std::runtime_error("surrogate gating serves two-state RyR models");
    if (h->d.site_gate) throw unsupported("surrogate gating serves one gating model per batch");
    if (n > 0) ck(cb_sg_steps(h->d, n, h->stream), "surrogate steps");
    return CASIM_OK;
    END_GUARD(h)
}

namespace {

// one surrogate window on h->stream: features, network, mouth values, `window` steps
cudaError_t sg_window(casim_h h, casim_sg net, double ca_ref, int window) {
    cudaError_t e = cb_sg_features(h->d, h->sg_maxch, h->sg_ld, h->sg_x, h->stream);
    const float* y = nullptr;
    int ld = 0;
    if (e == cudaSuccess) e = cb_sg_net_forward(net, h->sg_x, h->sg_rows, h->stream, &y, &ld);
    if (e == cudaSuccess) e = cb_sg_mouth(h->d, y, ld, ca_ref, h->stream);
    if (e == cudaSuccess) e = cb_sg_steps(h->d, window, h->stream);
    return e;
}

}  // namespace

namespace {

// n steps of surrogate-driven gating in windows (one window captured as a CUDA graph)
void sg_windows(casim_h h, casim_sg net, int max_channels, long long n, int window, double ca_ref) {
    if (!net || n < 0 || window < 1 || !(ca_ref > 0) || max_channels < 1) throw std::runtime_error("bad surrogate run arguments");
    if (h->d.m.cyto_type != CB_CYTO_POOL) throw std::runtime_error("surrogate gating needs the pool cytosol");
    if (h->d.m.ch_model == CB_SINGLE_SITE_MWC) throw std::runtime_error("surrogate gating serves two-state RyR models");
    const int ld = 3 * max_channels + 1 + h->d.m.n_buf;
    const int rows = (h->d.S + 127) / 128 * 128;
    if (!h->sg_x || h->sg_rows != rows || h->sg_ld != ld) {
        if (h->sg_x) cudaFree(h->sg_x);
        h->sg_x = nullptr;
        ck(cudaMalloc(&h->sg_x, sizeof(float) * (size_t)rows * ld), "cudaMalloc");
        ck(cudaMemset(h->sg_x, 0, sizeof(float) * (size_t)rows * ld), "cudaMemset");
        h->sg_rows = rows;
        h->sg_ld = ld;
    }
    h->sg_maxch = max_channels;
    ck(cb_sg_net_prepare(net, rows), "surrogate buffers");
    if (h->sg_exec && (h->sg_net != (void*)net || h->sg_window != window || h->sg_out != cb_sg_net_output(net))) {
        cudaGraphExecDestroy(h->sg_exec);
        h->sg_exec = nullptr;
    }
    long long done = 0;
    // the first full window runs eagerly (sets kernel attributes), then one
    // window is captured into a graph and replayed
    while (done < n) {
        const int k = (int)std::min<long long>(window, n - done);
        if (k == window && h->sg_exec) {
            ck(cudaGraphLaunch(h->sg_exec, h->stream), "cudaGraphLaunch");
        } else {
            ck(sg_window(h, net, ca_ref, k), "surrogate window");
            if (k == window && !h->sg_exec) {
                cudaGraph_t g = nullptr;
                ck(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
                const cudaError_t ew = sg_window(h, net, ca_ref, window);
                const cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
                ck(ew, "surrogate window capture");
                ck(ec, "cudaStreamEndCapture");
                const cudaError_t ei = cudaGraphInstantiate(&h->sg_exec, g, 0);
                cudaGraphDestroy(g);
                ck(ei, "cudaGraphInstantiate");
                h->sg_net = (void*)net;
                h->sg_window = window;
                h->sg_out = cb_sg_net_output(net);
            }
        }
        done += k;
    }
}

casim_status sg_net_status(casim_h h, casim_sg net) {
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    const cudaError_t en = cb_sg_net_error(net);
    if (en == cudaErrorLaunchTimeout) {
        h->err = "a tensor-core wait of the surrogate network gave up";
        return CASIM_ETIMEOUT;
    }
    ck(en, "surrogate network");
    return CASIM_OK;
}

void rd_steps(casim_h h, long long n) {
    long long launches = 0;
    if (h->path == CASIM_PATH_RESIDENT) ck(cb_resident_step(h->d, n, h->stream, &launches), "resident step");
    else ck(cb_plain_step(h->d, n, h->stream, &launches), "plain step");
}

}  // namespace

casim_status casim_b200_sg_run(casim_h h, casim_sg net, int32_t max_channels, int64_t n, int32_t window, double ca_ref) {
    GUARD(h)
    if (h->d.site_gate) throw unsupported("surrogate gating serves one gating model per batch");
    sg_windows(h, net, max_channels, n, window, ca_ref);
    return sg_net_status(h, net);
    END_GUARD(h)
}

casim_status casim_b200_sg_hybrid_run(casim_h h, casim_sg net, int32_t max_channels, int64_t n, int32_t window,
                                      int32_t windows_per_check, int32_t rd_correction_steps, double tol, double max_fail_fraction,
                                      double ca_ref, casim_sg_hybrid_stats* stats) {
    GUARD(h)
    if (h->d.site_gate) throw unsupported("surrogate gating serves one gating model per batch");
    if (windows_per_check < 1 || rd_correction_steps < 1 || !(tol > 0) || !(max_fail_fraction >= 0) || n < 0)
        throw std::runtime_error("bad hybrid run arguments");
    casim_sg_hybrid_stats st{};
    if (!h->sg_res) {
        void* p = nullptr;
        ck(cudaMalloc(&p, 2 * sizeof(unsigned long long)), "cudaMalloc");
        h->sg_res = (unsigned long long*)p;
    }
    bool surrogate = true;
    long long done = 0;
    const long long period = (long long)windows_per_check * window;
    while (done < n) {
        const long long k = std::min(period, n - done);
        if (surrogate) {
            sg_windows(h, net, max_channels, k, window, ca_ref);
            st.surrogate_steps += k;
        } else {
            rd_steps(h, k);
            st.rd_steps += k;
        }
        done += k;
        if (done >= n) break;
        // full-RD correction, then the residual check of the network against it
        const long long c = std::min<long long>(rd_correction_steps, n - done);
        rd_steps(h, c);
        st.rd_steps += c;
        done += c;
        const float* y = nullptr;
        int ld = 0;
        ck(cb_sg_features(h->d, h->sg_maxch, h->sg_ld, h->sg_x, h->stream), "surrogate features");
        ck(cb_sg_net_forward(net, h->sg_x, h->sg_rows, h->stream, &y, &ld), "surrogate forward");
        double worst = 0, frac = 0;
        ck(cb_sg_residual(h->d, y, ld, ca_ref, tol, h->sg_res, &worst, &frac, h->stream), "residual check");
        ++st.checks;
        st.last_residual = worst;
        st.last_fail_fraction = frac;
        surrogate = frac <= max_fail_fraction;
        if (!surrogate) ++st.fallbacks;
    }
    const casim_status r = sg_net_status(h, net);
    if (stats) *stats = st;
    return r;
    END_GUARD(h)
}

casim_status casim_b200_set_all_states(casim_h h, const int32_t* states) {
    GUARD(h)
    if (h->d.ch_micro) throw std::runtime_error("set_all_states sets two-state RyRs only");
    if (!states) throw std::runtime_error("states is null");
    for (long long c = 0; c < h->d.total_ch; ++c)
        if (states[c] != 0 && states[c] != 1) throw std::runtime_error("RyR states must be 0 or 1");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    ck(cudaMemcpy(h->d.ch_state, states, sizeof(int) * (size_t)h->d.total_ch, cudaMemcpyHostToDevice), "cudaMemcpy");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_get_all_states(casim_h h, int32_t* out) {
    GUARD(h)
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    ck(cudaMemcpy(out, h->d.ch_state, sizeof(int) * (size_t)h->d.total_ch, cudaMemcpyDeviceToHost), "cudaMemcpy");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_get_all_mouth(casim_h h, int32_t species, double* out) {
    GUARD(h)
    if (species < 0 || species >= h->d.NS) throw std::runtime_error("species out of range");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    std::vector<double> mo((size_t)h->d.total_ch * h->d.NS);
    ck(cudaMemcpy(mo.data(), h->d.mouth, mo.size() * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    for (long long c = 0; c < h->d.total_ch; ++c) out[c] = mo[(size_t)c * h->d.NS + species];
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_get_jsr(casim_h h, int32_t site, double* out) {
    GUARD(h)
    cb_site_scalars q;
    get_scalars(h, site, q);
    for (int i = 0; i < h->d.m.n_ions; ++i) out[i] = q.jsr_new[i];
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_get_total_current(casim_h h, int32_t site, double* out) {
    GUARD(h)
    cb_site_scalars q;
    get_scalars(h, site, q);
    for (int i = 0; i < h->d.m.n_ions; ++i) out[i] = q.total[i];
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_get_efflux(casim_h h, int32_t site, double* out) {
    GUARD(h)
    cb_site_scalars q;
    get_scalars(h, site, q);
    for (int i = 0; i < h->d.m.F; ++i) out[i] = q.efflux[i];
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_get_cyto(casim_h h, int32_t site, double* out) {
    GUARD(h)
    cb_site_scalars q;
    get_scalars(h, site, q);
    for (int i = 0; i < h->d.m.n_ions; ++i) out[i] = q.c_ions[i];
    for (int p = 0; p < h->d.m.c_n_pairs; ++p) out[h->d.m.n_ions + p] = q.c_pairs[p];
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_get_cyto_field(casim_h h, int32_t site, int32_t species, double* out) {
    GUARD(h)
    check_site(h, site);
    if (h->d.m.cyto_type != CB_CYTO_RD3D) throw std::runtime_error("the cytosol is not RD3D");
    if (species < 0 || species >= h->d.CS) throw std::runtime_error("species out of range");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    size_t rs = h->d.precision == 0 ? 8 : 4;
    std::vector<char> raw((size_t)h->d.nc * rs);
    const char* base = (const char*)h->d.cyto[h->d.ccur] + ((size_t)site * h->d.CS + species) * h->d.nc * rs;
    ck(cudaMemcpy(raw.data(), base, raw.size(), cudaMemcpyDeviceToHost), "cudaMemcpy");
    for (int n = 0; n < h->d.nc; ++n) out[n] = rs == 8 ? ((double*)raw.data())[n] : (double)((float*)raw.data())[n];
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_set_cyto_field(casim_h h, int32_t site, int32_t species, const double* in) {
    GUARD(h)
    check_site(h, site);
    if (h->d.m.cyto_type != CB_CYTO_RD3D) throw std::runtime_error("the cytosol is not RD3D");
    if (species < 0 || species >= h->d.CS) throw std::runtime_error("species out of range");
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    size_t rs = h->d.precision == 0 ? 8 : 4;
    std::vector<char> raw((size_t)h->d.nc * rs);
    for (int n = 0; n < h->d.nc; ++n) {
        if (rs == 8) ((double*)raw.data())[n] = in[n];
        else ((float*)raw.data())[n] = (float)in[n];
    }
    char* base = (char*)h->d.cyto[h->d.ccur] + ((size_t)site * h->d.CS + species) * h->d.nc * rs;
    ck(cudaMemcpy(base, raw.data(), raw.size(), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_get_draws(casim_h h, int32_t site, uint64_t* out) {
    GUARD(h)
    cb_site_scalars q;
    get_scalars(h, site, q);
    *out = q.draws;
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_get_release(casim_h h, int32_t site, double* out) {
    GUARD(h)
    cb_site_scalars q;
    get_scalars(h, site, q);
    *out = q.release;
    return CASIM_OK;
    END_GUARD(h)
}

casim_status casim_b200_check_finite(casim_h h, int32_t* bad_site) {
    GUARD(h)
    if (bad_site) *bad_site = -1;
    ck(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    const cb_model& m = h->d.m;
    size_t rs = h->d.precision == 0 ? 8 : 4;
    std::vector<cb_site> st(h->d.S);
    ck(cudaMemcpy(st.data(), h->d.sites, sizeof(cb_site) * h->d.S, cudaMemcpyDeviceToHost), "cudaMemcpy");
    std::vector<char> raw;
    for (int s = 0; s < h->d.S; ++s) {
        raw.resize((size_t)st[s].npad * m.F * rs);
        const char* base = (const char*)h->d.fields[h->d.cur] + (size_t)st[s].node_base * m.F * rs;
        ck(cudaMemcpy(raw.data(), base, raw.size(), cudaMemcpyDeviceToHost), "cudaMemcpy");
        // cleft fields, then (RD3D) the site's cytosol grid
        if (m.cyto_type == CB_CYTO_RD3D && h->d.nc > 0) {
            const size_t nf = raw.size(), nci = (size_t)h->d.CS * h->d.nc * rs;
            raw.resize(nf + nci);
            const char* cb = (const char*)h->d.cyto[h->d.ccur] + (size_t)s * nci;
            ck(cudaMemcpy(raw.data() + nf, cb, nci, cudaMemcpyDeviceToHost), "cudaMemcpy");
        }
        size_t n = raw.size() / rs;
        bool bad = false;
        for (size_t k = 0; k < n && !bad; ++k) {
            double v = rs == 8 ? ((double*)raw.data())[k] : (double)((float*)raw.data())[k];
            bad = !std::isfinite(v);
        }
        if (!bad) {
            // FP64 pool scalars: jSR, cytosol pool, release accumulator
            cb_site_scalars q;
            ck(cudaMemcpy(&q, h->d.sc + s, sizeof(q), cudaMemcpyDeviceToHost), "cudaMemcpy");
            for (int j = 0; j < m.n_ions; ++j) bad = bad || !std::isfinite(q.jsr[j]) || !std::isfinite(q.c_ions[j]);
            bad = bad || !std::isfinite(q.release);
        }
        if (bad) {
            if (bad_site) *bad_site = s;
            return set_err(h, CASIM_ENONFINITE, "non-finite value in site " + std::to_string(s));
        }
    }
    return CASIM_OK;
    END_GUARD(h)
}

}  // extern "C"

namespace {
__global__ void k_debug_rng(cbrng::State g, long long n, double* out) {
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (long long k = 0; k < n; ++k) out[k] = cbrng::u01d(g);
}
}  // namespace

extern "C" casim_status casim_b200_debug_rng(const uint32_t seed[6], int64_t n, double* out) {
    if (!seed || !out || n < 0) return set_err(nullptr, CASIM_EINVAL, "bad argument");
    {
        // the rules of RngStream's CheckSeed (CaSim/rngstream.cpp:200-234): a seed word at or
        // above its modulus, or three zero words in one component, is rejected
        const uint64_t s6[6] = {seed[0], seed[1], seed[2], seed[3], seed[4], seed[5]};
        if (!cbrng::seed_ok(s6)) return set_err(nullptr, CASIM_EINVAL, "debug_rng: not a valid MRG32k3a seed");
    }
    try {
        cbrng::State g;
        for (int i = 0; i < 6; ++i) g.s[i] = seed[i];
        double* d = nullptr;
        ck(cudaMalloc(&d, sizeof(double) * (size_t)std::max<int64_t>(n, 1)), "cudaMalloc");
        k_debug_rng<<<1, 1>>>(g, n, d);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(out, d, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost);
        cudaFree(d);
        ck(e, "debug_rng");
    } catch (const cuda_fail& e) {
        return set_err(nullptr, CASIM_ECUDA, e.what());
    }
    return CASIM_OK;
}
