// Device state of one batch of release sites and the launch entry points of
// the two stepping paths. Internal to libcasim_b200.so.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "model.h"

struct cb_dev {
    cb_model m;
    int S = 0;              // sites
    int precision = 0;      // 0 = FP64 fields, 1 = FP32 fields
    int min_cluster = 1;    // smallest thread-block cluster per site on the resident path
    int light_rows = 0;     // start from the lighter row partition of the edge and plane-0 blocks
    int NS = 0;             // mouth species per RyR: ions + pairs + free buffers
    int max_nodes = 0;      // largest padded node count of a site
    int max_ch = 0;
    int max_terms = 0;      // largest efflux term count of a site
    long long total_nodes = 0;  // sum of npad
    long long total_ch = 0;
    cb_site* sites = nullptr;         // [S]
    cb_site_scalars* sc = nullptr;    // [S]
    void* fields[2] = {nullptr, nullptr};  // ping-pong field storage (R = double or float)
    int cur = 0;                      // which of fields[] holds the current state
    void* curgrid = nullptr;          // RyR current per node (R), n_ions blocks per site
    int* ch_node = nullptr;           // local node index (x fastest) per RyR
    int* ch_owner = nullptr;          // 1 if the RyR is the highest-index one at its node
    int* ch_state = nullptr;          // open (1) / closed (0)
    int* ch_micro = nullptr;          // SingleSiteMWC: micro-state 0..59 per RyR (else unused)
    const struct cb_mwc_tab* mwc = nullptr;  // SingleSiteMWC: adjacency and initial distribution
    double* mouth = nullptr;          // [(ch)*NS + species]
    // RD3D cytosol
    int nc = 0;                       // nodes per site cytosol (mc^3)
    int CS = 0;                       // cytosol species: ions + cytosol pairs
    void* cyto[2] = {nullptr, nullptr};  // ping-pong, [site][species][node]
    int ccur = 0;
    double* cin = nullptr;            // efflux deposit into layer 0, [site][species][mc*mc]
    int* rim_cnode = nullptr;         // cytosol layer-0 node (i + mc*j) per rim entry
    int* dep_ptr = nullptr;           // per site (mc*mc + 1) CSR offsets into dep_term
    int* dep_term = nullptr;          // efflux term indices, oracle order
    // spline tables
    double* spx[2] = {nullptr, nullptr};
    double* spc[2] = {nullptr, nullptr};
    // bookkeeping
    int* err_flag = nullptr;          // device-side error word
    // resident path: work queue (sites by decreasing size), its counter and
    // the MRG32k3a jump table A^(2^k), k < 64; allocated on first use
    int* rs_order = nullptr;
    int* rs_counter = nullptr;
    unsigned long long* rs_pow2 = nullptr;
    struct cb_rs_plan* rs_plan = nullptr;  // host-side launch plan (resident.cu)
    // plain path, specialised stencils: (site, first column) of every cleft block;
    // st_nz = the cleft layers every site shares (0: mixed), -1 before the first step
    int2* st_tiles = nullptr;
    int st_ntiles = 0;
    int st_nz = -1;
    unsigned* st_chcol = nullptr;  // bit per cleft column (node_base + x + nx*y): holds a RyR
    // per-site gating models (plain path): gates[0] the batch's own, site_gate[s] the index
    cb_gate* gates = nullptr;
    int* site_gate = nullptr;
    int n_gates = 0;
    unsigned long long* pre_jump = nullptr;  // k_pre_r: MRG32k3a jumps A^(2l), l < 32
};

// plain path (plain.cu)
cudaError_t cb_plain_reset(cb_dev& d, cudaStream_t st);
cudaError_t cb_plain_init_opening(cb_dev& d, const int* d_first, int site_lo, int site_hi, cudaStream_t st);
cudaError_t cb_plain_update(cb_dev& d, cudaStream_t st, long long* launches);
cudaError_t cb_plain_step(cb_dev& d, long long n, cudaStream_t st, long long* launches);
// whether the plain path's specialised streaming kernels serve the batch's layout
bool cb_plain_streaming(cb_dev& d);
// whether the warp-parallel gating kernel (the one that serves per-site models) runs
bool cb_plain_gating_ready(cb_dev& d);
// one plain time step with ev[0..4] recorded around its four kernels
cudaError_t cb_plain_step_marked(cb_dev& d, cudaStream_t st, cudaEvent_t* ev);

// surrogate-driven gating without the RD step (plain.cu)
cudaError_t cb_sg_features(cb_dev& d, int max_ch, int ld, float* X, cudaStream_t st);
cudaError_t cb_sg_mouth(cb_dev& d, const float* Y, int ld, double ca_ref, cudaStream_t st);
cudaError_t cb_sg_steps(cb_dev& d, long long n, cudaStream_t st);
// residual check of the network's mouth Ca (Y) against the mouth Ca of the last RD Update at
// the open RyRs: the largest per-site relative error and the fraction of sites above tol
// (synchronises)
cudaError_t cb_sg_residual(const cb_dev& d, const float* Y, int ld, double ca_ref, double tol, unsigned long long* scratch,
                           double* worst, double* fail_fraction, cudaStream_t st);
cudaError_t cb_sg_steps_warp(cb_dev& d, long long n, cudaStream_t st, bool* used);  // sg_gate.cu
// analysis.cu: open-RyR trace sample j of every site; the release-event analysis of n samples
cudaError_t cb_trace_record(const cb_dev& d, uint16_t* trace, long long max_samples, long long j, cudaStream_t st);
cudaError_t cb_cre_analysis(const cb_dev& d, const uint16_t* trace, long long max_samples, long long n, double ts, double hd,
                            long long nh, int nadir, double* per_site, int* cls, int* h_all, int* h_q, int* h_b, int* h_s,
                            int* counts, cudaStream_t st);
// the surrogate network (surrogate.cu)
struct casim_surrogate_s;
cudaError_t cb_sg_net_prepare(struct casim_surrogate_s* net, int batch);
cudaError_t cb_sg_net_forward(struct casim_surrogate_s* net, const float* x, int batch, cudaStream_t st, const float** y, int* ld);
cudaError_t cb_sg_net_error(struct casim_surrogate_s* net);
const void* cb_sg_net_output(struct casim_surrogate_s* net);  // changes when its buffers are reallocated

// resident path (resident.cu)
bool cb_resident_fits(const cb_dev& d, int* threads, size_t* smem, std::string* why);
cudaError_t cb_resident_step(cb_dev& d, long long n, cudaStream_t st, long long* launches);
// measured choice of block and cluster size per class (state unchanged); a description of
// the choices into *report
cudaError_t cb_resident_autotune(cb_dev& d, long long steps, cudaStream_t st, std::string* report);
void cb_resident_free(cb_dev& d);
// MRG32k3a jump table d.rs_pow2: A^(2^k), k < 64, then the ring-refill jump (resident.cu)
cudaError_t cb_ensure_pow2(cb_dev& d);
