/*
 * CPU restatement of CaSim's release-site hot path: TEST INFRASTRUCTURE ONLY.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it,
 * and only as the checker (or as the timed CPU port), never as the product.
 *
 * Every site is an independent dyad with its own grid extents, RyR positions,
 * MRG32k3a stream and jSR/cytosol state. One step follows the reference loop
 * body CaSim/ParallelHybridSolver.cpp:421-429 followed by Update()
 * (CaSim/ParallelHybridSolver.cpp:159-175).
 */
#ifndef CASIM_ORACLE_H
#define CASIM_ORACLE_H
#include <stdint.h>

#define OR_MAX_IONS 4
#define OR_MAX_BUF 8
#define OR_MAX_PAIRS 16
#define OR_MAX_CBUF 12
#define OR_MAX_CPAIRS 24
#define OR_MAX_CHPAR 32
#define OR_MAX_SPLINE 1024

/* gating models (CaSim/PassiveIonChannel.cpp:10-26) */
enum { OR_SHEEP_CANNELL = 0, OR_TWO_STATE_MWC = 1, OR_TWO_STATE_AHTG = 2, OR_TWO_STATE_SPLINE = 3,
       OR_FOUR_STATE_MWC = 4, OR_SINGLE_SITE_MWC = 5 };
/* cytosol models */
enum { OR_CYTO_POOL = 0, OR_CYTO_RD3D = 1 };

typedef struct {
    int dim;                       /* 2: DyadRD2DCPU, 3: DyadRDCPU */
    double dx, dy, dz, z, R, dt, voltage;
    int n_ions;
    double D_ion[OR_MAX_IONS], Cb_ion[OR_MAX_IONS], extracell[OR_MAX_IONS];
    int has_sl[OR_MAX_IONS];
    double N1[OR_MAX_IONS], K1[OR_MAX_IONS], N2[OR_MAX_IONS], K2[OR_MAX_IONS];
    int n_buf;
    double Ctot[OR_MAX_BUF];
    int binds[OR_MAX_BUF * OR_MAX_IONS]; /* binds[b + i*n_buf] */
    int n_pairs;
    int pair_ion[OR_MAX_PAIRS], pair_buf[OR_MAX_PAIRS];
    double D_pair[OR_MAX_PAIRS], kon[OR_MAX_PAIRS], koff[OR_MAX_PAIRS], pair_init[OR_MAX_PAIRS];
    /* RyR */
    int ch_model;
    double ch_par[OR_MAX_CHPAR];
    double g[OR_MAX_IONS];
    int ca_idx, mg_idx;
    /* spline tables: per-interval cubic coefficients y = a + b t + c t^2 + d t^3, t = x - x_i */
    int sp_n[2];
    double sp_x[2][OR_MAX_SPLINE], sp_c[2][OR_MAX_SPLINE][4];
    double sp_left[2][3], sp_right[2][3]; /* extrapolation: value, slope, curvature/2 at ends */
    /* jSR (CaSim/SRPool.cpp) */
    int jsr_const;
    double CQ, V_jsr;
    int nCQ[OR_MAX_IONS];
    double K_CQ[OR_MAX_IONS], tau_refill[OR_MAX_IONS], jsr0[OR_MAX_IONS];
    double nsr[OR_MAX_IONS];
    /* cytosol */
    int cyto_type;
    /* pool (CaSim/CytosolPool.cpp): ions are the dyad ions */
    double c_bg[OR_MAX_IONS], c_onetau_ion[OR_MAX_IONS];
    int c_n_buf;
    double c_Ctot[OR_MAX_CBUF];
    int c_binds[OR_MAX_CBUF * OR_MAX_IONS];
    int c_n_pairs;
    double c_kon[OR_MAX_CPAIRS], c_koff[OR_MAX_CPAIRS], c_init[OR_MAX_CPAIRS], c_onetau_pair[OR_MAX_CPAIRS];
    double c_D_pair[OR_MAX_CPAIRS];
    int c_in_dyad[OR_MAX_CPAIRS];
    int c_dyad_pair[OR_MAX_CPAIRS]; /* dyad pair index for in-dyad cytosol pairs, else -1 */
    int c_serca[OR_MAX_IONS];
    double c_Jmax[OR_MAX_IONS], c_Kup[OR_MAX_IONS];
    /* rd3d cytosol: cube of mc^3 nodes, spacing hc (nm) */
    int mc;
    double hc;
} or_model;

typedef struct or_sim or_sim;

/* sites: nx, ny, nz per site; n_ch per site; ch_xyz: 3 ints per channel (grid
 * indices), packed site after site; seeds: 6 per site; jsr_init: n_ions per
 * site or NULL (model jsr0). */
or_sim* or_create(const or_model* m, int n_sites, const int* nx, const int* ny, const int* nz,
                  const int* n_ch, const int* ch_xyz, const uint32_t* seeds, const double* jsr_init);
void or_destroy(or_sim* s);
void or_reset(or_sim* s);
void or_init_opening(or_sim* s, int site, int channel);
void or_update(or_sim* s);
void or_start(or_sim* s, const int* first_channel);
void or_step(or_sim* s, long n_steps, int n_threads);

/* site-local node index used by the getters: reference order, y fastest in 2D
 * (y + ny*x) and z fastest in 3D (z + nz*(y + ny*x)). */
long or_site_nodes(const or_sim* s, int site);
/* species: 0..n_ions-1 ions, then pairs, then free buffers */
void or_get_field(const or_sim* s, int site, int species, double* out);
void or_get_mouth(const or_sim* s, int site, int species, double* out);
void or_get_states(const or_sim* s, int site, int* out);
/* SingleSiteMWC: micro-states 0..59 (45-59 open) */
void or_get_micro(const or_sim* s, int site, int* out);
void or_get_jsr(const or_sim* s, int site, double* out);           /* n_ions */
void or_get_total_current(const or_sim* s, int site, double* out); /* n_ions */
void or_get_efflux(const or_sim* s, int site, double* out);        /* n_ions + n_pairs */
void or_get_cyto(const or_sim* s, int site, double* out);          /* pool: n_ions + c_n_pairs */
long or_get_cyto_field(const or_sim* s, int site, int species, double* out); /* rd3d */
uint64_t or_draws(const or_sim* s, int site);                       /* runif() draws consumed */
double or_release(const or_sim* s, int site);                       /* accumulated Ca release */

/* MRG32k3a (L'Ecuyer 1999 / RngStreams 2002) helpers for tests */
void or_mrg_u01d(const uint32_t seed[6], long n, double* out);
void or_mrg_jump(const uint32_t seed[6], int log2_steps, long mult, uint32_t out[6]);
/* one quasi-stationary Gillespie scenario (CaSim/QuasyStationaryReleaseSite.cpp:89-133) */
long or_qs_run(const or_model* m, int n_ch, const double* added, double bg, double mg, double max_time, uint32_t* seed6,
               int first, long max_events, double* ev_t, int* ev_c, int* ev_s, uint64_t* draws);
#endif
