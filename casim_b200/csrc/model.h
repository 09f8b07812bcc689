// Resolved release-site model: species, kinetics, gating law, pools and the
// derived stencil constants. Plain-old-data so it can be passed by value to
// kernels (it lands in the constant bank) and copied to the host unchanged.
#pragma once
#include <stdint.h>

#define CB_MAX_IONS 4
#define CB_MAX_BUF 8
#define CB_MAX_PAIRS 12
#define CB_MAX_CBUF 12
#define CB_MAX_CPAIRS 16
#define CB_MAX_SPECIES (CB_MAX_IONS + CB_MAX_PAIRS)
#define CB_MAX_CSPECIES (CB_MAX_IONS + CB_MAX_CPAIRS)
#define CB_MAX_CHPAR 24
#define CB_MAX_CHANNELS 1024

// gating laws (CaSim/PassiveIonChannel.cpp:10-26)
enum { CB_SHEEP_CANNELL = 0, CB_TWO_STATE_MWC = 1, CB_TWO_STATE_AHTG = 2, CB_TWO_STATE_SPLINE = 3, CB_SINGLE_SITE_MWC = 4 };
enum { CB_CYTO_POOL = 0, CB_CYTO_RD3D = 1 };

// A two-state RyR gating model of some sites of a batch (per-site gating): the rate
// law and its parameters as in cb_model, and its spline tables (device pointers).
#define CB_MAX_GATES 8
struct cb_gate {
    int ch_model;
    double ch_par[24];
    int sp_n[2];
    const double* spx[2];
    const double* spc[2];
};

struct cb_model {
    int dim;  // 2 or 3
    double dx, dy, dz, z, R, dt, voltage;
    int n_ions, n_buf, n_pairs;
    int F;  // stored species: n_ions + n_pairs
    double D_ion[CB_MAX_IONS], Cb[CB_MAX_IONS], extracell[CB_MAX_IONS];
    int has_sl[CB_MAX_IONS];
    double N1[CB_MAX_IONS], K1[CB_MAX_IONS], N2[CB_MAX_IONS], K2[CB_MAX_IONS];
    double Ctot[CB_MAX_BUF];
    int pair_ion[CB_MAX_PAIRS], pair_buf[CB_MAX_PAIRS];
    double D_pair[CB_MAX_PAIRS], kon[CB_MAX_PAIRS], koff[CB_MAX_PAIRS], pair_init[CB_MAX_PAIRS];
    // RyR gating and conductance
    int ch_model;
    double ch_par[CB_MAX_CHPAR];
    double g[CB_MAX_IONS];
    int ca_idx, mg_idx;
    int sp_n[2];  // spline knots (tables live in device memory)
    // jSR (CaSim/SRPool.cpp)
    int jsr_const;
    double CQ, V_jsr;
    double nCQ[CB_MAX_IONS], K_CQ[CB_MAX_IONS], tau_refill[CB_MAX_IONS], jsr0[CB_MAX_IONS], nsr[CB_MAX_IONS];
    // cytosol
    int cyto_type;
    double c_bg[CB_MAX_IONS], c_onetau_ion[CB_MAX_IONS];
    int c_n_buf, c_n_pairs;
    double c_Ctot[CB_MAX_CBUF];
    int c_pair_ion[CB_MAX_CPAIRS], c_pair_buf[CB_MAX_CPAIRS];
    double c_kon[CB_MAX_CPAIRS], c_koff[CB_MAX_CPAIRS], c_init[CB_MAX_CPAIRS], c_onetau_pair[CB_MAX_CPAIRS];
    double c_D_pair[CB_MAX_CPAIRS];
    int c_in_dyad[CB_MAX_CPAIRS];
    int c_dyad_pair[CB_MAX_CPAIRS];   // dyad pair of an in-dyad cytosol pair, else -1
    int dyad_c_pair[CB_MAX_PAIRS];    // cytosol pair of a dyad pair, else -1
    int c_serca[CB_MAX_IONS];
    double c_Jmax[CB_MAX_IONS], c_Kup[CB_MAX_IONS];
    int mc;     // RD3D nodes per edge
    double hc;  // RD3D spacing, nm
    // derived
    double grad_mult;  // 3/(4 pi R^3)
    double sx, sy;     // edge face factors of the efflux
    double V_elem;     // DyadSeries::GetElementVolume
    double inv_dx2, inv_dy2, inv_dz2, inv_hc2, inv_hc3;
};

// Per-site scalars that live in HBM between launches (always FP64).
struct cb_site_scalars {
    double jsr[CB_MAX_IONS];      // SRPool ions
    double jsr_new[CB_MAX_IONS];  // SRPool ions_new
    double IjSR[CB_MAX_IONS];
    double nsr[CB_MAX_IONS];
    double total[CB_MAX_IONS];    // total SR current of the last Update
    double efflux[CB_MAX_SPECIES];
    double c_ions[CB_MAX_IONS];   // cytosol pool
    double c_pairs[CB_MAX_CPAIRS];
    double c_free[CB_MAX_CBUF];
    double c_bnd[CB_MAX_PAIRS];   // cytosol values of the dyad pairs (buffers_boundary)
    double release;               // accumulated jSR Ca release
    double jsr0[CB_MAX_IONS];
    unsigned long long draws;
    unsigned int rng[6];
    int pad;
};

// Packed site table entry (device resident, read-only during stepping).
// Fields of site s: species f, node n (x fastest: n = x + nx*(y + ny*z)) at
// fields[node_base*F + f*npad + n]; RyR currents at cur[node_base*n_ions + j*npad + n].
struct cb_site {
    int nx, ny, nz;
    int n_ch;
    int npad;              // node count rounded up to a multiple of 32
    int ch_off;            // first RyR of the site in the channel arrays
    long long node_base;   // sum of npad over the preceding sites
    int rim_off;           // RD3D: first rim entry of the site (rim -> cytosol node table)
    int term_off;          // RD3D: first deposit-list entry of the site
};
