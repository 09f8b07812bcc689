// Pool ODEs of one site, shared by the one-thread-per-site kernels of the
// plain path and the surrogate-driven gating.
#pragma once
#include "model.h"

// Cytosol pool ODE of one site (CaSim/CytosolPool.cpp:217-288).
__device__ __forceinline__ void cb_pool_step(const cb_model& m, cb_site_scalars& q, double dt) {
    double evo_i[CB_MAX_IONS], evo_p[CB_MAX_CPAIRS];
    int ipd = 0, is = 0;
    for (int j = 0; j < m.n_ions; ++j) {
        double react = 0;
        for (int p = 0; p < m.c_n_pairs; ++p) {
            if (m.c_pair_ion[p] != j) continue;
            double R1 = m.c_koff[p] * q.c_pairs[p] - m.c_kon[p] * q.c_ions[j] * q.c_free[m.c_pair_buf[p]];
            evo_p[p] = -R1;
            react += R1;
            if (m.c_in_dyad[p]) {
                evo_p[p] += q.efflux[m.n_ions + ipd];
                ++ipd;
            }
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
    for (int j = 0; j < m.n_ions; ++j) {
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

// jSR pool ODE of one site (CaSim/SRPool.cpp:70-89) with the site's own beta.
__device__ __forceinline__ void cb_jsr_step(const cb_model& m, cb_site_scalars& q, double dt) {
    if (m.jsr_const) return;
    double beta = 1;
    for (int j = 0; j < m.n_ions; ++j)
        beta += m.nCQ[j] * m.K_CQ[j] * m.CQ / ((m.K_CQ[j] + q.jsr[j]) * (m.K_CQ[j] + q.jsr[j]));
    for (int i = 0; i < m.n_ions; ++i) {
        double Iref = 1 / m.tau_refill[i] * (q.nsr[i] - q.jsr[i]);
        q.jsr_new[i] = q.jsr[i] + dt / beta * (Iref - q.IjSR[i] / m.V_jsr);
    }
    if (m.ca_idx >= 0) q.release += q.IjSR[m.ca_idx] * dt;
}

