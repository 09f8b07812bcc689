// 60-state single-site MWC RyR gating (CaSim/SingleSiteMWC.cpp, the Q-matrix model of
// CaSim/QMatrixModel.cpp). Micro-state s = idx + 15 * block: idx enumerates the
// (i Ca, j Mg) occupancies of the four sites (i + j <= 4, idx = 15 - (6-j)(5-j)/2 + i,
// CaSim/SingleSiteMWC.cpp:100-101). Block 0 is closed, block 1 closed with Mg on the
// inhibition site, block 2 the open conformation with Mg on it (still closed), block 3
// open: states 0-44 are closed and 45-59 open (:39-45).
//
// Gating per time step (CaSim/DyadChannels.cpp:118-119 with QMatrixModel::GetRate and
// MakeTransition, CaSim/QMatrixModel.cpp:20-36): the escape rate of the current state is
// the sum of its row over the adjacency list (in the list's order), a draw below rate * dt
// makes a transition, and a second draw picks the destination by the cumulative row.
#pragma once
#include <math.h>

#include "model.h"

constexpr int CB_MWC_N = 60;       // micro-states
constexpr int CB_MWC_OPEN = 45;    // first open micro-state
constexpr int CB_MWC_MAXADJ = 6;   // at most 4 binding moves and 2 conformational ones

// parameter slots in cb_model::ch_par (CaSim/SingleSiteMWC.cpp:5-37 reads them by name)
enum {
    MWC_fCa4I, MWC_fCa, MWC_KCa, MWC_alphaCa, MWC_konCa, MWC_fMg, MWC_KMg, MWC_konMg, MWC_alphaMg, MWC_alphaMgI,
    MWC_KO0, MWC_alphakco, MWC_alphakcoI, MWC_kco, MWC_KMgI, MWC_konMgI, MWC_fICa, MWC_fIMg, MWC_gMg, MWC_gCa, MWC_NPAR
};

// adjacency lists in the reference's order and the stationary distribution of the full
// Q at the initial mouth values (for InitOpening), built on the host
struct cb_mwc_tab {
    unsigned char nadj[CB_MWC_N];
    unsigned char adj[CB_MWC_N][CB_MWC_MAXADJ];
    double p_init[CB_MWC_N];
};

// (i, j, block) of micro-state s, decoded as CaSim/SingleSiteMWC.cpp:156-168 does
__host__ __device__ inline void cb_mwc_ij(int s, int& i, int& j, int& b) {
    b = s / 15;
    int r = s - 15 * b;
    for (j = 0; j <= 4; ++j) {
        if (r - (5 - j) < 0) {
            i = r;
            return;
        }
        r -= 5 - j;
    }
    i = 0;
    j = 4;
}

// Q[s][d] for d adjacent to s, the entries CaSim/SingleSiteMWC.cpp:100-151 (SetRow) sets,
// each with the reference's operand order
__host__ __device__ inline double cb_mwc_q(const double* P, int s, int d, double ca, double mg) {
    int i, j, b;
    cb_mwc_ij(s, i, j, b);
    const double fCa4I = P[MWC_fCa4I], fCa = P[MWC_fCa], konCa = P[MWC_konCa], alphaCa = P[MWC_alphaCa];
    const double fMg = P[MWC_fMg], konMg = P[MWC_konMg], alphaMg = P[MWC_alphaMg], alphaMgI = P[MWC_alphaMgI];
    const double kco = P[MWC_kco], alphakco = P[MWC_alphakco], alphakcoI = P[MWC_alphakcoI];
    const double konMgI = P[MWC_konMgI], fICa = P[MWC_fICa], fIMg = P[MWC_fIMg], gMg = P[MWC_gMg], gCa = P[MWC_gCa];
    const double koffCa = P[MWC_KCa] * konCa, koffMg = konMg * P[MWC_KMg], koc = P[MWC_KO0] * kco;
    const double koffMgI = P[MWC_KMgI] * P[MWC_KMgI] * konMgI;
    const int c = s - 15 * b, db = d / 15, c2 = d - 15 * db;
    if (db == b) {
        const int del = c2 - c;
        if (del == 1) {  // Ca binding
            const double k = (4 - i - j) * konCa * ca;
            if (b == 0 || b == 1) return k;
            if (b == 3) return k / pow(fCa, alphaCa);
            return i == 3 ? k / pow(fCa4I, alphaCa) : k / pow(fICa, alphaCa);
        }
        if (del == -1) {  // Ca unbinding
            if (b == 0) return i * koffCa;
            if (b == 3) return i * koffCa * pow(fCa, 1 - alphaCa);
            if (b == 1) return i * koffCa * gCa;
            return i == 4 ? i * koffCa * pow(fCa4I, 1 - alphaCa) * gCa : i * koffCa * pow(fICa, 1 - alphaCa) * gCa;
        }
        if (del > 0) {  // Mg binding (j + 1)
            const double k = (4 - i - j) * konMg * mg;
            if (b == 0) return k;
            if (b == 3) return k / pow(fMg, alphaMg);
            if (b == 1) return k / pow(gMg, alphaMgI);
            return k / (pow(fIMg, alphaMg) * pow(gMg, alphaMgI));
        }
        // Mg unbinding (j - 1)
        if (b == 0) return j * koffMg;
        if (b == 3) return j * koffMg * pow(fMg, 1 - alphaMg);
        if (b == 1) return j * koffMg * pow(gMg, 1 - alphaMgI);
        return j * koffMg * pow(fIMg, 1 - alphaMg) * pow(gMg, 1 - alphaMgI);
    }
    const double ff = pow(fCa, i) * pow(fMg, j);
    const double fIco = i == 4 ? pow(fICa, 3) * fCa4I : pow(fICa, i) * pow(fIMg, j);
    if (b == 0 && db == 1) return konMgI * pow(mg, 2) / pow(gMg, j);
    if (b == 1 && db == 0) return koffMgI * pow(gCa, i);
    if (b == 3 && db == 2) return konMgI * pow(mg, 2) / pow(fIMg / fMg * gMg, j);
    if (b == 2 && db == 3) return i == 4 ? koffMgI * pow(fICa / fCa * gCa, 3) * fCa4I / fCa : koffMgI * pow(fICa / fCa * gCa, i);
    if (b == 0 && db == 3) return kco / pow(ff, alphakco);
    if (b == 3 && db == 0) return koc * pow(ff, 1 - alphakco);
    if (b == 1 && db == 2) return kco / pow(fIco, alphakcoI);
    return koc * pow(fIco, 1 - alphakcoI);  // b == 2, db == 1
}

// escape rate of s (CaSim/SingleSiteMWC.cpp:162-165)
__host__ __device__ inline double cb_mwc_exit(const double* P, const cb_mwc_tab& t, int s, double ca, double mg) {
    double r = 0;
    for (int k = 0; k < t.nadj[s]; ++k) r += cb_mwc_q(P, s, t.adj[s][k], ca, mg);
    return r;
}

// destination of a transition out of s for the draw u (CaSim/QMatrixModel.cpp:26-35:
// the first neighbour whose cumulative rate over the escape rate reaches u; none keeps s)
__host__ __device__ inline int cb_mwc_next(const double* P, const cb_mwc_tab& t, int s, double ca, double mg, double exit_rate,
                                           double u) {
    double cum = 0;
    for (int k = 0; k < t.nadj[s]; ++k) {
        const int d = t.adj[s][k];
        cum += cb_mwc_q(P, s, d, ca, mg);
        if (cum / exit_rate >= u) return d;
    }
    return s;
}

// micro-state of a macro state (0 closed, 1 open) drawn from the stationary distribution
// (CaSim/QMatrixModel.cpp:38-58); none reached keeps s
__host__ __device__ inline int cb_mwc_pick(const cb_mwc_tab& t, int macro, double u, int s) {
    double total = 0;
    for (int i = 0; i < CB_MWC_N; ++i) total += ((i >= CB_MWC_OPEN) == (macro != 0)) * t.p_init[i];
    double c = 0;
    for (int i = 0; i < CB_MWC_N; ++i) {
        c += ((i >= CB_MWC_OPEN) == (macro != 0)) * t.p_init[i];
        if (c / total >= u) return i;
    }
    return s;
}

// host: the table for parameters P and initial mouth Ca / Mg
void cb_mwc_build(const double* P, double ca0, double mg0, cb_mwc_tab& t);
