// Device-side rate laws and small helpers shared by the plain and resident paths.
#pragma once
#include "model.h"

// Transition rate (per ms) of a two-state RyR in `state` given mouth Ca/Mg.
//   SheepCannell      CaSim/SheepCannell.cpp:12-18
//   TwoStatePoModel   CaSim/TwoStatePoModel.cpp:3-8 with Po from
//   TwoStateMWC       CaSim/TwoStateMWC.cpp:15-23
//   TwoStateaHTG      CaSim/TwoStateaHTG.cpp:18-29
//   TwoStateSpline    CaSim/TwoStateSplineModel.cpp:28-34 (natural cubic spline of the tables)
__device__ __forceinline__ double cb_spline(const double* __restrict__ x, const double* __restrict__ c, int n, double v) {
    if (v <= x[0]) return c[0] + c[1] * (v - x[0]);
    if (v >= x[n - 1]) return c[4 * (n - 1)] + c[4 * (n - 1) + 1] * (v - x[n - 1]);
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (x[mid] <= v) lo = mid;
        else hi = mid;
    }
    double h = v - x[lo];
    const double* q = c + 4 * lo;
    return ((q[3] * h + q[2]) * h + q[1]) * h + q[0];
}

// x^e for the rate laws: exponents that are multiples of 1/2 up to 8 (the power laws of the
// shipped configs, 2.5 and 0.5) by repeated squaring and one sqrt, x^(n + 1/2) = x^n sqrt(x);
// any other exponent by pow. Both agree with pow to a few ulp, far below what could move a
// gating decision u < rate*dt.
__device__ __forceinline__ double cb_pow(double x, double e) {
    const double e2 = 2.0 * e;
    if (e2 >= 0.0 && e2 <= 16.0 && e2 == (double)(int)e2 && x >= 0.0) {
        int n = (int)e2 >> 1;
        double r = (int)e2 & 1 ? sqrt(x) : 1.0, b = x;
        while (n) {
            if (n & 1) r *= b;
            b *= b;
            n >>= 1;
        }
        return r;
    }
    return pow(x, e);
}

// MODEL >= 0 fixes the rate law at compile time (kernels instantiated per model);
// the default reads it from m.ch_model.
// G: cb_model, or a cb_gate of a per-site gating model (the same ch_model, ch_par and
// sp_n members).
template <int MODEL = -1, typename G = cb_model>
__device__ __forceinline__ double cb_rate(const G& m, const double* __restrict__ spx0, const double* __restrict__ spc0,
                                          const double* __restrict__ spx1, const double* __restrict__ spc1, int state, double ca,
                                          double mg) {
    const double* p = m.ch_par;
    switch (MODEL >= 0 ? MODEL : m.ch_model) {
    case CB_SHEEP_CANNELL: {
        // one power per lane whatever the state (no divergence between open and
        // closed channels); x^0 == 1 exactly, so a zero exponent skips it
        const double k0 = state ? p[3] : p[0];
        const double ex = state ? p[4] : p[1];
        const double k = k0 * (ex == 0.0 ? 1.0 : cb_pow(ca * 1e-3, ex));
        return (state ? k : (p[2] < k ? p[2] : k)) * 1e-3;
    }
    case CB_TWO_STATE_MWC: {
        double kclose = p[6];
        if (state) return kclose;
        double inac = p[5] * p[5] / (p[5] * p[5] + mg * mg);
        double a = ca + p[1] * p[0] * (1 + mg / (p[2] * p[3]));
        double b = p[0] * (ca + p[1] * (1 + mg / p[3]));
        double a2 = a * a, b2 = b * b;
        double open = a2 * a2;
        double close = p[4] * (b2 * b2);
        double P = inac * open / (open + close);
        return kclose * P / (1 - P);
    }
    case CB_TWO_STATE_AHTG: {
        double fCa = p[0], KCa = p[1], fMg = p[2], KMg = p[3], KO0 = p[4], KMgI = p[5], KCL = p[6], KI = p[7], KOL = p[8];
        double kclose = p[9];
        if (state) return kclose;
        double mult = KMgI * KMgI / (KMgI * KMgI + mg * mg);
        double up = (KCL * KI * (pow(ca, 4) * pow(fMg, 4) * pow(fCa, 4) * pow(KMg, 4) * KO0 + pow(ca * fMg * KMg + fCa * (mg + fMg * KMg) * KCa, 4) * KOL));
        double down = (4 * pow(ca, 3) * pow(fMg, 3) * fCa * pow(KMg, 3) * KCa * KCL * KI * (mg + fMg * KMg + fMg * pow(fCa, 3) * (mg + KMg) * KO0) * KOL +
                       6 * pow(ca, 2) * pow(fMg, 2) * pow(fCa, 2) * pow(KMg, 2) * pow(KCa, 2) * KCL * KI * (pow(mg + fMg * KMg, 2) + pow(fMg, 2) * pow(fCa, 2) * pow(mg + KMg, 2) * KO0) * KOL +
                       4 * ca * fMg * pow(fCa, 3) * KMg * pow(KCa, 3) * KCL * KI * (pow(mg + fMg * KMg, 3) + pow(fMg, 3) * fCa * pow(mg + KMg, 3) * KO0) * KOL +
                       pow(fCa, 4) * pow(KCa, 4) * KCL * KI * (pow(mg + fMg * KMg, 4) + pow(fMg, 4) * pow(mg + KMg, 4) * KO0) * KOL +
                       pow(ca, 4) * pow(fMg, 4) * pow(KMg, 4) * (KCL * KI * KOL + pow(fCa, 4) * KO0 * (1 + KI + KCL * KI + KCL * KI * KOL)));
        double P = mult * up / down;
        return kclose * P / (1 - P);
    }
    case CB_TWO_STATE_SPLINE:
        return state ? cb_spline(spx1, spc1, m.sp_n[1], ca) : cb_spline(spx0, spc0, m.sp_n[0], ca);
    default:
        return 0.0;
    }
}

// Rim enumeration of a cleft (x, y) plane: x = 0 column, x = nx-1 column,
// then the y = 0 and y = ny-1 rows without their corners.
__host__ __device__ __forceinline__ int cb_rim_count(int nx, int ny) { return 2 * ny + 2 * (nx - 2); }
__host__ __device__ __forceinline__ void cb_rim_xy(int r, int nx, int ny, int& x, int& y) {
    if (r < ny) {
        x = 0;
        y = r;
    } else if (r < 2 * ny) {
        x = nx - 1;
        y = r - ny;
    } else if (r < 2 * ny + nx - 2) {
        x = r - 2 * ny + 1;
        y = 0;
    } else {
        x = r - (2 * ny + nx - 2) + 1;
        y = ny - 1;
    }
}
// RD3D: the layer-0 cytosol node (i + mc*j) nearest below cleft node (x, y), clamped to
// the updated range; both grids are centred on each other. Host and device evaluate the
// same expressions to the same node: each step is one correctly rounded operation (the
// products by 0.5 of small integers are exact).
__host__ __device__ __forceinline__ int cb_rim_cnode(int x, int y, int nx, int ny, double dx, double dy, double hc, int mc) {
    const double px = (x - 0.5 * (nx - 1)) * dx, py = (y - 0.5 * (ny - 1)) * dy;
    int ci = (int)floor(px / hc + 0.5 * (mc - 1) + 0.5);
    int cj = (int)floor(py / hc + 0.5 * (mc - 1) + 0.5);
    ci = ci < 1 ? 1 : (ci > mc - 2 ? mc - 2 : ci);
    cj = cj < 1 ? 1 : (cj > mc - 2 ? mc - 2 : cj);
    return ci + mc * cj;
}
__host__ __device__ __forceinline__ int cb_rim_index(int x, int y, int nx, int ny) {
    if (x == 0) return y;
    if (x == nx - 1) return ny + y;
    if (y == 0) return 2 * ny + (x - 1);
    return 2 * ny + (nx - 2) + (x - 1);
}

// Efflux terms of one site in the reference's loop order
// (CaSim/DyadRD2DCPU.cpp:315-349, CaSim/DyadRDCPU.cpp:337-368):
// x-edges (x = 0 then x = nx-1) over y = 1..ny-2, then y-edges (y = 0 then
// y = ny-1) over x = 0..nx-1; z = 0..zmax-1 innermost.
__host__ __device__ __forceinline__ int cb_efflux_terms(int nx, int ny, int zmax) { return (2 * (ny - 2) + 2 * nx) * zmax; }
// returns the face factor selector (0: x-edge, 1: y-edge) and the three nodes (edge, 1 in, 2 in)
__host__ __device__ __forceinline__ int cb_efflux_term(int t, int nx, int ny, int zmax, int& x0, int& y0, int& x1, int& y1,
                                                      int& x2, int& y2, int& z) {
    z = t % zmax;
    int a = t / zmax;
    int nxe = ny - 2;
    if (a < 2 * nxe) {
        int e = a / nxe;
        int yy = 1 + a % nxe;
        x0 = e == 0 ? 0 : nx - 1;
        x1 = e == 0 ? 1 : nx - 2;
        x2 = e == 0 ? 2 : nx - 3;
        y0 = y1 = y2 = yy;
        return 0;
    }
    a -= 2 * nxe;
    int e = a / nx;
    int xx = a % nx;
    y0 = e == 0 ? 0 : ny - 1;
    y1 = e == 0 ? 1 : ny - 2;
    y2 = e == 0 ? 2 : ny - 3;
    x0 = x1 = x2 = xx;
    return 1;
}
