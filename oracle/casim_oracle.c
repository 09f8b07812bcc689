/*
 * CPU restatement of CaSim's release-site hot path (TEST INFRASTRUCTURE ONLY:
 * the checker for the CUDA product path and the CPU "port" baseline; the
 * product never links or calls it).
 *
 * Restated from the reference (paths relative to the reference project):
 *   dyad RD step, 2D     CaSim/DyadRD2DCPU.cpp:394-490  (_EvolutionOp, _GetFreeBuffers, _UpdateEvo, RunRD)
 *   dyad RD step, 3D     CaSim/DyadRDCPU.cpp:404-506    (mirrored z faces :410-411, SL on top layer :480)
 *   mouth gather         CaSim/DyadRD2DCPU.cpp:361-380
 *   Dirichlet edges      CaSim/DyadRD2DCPU.cpp:274-303
 *   lateral efflux       CaSim/DyadRD2DCPU.cpp:305-350, CaSim/DyadRDCPU.cpp:322-369
 *   RyR currents         CaSim/DyadRD2DCPU.cpp:243-264 + CaSim/PassiveIonChannel.cpp:28-34
 *   gating MC            CaSim/DyadChannels.cpp:97-130, InitOpening :83-95
 *   rate laws            CaSim/SheepCannell.cpp:12-18, CaSim/TwoStatePoModel.cpp:3-8,
 *                        CaSim/TwoStateMWC.cpp:15-23, CaSim/TwoStateaHTG.cpp:18-29
 *   jSR pool             CaSim/SRPool.cpp:55-89
 *   cytosol pool         CaSim/CytosolPool.cpp:217-288
 *   RNG                  CaSim/rngstream.cpp:242-283 (MRG32k3a with incPrec = true, U01d)
 *
 * Deliberate differences from the reference (each one listed here):
 *   - each site draws from its own MRG32k3a stream (the reference hands one
 *     stream to each OpenMP thread); with one site per run they coincide;
 *   - SRPool's beta and NSR lookups use the site's own values (the reference
 *     indexes another site's jSR Ca for NumBatch > 1, CaSim/SRPool.cpp:75,80);
 *   - total SR current is cleared for every ion each Update (the reference
 *     clears ion 0 only, CaSim/DyadRD2DCPU.cpp:247; identical while the
 *     other ions' conductances are zero, as in every shipped config);
 *   - the RD3D cytosol (a 3D Cartesian cytosol coupled to the cleft rim) has
 *     no reference counterpart and follows this project's own definition:
 *     Update(n) sets the rim from the cytosol as it was at the start of step
 *     n (before the cytosol's own step n), and the efflux of Update(n) is
 *     deposited into cytosol layer 0 during step n + 1.
 * Arithmetic is written in the reference's operation order so that the FP64
 * restatement tracks the reference to rounding.
 */
#include "casim_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- MRG32k3a */
#define M1 4294967087ULL
#define M2 4294944443ULL
#define A12 1403580ULL
#define A13N 810728ULL
#define A21 527612ULL
#define A23N 1370589ULL

typedef struct {
    uint64_t s[6];
} mrg_t;

static double mrg_u01(mrg_t* g) {
    /* component 1: x_n = (a12 x_{n-2} - a13 x_{n-3}) mod m1 */
    /* each product is < 2^53; reduce them separately so nothing exceeds 2^64 */
    uint64_t p1 = ((A12 * g->s[1]) % M1 + M1 - (A13N * g->s[0]) % M1) % M1;
    g->s[0] = g->s[1];
    g->s[1] = g->s[2];
    g->s[2] = p1;
    /* component 2: y_n = (a21 y_{n-1} - a23 y_{n-3}) mod m2 */
    uint64_t p2 = ((A21 * g->s[5]) % M2 + M2 - (A23N * g->s[3]) % M2) % M2;
    g->s[3] = g->s[4];
    g->s[4] = g->s[5];
    g->s[5] = p2;
    const double norm = 1.0 / ((double)M1 + 1.0);
    double d1 = (double)p1, d2 = (double)p2;
    return (p1 > p2) ? (d1 - d2) * norm : (d1 - d2 + (double)M1) * norm;
}

/* RandU01 with incPrec = true: two U01 per draw (CaSim/rngstream.cpp:271-283) */
static double mrg_u01d(mrg_t* g) {
    const double fact = 5.9604644775390625e-8; /* 2^-24 */
    double u = mrg_u01(g);
    u += mrg_u01(g) * fact;
    return (u < 1.0) ? u : (u - 1.0);
}

/* 3x3 matrices mod m, used for jump-ahead; built from the recurrences above */
typedef struct {
    uint64_t a[3][3];
} mat3;

static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) { return (uint64_t)(((__uint128_t)a * b) % m); }

static mat3 matmul(mat3 x, mat3 y, uint64_t m) {
    mat3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            uint64_t acc = 0;
            for (int k = 0; k < 3; ++k) acc = (acc + mulmod(x.a[i][k], y.a[k][j], m)) % m;
            r.a[i][j] = acc;
        }
    return r;
}

static void matvec(mat3 x, uint64_t* v, uint64_t m) {
    uint64_t r[3];
    for (int i = 0; i < 3; ++i) {
        uint64_t acc = 0;
        for (int k = 0; k < 3; ++k) acc = (acc + mulmod(x.a[i][k], v[k], m)) % m;
        r[i] = acc;
    }
    v[0] = r[0];
    v[1] = r[1];
    v[2] = r[2];
}

static mat3 base1(void) {
    mat3 r = {{{0, 1, 0}, {0, 0, 1}, {M1 - A13N, A12, 0}}};
    return r;
}
static mat3 base2(void) {
    mat3 r = {{{0, 1, 0}, {0, 0, 1}, {M2 - A23N, 0, A21}}};
    return r;
}

/* advance a state by mult * 2^log2_steps steps */
void or_mrg_jump(const uint32_t seed[6], int log2_steps, long mult, uint32_t out[6]) {
    mat3 a1 = base1(), a2 = base2();
    for (int e = 0; e < log2_steps; ++e) {
        a1 = matmul(a1, a1, M1);
        a2 = matmul(a2, a2, M2);
    }
    uint64_t v1[3] = {seed[0], seed[1], seed[2]}, v2[3] = {seed[3], seed[4], seed[5]};
    for (long k = 0; k < mult; ++k) {
        matvec(a1, v1, M1);
        matvec(a2, v2, M2);
    }
    for (int i = 0; i < 3; ++i) {
        out[i] = (uint32_t)v1[i];
        out[i + 3] = (uint32_t)v2[i];
    }
}

void or_mrg_u01d(const uint32_t seed[6], long n, double* out) {
    mrg_t g;
    for (int i = 0; i < 6; ++i) g.s[i] = seed[i];
    for (long k = 0; k < n; ++k) out[k] = mrg_u01d(&g);
}

/* ---------------------------------------------------------------- state */
typedef struct {
    int nx, ny, nz;
    long N;
    int n_ch;
    int* cx; /* channel grid indices */
    int* cy;
    int* cz;
    double* ions;  /* [n_ions][N] */
    double* pairs; /* [n_pairs][N] */
    double* freeb; /* [n_buf][N] */
    double* evo_i;
    double* evo_p;
    double* cur;   /* [n_ions][N] currents grid */
    int* state;    /* [n_ch] open (1) / closed (0) */
    int* micro;    /* [n_ch] SingleSiteMWC micro-state 0..59 */
    double* mouth; /* [(n_ions + n_pairs + n_buf)][n_ch] */
    double efflux[OR_MAX_IONS + OR_MAX_PAIRS];
    double total[OR_MAX_IONS];
    /* jSR */
    double jsr[OR_MAX_IONS], jsr_new[OR_MAX_IONS], jsr0[OR_MAX_IONS], IjSR[OR_MAX_IONS], nsr[OR_MAX_IONS];
    double release;
    /* cytosol pool */
    double c_ions[OR_MAX_IONS], c_pairs[OR_MAX_CPAIRS], c_free[OR_MAX_CBUF], c_bnd[OR_MAX_PAIRS];
    /* rd3d cytosol */
    double* cf;      /* [(n_ions + c_n_pairs)][mc^3] */
    double* cf_prev; /* cytosol at the start of the current step (read by Update) */
    double* cf_evo;
    double* cf_in;   /* efflux deposit [(n_ions + c_n_pairs)][mc^3] */
    int* rim_map;    /* cytosol node for each cleft (x,y) rim position, [nx*ny] */
    mrg_t rng;
    uint64_t draws;
} site_t;

struct or_sim {
    or_model m;
    int S;
    site_t* site;
    /* SingleSiteMWC: adjacency lists and the stationary distribution at the initial ions */
    int mwc_nadj[60], mwc_adj[60][6];
    double mwc_p[60];
};

/* ------------------------------------------------ SingleSiteMWC (60 states)
 * CaSim/SingleSiteMWC.cpp with QMatrixModel (CaSim/QMatrixModel.cpp). Parameter slots
 * of ch_par: fCa4I fCa KCa alphaCa konCa fMg KMg konMg alphaMg alphaMgI KO0 alphakco
 * alphakcoI kco KMgI konmgI fICa fIMg gMg gCa. */
static int mwc_index(int i, int j) { return 15 - (6 - j) * (5 - j) / 2 + i; }

/* the entries of the four blocks' rows for occupancy (i Ca, j Mg), SetRow
 * (CaSim/SingleSiteMWC.cpp:100-151) */
static void mwc_set_row(const double* P, int i, double ca, int j, double mg, double Q[60][60]) {
    double fCa4I = P[0], fCa = P[1], KCa = P[2], alphaCa = P[3], konCa = P[4], fMg = P[5], KMg = P[6], konMg = P[7];
    double alphaMg = P[8], alphaMgI = P[9], KO0 = P[10], alphakco = P[11], alphakcoI = P[12], kco = P[13], KMgI = P[14];
    double konMgI = P[15], fICa = P[16], fIMg = P[17], gMg = P[18], gCa = P[19];
    double koffCa = KCa * konCa, koffMg = konMg * KMg, koc = KO0 * kco, koffMgI = KMgI * KMgI * konMgI;
    double ff = pow(fCa, i) * pow(fMg, j);
    double fIco = pow(fICa, i) * pow(fIMg, j);
    int c = mwc_index(i, j), c2;
    if (i + j < 4) {
        c2 = mwc_index(i + 1, j);
        Q[c][c2] = (4 - i - j) * konCa * ca;
        Q[c + 45][c2 + 45] = (4 - i - j) * konCa * ca / pow(fCa, alphaCa);
        Q[c + 15][c2 + 15] = (4 - i - j) * konCa * ca;
        Q[c + 30][c2 + 30] = (4 - i - j) * konCa * ca / pow(i == 3 ? fCa4I : fICa, alphaCa);
    }
    if (i > 0) {
        c2 = mwc_index(i - 1, j);
        Q[c][c2] = i * koffCa;
        Q[c + 45][c2 + 45] = i * koffCa * pow(fCa, 1 - alphaCa);
        Q[c + 15][c2 + 15] = i * koffCa * gCa;
        Q[c + 30][c2 + 30] = i * koffCa * pow(i == 4 ? fCa4I : fICa, 1 - alphaCa) * gCa;
    }
    if (i + j < 4) {
        c2 = mwc_index(i, j + 1);
        Q[c][c2] = (4 - i - j) * konMg * mg;
        Q[c + 45][c2 + 45] = (4 - i - j) * konMg * mg / pow(fMg, alphaMg);
        Q[c + 15][c2 + 15] = (4 - i - j) * konMg * mg / pow(gMg, alphaMgI);
        Q[c + 30][c2 + 30] = (4 - i - j) * konMg * mg / (pow(fIMg, alphaMg) * pow(gMg, alphaMgI));
    }
    if (j > 0) {
        c2 = mwc_index(i, j - 1);
        Q[c][c2] = j * koffMg;
        Q[c + 45][c2 + 45] = j * koffMg * pow(fMg, 1 - alphaMg);
        Q[c + 15][c2 + 15] = j * koffMg * pow(gMg, 1 - alphaMgI);
        Q[c + 30][c2 + 30] = j * koffMg * pow(fIMg, 1 - alphaMg) * pow(gMg, 1 - alphaMgI);
    }
    Q[c][c + 15] = konMgI * pow(mg, 2) / pow(gMg, j);
    Q[c + 15][c] = koffMgI * pow(gCa, i);
    Q[c + 45][c + 30] = konMgI * pow(mg, 2) / pow(fIMg / fMg * gMg, j);
    if (i == 4)
        Q[c + 30][c + 45] = koffMgI * pow(fICa / fCa * gCa, 3) * fCa4I / fCa;
    else
        Q[c + 30][c + 45] = koffMgI * pow(fICa / fCa * gCa, i);
    Q[c][c + 45] = kco / pow(ff, alphakco);
    Q[c + 45][c] = koc * pow(ff, 1 - alphakco);
    if (i == 4) fIco = pow(fICa, 3) * fCa4I;
    Q[c + 15][c + 30] = kco / pow(fIco, alphakcoI);
    Q[c + 30][c + 15] = koc * pow(fIco, 1 - alphakcoI);
}

/* adjacency lists in the order CaSim/SingleSiteMWC.cpp:55-89 builds them */
static void mwc_adjacency(or_sim* s) {
    for (int k = 0; k < 60; ++k) s->mwc_nadj[k] = 0;
#define MWC_PUSH(x, y) (s->mwc_adj[x][s->mwc_nadj[x]++] = (y))
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5 - i; ++j) {
            int c = mwc_index(i, j);
            int nb[4], n = 0;
            if (i + j < 4) nb[n++] = mwc_index(i + 1, j);
            if (i > 0) nb[n++] = mwc_index(i - 1, j);
            if (i + j < 4) nb[n++] = mwc_index(i, j + 1);
            if (j > 0) nb[n++] = mwc_index(i, j - 1);
            for (int k = 0; k < n; ++k) {
                MWC_PUSH(c, nb[k]);
                MWC_PUSH(c + 45, nb[k] + 45);
                MWC_PUSH(c + 15, nb[k] + 15);
                MWC_PUSH(c + 30, nb[k] + 30);
            }
            MWC_PUSH(c, c + 15);
            MWC_PUSH(c + 15, c);
            MWC_PUSH(c + 45, c + 30);
            MWC_PUSH(c + 30, c + 45);
            MWC_PUSH(c, c + 45);
            MWC_PUSH(c + 45, c);
            MWC_PUSH(c + 15, c + 30);
            MWC_PUSH(c + 30, c + 15);
        }
#undef MWC_PUSH
}

/* (i, j) of micro-state s (CaSim/SingleSiteMWC.cpp:156-168) */
static void mwc_occupancy(int s, int* i, int* j) {
    int r = s % 15;
    for (int jj = 0; jj <= 4; ++jj) {
        if (r - (5 - jj) < 0) {
            *i = r;
            *j = jj;
            return;
        }
        r -= 5 - jj;
    }
    *i = 0;
    *j = 4;
}

/* escape rate of s and its row over the adjacency list (GetRate, CaSim/QMatrixModel.cpp:20-24) */
static double mwc_row(const or_sim* s, int st, double ca, double mg, double* row) {
    static __thread double Q[60][60];
    int i, j;
    mwc_occupancy(st, &i, &j);
    mwc_set_row(s->m.ch_par, i, ca, j, mg, Q);
    double r = 0;
    for (int k = 0; k < s->mwc_nadj[st]; ++k) {
        row[k] = Q[st][s->mwc_adj[st][k]];
        r += row[k];
    }
    return r;
}

/* stationary distribution of the full Q at (ca, mg): the least-squares solution of
 * p [Q | 1] = [0 | 1], i.e. (S S^T) p = 1 with S = [Q | 1] (CaSim/QMatrixModel.cpp:38-47),
 * by Gaussian elimination with partial pivoting */
static void mwc_stationary(or_sim* s, double ca, double mg) {
    static double Q[60][60], M[60][60], b[60];
    memset(Q, 0, sizeof(Q));
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5 - i; ++j) mwc_set_row(s->m.ch_par, i, ca, j, mg, Q);
    for (int r = 0; r < 60; ++r) {
        double sum = 0;
        for (int k = 0; k < s->mwc_nadj[r]; ++k) sum += Q[r][s->mwc_adj[r][k]];
        Q[r][r] = -sum;
    }
    for (int a = 0; a < 60; ++a) {
        for (int c = 0; c < 60; ++c) {
            double v = 1.0;
            for (int k = 0; k < 60; ++k) v += Q[a][k] * Q[c][k];
            M[a][c] = v;
        }
        b[a] = 1.0;
    }
    for (int c = 0; c < 60; ++c) {
        int piv = c;
        for (int r = c + 1; r < 60; ++r)
            if (fabs(M[r][c]) > fabs(M[piv][c])) piv = r;
        if (piv != c) {
            for (int k = 0; k < 60; ++k) {
                double t = M[c][k];
                M[c][k] = M[piv][k];
                M[piv][k] = t;
            }
            double t = b[c];
            b[c] = b[piv];
            b[piv] = t;
        }
        for (int r = c + 1; r < 60; ++r) {
            double f = M[r][c] / M[c][c];
            if (f == 0) continue;
            for (int k = c; k < 60; ++k) M[r][k] -= f * M[c][k];
            b[r] -= f * b[c];
        }
    }
    for (int r = 59; r >= 0; --r) {
        double v = b[r];
        for (int k = r + 1; k < 60; ++k) v -= M[r][k] * s->mwc_p[k];
        s->mwc_p[r] = v / M[r][r];
    }
}

/* SetMacroState (CaSim/QMatrixModel.cpp:48-58): a micro-state of macro state `open` */
static int mwc_macro_pick(const or_sim* s, int open, double u, int cur) {
    double total = 0, acc = 0;
    for (int i = 0; i < 60; ++i) total += ((i >= 45) == open) * s->mwc_p[i];
    for (int i = 0; i < 60; ++i) {
        acc += ((i >= 45) == open) * s->mwc_p[i];
        if (acc / total >= u) return i;
    }
    return cur;
}

static inline long IDX(const site_t* t, int x, int y, int z) { return z + (long)t->nz * (y + (long)t->ny * x); }

or_sim* or_create(const or_model* m, int n_sites, const int* nx, const int* ny, const int* nz,
                  const int* n_ch, const int* ch_xyz, const uint32_t* seeds, const double* jsr_init) {
    or_sim* s = (or_sim*)calloc(1, sizeof(or_sim));
    s->m = *m;
    s->S = n_sites;
    s->site = (site_t*)calloc((size_t)n_sites, sizeof(site_t));
    long ch_off = 0;
    for (int k = 0; k < n_sites; ++k) {
        site_t* t = &s->site[k];
        t->nx = nx[k];
        t->ny = ny[k];
        t->nz = m->dim == 2 ? 1 : nz[k];
        t->N = (long)t->nx * t->ny * t->nz;
        t->n_ch = n_ch[k];
        t->cx = (int*)malloc(sizeof(int) * (size_t)(t->n_ch + 1));
        t->cy = (int*)malloc(sizeof(int) * (size_t)(t->n_ch + 1));
        t->cz = (int*)malloc(sizeof(int) * (size_t)(t->n_ch + 1));
        for (int c = 0; c < t->n_ch; ++c) {
            t->cx[c] = ch_xyz[3 * (ch_off + c) + 0];
            t->cy[c] = ch_xyz[3 * (ch_off + c) + 1];
            t->cz[c] = ch_xyz[3 * (ch_off + c) + 2];
        }
        ch_off += t->n_ch;
        t->ions = (double*)calloc((size_t)(m->n_ions * t->N), sizeof(double));
        t->pairs = (double*)calloc((size_t)(m->n_pairs * t->N + 1), sizeof(double));
        t->freeb = (double*)calloc((size_t)(m->n_buf * t->N + 1), sizeof(double));
        t->evo_i = (double*)calloc((size_t)(m->n_ions * t->N), sizeof(double));
        t->evo_p = (double*)calloc((size_t)(m->n_pairs * t->N + 1), sizeof(double));
        t->cur = (double*)calloc((size_t)(m->n_ions * t->N), sizeof(double));
        t->state = (int*)calloc((size_t)(t->n_ch + 1), sizeof(int));
        t->micro = (int*)calloc((size_t)(t->n_ch + 1), sizeof(int));
        t->mouth = (double*)calloc((size_t)((m->n_ions + m->n_pairs + m->n_buf) * (t->n_ch + 1)), sizeof(double));
        for (int i = 0; i < 6; ++i) t->rng.s[i] = seeds[6 * k + i];
        for (int i = 0; i < m->n_ions; ++i) t->jsr0[i] = jsr_init ? jsr_init[(long)k * m->n_ions + i] : m->jsr0[i];
        if (m->cyto_type == OR_CYTO_RD3D) {
            long nc = (long)m->mc * m->mc * m->mc;
            int ns = m->n_ions + m->c_n_pairs;
            t->cf = (double*)calloc((size_t)(ns * nc), sizeof(double));
            t->cf_prev = (double*)calloc((size_t)(ns * nc), sizeof(double));
            t->cf_evo = (double*)calloc((size_t)(ns * nc), sizeof(double));
            t->cf_in = (double*)calloc((size_t)(ns * nc), sizeof(double));
            t->rim_map = (int*)calloc((size_t)(t->nx * t->ny), sizeof(int));
            /* cleft lateral position relative to its centre -> nearest cytosol
             * node of layer k = 0, clamped to the updated range [1, mc-2] */
            for (int x = 0; x < t->nx; ++x)
                for (int y = 0; y < t->ny; ++y) {
                    double px = (x - 0.5 * (t->nx - 1)) * m->dx, py = (y - 0.5 * (t->ny - 1)) * m->dy;
                    int ci = (int)floor(px / m->hc + 0.5 * (m->mc - 1) + 0.5);
                    int cj = (int)floor(py / m->hc + 0.5 * (m->mc - 1) + 0.5);
                    if (ci < 1) ci = 1;
                    if (ci > m->mc - 2) ci = m->mc - 2;
                    if (cj < 1) cj = 1;
                    if (cj > m->mc - 2) cj = m->mc - 2;
                    t->rim_map[x * t->ny + y] = ci + m->mc * cj;
                }
        }
    }
    if (m->ch_model == OR_SINGLE_SITE_MWC) {
        /* InitOpening reads the channel map's initial values: the ions' concentrations
           (CaSim/DyadChannels.h:25-58) */
        mwc_adjacency(s);
        mwc_stationary(s, m->Cb_ion[m->ca_idx], m->Cb_ion[m->mg_idx]);
    }
    return s;
}

void or_destroy(or_sim* s) {
    if (!s) return;
    for (int k = 0; k < s->S; ++k) {
        site_t* t = &s->site[k];
        free(t->cx); free(t->cy); free(t->cz);
        free(t->ions); free(t->pairs); free(t->freeb); free(t->evo_i); free(t->evo_p);
        free(t->cur); free(t->state); free(t->micro); free(t->mouth);
        free(t->cf); free(t->cf_prev); free(t->cf_evo); free(t->cf_in); free(t->rim_map);
    }
    free(s->site);
    free(s);
}

/* ---------------------------------------------------------------- reset */
void or_reset(or_sim* s) {
    const or_model* m = &s->m;
    for (int k = 0; k < s->S; ++k) {
        site_t* t = &s->site[k];
        /* CaSim/DyadRD2DCPU.cpp:319-344 */
        for (long n = 0; n < t->N; ++n) {
            int ip = 0;
            for (int j = 0; j < m->n_ions; ++j) {
                t->ions[j * t->N + n] = m->Cb_ion[j];
                t->cur[j * t->N + n] = 0;
                for (int b = 0; b < m->n_buf; ++b) {
                    if (j == 0) t->freeb[b * t->N + n] = m->Ctot[b];
                    if (m->binds[b + j * m->n_buf]) {
                        double v = m->pair_init[ip];
                        t->pairs[ip * t->N + n] = v;
                        t->freeb[b * t->N + n] -= v;
                        ++ip;
                    }
                }
            }
        }
        /* CaSim/SRPool.cpp:111-124 */
        for (int i = 0; i < m->n_ions; ++i) {
            t->jsr[i] = t->jsr0[i];
            t->jsr_new[i] = t->jsr0[i];
            t->IjSR[i] = 0;
            t->nsr[i] = t->jsr0[i]; /* SRPool's ions_NSR starts at the jSR initial values (SRPool.cpp:40-45) */
        }
        t->release = 0;
        /* CaSim/CytosolPool.cpp:373-398 */
        for (int j = 0; j < m->n_ions; ++j) t->c_ions[j] = m->c_bg[j];
        {
            int ip = 0, ipd = 0;
            for (int j = 0; j < m->n_ions; ++j)
                for (int b = 0; b < m->c_n_buf; ++b) {
                    if (j == 0) t->c_free[b] = m->c_Ctot[b];
                    if (m->c_binds[b + j * m->c_n_buf]) {
                        double v = m->c_init[ip];
                        t->c_pairs[ip] = v;
                        if (m->c_in_dyad[ip]) t->c_bnd[ipd++] = v;
                        t->c_free[b] -= v;
                        ++ip;
                    }
                }
        }
        if (m->cyto_type == OR_CYTO_RD3D) {
            long nc = (long)m->mc * m->mc * m->mc;
            int ns = m->n_ions + m->c_n_pairs;
            for (int sp = 0; sp < ns; ++sp) {
                double v = sp < m->n_ions ? m->c_bg[sp] : m->c_init[sp - m->n_ions];
                for (long n = 0; n < nc; ++n) {
                    t->cf[sp * nc + n] = v;
                    t->cf_prev[sp * nc + n] = v;
                    t->cf_in[sp * nc + n] = 0;
                }
            }
        }
        for (int c = 0; c < t->n_ch; ++c) t->state[c] = 0;
        for (int q = 0; q < m->n_ions + m->n_pairs; ++q) t->efflux[q] = 0;
        for (int i = 0; i < m->n_ions; ++i) t->total[i] = 0;
        t->draws = 0;
    }
}

static double runif(site_t* t) {
    t->draws++;
    return mrg_u01d(&t->rng);
}

/* CaSim/DyadChannels.cpp:83-95 (two-state models: every channel closed, one
 * draw each, then the chosen channel opened with one more draw) */
void or_init_opening(or_sim* s, int site, int channel) {
    site_t* t = &s->site[site];
    const int mwc = s->m.ch_model == OR_SINGLE_SITE_MWC;
    for (int c = 0; c < t->n_ch; ++c) {
        double u = runif(t);
        t->state[c] = 0;
        if (mwc) t->micro[c] = mwc_macro_pick(s, 0, u, t->micro[c]);
    }
    double u = runif(t);
    if (channel >= 0 && channel < t->n_ch) {
        t->state[channel] = 1;
        if (mwc) {
            t->micro[channel] = mwc_macro_pick(s, 1, u, t->micro[channel]);
            t->state[channel] = t->micro[channel] >= 45;
        }
    }
}

/* ---------------------------------------------------------------- rates */
static double spline_eval(const or_model* m, int w, double x) {
    int n = m->sp_n[w];
    const double* X = m->sp_x[w];
    if (x <= X[0]) {
        double h = x - X[0];
        return m->sp_left[w][0] + h * (m->sp_left[w][1] + h * m->sp_left[w][2]);
    }
    if (x >= X[n - 1]) {
        double h = x - X[n - 1];
        return m->sp_right[w][0] + h * (m->sp_right[w][1] + h * m->sp_right[w][2]);
    }
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (X[mid] <= x) lo = mid; else hi = mid;
    }
    double h = x - X[lo];
    const double* c = m->sp_c[w][lo];
    return ((c[3] * h + c[2]) * h + c[1]) * h + c[0];
}

/* transition rate (per ms) of a channel in `state`, given its mouth values */
static double rate(const or_model* m, int state, const double* mouth_ions, const double* jsr) {
    const double* p = m->ch_par;
    double ca = m->ca_idx >= 0 ? mouth_ions[m->ca_idx] : 0.0;
    double mg = m->mg_idx >= 0 ? mouth_ions[m->mg_idx] : 0.0;
    (void)jsr;
    switch (m->ch_model) {
    case OR_SHEEP_CANNELL: {
        /* p: kopen0, ncaopen, kopenmax, kclose0, ncaclose */
        if (state) return p[3] * pow(ca * 1e-3, p[4]) * 1e-3;
        double ko = p[0] * pow(ca * 1e-3, p[1]);
        return (ko < p[2] ? ko : p[2]) * 1e-3;
    }
    case OR_TWO_STATE_MWC: {
        /* p: fCa, KCa, fMg, KMg, KO0, KMgI, kclose */
        double kclose = p[6];
        if (state) return kclose;
        double inac = p[5] * p[5] / (p[5] * p[5] + mg * mg);
        double open = pow(ca + p[1] * p[0] * (1 + mg / (p[2] * p[3])), 4);
        double close = p[4] * pow(p[0] * (ca + p[1] * (1 + mg / p[3])), 4);
        double P = inac * open / (open + close);
        return kclose * P / (1 - P);
    }
    case OR_TWO_STATE_AHTG: {
        /* p: fCa, KCa, fMg, KMg, KO0, KMgI, KCL, KI, KOL, kclose */
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
    case OR_TWO_STATE_SPLINE:
        return state ? spline_eval(m, 1, ca) : spline_eval(m, 0, ca);
    default:
        return 0;
    }
}

/* ---------------------------------------------------------------- steps */
static inline double d2(double l, double c, double r, double h) { return (r - 2 * c + l) / (h * h); }

/* CaSim/DyadRD2DCPU.cpp:394-490 and CaSim/DyadRDCPU.cpp:404-506 */
static void dyad_rd(const or_model* m, site_t* t, double dt) {
    const long N = t->N;
    const int nx = t->nx, ny = t->ny, nz = t->nz;
    for (int x = 1; x < nx - 1; ++x)
        for (int y = 1; y < ny - 1; ++y)
            for (int z = 0; z < nz; ++z) {
                long c = IDX(t, x, y, z), xl = IDX(t, x - 1, y, z), xr = IDX(t, x + 1, y, z);
                long yl = IDX(t, x, y - 1, z), yr = IDX(t, x, y + 1, z);
                long zl = 0, zr = 0;
                if (m->dim == 3) {
                    zl = z == 0 ? IDX(t, x, y, z + 1) : IDX(t, x, y, z - 1);
                    zr = z == nz - 1 ? IDX(t, x, y, z - 1) : IDX(t, x, y, z + 1);
                }
                for (int j = 0; j < m->n_ions; ++j) {
                    const double* u = t->ions + j * N;
                    double v = u[c];
                    double lap = d2(u[xl], v, u[xr], m->dx) + d2(u[yl], v, u[yr], m->dy);
                    if (m->dim == 3) lap = lap + d2(u[zl], v, u[zr], m->dz);
                    t->evo_i[j * N + c] = m->D_ion[j] * lap;
                }
                for (int p = 0; p < m->n_pairs; ++p) {
                    const double* u = t->pairs + p * N;
                    double v = u[c];
                    double lap = d2(u[xl], v, u[xr], m->dx) + d2(u[yl], v, u[yr], m->dy);
                    if (m->dim == 3) lap = lap + d2(u[zl], v, u[zr], m->dz);
                    t->evo_p[p * N + c] = m->D_pair[p] * lap;
                }
                int ip = 0;
                for (int j = 0; j < m->n_ions; ++j) {
                    double R = 0;
                    for (int b = 0; b < m->n_buf; ++b)
                        if (m->binds[b + j * m->n_buf]) {
                            double R1 = m->koff[ip] * t->pairs[ip * N + c] - m->kon[ip] * t->ions[j * N + c] * t->freeb[b * N + c];
                            t->evo_p[ip * N + c] += -R1;
                            R += R1;
                            ++ip;
                        }
                    t->evo_i[j * N + c] += R;
                }
            }
    for (int x = 1; x < nx - 1; ++x)
        for (int y = 1; y < ny - 1; ++y)
            for (int z = 0; z < nz; ++z) {
                long c = IDX(t, x, y, z);
                int sl_layer = (m->dim == 2) || (z == nz - 1);
                for (int j = 0; j < m->n_ions; ++j) {
                    long q = j * N + c;
                    t->evo_i[q] += t->cur[q];
                    if (sl_layer && m->has_sl[j]) {
                        double s1 = m->K1[j] + t->ions[q];
                        double s2 = m->K2[j] + t->ions[q];
                        t->evo_i[q] *= 1 / (1 + m->N1[j] * m->K1[j] / (s1 * s1) + m->N2[j] * m->K2[j] / (s2 * s2));
                    }
                    t->ions[q] += t->evo_i[q] * dt;
                }
                for (int p = 0; p < m->n_pairs; ++p) t->pairs[p * N + c] += t->evo_p[p * N + c] * dt;
                int ip = 0;
                for (int j = 0; j < m->n_ions; ++j) {
                    if (j == 0)
                        for (int b = 0; b < m->n_buf; ++b) t->freeb[b * N + c] = m->Ctot[b];
                    for (int b = 0; b < m->n_buf; ++b)
                        if (m->binds[b + j * m->n_buf]) {
                            t->freeb[b * N + c] -= t->pairs[ip * N + c];
                            ++ip;
                        }
                }
            }
}

/* CaSim/CytosolPool.cpp:217-288; dyad efflux layout [species] for this site */
static void cyto_pool(const or_model* m, site_t* t, double dt) {
    double evo_i[OR_MAX_IONS], evo_p[OR_MAX_CPAIRS];
    int ip = 0, ipd = 0, is = 0;
    for (int j = 0; j < m->n_ions; ++j) {
        double react = 0;
        for (int b = 0; b < m->c_n_buf; ++b)
            if (m->c_binds[b + j * m->c_n_buf]) {
                double R1 = m->c_koff[ip] * t->c_pairs[ip] - m->c_kon[ip] * t->c_ions[j] * t->c_free[b];
                evo_p[ip] = -R1;
                react += R1;
                if (m->c_in_dyad[ip]) {
                    evo_p[ip] += t->efflux[m->n_ions + ipd];
                    ++ipd;
                }
                ++ip;
            }
        evo_i[j] = react + t->efflux[j];
        if (m->c_serca[j]) {
            double i2 = t->c_ions[j] * t->c_ions[j];
            double K2 = m->c_Kup[is] * m->c_Kup[is];
            double b2 = m->c_bg[is] * m->c_bg[is];
            evo_i[j] -= m->c_Jmax[is] * (i2 / (i2 + K2) - b2 / (b2 + K2));
            ++is;
        }
    }
    for (int j = 0; j < m->n_ions; ++j) {
        evo_i[j] -= m->c_onetau_ion[j] * (t->c_ions[j] - m->c_bg[j]);
        t->c_ions[j] += evo_i[j] * dt;
    }
    ipd = 0;
    for (int p = 0; p < m->c_n_pairs; ++p) {
        evo_p[p] -= m->c_onetau_pair[p] * (t->c_pairs[p] - m->c_init[p]);
        t->c_pairs[p] += evo_p[p] * dt;
        if (m->c_in_dyad[p]) t->c_bnd[ipd++] = t->c_pairs[p];
    }
    ip = 0;
    for (int j = 0; j < m->n_ions; ++j) {
        if (j == 0)
            for (int b = 0; b < m->c_n_buf; ++b) t->c_free[b] = m->c_Ctot[b];
        for (int b = 0; b < m->c_n_buf; ++b)
            if (m->c_binds[b + j * m->c_n_buf]) {
                t->c_free[b] -= t->c_pairs[ip];
                ++ip;
            }
    }
}

/* RD3D cytosol: explicit Euler on an mc^3 cube (this project's definition).
 * Faces x = 0, x = mc-1, y = 0, y = mc-1, z = mc-1 hold the resting values;
 * the z = 0 face is no-flux (mirror) and receives the dyad efflux deposit.
 * Reactions and SERCA as in the pool; no leak term. */
static void cyto_rd3d(const or_model* m, site_t* t, double dt) {
    const int mc = m->mc;
    const long nc = (long)mc * mc * mc;
    const double h = m->hc;
    const int ns = m->n_ions + m->c_n_pairs;
    memcpy(t->cf_prev, t->cf, sizeof(double) * (size_t)(ns * nc));
    for (int k = 0; k < mc - 1; ++k)
        for (int j = 1; j < mc - 1; ++j)
            for (int i = 1; i < mc - 1; ++i) {
                long c = i + (long)mc * (j + (long)mc * k);
                long xl = c - 1, xr = c + 1, yl = c - mc, yr = c + mc;
                long zl = k == 0 ? c + (long)mc * mc : c - (long)mc * mc, zr = c + (long)mc * mc;
                for (int sp = 0; sp < m->n_ions + m->c_n_pairs; ++sp) {
                    const double* u = t->cf + sp * nc;
                    double D = sp < m->n_ions ? m->D_ion[sp] : m->c_D_pair[sp - m->n_ions];
                    double v = u[c];
                    t->cf_evo[sp * nc + c] = D * (d2(u[xl], v, u[xr], h) + d2(u[yl], v, u[yr], h) + d2(u[zl], v, u[zr], h));
                }
                /* free buffers at this node */
                double fr[OR_MAX_CBUF];
                for (int b = 0; b < m->c_n_buf; ++b) fr[b] = m->c_Ctot[b];
                {
                    int ip = 0;
                    for (int j2 = 0; j2 < m->n_ions; ++j2)
                        for (int b = 0; b < m->c_n_buf; ++b)
                            if (m->c_binds[b + j2 * m->c_n_buf]) {
                                fr[b] -= t->cf[(m->n_ions + ip) * nc + c];
                                ++ip;
                            }
                }
                int ip = 0, is = 0;
                for (int j2 = 0; j2 < m->n_ions; ++j2) {
                    double react = 0;
                    double ion = t->cf[j2 * nc + c];
                    for (int b = 0; b < m->c_n_buf; ++b)
                        if (m->c_binds[b + j2 * m->c_n_buf]) {
                            double B = t->cf[(m->n_ions + ip) * nc + c];
                            double R1 = m->c_koff[ip] * B - m->c_kon[ip] * ion * fr[b];
                            t->cf_evo[(m->n_ions + ip) * nc + c] += -R1;
                            react += R1;
                            ++ip;
                        }
                    t->cf_evo[j2 * nc + c] += react;
                    if (m->c_serca[j2]) {
                        double i2 = ion * ion;
                        double K2 = m->c_Kup[is] * m->c_Kup[is];
                        double b2 = m->c_bg[is] * m->c_bg[is];
                        t->cf_evo[j2 * nc + c] -= m->c_Jmax[is] * (i2 / (i2 + K2) - b2 / (b2 + K2));
                        ++is;
                    }
                }
            }
    for (int k = 0; k < mc - 1; ++k)
        for (int j = 1; j < mc - 1; ++j)
            for (int i = 1; i < mc - 1; ++i) {
                long c = i + (long)mc * (j + (long)mc * k);
                for (int sp = 0; sp < m->n_ions + m->c_n_pairs; ++sp) {
                    double e = t->cf_evo[sp * nc + c];
                    if (k == 0) e += t->cf_in[sp * nc + c];
                    t->cf[sp * nc + c] += e * dt;
                }
            }
}

/* CaSim/SRPool.cpp:70-89 with the site's own beta and NSR values */
static void sr_run(const or_model* m, site_t* t, double dt) {
    if (m->jsr_const) return;
    double beta = 1;
    for (int j = 0; j < m->n_ions; ++j)
        beta += m->nCQ[j] * m->K_CQ[j] * m->CQ / ((m->K_CQ[j] + t->jsr[j]) * (m->K_CQ[j] + t->jsr[j]));
    for (int i = 0; i < m->n_ions; ++i) {
        double Iref = 1 / m->tau_refill[i] * (t->nsr[i] - t->jsr[i]);
        t->jsr_new[i] = t->jsr[i] + dt / beta * (Iref - t->IjSR[i] / m->V_jsr);
    }
    if (m->ca_idx >= 0) t->release += t->IjSR[m->ca_idx] * dt;
}

/* CaSim/DyadChannels.cpp:97-130 for two-state models */
static void run_mc(const or_sim* s, const or_model* m, site_t* t, double dt) {
    int nsp = m->n_ions + m->n_pairs + m->n_buf;
    double mi[OR_MAX_IONS];
    (void)nsp;
    for (int c = 0; c < t->n_ch; ++c) {
        for (int j = 0; j < m->n_ions; ++j) mi[j] = t->mouth[j * t->n_ch + c];
        if (m->ch_model == OR_SINGLE_SITE_MWC) {
            /* QMatrixModel::GetRate / MakeTransition (CaSim/QMatrixModel.cpp:20-36) */
            double row[6];
            int st = t->micro[c];
            double r = mwc_row(s, st, mi[m->ca_idx], mi[m->mg_idx], row);
            if (runif(t) < r * dt) {
                double u = runif(t), acc = 0;
                for (int k = 0; k < s->mwc_nadj[st]; ++k) {
                    acc += row[k];
                    if (acc / r >= u) {
                        t->micro[c] = s->mwc_adj[st][k];
                        break;
                    }
                }
                t->state[c] = t->micro[c] >= 45;
            }
            continue;
        }
        double r = rate(m, t->state[c], mi, t->jsr_new);
        if (runif(t) < r * dt) {
            (void)runif(t);
            t->state[c] = 1 - t->state[c];
        }
    }
}

/* Update(): mouth gather, Dirichlet edges, efflux, currents (CaSim/DyadRD2DCPU.cpp:382-392) */
static void dyad_update(const or_model* m, site_t* t) {
    const long N = t->N;
    const int nx = t->nx, ny = t->ny, nz = t->nz;
    /* mouth values: ions, pairs, free buffers */
    for (int c = 0; c < t->n_ch; ++c) {
        long q = IDX(t, t->cx[c], t->cy[c], t->cz[c]);
        for (int j = 0; j < m->n_ions; ++j) t->mouth[j * t->n_ch + c] = t->ions[j * N + q];
        for (int p = 0; p < m->n_pairs; ++p) t->mouth[(m->n_ions + p) * t->n_ch + c] = t->pairs[p * N + q];
        for (int b = 0; b < m->n_buf; ++b) t->mouth[(m->n_ions + m->n_pairs + b) * t->n_ch + c] = t->freeb[b * N + q];
    }
    /* Dirichlet edges from the cytosol */
    for (int pass = 0; pass < 2; ++pass) {
        for (int e = 0; e < 2; ++e) {
            int lim = pass == 0 ? ny : nx;
            for (int a = 0; a < lim; ++a)
                for (int z = 0; z < nz; ++z) {
                    int x = pass == 0 ? (e == 0 ? 0 : nx - 1) : a;
                    int y = pass == 0 ? a : (e == 0 ? 0 : ny - 1);
                    long q = IDX(t, x, y, z);
                    if (m->cyto_type == OR_CYTO_POOL) {
                        for (int j = 0; j < m->n_ions; ++j) t->ions[j * N + q] = t->c_ions[j];
                        for (int p = 0; p < m->n_pairs; ++p) t->pairs[p * N + q] = t->c_bnd[p];
                    } else {
                        long cn = t->rim_map[x * ny + y];
                        long nc = (long)m->mc * m->mc * m->mc;
                        for (int j = 0; j < m->n_ions; ++j) t->ions[j * N + q] = t->cf_prev[j * nc + cn];
                        for (int p = 0; p < m->n_pairs; ++p) {
                            int cp = -1;
                            for (int r = 0; r < m->c_n_pairs; ++r)
                                if (m->c_dyad_pair[r] == p) cp = r;
                            t->pairs[p * N + q] = cp >= 0 ? t->cf_prev[(m->n_ions + cp) * nc + cn] : m->pair_init[p];
                        }
                    }
                }
        }
    }
    /* efflux (CaSim/DyadRD2DCPU.cpp:305-350, CaSim/DyadRDCPU.cpp:322-369) */
    double gm = 3.0 / (4 * acos(-1) * m->R * m->R * m->R);
    double sx, sy;
    if (m->dim == 2) {
        sx = m->dy * m->z / m->dx;
        sy = m->dx * m->z / m->dy;
    } else {
        sx = m->dy * m->dz / m->dx;
        sy = m->dx * m->dz / m->dy;
    }
    int zmax = m->dim == 2 ? 1 : nz - 1;
    const int nsp = m->n_ions + m->n_pairs;
    long nc = m->cyto_type == OR_CYTO_RD3D ? (long)m->mc * m->mc * m->mc : 0;
    if (m->cyto_type == OR_CYTO_RD3D)
        for (long q = 0; q < (long)(m->n_ions + m->c_n_pairs) * nc; ++q) t->cf_in[q] = 0;
    double vinv = m->cyto_type == OR_CYTO_RD3D ? 1.0 / (m->hc * m->hc * m->hc) : 0.0;
    for (int q = 0; q < nsp; ++q) t->efflux[q] = 0;
    for (int pass = 0; pass < 2; ++pass) {
        double sf = pass == 0 ? sx : sy;
        for (int e = 0; e < 2; ++e) {
            int lo = pass == 0 ? 1 : 0, hi = pass == 0 ? ny - 1 : nx;
            for (int a = lo; a < hi; ++a)
                for (int z = 0; z < zmax; ++z) {
                    int x0, y0, x1, y1, x2, y2;
                    if (pass == 0) {
                        x0 = e == 0 ? 0 : nx - 1; x1 = e == 0 ? 1 : nx - 2; x2 = e == 0 ? 2 : nx - 3;
                        y0 = y1 = y2 = a;
                    } else {
                        y0 = e == 0 ? 0 : ny - 1; y1 = e == 0 ? 1 : ny - 2; y2 = e == 0 ? 2 : ny - 3;
                        x0 = x1 = x2 = a;
                    }
                    long q0 = IDX(t, x0, y0, z), q1 = IDX(t, x1, y1, z), q2 = IDX(t, x2, y2, z);
                    for (int sp = 0; sp < nsp; ++sp) {
                        const double* u = sp < m->n_ions ? t->ions + sp * N : t->pairs + (sp - m->n_ions) * N;
                        double D = sp < m->n_ions ? m->D_ion[sp] : m->D_pair[sp - m->n_ions];
                        if (m->cyto_type == OR_CYTO_POOL) {
                            t->efflux[sp] += D * gm * sf * (2 * u[q1] - 1.5 * u[q0] - 0.5 * u[q2]);
                        } else {
                            double term = D * sf * (2 * u[q1] - 1.5 * u[q0] - 0.5 * u[q2]);
                            t->efflux[sp] += term * vinv;
                            int cs = -1;
                            if (sp < m->n_ions) cs = sp;
                            else
                                for (int r = 0; r < m->c_n_pairs; ++r)
                                    if (m->c_dyad_pair[r] == sp - m->n_ions) cs = m->n_ions + r;
                            if (cs >= 0) t->cf_in[cs * nc + t->rim_map[x0 * ny + y0]] += term * vinv;
                        }
                    }
                }
        }
    }
    /* currents (CaSim/DyadRD2DCPU.cpp:243-264) */
    for (int j = 0; j < m->n_ions; ++j) t->total[j] = 0;
    for (int c = 0; c < t->n_ch; ++c) {
        long q = IDX(t, t->cx[c], t->cy[c], t->cz[c]);
        for (int j = 0; j < m->n_ions; ++j) {
            double flux = t->state[c] * (m->g[j] * (t->jsr_new[j] - t->ions[j * N + q]));
            t->cur[j * N + q] = flux;
            t->total[j] += flux;
        }
    }
}

static void sr_update(const or_model* m, site_t* t, double V_elem) {
    if (m->jsr_const) return;
    for (int i = 0; i < m->n_ions; ++i) {
        t->IjSR[i] = t->total[i] * V_elem;
        t->nsr[i] = m->nsr[i];
        t->jsr[i] = t->jsr_new[i];
    }
}

static double element_volume(const or_model* m) {
    return m->dim == 2 ? m->dx * m->dy * m->z : 0.5 * m->dx * m->dy * m->dz;
}

void or_update(or_sim* s) {
    const or_model* m = &s->m;
    double ve = element_volume(m);
    for (int k = 0; k < s->S; ++k) {
        dyad_update(m, &s->site[k]);
        sr_update(m, &s->site[k], ve);
    }
}

void or_start(or_sim* s, const int* first_channel) {
    or_reset(s);
    for (int k = 0; k < s->S; ++k) or_init_opening(s, k, first_channel[k]);
    or_update(s);
}

void or_step(or_sim* s, long n_steps, int n_threads) {
    const or_model* m = &s->m;
    double ve = element_volume(m);
    (void)n_threads;
    for (long it = 0; it < n_steps; ++it) {
#pragma omp parallel for num_threads(n_threads > 0 ? n_threads : 1) schedule(dynamic, 1)
        for (int k = 0; k < s->S; ++k) {
            site_t* t = &s->site[k];
            if (m->cyto_type == OR_CYTO_POOL) cyto_pool(m, t, m->dt);
            else cyto_rd3d(m, t, m->dt);
            dyad_rd(m, t, m->dt);
            sr_run(m, t, m->dt);
            run_mc(s, m, t, m->dt);
            dyad_update(m, t);
            sr_update(m, t, ve);
        }
    }
}

/* ---------------------------------------------------------------- getters */
long or_site_nodes(const or_sim* s, int site) { return s->site[site].N; }

void or_get_field(const or_sim* s, int site, int species, double* out) {
    const or_model* m = &s->m;
    const site_t* t = &s->site[site];
    const double* src;
    if (species < m->n_ions) src = t->ions + species * t->N;
    else if (species < m->n_ions + m->n_pairs) src = t->pairs + (species - m->n_ions) * t->N;
    else src = t->freeb + (species - m->n_ions - m->n_pairs) * t->N;
    memcpy(out, src, sizeof(double) * (size_t)t->N);
}

void or_get_mouth(const or_sim* s, int site, int species, double* out) {
    const site_t* t = &s->site[site];
    memcpy(out, t->mouth + species * t->n_ch, sizeof(double) * (size_t)t->n_ch);
}

void or_get_states(const or_sim* s, int site, int* out) {
    const site_t* t = &s->site[site];
    memcpy(out, t->state, sizeof(int) * (size_t)t->n_ch);
}

void or_get_micro(const or_sim* s, int site, int* out) {
    const site_t* t = &s->site[site];
    memcpy(out, t->micro, sizeof(int) * (size_t)t->n_ch);
}

void or_get_jsr(const or_sim* s, int site, double* out) {
    for (int i = 0; i < s->m.n_ions; ++i) out[i] = s->site[site].jsr_new[i];
}

void or_get_total_current(const or_sim* s, int site, double* out) {
    for (int i = 0; i < s->m.n_ions; ++i) out[i] = s->site[site].total[i];
}

void or_get_efflux(const or_sim* s, int site, double* out) {
    for (int i = 0; i < s->m.n_ions + s->m.n_pairs; ++i) out[i] = s->site[site].efflux[i];
}

void or_get_cyto(const or_sim* s, int site, double* out) {
    const site_t* t = &s->site[site];
    for (int i = 0; i < s->m.n_ions; ++i) out[i] = t->c_ions[i];
    for (int p = 0; p < s->m.c_n_pairs; ++p) out[s->m.n_ions + p] = t->c_pairs[p];
}

long or_get_cyto_field(const or_sim* s, int site, int species, double* out) {
    const or_model* m = &s->m;
    if (m->cyto_type != OR_CYTO_RD3D) return 0;
    long nc = (long)m->mc * m->mc * m->mc;
    if (out) memcpy(out, s->site[site].cf + species * nc, sizeof(double) * (size_t)nc);
    return nc;
}

uint64_t or_draws(const or_sim* s, int site) { return s->site[site].draws; }
double or_release(const or_sim* s, int site) { return s->site[site].release; }

/* ------------------------------------------ quasi-stationary release site (Gillespie)
 * One scenario of CaSim/QuasyStationaryReleaseSite.cpp:89-133 with two-state channels:
 * every channel set closed (one draw each), `first` opened (one draw); then, while a
 * channel is open and t < max_time: mouth Ca c_j = sum over open i of added[i][j] (in
 * channel order) + bg, rates at (c_j, mg), total in channel order, t += -log(u) / total
 * (ParallelRng::rexp), channel picked by the running share p <= r <= p + rate/total, its
 * transition (one more draw). The stream state in seed6 is advanced in place. Events
 * (time, channel, new state) beyond max_events are counted but not stored. Returns the
 * event count. */
long or_qs_run(const or_model* m, int n_ch, const double* added, double bg, double mg, double max_time, uint32_t* seed6,
               int first, long max_events, double* ev_t, int* ev_c, int* ev_s, uint64_t* draws) {
    mrg_t g;
    for (int i = 0; i < 6; ++i) g.s[i] = seed6[i];
    int* st = (int*)calloc((size_t)n_ch, sizeof(int));
    double* rt = (double*)malloc(sizeof(double) * (size_t)n_ch);
    double ions[OR_MAX_IONS] = {0};
    uint64_t nd = 0;
    for (int i = 0; i < n_ch; ++i) {
        mrg_u01d(&g);
        st[i] = 0;
    }
    mrg_u01d(&g);
    st[first] = 1;
    nd = (uint64_t)n_ch + 1;
    int n_open = 1;
    double t = 0;
    long ne = 0;
    while (n_open >= 1 && t < max_time) {
        double total = 0;
        for (int j = 0; j < n_ch; ++j) {
            double c = 0;
            for (int i = 0; i < n_ch; ++i) c += st[i] * added[(long)i * n_ch + j];
            c += bg;
            ions[m->ca_idx] = c;
            if (m->mg_idx >= 0) ions[m->mg_idx] = mg;
            rt[j] = rate(m, st[j], ions, NULL);
        }
        for (int j = 0; j < n_ch; ++j) total += rt[j];
        double theta = 1 / total;
        t += -log(mrg_u01d(&g)) * theta;
        double r = mrg_u01d(&g);
        double p = 0;
        int idx = 0;
        for (int i = 0; i < n_ch; ++i) {
            if (p <= r && r <= p + rt[i] / total) {
                idx = i;
                break;
            }
            p += rt[i] / total;
        }
        mrg_u01d(&g);
        nd += 3;
        st[idx] = 1 - st[idx];
        n_open += st[idx] ? 1 : -1;
        if (ne < max_events) {
            ev_t[ne] = t;
            ev_c[ne] = idx;
            ev_s[ne] = st[idx];
        }
        ++ne;
    }
    for (int i = 0; i < 6; ++i) seed6[i] = (uint32_t)g.s[i];
    if (draws) *draws = nd;
    free(st);
    free(rt);
    return ne;
}
