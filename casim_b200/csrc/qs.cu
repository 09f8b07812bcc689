// Quasi-stationary release sites: the reference's ParallelSolver path
// (CaSim/ParallelSolver.cpp:51-143) batched on the device.
//
// A site is a set of RyRs at fixed positions whose mouth Ca is the
// quasi-stationary solution of linearised buffered diffusion around point
// sources (Naraghi & Neher 1997; CaSim/LinearNaraghiNeher.cpp:9-75): the Ca at
// channel j is the background plus, for every open channel i, a precomputed
// increment added[i][j]. Gating is simulated exactly with Gillespie's method
// (CaSim/QuasyStationaryReleaseSite.cpp:89-133): the total rate of the
// channels at their mouth Ca, an exponential waiting time, a channel picked by
// its share of the total rate, its transition; until no channel is open or
// the time limit is reached.
//
// Device work, sites of up to 32 RyRs: one scenario per lane (k_qs_lane, the open set a
// bitmask in a register, the reference's operations in its order per lane). Larger
// sites: persistent warps, each taking the next scenario off a counter
// when its last one ends (event counts run from 1 to hundreds, so a static
// warp-per-scenario grid idles behind its longest scenario). Per event, lanes
// form the mouth Ca and the rate of one channel each (the Ca summed over the
// open channels, read off a bitmask, in channel order as the reference sums
// it), lane 0 sums the total rate in channel order, the lanes divide every rate
// by it (the shares the reference's pick forms), and lane 0 takes the draws and
// walks the shares in order, so that every floating-point operation follows
// the reference's order. Each scenario has its own MRG32k3a stream. The
// increments are computed on the host (a symmetric eigenproblem, below).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <nlohmann/json.hpp>
#include <string>
#include <vector>

#include "../../include/casim_b200.h"
#include "model.h"
#include "mrg32k3a.cuh"
#include "physics.cuh"

using json = nlohmann::json;

struct casim_qs_s {
    cb_model m{};        // gating law (ch_model, ch_par), ca_idx 0 and mg_idx 1
    int n_ch = 0, n_scen = 0;
    double bg = 0, mg = 0, max_time = 0;
    long long max_events = 0;
    std::vector<double> added;           // [i][j]: Ca at channel j from open channel i (uM)
    std::vector<uint32_t> seeds;         // 6 per scenario: the stream state for the next run
    double* d_added = nullptr;
    uint32_t* d_seed = nullptr;
    int* d_first = nullptr;
    double* d_t = nullptr;               // [scenario][max_events] event times
    int* d_ev = nullptr;                 // channel | new state << 30
    long long* d_nev = nullptr;
    unsigned long long* d_draws = nullptr;
    int* d_flags = nullptr;              // per scenario: 1 = event storage ran out, 2 = stopped at the cap
    int* d_next = nullptr;               // next scenario to take (persistent warps)
    int grid = 0;                        // resident blocks of k_qs_run
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0;
    bool ran = false;
    std::string err;
};

namespace {

std::string g_qs_create_err;

casim_status qs_fail(casim_qs h, casim_status s, const std::string& msg) {
    if (h) h->err = msg;
    else g_qs_create_err = msg;
    return s;
}

struct qs_error : std::runtime_error {
    casim_status code;
    qs_error(casim_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw qs_error(CASIM_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

double jnum(const json& j, const char* key, const char* where) {
    if (!j.contains(key) || !j.at(key).is_number()) throw qs_error(CASIM_EINVAL, std::string(where) + ": missing number \"" + key + "\"");
    return j.at(key).get<double>();
}

// Jacobi eigenvalue iteration for a small symmetric matrix (Golub & Van Loan, "Matrix
// Computations", cyclic Jacobi): A = Q diag(w) Q^T; A is overwritten.
void jacobi_eigen(std::vector<double>& A, int n, std::vector<double>& w, std::vector<double>& Q) {
    Q.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) Q[i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0, diag = 0;
        for (int p = 0; p < n; ++p)
            for (int q = 0; q < n; ++q) (p == q ? diag : off) += A[p * n + q] * A[p * n + q];
        if (off <= 1e-30 * (diag + 1e-300)) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[p * n + q];
                if (apq == 0.0) continue;
                const double theta = (A[q * n + q] - A[p * n + p]) / (2 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                const double c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < n; ++k) {  // columns p, q
                    const double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - s * akq;
                    A[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {  // rows p, q
                    const double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - s * aqk;
                    A[q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double qkp = Q[k * n + p], qkq = Q[k * n + q];
                    Q[k * n + p] = c * qkp - s * qkq;
                    Q[k * n + q] = s * qkp + c * qkq;
                }
            }
    }
    w.resize(n);
    for (int i = 0; i < n; ++i) w[i] = A[i * n + i];
}

// x = M^-1 b by Gaussian elimination with partial pivoting (M n x n, row-major)
std::vector<double> solve_dense(std::vector<double> M, std::vector<double> b, int n) {
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(M[r * n + c]) > std::fabs(M[piv * n + c])) piv = r;
        if (M[piv * n + c] == 0.0) throw qs_error(CASIM_EINVAL, "Naraghi-Neher eigenvectors are singular");
        if (piv != c) {
            for (int k = 0; k < n; ++k) std::swap(M[c * n + k], M[piv * n + k]);
            std::swap(b[c], b[piv]);
        }
        for (int r = c + 1; r < n; ++r) {
            const double f = M[r * n + c] / M[c * n + c];
            for (int k = c; k < n; ++k) M[r * n + k] -= f * M[c * n + k];
            b[r] -= f * b[c];
        }
    }
    std::vector<double> x(n);
    for (int r = n - 1; r >= 0; --r) {
        double acc = b[r];
        for (int k = r + 1; k < n; ++k) acc -= M[r * n + k] * x[k];
        x[r] = acc / M[r * n + r];
    }
    return x;
}

// Quasi-stationary Ca increments of the linearised buffered diffusion around a point
// source (the quantities of CaSim/LinearNaraghiNeher.cpp:9-75). With buffers b (mobile:
// D_b > 0), kappa_b = B_b K_b / (K_b + c0)^2 and tau_b = 1 / (koff_b + kon_b c0), the
// system D u'' = -A u has A with A(b,b) = -1/tau_b, A(b,Ca) = kappa_b/tau_b,
// A(Ca,b) = 1/tau_b, A(Ca,Ca) = -sum kappa_b/tau_b. A = W S with W = diag(kappa, 1) and S
// symmetric, so B = -D^-1 A = -G S (G = D^-1 W, positive diagonal) is similar to the
// symmetric -G^1/2 S G^1/2: its eigenvalues mu are real, its eigenvectors G^1/2 Q. The
// smallest eigenvalue (the conserved mode) goes last, as the reference orders them; the
// amplitudes a solve E a = (0, .., I / (4 pi F D_Ca)); the Ca increment at distance r is
// sum_k a_k E(Ca, k) exp(-r sqrt|mu_k| 1e-8) / r * 1e-4, and ca_open at the source itself.
std::vector<double> naraghi_neher(const std::vector<double>& kon, const std::vector<double>& koff, const std::vector<double>& D,
                                  const std::vector<double>& tot, double c0, double dca, double current, double ca_open,
                                  const std::vector<double>& px, const std::vector<double>& py) {
    const int nb = (int)kon.size(), n = nb + 1;
    std::vector<double> kap(nb), tau(nb);
    for (int b = 0; b < nb; ++b) {
        if (!(D[b] > 0)) throw qs_error(CASIM_EINVAL, "Naraghi-Neher buffers must diffuse (D > 0)");
        const double K = koff[b] / kon[b];
        kap[b] = tot[b] * K / ((K + c0) * (K + c0));
        tau[b] = 1 / (koff[b] + kon[b] * c0);
    }
    std::vector<double> S((size_t)n * n, 0.0), g(n);
    double scc = 0;
    for (int b = 0; b < nb; ++b) {
        S[b * n + b] = -1 / (kap[b] * tau[b]);
        S[b * n + nb] = S[nb * n + b] = 1 / tau[b];
        scc -= kap[b] / tau[b];
        g[b] = kap[b] / D[b];
    }
    S[nb * n + nb] = scc;
    g[nb] = 1 / dca;
    std::vector<double> M((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) M[i * n + j] = -std::sqrt(g[i]) * S[i * n + j] * std::sqrt(g[j]);
    std::vector<double> mu, Q;
    jacobi_eigen(M, n, mu, Q);
    std::vector<double> E((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) E[i * n + k] = std::sqrt(g[i]) * Q[i * n + k];
    int kmin = 0;
    for (int k = 1; k < n; ++k)
        if (mu[k] < mu[kmin]) kmin = k;
    std::swap(mu[kmin], mu[n - 1]);
    for (int i = 0; i < n; ++i) std::swap(E[i * n + kmin], E[i * n + n - 1]);
    const double far = 96485.33e-6, pi = std::acos(-1.0);
    std::vector<double> u(n, 0.0);
    u[n - 1] = current / (4 * pi * far * dca);
    const std::vector<double> a = solve_dense(E, u, n);
    const int nc = (int)px.size();
    std::vector<double> added((size_t)nc * nc);
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
            const double r = std::sqrt((px[i] - px[j]) * (px[i] - px[j]) + (py[i] - py[j]) * (py[i] - py[j]));
            double d = 0;
            if (r > 1e-6) {
                for (int k = 0; k < n; ++k) d += 1 / r * a[k] * std::exp(-r * std::sqrt(std::fabs(mu[k])) * 1e-8) * E[(n - 1) * n + k] * 1e-4;
            } else {
                d = ca_open;
            }
            added[(size_t)i * nc + j] = d;
        }
    return added;
}

constexpr int QS_WARPS = 4;  // warps per block

// Shared memory of one warp: rates (then shares) and the open-channel bitmask, padded
// to 16 bytes so that every warp's rates start 8-byte aligned.
__host__ __device__ inline size_t qs_warp_bytes(int n_ch) {
    return (sizeof(double) * n_ch + sizeof(unsigned) * ((n_ch + 31) / 32) + 15) / 16 * 16;
}

// Scenarios on persistent warps (CaSim/QuasyStationaryReleaseSite.cpp:89-133).
template <int MODEL>
__global__ void __launch_bounds__(32 * QS_WARPS) k_qs_run(cb_model m, int n_ch, const double* __restrict__ added, double bg, double mg,
                                                          double max_time, int n_scen, const int* __restrict__ first,
                                                          uint32_t* __restrict__ seeds, long long max_events,
                                                          double* __restrict__ ev_t, int* __restrict__ ev_c,
                                                          long long* __restrict__ nev, unsigned long long* __restrict__ draws,
                                                          int* __restrict__ flags, int* __restrict__ next) {
    extern __shared__ __align__(16) unsigned char qs_smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int nw = (n_ch + 31) / 32;
    double* rt = (double*)(qs_smem + qs_warp_bytes(n_ch) * wib);  // rate, then share, of each channel
    unsigned* om = (unsigned*)(rt + n_ch);                          // bit i: channel i open
    for (;;) {
        int s = 0;
        if (lane == 0) s = atomicAdd(next, 1);
        s = __shfl_sync(0xffffffffu, s, 0);
        if (s >= n_scen) return;
        cbrng::State g;
        for (int i = 0; i < 6; ++i) g.s[i] = seeds[6 * (size_t)s + i];
        // every channel set closed (one draw each), then the first one opened (one more draw)
        // (CaSim/QuasyStationaryReleaseSite.cpp:93-98; SetMacroState consumes its draw)
        const int f0 = first[s];
        for (int w = lane; w < nw; w += 32) om[w] = w == (f0 >> 5) ? 1u << (f0 & 31) : 0u;
        if (lane == 0)
            for (int i = 0; i <= n_ch; ++i) cbrng::u01d_fold(g);
        __syncwarp();
        double t = 0;
        int n_open = 1;
        long long ne = 0;
        double* et = ev_t + (size_t)s * max_events;
        int* ec = ev_c + (size_t)s * max_events;
        int overflow = 0;
        // the loop ends when no channel is open or time runs out; as a guard against rates that
        // would take it to absurd event counts, it also stops after 64 x max_events events
        const long long cap = 64 * max_events;
        while (n_open >= 1 && t < max_time && ne < cap) {
            // mouth Ca (the increments of the open channels in channel order, then the
            // background) and rate; a closed channel adds 0 * increment = +0 there
            for (int j = lane; j < n_ch; j += 32) {
                double c = 0;
                for (int w = 0; w < nw; ++w)
                    for (unsigned b = om[w]; b; b &= b - 1) c += added[(size_t)(32 * w + __ffs(b) - 1) * n_ch + j];
                c += bg;
                const int sj = (om[j >> 5] >> (j & 31)) & 1;
                rt[j] = cb_rate<MODEL>(m, nullptr, nullptr, nullptr, nullptr, sj, c, mg);
            }
            __syncwarp();
            double total = 0;
            if (lane == 0)
                for (int j = 0; j < n_ch; ++j) total += rt[j];
            total = __shfl_sync(0xffffffffu, total, 0);
            __syncwarp();
            for (int j = lane; j < n_ch; j += 32) rt[j] = rt[j] / total;
            __syncwarp();
            if (lane == 0) {
                // ParallelRng::rexp(1 / total): -log(runif()) * theta (CaSim/ParallelRng.cpp)
                const double theta = 1 / total;
                t += -log(cbrng::u01d_fold(g)) * theta;
                const double r = cbrng::u01d_fold(g);
                double p = 0;
                int idx = 0;
                for (int i = 0; i < n_ch; ++i) {
                    const double q = rt[i];
                    if (p <= r && r <= p + q) {
                        idx = i;
                        break;
                    }
                    p += q;
                }
                cbrng::u01d_fold(g);  // MakeTransition(runif()): a two-state channel flips
                const unsigned bit = 1u << (idx & 31);
                om[idx >> 5] ^= bit;
                const int now = (om[idx >> 5] & bit) ? 1 : 0;
                n_open += now ? 1 : -1;
                if (ne < max_events) {
                    et[ne] = t;
                    ec[ne] = idx | (now << 30);
                } else {
                    overflow = 1;
                }
                ++ne;
            }
            // the loop condition reads t, n_open and ne: every lane takes lane 0's values
            t = __shfl_sync(0xffffffffu, t, 0);
            n_open = __shfl_sync(0xffffffffu, n_open, 0);
            ne = __shfl_sync(0xffffffffu, ne, 0);
            __syncwarp();
        }
        if (lane == 0) {
            for (int i = 0; i < 6; ++i) seeds[6 * (size_t)s + i] = g.s[i];
            nev[s] = ne;
            draws[s] = (unsigned long long)n_ch + 1 + 3ull * ne;
            flags[s] = overflow | (ne >= cap && n_open >= 1 && t < max_time ? 2 : 0);
        }
        __syncwarp();
    }
}

// Sites of at most 32 RyRs: one scenario per lane. The open set is a bitmask in a
// register; each event every running lane forms the mouth Ca of all RyRs (the increments
// of the open RyRs in RyR order, a closed RyR adding +0 as the reference's 0 * increment
// does), the rates (kept in shared memory, a column per lane), the total in RyR order,
// the draws and the pick by shares rt[i] / total in order: the reference's operations
// in its order, for 32 scenarios at once. Lanes take the next scenario off the counter
// when theirs ends.
constexpr int QSL_WARPS = 4;
__host__ __device__ inline size_t qsl_smem(int n_ch) {
    return sizeof(double) * ((size_t)n_ch * n_ch + (size_t)QSL_WARPS * 32 * n_ch);
}

template <int MODEL>
__global__ void __launch_bounds__(32 * QSL_WARPS) k_qs_lane(cb_model m, int n_ch, const double* __restrict__ added, double bg, double mg,
                                                            double max_time, int n_scen, const int* __restrict__ first,
                                                            uint32_t* __restrict__ seeds, long long max_events,
                                                            double* __restrict__ ev_t, int* __restrict__ ev_c,
                                                            long long* __restrict__ nev, unsigned long long* __restrict__ draws,
                                                            int* __restrict__ flags, int* __restrict__ next) {
    extern __shared__ __align__(16) unsigned char qsl_raw[];
    double* A = (double*)qsl_raw;  // [i][j]: the increments
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double* rt = A + (size_t)n_ch * n_ch + (size_t)wib * 32 * n_ch;  // [j][lane]
    for (int k = threadIdx.x; k < n_ch * n_ch; k += blockDim.x) A[k] = added[k];
    __syncthreads();
    const long long cap = 64 * max_events;
    int s = -1;
    bool running = false;
    cbrng::State g;
    unsigned mask = 0;
    int n_open = 0;
    long long ne = 0;
    double t = 0;
    int overflow = 0;
    double* et = nullptr;
    int* ec = nullptr;
    for (;;) {
        if (!running) {
            if (s >= 0) {
                for (int i = 0; i < 6; ++i) seeds[6 * (size_t)s + i] = g.s[i];
                nev[s] = ne;
                draws[s] = (unsigned long long)n_ch + 1 + 3ull * ne;
                flags[s] = overflow | (ne >= cap && n_open >= 1 && t < max_time ? 2 : 0);
            }
            s = atomicAdd(next, 1);
            if (s >= n_scen) break;
            for (int i = 0; i < 6; ++i) g.s[i] = seeds[6 * (size_t)s + i];
            // every channel set closed (one draw each), then the first one opened (one more
            // draw) (CaSim/QuasyStationaryReleaseSite.cpp:93-98)
            for (int i = 0; i <= n_ch; ++i) cbrng::u01d_fold(g);
            mask = 1u << first[s];
            n_open = 1;
            ne = 0;
            t = 0;
            overflow = 0;
            et = ev_t + (size_t)s * max_events;
            ec = ev_c + (size_t)s * max_events;
            running = t < max_time;
            if (!running) continue;
        }
        // four RyRs at a time: four independent sums (each in RyR order) keep the FP64
        // pipeline busy; the total then adds the rates in RyR order
        for (int j0 = 0; j0 < n_ch; j0 += 4) {
            double c[4] = {0, 0, 0, 0};
            for (int i = 0; i < n_ch; ++i) {
                const bool on = (mask >> i) & 1u;
                const double* a = A + i * n_ch + j0;
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (j0 + k < n_ch) c[k] += on ? a[k] : 0.0;
            }
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (j0 + k < n_ch) {
                    const int j = j0 + k;
                    rt[j * 32 + lane] = cb_rate<MODEL>(m, nullptr, nullptr, nullptr, nullptr, (int)((mask >> j) & 1u), c[k] + bg, mg);
                }
        }
        double total = 0;
        for (int j = 0; j < n_ch; ++j) total += rt[j * 32 + lane];
        // ParallelRng::rexp(1 / total): -log(runif()) * theta (CaSim/ParallelRng.cpp)
        const double theta = 1 / total;
        t += -log(cbrng::u01d_fold(g)) * theta;
        const double r = cbrng::u01d_fold(g);
        double p = 0;
        int idx = 0;
        for (int i = 0; i < n_ch; ++i) {
            const double q = rt[i * 32 + lane] / total;
            if (p <= r && r <= p + q) {
                idx = i;
                break;
            }
            p += q;
        }
        cbrng::u01d_fold(g);  // MakeTransition(runif()): a two-state channel flips
        mask ^= 1u << idx;
        const int now = (mask >> idx) & 1u;
        n_open += now ? 1 : -1;
        if (ne < max_events) {
            et[ne] = t;
            ec[ne] = idx | (now << 30);
        } else {
            overflow = 1;
        }
        ++ne;
        running = n_open >= 1 && t < max_time && ne < cap;
    }
}

using qs_kernel_t = decltype(&k_qs_run<0>);
qs_kernel_t qs_kernel(int model, bool lane) {
    switch (model) {
    case CB_TWO_STATE_MWC: return lane ? k_qs_lane<CB_TWO_STATE_MWC> : k_qs_run<CB_TWO_STATE_MWC>;
    case CB_TWO_STATE_AHTG: return lane ? k_qs_lane<CB_TWO_STATE_AHTG> : k_qs_run<CB_TWO_STATE_AHTG>;
    default: return lane ? k_qs_lane<CB_SHEEP_CANNELL> : k_qs_run<CB_SHEEP_CANNELL>;
    }
}

// Release-event metrics of each scenario's trace (CaSim/IndChannelCREAnalyzer.cpp:64-118):
// the trace is the row at t = 0 (one open channel) and one row per event; amplitude = most
// open channels (first maximum), time to peak, time to end = last row's time, integral of
// the open count (each row's count times the time to the next row), its mean.
__global__ void k_qs_metrics(int n_scen, long long max_events, const double* __restrict__ ev_t, const int* __restrict__ ev_c,
                             const long long* __restrict__ nev, int nadir, double* __restrict__ out, int* __restrict__ cls) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_scen) return;
    const long long n = min(nev[s], max_events);
    const double* et = ev_t + (size_t)s * max_events;
    const int* ec = ev_c + (size_t)s * max_events;
    int open = 1;
    double amp = 1, ttp = 0, q = 0, tprev = 0;
    for (long long k = 0; k < n; ++k) {
        const double tk = et[k];
        q += open * (tk - tprev);
        open += (ec[k] >> 30) ? 1 : -1;
        if (open > amp) {
            amp = open;
            ttp = tk;
        }
        tprev = tk;
    }
    const double tte = tprev;
    double* o = out + (size_t)s * 5;
    o[0] = amp;
    o[1] = ttp;
    o[2] = tte;
    o[3] = q;
    o[4] = q / tte;
    atomicAdd(cls + (amp == 1 ? 0 : amp <= nadir ? 1 : 2), 1);
}

}  // namespace

extern "C" {

casim_status casim_b200_qs_create(const char* json_text, const char* base_dir, int32_t n_scenarios, const uint32_t* seeds,
                                  int64_t max_events, casim_qs* out) {
    if (!json_text || !out || n_scenarios < 1 || max_events < 1) return qs_fail(nullptr, CASIM_EINVAL, "qs_create: bad argument");
    *out = nullptr;
    auto* h = new casim_qs_s();
    try {
        json file;
        try {
            file = json::parse(json_text);
        } catch (const std::exception& e) {
            throw qs_error(CASIM_EINVAL, std::string("JSON: ") + e.what());
        }
        if (!file.contains("Calcium Release Site")) throw qs_error(CASIM_EINVAL, "missing \"Calcium Release Site\"");
        const json& crs = file["Calcium Release Site"];
        const std::string name = crs.value("Name", std::string("LinearNaraghiNeher"));
        if (name != "LinearNaraghiNeher") throw qs_error(CASIM_EUNSUPPORTED, "stationary model \"" + name + "\" is not built");
        h->max_time = jnum(crs, "Max Time", "Calcium Release Site");
        const json& par = crs.at("Parameters");
        const json& chs = par.at("Channels");
        if (chs.size() != 1) throw qs_error(CASIM_EINVAL, "stationary diffusion models take exactly one ion channel");
        const json& ch = chs.begin().value();
        const std::string model = ch.at("Model").get<std::string>();
        const json cp = ch.contains("Parameters") ? ch.at("Parameters") : json::object();
        auto P = [&](const char* k) { return jnum(cp, k, "Channels.Parameters"); };
        std::vector<double> v;
        if (model == "TwoStateMWC") {
            h->m.ch_model = CB_TWO_STATE_MWC;
            v = {P("fCa"), P("KCa"), P("fMg"), P("KMg"), P("KO0"), P("KMgI"), P("kclose")};
        } else if (model == "TwoStateaHTG") {
            h->m.ch_model = CB_TWO_STATE_AHTG;
            v = {P("fCa"), P("KCa"), P("fMg"), P("KMg"), P("KO0"), P("KMgI"), P("KCL"), P("KI"), P("KOL"), P("kclose")};
        } else if (model == "SheepCannell") {
            h->m.ch_model = CB_SHEEP_CANNELL;
            v = {P("kopen0"), P("ncaopen"), P("kopenmax"), P("kclose0"), P("ncaclose")};
        } else {
            throw qs_error(CASIM_EUNSUPPORTED, "gating model \"" + model + "\" is not built for quasi-stationary sites "
                                              "(TwoStateMWC, TwoStateaHTG, SheepCannell)");
        }
        for (size_t k = 0; k < v.size(); ++k) h->m.ch_par[k] = v[k];
        h->m.ca_idx = 0;
        h->m.mg_idx = 1;
        // channel positions (nm)
        std::string cf = ch.at("Coordinates").get<std::string>();
        if (base_dir && *base_dir && !cf.empty() && cf[0] != '/') cf = std::string(base_dir) + "/" + cf;
        std::ifstream in(cf);
        if (!in) throw qs_error(CASIM_EINVAL, "cannot read coordinates \"" + cf + "\"");
        std::vector<double> px, py;
        double x, y;
        while (in >> x >> y) {
            px.push_back(x);
            py.push_back(y);
        }
        if (px.empty() || px.size() > 1024) throw qs_error(CASIM_EINVAL, "1 to 1024 channels are supported");
        h->n_ch = (int)px.size();
        const json& cleft = par.at("Dyadic Cleft");
        const json& ions = cleft.at("Ions");
        h->bg = jnum(ions.at("Calcium"), "Concentration", "Ions.Calcium");
        const double dca = jnum(ions.at("Calcium"), "D", "Ions.Calcium");
        h->mg = ions.contains("Magnesium") ? jnum(ions.at("Magnesium"), "Concentration", "Ions.Magnesium") : 0.0;
        if (h->m.ch_model != CB_SHEEP_CANNELL && !ions.contains("Magnesium"))
            throw qs_error(CASIM_EINVAL, "gating model " + model + " needs a Magnesium ion");
        std::vector<double> kon, koff, D, tot;
        if (cleft.contains("Buffers"))
            for (auto& el : cleft.at("Buffers").items()) {  // name order, as the reference's std::map
                kon.push_back(jnum(el.value(), "kon", "Buffers"));
                koff.push_back(jnum(el.value(), "koff", "Buffers"));
                D.push_back(jnum(el.value(), "D", "Buffers"));
                tot.push_back(jnum(el.value(), "Total Concentration", "Buffers"));
            }
        h->added = naraghi_neher(kon, koff, D, tot, h->bg, dca, jnum(ch, "Current", "Channels"), jnum(par, "Open Concentration", "Parameters"),
                                 px, py);
        h->n_scen = n_scenarios;
        h->max_events = max_events;
        h->seeds.resize((size_t)6 * n_scenarios);
        if (seeds) {
            for (int s = 0; s < n_scenarios; ++s) {
                uint64_t s6[6];
                for (int q = 0; q < 6; ++q) s6[q] = seeds[6 * s + q];
                if (!cbrng::seed_ok(s6)) throw qs_error(CASIM_EINVAL, "seed of scenario " + std::to_string(s) + " is not a valid MRG32k3a seed");
                for (int q = 0; q < 6; ++q) h->seeds[6 * s + q] = (uint32_t)s6[q];
            }
        } else {
            // scenario s draws from stream s of the package seed 12345 x 6 (2^127 apart)
            cbrng::State g;
            for (int q = 0; q < 6; ++q) g.s[q] = 12345u;
            for (int s = 0; s < n_scenarios; ++s) {
                for (int q = 0; q < 6; ++q) h->seeds[6 * s + q] = g.s[q];
                cbrng::jump_pow2(g, 127, 1);
            }
        }
    } catch (const qs_error& e) {
        casim_b200_qs_destroy(h);
        return qs_fail(nullptr, e.code, e.what());
    } catch (const std::exception& e) {
        casim_b200_qs_destroy(h);
        return qs_fail(nullptr, CASIM_EINVAL, e.what());
    }
    *out = h;
    return CASIM_OK;
}

casim_status casim_b200_qs_destroy(casim_qs h) {
    if (!h) return CASIM_OK;
    if (!h->stream) {  // never ran: nothing on the device
        delete h;
        return CASIM_OK;
    }
    cudaStreamSynchronize(h->stream);
    cudaFree(h->d_added);
    cudaFree(h->d_seed);
    cudaFree(h->d_first);
    cudaFree(h->d_t);
    cudaFree(h->d_ev);
    cudaFree(h->d_nev);
    cudaFree(h->d_draws);
    cudaFree(h->d_flags);
    cudaFree(h->d_next);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return CASIM_OK;
}

casim_status casim_b200_qs_last_error(casim_qs h, char* buf, size_t n) {
    if (!buf || !n) return CASIM_EINVAL;
    const std::string& e = h ? h->err : g_qs_create_err;
    const size_t k = std::min(n - 1, e.size());
    std::memcpy(buf, e.data(), k);
    buf[k] = 0;
    return CASIM_OK;
}

casim_status casim_b200_qs_info(casim_qs h, int32_t* n_channels, int32_t* n_scenarios, double* max_time) {
    if (!h) return CASIM_EINVAL;
    if (n_channels) *n_channels = h->n_ch;
    if (n_scenarios) *n_scenarios = h->n_scen;
    if (max_time) *max_time = h->max_time;
    return CASIM_OK;
}

casim_status casim_b200_qs_increments(casim_qs h, double* out) {
    if (!h || !out) return CASIM_EINVAL;
    std::memcpy(out, h->added.data(), sizeof(double) * h->added.size());
    return CASIM_OK;
}

casim_status casim_b200_qs_run(casim_qs h, const int32_t* first_channel) {
    if (!h || !first_channel) return CASIM_EINVAL;
    for (int s = 0; s < h->n_scen; ++s)
        if (first_channel[s] < 0 || first_channel[s] >= h->n_ch) return qs_fail(h, CASIM_EINVAL, "first channel out of range");
    try {
        if (!h->stream) {
            // device state on the first run (creating a handle needs no device)
            ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            ck(cudaEventCreate(&h->ev0), "cudaEventCreate");
            ck(cudaEventCreate(&h->ev1), "cudaEventCreate");
            const size_t S = (size_t)h->n_scen;
            ck(cudaMalloc(&h->d_added, sizeof(double) * h->added.size()), "cudaMalloc");
            ck(cudaMalloc(&h->d_seed, sizeof(uint32_t) * 6 * S), "cudaMalloc");
            ck(cudaMalloc(&h->d_first, sizeof(int) * S), "cudaMalloc");
            ck(cudaMalloc(&h->d_t, sizeof(double) * S * h->max_events), "cudaMalloc");
            ck(cudaMalloc(&h->d_ev, sizeof(int) * S * h->max_events), "cudaMalloc");
            ck(cudaMalloc(&h->d_nev, sizeof(long long) * S), "cudaMalloc");
            ck(cudaMalloc(&h->d_draws, sizeof(unsigned long long) * S), "cudaMalloc");
            ck(cudaMalloc(&h->d_flags, sizeof(int) * S), "cudaMalloc");
            ck(cudaMalloc(&h->d_next, sizeof(int)), "cudaMalloc");
            ck(cudaMemcpy(h->d_added, h->added.data(), sizeof(double) * h->added.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
            ck(cudaMemcpy(h->d_seed, h->seeds.data(), sizeof(uint32_t) * 6 * S, cudaMemcpyHostToDevice), "cudaMemcpy");
        }
        ck(cudaMemcpyAsync(h->d_first, first_channel, sizeof(int) * h->n_scen, cudaMemcpyHostToDevice, h->stream), "cudaMemcpy");
        // up to 32 RyRs: a scenario per lane; more: a scenario per warp
        const bool lane = h->n_ch <= 32;
        const size_t smem = lane ? qsl_smem(h->n_ch) : QS_WARPS * qs_warp_bytes(h->n_ch);
        const qs_kernel_t kern = qs_kernel(h->m.ch_model, lane);
        if (smem > 48 * 1024) ck(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "cudaFuncSetAttribute");
        if (!h->grid) {
            int dev = 0, sms = 0, per_sm = 0;
            ck(cudaGetDevice(&dev), "cudaGetDevice");
            ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
            ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * QS_WARPS, smem), "cudaOccupancy");
            h->grid = std::max(1, sms * per_sm);
        }
        // one scenario per lane: as many resident lanes as the batch fills (a warp runs until
        // its longest scenario ends, so large batches, several scenarios per lane, balance best)
        const int blocks = std::min(h->grid, lane ? (h->n_scen + 32 * QSL_WARPS - 1) / (32 * QSL_WARPS)
                                                  : (h->n_scen + QS_WARPS - 1) / QS_WARPS);
        ck(cudaMemsetAsync(h->d_next, 0, sizeof(int), h->stream), "cudaMemsetAsync");
        ck(cudaEventRecord(h->ev0, h->stream), "cudaEventRecord");
        kern<<<blocks, 32 * QS_WARPS, smem, h->stream>>>(h->m, h->n_ch, h->d_added, h->bg, h->mg, h->max_time, h->n_scen, h->d_first,
                                                         h->d_seed, h->max_events, h->d_t, h->d_ev, h->d_nev, h->d_draws, h->d_flags,
                                                         h->d_next);
        ck(cudaGetLastError(), "k_qs_run");
        ck(cudaEventRecord(h->ev1, h->stream), "cudaEventRecord");
        ck(cudaStreamSynchronize(h->stream), "k_qs_run");
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "cudaEventElapsedTime");
        h->last_ms = ms;
        h->ran = true;
        std::vector<int> flags(h->n_scen);
        ck(cudaMemcpy(flags.data(), h->d_flags, sizeof(int) * h->n_scen, cudaMemcpyDeviceToHost), "cudaMemcpy");
        // a scenario stopped at the cap outranks one whose trace was only truncated
        int capped = -1, truncated = -1;
        for (int s = h->n_scen - 1; s >= 0; --s) {
            if (flags[s] & 2) capped = s;
            if (flags[s] & 1) truncated = s;
        }
        if (capped >= 0)
            return qs_fail(h, CASIM_ETIMEOUT, "scenario " + std::to_string(capped) + " reached 64 x max_events events before its "
                                              "end; it was stopped there");
        if (truncated >= 0)
            return qs_fail(h, CASIM_EUNSUPPORTED, "scenario " + std::to_string(truncated) + " had more events than max_events; "
                                                  "its trace is truncated (the run itself is complete)");
    } catch (const qs_error& e) {
        return qs_fail(h, e.code, e.what());
    }
    return CASIM_OK;
}

casim_status casim_b200_qs_last_run_ms(casim_qs h, double* out) {
    if (!h || !out) return CASIM_EINVAL;
    *out = h->last_ms;
    return CASIM_OK;
}

casim_status casim_b200_qs_event_count(casim_qs h, int32_t scenario, int64_t* n) {
    if (!h || !n || scenario < 0 || scenario >= h->n_scen) return CASIM_EINVAL;
    if (!h->ran) return qs_fail(h, CASIM_EINVAL, "no run yet");
    long long v = 0;
    if (cudaMemcpy(&v, h->d_nev + scenario, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return qs_fail(h, CASIM_ECUDA, "cudaMemcpy");
    *n = v;
    return CASIM_OK;
}

casim_status casim_b200_qs_events(casim_qs h, int32_t scenario, double* t, int32_t* channel, int32_t* state) {
    if (!h || scenario < 0 || scenario >= h->n_scen) return CASIM_EINVAL;
    int64_t n = 0;
    casim_status s = casim_b200_qs_event_count(h, scenario, &n);
    if (s != CASIM_OK) return s;
    n = std::min<int64_t>(n, h->max_events);
    std::vector<double> tt(n);
    std::vector<int> cc(n);
    const size_t off = (size_t)scenario * h->max_events;
    if (cudaMemcpy(tt.data(), h->d_t + off, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(cc.data(), h->d_ev + off, sizeof(int) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return qs_fail(h, CASIM_ECUDA, "cudaMemcpy");
    for (int64_t k = 0; k < n; ++k) {
        if (t) t[k] = tt[k];
        if (channel) channel[k] = cc[k] & ((1 << 30) - 1);
        if (state) state[k] = cc[k] >> 30;
    }
    return CASIM_OK;
}

casim_status casim_b200_qs_draws(casim_qs h, int32_t scenario, uint64_t* out) {
    if (!h || !out || scenario < 0 || scenario >= h->n_scen) return CASIM_EINVAL;
    unsigned long long v = 0;
    if (cudaMemcpy(&v, h->d_draws + scenario, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return qs_fail(h, CASIM_ECUDA, "cudaMemcpy");
    *out = v;
    return CASIM_OK;
}

casim_status casim_b200_qs_analysis(casim_qs h, int32_t nadir, double* per_scenario, int32_t* class_counts) {
    if (!h || !per_scenario || !class_counts) return CASIM_EINVAL;
    if (!h->ran) return qs_fail(h, CASIM_EINVAL, "no run yet");
    double* d_out = nullptr;
    int* d_cls = nullptr;
    try {
        ck(cudaMalloc(&d_out, sizeof(double) * 5 * h->n_scen), "cudaMalloc");
        ck(cudaMalloc(&d_cls, sizeof(int) * 3), "cudaMalloc");
        ck(cudaMemsetAsync(d_cls, 0, sizeof(int) * 3, h->stream), "cudaMemset");
        k_qs_metrics<<<(h->n_scen + 127) / 128, 128, 0, h->stream>>>(h->n_scen, h->max_events, h->d_t, h->d_ev, h->d_nev, nadir, d_out, d_cls);
        ck(cudaGetLastError(), "k_qs_metrics");
        ck(cudaMemcpyAsync(per_scenario, d_out, sizeof(double) * 5 * h->n_scen, cudaMemcpyDeviceToHost, h->stream), "cudaMemcpy");
        ck(cudaMemcpyAsync(class_counts, d_cls, sizeof(int) * 3, cudaMemcpyDeviceToHost, h->stream), "cudaMemcpy");
        ck(cudaStreamSynchronize(h->stream), "k_qs_metrics");
    } catch (const qs_error& e) {
        cudaFree(d_out);
        cudaFree(d_cls);
        return qs_fail(h, e.code, e.what());
    }
    cudaFree(d_out);
    cudaFree(d_cls);
    return CASIM_OK;
}

}  // extern "C"
