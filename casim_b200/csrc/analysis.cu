// Decimated open-RyR traces and the release-event analysis on the device.
//
// The reference keeps the channel states of every output step on the host (HDF5,
// CaSim/ParallelHybridSolver.cpp:316-337) and analyses the traces there with
// IndChannelCREAnalyzer::RunAnalysis (CaSim/IndChannelCREAnalyzer.cpp:53-138): per
// trace the amplitude (largest number of open RyRs), the time to peak, the time to end,
// the integral of the open count and its mean, and time histograms of the open count
// over all traces and over quarks (amplitude 1), blips (amplitude <= nadir) and sparks.
// Here the open count of every site is recorded on the device every `every` time steps
// (u16 per site and sample), and the analysis runs on the recorded samples with the
// reference's arithmetic: sample j at t_j = j * Ts, histogram bins of width hd, bin
// index (long long)(t / hd), the last interval of a trace empty, column 0 of each
// histogram replaced by the class count minus the other columns
// (CaSim/IndChannelCREAnalyzer.cpp:23-40).
#include "engine.h"

namespace {

// open RyRs of every site into sample j: a warp per site
__global__ void k_trace_record(const cb_site* __restrict__ sites, const int* __restrict__ ch_state, int S, uint16_t* __restrict__ trace,
                               long long max_samples, long long j) {
    const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (s >= S) return;
    const cb_site st = sites[s];
    int n = 0;
    for (int c = lane; c < st.n_ch; c += 32) n += ch_state[st.ch_off + c] != 0;
    n = __reduce_add_sync(0xffffffffu, n);
    if (lane == 0) trace[(size_t)s * max_samples + j] = (uint16_t)n;
}

// per site, in sample order (CaSim/IndChannelCREAnalyzer.cpp:71-83, 120-122):
// amp, ttp, tte, integral of the open count, its mean; and the site's class
__global__ void k_cre_metrics(const uint16_t* __restrict__ trace, int S, long long max_samples, long long n, double ts, int nadir,
                              double* __restrict__ out, int* __restrict__ cls, int* __restrict__ counts) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const uint16_t* tr = trace + (size_t)s * max_samples;
    double amp = 0, ttp = 0, q = 0;
    for (long long j = 0; j < n; ++j) {
        const int no = tr[j];
        const double t = (double)j * ts;
        if (no > amp) {
            amp = no;
            ttp = t;
        }
        const long long nx = j + 1 < n ? j + 1 : n - 1;
        q += no * ((double)nx * ts - t);
    }
    const double tte = (double)(n - 1) * ts;
    double* o = out + (size_t)s * 5;
    o[0] = amp;
    o[1] = ttp;
    o[2] = tte;
    o[3] = q;
    o[4] = q / tte;
    const int c = amp == 1 ? 0 : amp <= nadir ? 1 : 2;
    cls[s] = c;
    atomicAdd(counts + c, 1);
}

// sample j of site s fills bins [cur, end] at its open count
// (CaSim/IndChannelCREAnalyzer.cpp:17-21, 78-82)
__global__ void k_cre_hist(const uint16_t* __restrict__ trace, int S, long long max_samples, long long n, double ts, double hd,
                           long long nh, int mch, int nadir, const int* __restrict__ cls, int* __restrict__ h_all,
                           int* __restrict__ h_q, int* __restrict__ h_b, int* __restrict__ h_s) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (long long)S * n) return;
    const int s = (int)(g / n);
    const long long j = g - (long long)s * n;
    const int no = trace[(size_t)s * max_samples + j];
    const long long cur = j == 0 ? 0 : (long long)((double)j * ts / hd) + 1;
    const long long nx = j + 1 < n ? j + 1 : n - 1;
    long long end = (long long)((double)nx * ts / hd);
    if (end > nh) end = nh;
    const int c = cls[s];
    int* hc = c == 0 ? h_q : c == 1 ? h_b : h_s;
    const int wc = c == 0 ? 2 : c == 1 ? nadir + 1 : mch + 1;
    for (long long k = cur; k <= end; ++k) {
        atomicAdd(h_all + k * (mch + 1) + no, 1);
        atomicAdd(hc + k * wc + no, 1);
    }
}

// column 0: the class's traces minus those counted in the other columns
// (CaSim/IndChannelCREAnalyzer.cpp:32-38)
__global__ void k_cre_zero_column(int* __restrict__ h, long long rows, int w, const int* __restrict__ count, int total) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    int* r = h + i * w;
    int t = 0;
    for (int k = 1; k < w; ++k) t += r[k];
    r[0] = (count ? *count : total) - t;
}

}  // namespace

cudaError_t cb_trace_record(const cb_dev& d, uint16_t* trace, long long max_samples, long long j, cudaStream_t st) {
    if (j < 0 || j >= max_samples) return cudaErrorInvalidValue;
    k_trace_record<<<(d.S + 7) / 8, 256, 0, st>>>(d.sites, d.ch_state, d.S, trace, max_samples, j);
    return cudaGetLastError();
}

cudaError_t cb_cre_analysis(const cb_dev& d, const uint16_t* trace, long long max_samples, long long n, double ts, double hd,
                            long long nh, int nadir, double* per_site, int* cls, int* h_all, int* h_q, int* h_b, int* h_s,
                            int* counts, cudaStream_t st) {
    const int mch = d.max_ch;
    cudaError_t e;
    if ((e = cudaMemsetAsync(counts, 0, 3 * sizeof(int), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(h_all, 0, (size_t)(nh + 1) * (mch + 1) * sizeof(int), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(h_q, 0, (size_t)(nh + 1) * 2 * sizeof(int), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(h_b, 0, (size_t)(nh + 1) * (nadir + 1) * sizeof(int), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(h_s, 0, (size_t)(nh + 1) * (mch + 1) * sizeof(int), st)) != cudaSuccess) return e;
    k_cre_metrics<<<(d.S + 127) / 128, 128, 0, st>>>(trace, d.S, max_samples, n, ts, nadir, per_site, cls, counts);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const long long work = (long long)d.S * n;
    k_cre_hist<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(trace, d.S, max_samples, n, ts, hd, nh, mch, nadir, cls, h_all, h_q,
                                                                 h_b, h_s);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const unsigned gb = (unsigned)((nh + 1 + 127) / 128);
    k_cre_zero_column<<<gb, 128, 0, st>>>(h_all, nh + 1, mch + 1, nullptr, d.S);
    k_cre_zero_column<<<gb, 128, 0, st>>>(h_q, nh + 1, 2, counts + 0, 0);
    k_cre_zero_column<<<gb, 128, 0, st>>>(h_b, nh + 1, nadir + 1, counts + 1, 0);
    k_cre_zero_column<<<gb, 128, 0, st>>>(h_s, nh + 1, mch + 1, counts + 2, 0);
    return cudaGetLastError();
}
