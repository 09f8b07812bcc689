/*
 * C API around the reference's OWN CPU classes, compiled from the sources
 * where they lie (see oracle/Makefile). Test infrastructure only: it lets the
 * tests and the CPU-baseline leg of the benchmark drive the unmodified
 * reference hot path without HDF5.
 *
 * The driver restates only the orchestration of ParallelHybridSolver, which
 * cannot be compiled here (it needs H5Cpp.h):
 *   compartment construction  CaSim/ParallelHybridSolver.cpp:13-131
 *   ResetSystem               CaSim/ParallelHybridSolver.cpp:149-157
 *   Update                    CaSim/ParallelHybridSolver.cpp:159-175
 *   one loop iteration        CaSim/ParallelHybridSolver.cpp:421-429 (RunSimulationsCPU)
 *   initial channel choice    CaSim/ParallelHybridSolver.cpp:411-417
 * Everything numeric runs inside the reference classes themselves.
 */
#include <nlohmann/json.hpp>
#include <omp.h>
#include <cstring>
#include <string>
#include <vector>
#include <memory>

#include "NSRConstPool.h"
#include "SRPool.h"
#include "CytosolPool.h"
#include "DyadRD2DCPU.h"
#include "DyadRDCPU.h"

using json = nlohmann::json;

namespace {

struct RefSim {
    json file;
    int n_threads = 1;
    int n_cores = 1;
    double dt = 0;
    double V = 0;
    std::unique_ptr<NSRSeries> nsr;
    std::unique_ptr<SRSeries> sr;
    std::unique_ptr<DyadSeries> dyad;
    std::unique_ptr<CytosolSeries> cytosol;
    std::string err;
};

thread_local std::string g_err;

long copy_out(const std::vector<double>& v, double* out, long n) {
    if (out) {
        long m = (long)v.size() < n ? (long)v.size() : n;
        std::memcpy(out, v.data(), sizeof(double) * (size_t)m);
    }
    return (long)v.size();
}

}  // namespace

extern "C" {

const char* casimref_last_error() { return g_err.c_str(); }

void* casimref_create(const char* json_text, int n_batch, int n_cores) {
    try {
        auto s = std::make_unique<RefSim>();
        s->file = json::parse(json_text);
        json& file = s->file;
        s->n_threads = n_batch;
        s->n_cores = n_cores > 0 ? n_cores : 1;
        double dt = file["dt, ns"];
        s->dt = dt * 1e-6;
        if (file["nSR"]["Type"] == "ConstPool")
            s->nsr = std::make_unique<NSRConstPool>(file["nSR"], n_batch);
        std::string dtype = file["Dyad"]["Type"];
        if (dtype == "CPU3D" || dtype == "3D")
            s->dyad = std::make_unique<DyadRDCPU>(file["Dyad"], file["jSR"], n_batch);
        else
            s->dyad = std::make_unique<DyadRD2DCPU>(file["Dyad"], file["jSR"], n_batch);
        if (file["nSR"]["Type"] == "ConstPool")
            s->cytosol = std::make_unique<CytosolPool>(file["Cytosol"], file["Dyad"], file["nSR"], n_batch);
        else
            s->cytosol = std::make_unique<CytosolPool>(file["Cytosol"], file["Dyad"], n_batch);
        s->dyad->IsCytosolGPU(s->cytosol->UsesGPU());
        s->sr = std::make_unique<SRPool>(file["jSR"], n_batch, s->dyad->GetElementVolume(),
                                         s->dyad->GetNumSRChannels(), s->dyad->GetListofIons());
        return s.release();
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void casimref_destroy(void* h) { delete static_cast<RefSim*>(h); }

int casimref_num_channels(void* h) { return static_cast<RefSim*>(h)->dyad->GetNumSRChannels(); }

double casimref_element_volume(void* h) { return static_cast<RefSim*>(h)->dyad->GetElementVolume(); }

int casimref_dims(void* h, long* out, int n) {
    auto d = static_cast<RefSim*>(h)->dyad->GetDimensions();
    for (int i = 0; i < n && i < (int)d.size(); ++i) out[i] = (long)d[i];
    return (int)d.size();
}

void casimref_reset(void* h) {
    auto* s = static_cast<RefSim*>(h);
    s->nsr->Reset();
    s->sr->Reset();
    s->dyad->Reset();
    s->cytosol->Reset();
}

void casimref_init_opening(void* h, int site, int channel) {
    static_cast<RefSim*>(h)->dyad->InitOpening(site, channel);
}

void casimref_update(void* h) {
    auto* s = static_cast<RefSim*>(h);
    double* ions_cyto = nullptr;
    double* bufs_cyto = nullptr;
    double* currents = nullptr;
    s->cytosol->GetIonsBuffersandV(ions_cyto, bufs_cyto, s->V);
    s->dyad->Update(ions_cyto, bufs_cyto, s->sr->GetIons(), s->cytosol->GetExtraCellularIons(), s->V);
    s->dyad->GetEffluxes(currents);
    s->cytosol->Update(currents, s->nsr->GetIons());
    s->sr->Update(s->dyad->GetTotalSRCurrent(), s->nsr->GetIons());
    s->nsr->Update(ions_cyto, s->sr->GetIons());
}

/* ResetSystem + InitOpening for every site + Update, as at the start of each
 * batch in RunSimulationsCPU. first_channel[k] is the channel forced open in
 * site k. */
void casimref_start(void* h, const int* first_channel) {
    auto* s = static_cast<RefSim*>(h);
    casimref_reset(h);
    for (int k = 0; k < s->n_threads; ++k) s->dyad->InitOpening(k, first_channel[k]);
    casimref_update(h);
}

void casimref_step(void* h, long n_steps) {
    auto* s = static_cast<RefSim*>(h);
    const int nt = s->n_threads;
    const double dt = s->dt;
    for (long it = 0; it < n_steps; ++it) {
#pragma omp parallel for num_threads(s->n_cores)
        for (int k = 0; k < nt; ++k) {
            s->cytosol->RunRD(dt, k);
            s->dyad->RunRD(dt, k);
            s->sr->Run(dt, k);
            s->dyad->RunMC(dt, k);
        }
        casimref_update(h);
    }
}

/* what: "dyad:<species>" (reference field layout), "cyto:<species>",
 * "mouth:<ion>" (GetIonsNearChannels), "sr" (jSR ions, SRPool layout),
 * "efflux", "total_sr_current". Returns the full length; copies min(len, n). */
long casimref_get(void* h, const char* what, double* out, long n) {
    auto* s = static_cast<RefSim*>(h);
    std::string w(what);
    try {
        if (w.rfind("dyad:", 0) == 0) {
            std::vector<std::string> names{w.substr(5)};
            // GetConcentrations is keyed by ion name or by buffer name
            auto m = s->dyad->GetConcentrations(names);
            auto it = m.find(w.substr(5));
            if (it != m.end()) return copy_out(it->second, out, n);
            return -1;
        }
        if (w.rfind("dyadbuf:", 0) == 0) {
            // "dyadbuf:<buffer>|<ion>-<buffer>"
            std::string rest = w.substr(8);
            auto bar = rest.find('|');
            std::vector<std::string> names{rest.substr(0, bar)};
            auto m = s->dyad->GetConcentrations(names);
            auto it = m.find(rest.substr(bar + 1));
            if (it != m.end()) return copy_out(it->second, out, n);
            return -1;
        }
        if (w.rfind("cyto:", 0) == 0) {
            std::vector<std::string> names{w.substr(5)};
            auto m = s->cytosol->GetConcentrations(names);
            auto it = m.find(w.substr(5));
            if (it != m.end()) return copy_out(it->second, out, n);
            return -1;
        }
        if (w.rfind("cytobuf:", 0) == 0) {
            std::string rest = w.substr(8);
            auto bar = rest.find('|');
            std::vector<std::string> names{rest.substr(0, bar)};
            auto m = s->cytosol->GetConcentrations(names);
            auto it = m.find(rest.substr(bar + 1));
            if (it != m.end()) return copy_out(it->second, out, n);
            return -1;
        }
        if (w.rfind("mouth:", 0) == 0) {
            std::vector<std::string> names;
            auto m = s->dyad->GetIonsNearChannels(names);
            auto it = m.find(w.substr(6));
            if (it != m.end()) return copy_out(it->second, out, n);
            return -1;
        }
        if (w == "sr") return copy_out(s->sr->GetIons(), out, n);
        if (w == "total_sr_current") return copy_out(s->dyad->GetTotalSRCurrent(), out, n);
        if (w == "efflux") {
            double* p = nullptr;
            s->dyad->GetEffluxes(p);
            // length: (n_ions + n_ion_buffer_pairs) * n_threads; the caller passes it
            if (out && p) std::memcpy(out, p, sizeof(double) * (size_t)n);
            return n;
        }
    } catch (const std::exception& e) {
        g_err = e.what();
    }
    return -1;
}

long casimref_get_states(void* h, int* out, long n) {
    auto* s = static_cast<RefSim*>(h);
    std::vector<std::string> names;
    auto m = s->dyad->GetChannelsStates(names);
    auto& v = m["RyR"];
    long c = (long)v.size() < n ? (long)v.size() : n;
    if (out) std::memcpy(out, v.data(), sizeof(int) * (size_t)c);
    return (long)v.size();
}

}  // extern "C"

#include "rngstream.h"
extern "C" void casimref_rng_draws(const unsigned long* seed6, long n, double* out) {
    /* the reference's own RngStream (CaSim/rngstream.cpp): package seed, first stream */
    RngStream::SetPackageSeed(seed6);
    RngStream g;
    for (long k = 0; k < n; ++k) out[k] = g.RandU01();
}

// The reference's own release analysis (CaSim/IndChannelCREAnalyzer.cpp:53-138) over
// n_scen traces given as events: times [sum(n_events)] and the open (1) / closed (0)
// state of each of n_ch channels per event [sum(n_events)][n_ch]. Two-state channels:
// the state-to-open map of every channel is {0, 1}. It writes dir/analysis/*.txt.
#include "IndChannelCREAnalyzer.h"
#undef min
#undef max
extern "C" int casimref_cre_analysis(const char* dir, int n_scen, const int* n_events, const double* times, const int* states,
                                     int n_ch, double max_time, int nadir) {
    try {
        std::vector<std::vector<std::vector<double>>> data(n_scen);
        long q = 0;
        for (int i = 0; i < n_scen; ++i) {
            data[i].resize(n_events[i]);
            for (int j = 0; j < n_events[i]; ++j, ++q) {
                std::vector<double> row(1 + n_ch);
                row[0] = times[q];
                for (int c = 0; c < n_ch; ++c) row[1 + c] = states[q * n_ch + c];
                data[i][j] = row;
            }
        }
        std::vector<std::vector<int>> channels(n_ch, std::vector<int>{0, 1});
        std::string name(dir);
        IndChannelCREAnalyzer a;
        a.RunAnalysis(name, data, channels, max_time, 1, nadir);  // one thread: its class counters are not atomic
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}
