/*
 * Driver around the reference's OWN quasi-stationary release site
 * (CaSim/QuasyStationaryReleaseSite.cpp, CaSim/StationaryDiffusionModel.cpp, the
 * two-state models, CaSim/ParallelRng.cpp), compiled in place by oracle/Makefile.
 * Test infrastructure only.
 *
 * The reference's LinearNaraghiNeher constructor needs Eigen, which is absent; this
 * file stands in for that one constructor: it installs increments given by the
 * caller (qsref_set_increments, computed by the CPU restatement), so that the
 * Gillespie loop, the rate laws and the RNG consumption that run are the
 * reference's own (CaSim/QuasyStationaryReleaseSite.cpp:89-133). One ParallelRng
 * with the given package seed, scenarios run one after another on one thread, as a
 * one-thread ParallelSolver does (CaSim/ParallelSolver.cpp:51-70).
 */
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "LinearNaraghiNeher.h"
#include "QuasyStationaryReleaseSite.h"

namespace {
std::vector<std::vector<double>> g_increments;
thread_local std::string g_qs_err;
}  // namespace

LinearNaraghiNeher::LinearNaraghiNeher(std::map<std::string, std::map<std::string, double>>&, std::vector<std::shared_ptr<Point>>&,
                                       double, double ca_0, double, double) {
    background = ca_0;
    added_concentrations = g_increments;
}

extern "C" {

void qsref_set_increments(int n, const double* a) {
    g_increments.assign(n, std::vector<double>(n));
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) g_increments[i][j] = a[(long)i * n + j];
}

const char* qsref_last_error() { return g_qs_err.c_str(); }

// runs n_scen scenarios (scenario k opens first[k]); for each: the channel-state rows
// (t, states...) as the reference records them. Returns the total number of rows, or -1.
long qsref_run(const char* json_text, const unsigned long* seed6, int n_scen, const int* first, double* rows_t, int* rows_states,
               int* rows_per_scen, long max_rows) {
    try {
        auto file = nlohmann::json::parse(json_text);
        QuasyStationaryReleaseSite site(file);
        unsigned long s6[6];
        for (int i = 0; i < 6; ++i) s6[i] = seed6[i];
        ParallelRng rng(s6);
        const int nc = site.GetNChannels();
        long total = 0;
        for (int k = 0; k < n_scen; ++k) {
            datavector ch, dc, lumen, cyt;
            site.RunSimulation(ch, dc, lumen, cyt, first[k], &rng);
            const auto& rows = ch.begin()->second;
            rows_per_scen[k] = (int)rows.size();
            for (const auto& r : rows) {
                if (total < max_rows) {
                    rows_t[total] = r[0];
                    for (int c = 0; c < nc; ++c) rows_states[total * nc + c] = (int)r[c + 1];
                }
                ++total;
            }
        }
        return total;
    } catch (const std::exception& e) {
        g_qs_err = e.what();
        return -1;
    }
}

}  // extern "C"
