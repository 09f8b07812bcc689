/*
 * Test driver for include/casim_b200_dyad_series.hpp (test infrastructure, never
 * the product): compiles the DyadRDB200 adapter against the reference's own
 * DyadSeries.h (CaSim/DyadSeries.h:9-44) and drives one batch through it the way
 * ParallelHybridSolver drives a dyad (CaSim/ParallelHybridSolver.cpp:373-405,
 * with the B200 dyad owning the pools): ResetSystem, InitOpening per site, Update,
 * then per time step RunRD(dt, 0), RunMC per site and Update; then reads the
 * outputs through the DyadSeries getters.
 */
#include <cstring>
#include <string>
#include <vector>

#include "casim_b200_dyad_series.hpp"

extern "C" int adapter_run(const char* json_text, const char* base_dir, int n_batch, int n_steps, const int* first,
                           double* ca_out, int* states_out, double* mouth_out, double* total_out, double* efflux_out,
                           double* scalars_out, char* err, int n_err) {
    try {
        nlohmann::json j = nlohmann::json::parse(json_text);
        DyadSeries* dyad = new DyadRDB200(j, n_batch, base_dir);
        const double dt = (double)j["dt, ns"] * 1e-6;
        double* ions_cyto = nullptr;
        double* bufs_cyto = nullptr;
        double V = 0;
        const std::vector<double> jsr, extracell;
        dyad->IsCytosolGPU(true);
        dyad->Reset();
        for (int k = 0; k < n_batch; ++k) dyad->InitOpening(k, first[k]);
        dyad->Update(ions_cyto, bufs_cyto, jsr, extracell, V);
        for (int s = 1; s <= n_steps; ++s) {
            dyad->RunRD(dt, 0);
            for (int k = 0; k < n_batch; ++k) dyad->RunMC(dt, k);
            dyad->Update(ions_cyto, bufs_cyto, jsr, extracell, V);
        }
        std::vector<std::string> names{"Calcium"};
        auto conc = dyad->GetConcentrations(names).at("Calcium");
        std::memcpy(ca_out, conc.data(), sizeof(double) * conc.size());
        auto st = dyad->GetChannelsStates(names).at("RyR");
        std::memcpy(states_out, st.data(), sizeof(int) * st.size());
        auto mo = dyad->GetIonsNearChannels(names).at("Calcium");
        std::memcpy(mouth_out, mo.data(), sizeof(double) * mo.size());
        auto tc = dyad->GetTotalSRCurrent();
        std::memcpy(total_out, tc.data(), sizeof(double) * tc.size());
        double* ef = nullptr;
        dyad->GetEffluxes(ef);
        std::memcpy(efflux_out, ef, sizeof(double) * dyad->GetListofIons().size() * n_batch);
        auto dims = dyad->GetDimensions();
        scalars_out[0] = dyad->GetNumSRChannels();
        scalars_out[1] = dyad->UsesGPU() ? 1 : 0;
        scalars_out[2] = dyad->GetElementVolume();
        scalars_out[3] = dyad->GetL();
        scalars_out[4] = (double)dyad->GetListofIons().size();
        scalars_out[5] = (double)dims.size();
        scalars_out[6] = dims.size() > 3 ? (double)(dims[2] * dims[3]) : 0;
        scalars_out[7] = (double)dyad->GetChannelsDimensions()[2];
        delete dyad;
    } catch (const std::exception& e) {
        std::strncpy(err, e.what(), (size_t)n_err - 1);
        err[n_err - 1] = 0;
        return 1;
    }
    return 0;
}
