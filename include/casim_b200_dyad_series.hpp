/*
 * DyadRDB200: the reference's DyadSeries interface (CaSim/DyadSeries.h:9-44)
 * implemented on top of the casim_b200 C ABI, so that ParallelHybridSolver
 * (CaSim/ParallelHybridSolver.cpp:59-130 factories, :133-147 dispatch) can hold
 * a B200 batch as its dyad. Header-only; compile it inside the reference tree
 * (DyadSeries.h and nlohmann/json on the include path) and link
 * libcasim_b200.so.
 *
 * The batch owns the whole release site on the device: cleft, RyR gating and
 * their MRG32k3a streams, jSR and cytosol. A solver drives it per batch as
 * ResetSystem (Reset) -> InitOpening per site -> Update -> per time step
 * RunRD + Update, and reads outputs through the Get* maps at its output
 * cadence:
 *   Reset        casim_b200_reset (CaSim/ParallelHybridSolver.cpp:149-157)
 *   InitOpening  casim_b200_init_opening (CaSim/DyadChannels.cpp:83-95)
 *   Update       casim_b200_update after Reset/InitOpening, where the reference
 *                couples the compartments (CaSim/ParallelHybridSolver.cpp:159-175);
 *                after RunRD only a synchronisation: casim_b200_step already ran it
 *   RunRD        casim_b200_step(h, 1): cytosol, cleft RD, jSR, gating and the
 *                coupling of one time step for every site (the GPU classes step all
 *                sites in RunRD(dt, 0) as well, CaSim/DyadRDMP2D.cu:796-803)
 *   RunMC        nothing: the gating ran inside RunRD, on the device
 * The time step is the JSON's "dt, ns"; the dt arguments are not used.
 * Optional JSON block "B200": {"Precision": "fp32" | "fp64", "Path": "auto" |
 * "plain" | "resident"} (default fp32, auto).
 */
#pragma once

#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "DyadSeries.h"
#include "casim_b200.h"

class DyadRDB200 : public DyadSeries {
    casim_h h_ = nullptr;
    casim_info info_{};
    int n_sites_ = 0;
    int nx_ = 0, ny_ = 0, nz_ = 1;
    double radius_ = 0;
    bool update_pending_ = true;  // an Update after Reset/InitOpening couples the new state
    std::vector<std::string> species_;  // ions, then ion-buffer pairs
    std::vector<double> efflux_, total_;

    void check(casim_status s) const {
        if (s != CASIM_OK) {
            char buf[512];
            casim_b200_last_error(h_, buf, sizeof buf);
            throw std::runtime_error(std::string("casim_b200: ") + buf);
        }
    }
    int nodes() const { return nx_ * ny_ * nz_; }

public:
    // file: the whole Parameters.json (NumBatch sites); base_dir resolves relative file names
    DyadRDB200(const nlohmann::json& file, int nthreads, const std::string& base_dir = ".") : n_sites_(nthreads) {
        nlohmann::json j = file;
        j["NumBatch"] = nthreads;
        casim_precision prec = CASIM_FP32;
        casim_path path = CASIM_PATH_AUTO;
        if (j.contains("B200")) {
            const auto& b = j["B200"];
            if (b.contains("Precision") && b["Precision"] == "fp64") prec = CASIM_FP64;
            if (b.contains("Path")) path = b["Path"] == "plain" ? CASIM_PATH_PLAIN : b["Path"] == "resident" ? CASIM_PATH_RESIDENT : CASIM_PATH_AUTO;
        }
        check(casim_b200_create(j.dump().c_str(), base_dir.c_str(), prec, path, nullptr, &h_));
        check(casim_b200_info(h_, &info_));
        const auto& d = j["Dyad"];
        nx_ = (int)((double)d["x"] / (double)d["dx"] + 1);
        ny_ = (int)((double)d["y"] / (double)d["dy"] + 1);
        nz_ = info_.dim == 3 ? (int)((double)d["z"] / (double)d["dz"] + 1) : 1;
        radius_ = d["Radius"];
        n_channels = info_.max_channels;
        is_cytosol_cpu = false;
        dyad_dims = info_.dim == 3 ? std::vector<uint64_t>{0, (uint64_t)n_sites_, (uint64_t)nx_, (uint64_t)ny_, (uint64_t)nz_}
                                   : std::vector<uint64_t>{0, (uint64_t)n_sites_, (uint64_t)nx_, (uint64_t)ny_};
        channels_dims = {0, (uint64_t)n_sites_, (uint64_t)n_channels};
        channels_ions_dims = channels_dims;
        for (int k = 0; k < info_.n_ions + info_.n_pairs; ++k) {
            char buf[256];
            check(casim_b200_species_name(h_, k, buf, sizeof buf));
            species_.push_back(buf);
        }
        efflux_.resize((size_t)(info_.n_ions + info_.n_pairs) * n_sites_);
        total_.resize((size_t)info_.n_ions * n_sites_);
    }
    ~DyadRDB200() { casim_b200_destroy(h_); }
    DyadRDB200(const DyadRDB200&) = delete;
    DyadRDB200& operator=(const DyadRDB200&) = delete;
    casim_h handle() const { return h_; }

    int GetNumSRChannels() override { return n_channels; }
    bool UsesGPU() override { return true; }
    void Reset() override {
        check(casim_b200_reset(h_));
        update_pending_ = true;
    }
    void InitOpening(int site, int channel) override {
        check(casim_b200_init_opening(h_, site, channel));
        update_pending_ = true;
    }
    double GetElementVolume() override { return info_.element_volume; }
    std::vector<std::string> GetListofIons() override {
        return std::vector<std::string>(species_.begin(), species_.begin() + info_.n_ions);
    }
    // [species + F*site], F = ions + ion-buffer pairs (CaSim/DyadRD2DCPU.cpp:305-350)
    void GetEffluxes(double*& out) override {
        const int F = info_.n_ions + info_.n_pairs;
        for (int k = 0; k < n_sites_; ++k) check(casim_b200_get_efflux(h_, k, &efflux_[(size_t)k * F]));
        out = efflux_.data();
    }
    // [site + ion*S] (CaSim/DyadRD2DCPU.cpp:243-264)
    std::vector<double> GetTotalSRCurrent() override {
        std::vector<double> t(info_.n_ions);
        for (int k = 0; k < n_sites_; ++k) {
            check(casim_b200_get_total_current(h_, k, t.data()));
            for (int i = 0; i < info_.n_ions; ++i) total_[k + (size_t)i * n_sites_] = t[i];
        }
        return total_;
    }
    void RunMC(double, int) override {}
    void Update(double*&, double*&, const std::vector<double>&, const std::vector<double>&, double&) override {
        if (update_pending_) check(casim_b200_update(h_));
        else check(casim_b200_synchronize(h_));
        update_pending_ = false;
    }
    double GetL() override { return radius_; }
    void RunRD(double, int) override {
        if (update_pending_) check(casim_b200_update(h_));
        check(casim_b200_step(h_, 1));
        update_pending_ = false;
    }
    // name -> [site][node] in the reference's node order, for the ions and the buffers
    // (as "<ion>-<buffer>") named in values (CaSim/DyadRD2DCPU.cpp:500-523)
    std::map<std::string, std::vector<double>> GetConcentrations(std::vector<std::string>& values) override {
        std::map<std::string, std::vector<double>> out;
        for (size_t k = 0; k < species_.size(); ++k) {
            const std::string& name = species_[k];
            const std::string key = (int)k < info_.n_ions ? name : name.substr(name.find('-') + 1);
            bool want = false;
            for (const auto& v : values) want = want || v == key;
            if (!want) continue;
            std::vector<double> all((size_t)n_sites_ * nodes());
            for (int s = 0; s < n_sites_; ++s) check(casim_b200_get_field(h_, s, (int32_t)k, &all[(size_t)s * nodes()]));
            out[name] = std::move(all);
        }
        return out;
    }
    // "RyR" -> [site][channel] model states (micro-states of 60-state models)
    std::map<std::string, std::vector<int>> GetChannelsStates(std::vector<std::string>&) override {
        std::vector<int> st((size_t)n_sites_ * n_channels);
        std::vector<int32_t> one(n_channels);
        bool micro = true;
        for (int s = 0; s < n_sites_ && micro; ++s) {
            micro = casim_b200_get_micro_states(h_, s, one.data()) == CASIM_OK;
            if (micro)
                for (int c = 0; c < n_channels; ++c) st[(size_t)s * n_channels + c] = one[c];
        }
        if (!micro) {
            std::vector<int32_t> all((size_t)n_sites_ * n_channels);
            check(casim_b200_get_all_states(h_, all.data()));
            for (size_t i = 0; i < all.size(); ++i) st[i] = all[i];
        }
        return {{"RyR", st}};
    }
    // ion -> [site][channel] mouth values of the last Update (CaSim/DyadRD2DCPU.cpp:536-544)
    std::map<std::string, std::vector<double>> GetIonsNearChannels(std::vector<std::string>&) override {
        std::map<std::string, std::vector<double>> out;
        for (int i = 0; i < info_.n_ions; ++i) {
            std::vector<double> m((size_t)n_sites_ * n_channels);
            check(casim_b200_get_all_mouth(h_, i, m.data()));
            out[species_[i]] = std::move(m);
        }
        return out;
    }
};
