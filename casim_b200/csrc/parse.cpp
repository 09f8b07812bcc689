// Reference-schema Parameters.json -> cb_model + packed site table.
//
// Follows the reference's construction order so species, pairs and initial
// values line up with it:
//   ions / buffers / pairs     CaSim/DyadRD2DCPU.cpp:24-99 (nlohmann objects iterate in
//                              sorted key order: the default object type is std::map)
//   buffer equilibria          CaSim/DyadRD2DCPU.cpp:47-81, 157-187 (Gauss-Jordan, floating abs)
//   sarcolemmal buffer         CaSim/DyadRD2DCPU.cpp:100-115
//   RyR grid positions         CaSim/DyadRD2DCPU.cpp:121-135 + CaSim/Point.cpp:17-23
//   seeds                      CaSim/DyadChannels.cpp:16-25, CaSim/ParallelRng.cpp:13-16
//   jSR pool                   CaSim/SRPool.cpp:3-46
//   cytosol pool               CaSim/CytosolPool.cpp:1-155
#include "parse.h"

#include <cmath>
#include <fstream>
#include <map>
#include <nlohmann/json.hpp>
#include <sstream>
#include <stdexcept>

#include "../../include/casim_b200.h"
#include "mrg32k3a.cuh"
#include "mwc.h"
#include <cstring>

using json = nlohmann::json;

namespace {

[[noreturn]] void fail(const std::string& msg) { throw std::runtime_error(msg); }

const json& need(const json& j, const char* key, const char* where) {
    if (!j.is_object() || !j.contains(key)) fail(std::string("missing key \"") + key + "\" in " + where);
    return j.at(key);
}

double num(const json& j, const char* key, const char* where) {
    const json& v = need(j, key, where);
    if (!v.is_number()) fail(std::string("key \"") + key + "\" in " + where + " must be a number");
    return v.get<double>();
}

double num_or(const json& j, const char* key, double dflt) {
    if (j.is_object() && j.contains(key) && j.at(key).is_number()) return j.at(key).get<double>();
    return dflt;
}

// Gauss-Jordan elimination with partial pivoting, the algorithm of the
// reference's GaussElimination (CaSim/DyadRD2DCPU.cpp:157-187) with a
// floating-point |.|.
std::vector<double> gauss_jordan(std::vector<std::vector<double>> a) {
    int n = (int)a.size();
    int m = (int)a[0].size() - 1;
    std::vector<int> where(m, -1);
    for (int col = 0, row = 0; col < m && row < n; ++col) {
        int sel = row;
        for (int i = row; i < n; ++i)
            if (std::fabs(a[i][col]) > std::fabs(a[sel][col])) sel = i;
        if (std::fabs(a[sel][col]) < 1e-10) continue;
        for (int i = col; i <= m; ++i) std::swap(a[sel][i], a[row][i]);
        where[col] = row;
        for (int i = 0; i < n; ++i)
            if (i != row) {
                double c = a[i][col] / a[row][col];
                for (int j = col; j <= m; ++j) a[i][j] -= a[row][j] * c;
            }
        ++row;
    }
    std::vector<double> ans(m, 0.0);
    for (int i = 0; i < m; ++i)
        if (where[i] != -1) ans[i] = a[where[i]][m] / a[where[i]][i];
    return ans;
}

// Bound concentrations of one buffer at equilibrium with the resting ions.
std::map<std::string, double> equilibrium(const std::vector<std::pair<std::string, double>>& ions, const json& buf,
                                          bool start_eq) {
    std::map<std::string, double> out;
    const json& kin = need(buf, "Ions", "buffer");
    int n = (int)kin.size();
    std::vector<std::pair<std::string, double>> bound;
    for (auto& ic : ions)
        if (kin.contains(ic.first)) bound.push_back(ic);
    for (auto& b : bound) out[b.first] = 0.0;
    if (!start_eq || n == 0 || bound.empty()) return out;
    double ctot = num(buf, "Total Concentration", "buffer");
    std::vector<std::vector<double>> a(n, std::vector<double>(n + 1, 0.0));
    for (int it = 0; it < (int)bound.size() && it < n; ++it) {
        const json& k = kin.at(bound[it].first);
        double kon = num(k, "kon", "buffer ion"), koff = num(k, "koff", "buffer ion");
        for (int I = 0; I < n; ++I) {
            a[it][I] = kon * bound[it].second;
            if (I == it) a[it][I] += koff;
        }
        a[it][n] = kon * bound[it].second * ctot;
    }
    auto c = gauss_jordan(a);
    for (int t = 0; t < (int)bound.size(); ++t) out[bound[t].first] = c[t];
    return out;
}

int grid_index(double coord, double h) { return (int)((coord + 0.5 * h) / h); }

// Natural cubic spline through (x, y): per interval a + b t + c t^2 + d t^3.
void natural_spline(const std::vector<double>& x, const std::vector<double>& y, std::vector<double>& coef) {
    int n = (int)x.size();
    if (n < 3) fail("spline table needs at least 3 points");
    for (int i = 1; i < n; ++i)
        if (!(x[i] > x[i - 1])) fail("spline knots must increase strictly");
    // second derivatives M: tridiagonal system with M0 = M_{n-1} = 0
    std::vector<double> M(n, 0.0), cp(n, 0.0), dp(n, 0.0);
    for (int i = 1; i < n - 1; ++i) {
        double h0 = x[i] - x[i - 1], h1 = x[i + 1] - x[i];
        double a = h0 / 6.0, b = (h0 + h1) / 3.0, c = h1 / 6.0;
        double r = (y[i + 1] - y[i]) / h1 - (y[i] - y[i - 1]) / h0;
        double denom = b - a * cp[i - 1];
        cp[i] = c / denom;
        dp[i] = (r - a * dp[i - 1]) / denom;
    }
    for (int i = n - 2; i >= 1; --i) M[i] = dp[i] - cp[i] * M[i + 1];
    coef.assign(4 * (size_t)n, 0.0);
    for (int i = 0; i < n - 1; ++i) {
        double h = x[i + 1] - x[i];
        coef[4 * i + 0] = y[i];
        coef[4 * i + 1] = (y[i + 1] - y[i]) / h - h * (2 * M[i] + M[i + 1]) / 6.0;
        coef[4 * i + 2] = M[i] / 2.0;
        coef[4 * i + 3] = (M[i + 1] - M[i]) / (6.0 * h);
    }
    // last knot: value and end slope, for linear extrapolation to the right
    double h = x[n - 1] - x[n - 2];
    coef[4 * (n - 1) + 0] = y[n - 1];
    coef[4 * (n - 1) + 1] = coef[4 * (n - 2) + 1] + 2 * coef[4 * (n - 2) + 2] * h + 3 * coef[4 * (n - 2) + 3] * h * h;
}

std::string join(const std::string& dir, const std::string& p) {
    if (p.empty() || p[0] == '/' || dir.empty()) return p;
    return dir + "/" + p;
}

// dense solve with partial pivoting (row swaps), then back substitution
std::vector<double> solve_pivoted(std::vector<std::vector<double>> a, std::vector<double> b) {
    const int n = (int)b.size();
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
        std::swap(a[c], a[piv]);
        std::swap(b[c], b[piv]);
        for (int r = c + 1; r < n; ++r) {
            const double f = a[r][c] / a[c][c];
            if (f == 0) continue;
            for (int k = c; k < n; ++k) a[r][k] -= f * a[c][k];
            b[r] -= f * b[c];
        }
    }
    std::vector<double> x(n, 0.0);
    for (int r = n - 1; r >= 0; --r) {
        double v = b[r];
        for (int k = r + 1; k < n; ++k) v -= a[r][k] * x[k];
        x[r] = v / a[r][r];
    }
    return x;
}

void read_table(const std::string& path, std::vector<double>& a, std::vector<double>& b) {
    std::ifstream in(path);
    if (!in) fail("cannot open " + path);
    double u, v;
    while (in >> u >> v) {
        a.push_back(u);
        b.push_back(v);
    }
}

}  // namespace

double cb_cfl_number(const cb_model& m) {
    double lat = 2.0 / (m.dx * m.dx) + 2.0 / (m.dy * m.dy) + (m.dim == 3 ? 2.0 / (m.dz * m.dz) : 0.0);
    double dmax = 0;
    for (int i = 0; i < m.n_ions; ++i) dmax = std::max(dmax, m.D_ion[i]);
    for (int p = 0; p < m.n_pairs; ++p) dmax = std::max(dmax, m.D_pair[p]);
    double cfl = m.dt * dmax * lat;
    if (m.cyto_type == CB_CYTO_RD3D) {
        double dc = 0;
        for (int i = 0; i < m.n_ions; ++i) dc = std::max(dc, m.D_ion[i]);
        for (int p = 0; p < m.c_n_pairs; ++p) dc = std::max(dc, m.c_D_pair[p]);
        cfl = std::max(cfl, m.dt * dc * 6.0 / (m.hc * m.hc));
    }
    return cfl;
}

cb_config cb_parse_config(const std::string& json_text, const std::string& base_dir, const casim_site_table* tab) {
    json j;
    try {
        j = json::parse(json_text);
    } catch (const std::exception& e) {
        fail(std::string("JSON parse error: ") + e.what());
    }
    cb_config cfg;
    cb_model& m = cfg.m;
    const json& d = need(j, "Dyad", "Parameters");
    std::string dtype = d.contains("Type") ? d.at("Type").get<std::string>() : "2D";
    m.dim = dtype.find("3D") != std::string::npos ? 3 : 2;
    m.dx = num(d, "dx", "Dyad");
    m.dy = num(d, "dy", "Dyad");
    m.dz = m.dim == 3 ? num(d, "dz", "Dyad") : num_or(d, "dz", 1.0);
    m.z = num(d, "z", "Dyad");
    m.R = num(d, "Radius", "Dyad");
    m.voltage = num_or(d, "Voltage", 0.0);
    m.dt = num(j, "dt, ns", "Parameters") * 1e-6;
    if (!(m.dx > 0 && m.dy > 0 && m.dz > 0 && m.dt > 0 && m.R > 0)) fail("dx, dy, dz, dt and Radius must be positive");
    cfg.num_batch = j.contains("NumBatch") ? j.at("NumBatch").get<int>() : 1;
    if (j.contains("B200") && j.at("B200").contains("MinClusterSize")) {
        cfg.min_cluster = j.at("B200").at("MinClusterSize").get<int>();
        if (cfg.min_cluster != 1 && cfg.min_cluster != 2 && cfg.min_cluster != 4 && cfg.min_cluster != 8 && cfg.min_cluster != 16)
            fail("B200.MinClusterSize must be 1, 2, 4, 8 or 16");
    }
    if (j.contains("B200") && j.at("B200").contains("GenericKernels")) {
        cfg.generic_kernels = j.at("B200").at("GenericKernels").get<bool>() ? 1 : 0;
    }
    if (j.contains("B200") && j.at("B200").contains("LightEdgeRows")) {
        cfg.light_rows = j.at("B200").at("LightEdgeRows").get<bool>() ? 1 : 0;
    }

    // ions (sorted keys)
    const json& ions = need(d, "Ions", "Dyad");
    std::vector<std::pair<std::string, double>> ion_cb;
    for (auto& el : ions.items()) {
        if (m.n_ions >= CB_MAX_IONS) fail("too many ions (max 4)");
        int i = m.n_ions++;
        cfg.ion_names.push_back(el.key());
        m.D_ion[i] = num(el.value(), "D", "Dyad ion");
        m.Cb[i] = num(el.value(), "Concentration", "Dyad ion");
        m.extracell[i] = num_or(el.value(), "Extracell", 0.0);
        ion_cb.push_back({el.key(), m.Cb[i]});
    }
    if (m.n_ions == 0) fail("Dyad needs at least one ion");
    m.ca_idx = m.mg_idx = -1;
    for (int i = 0; i < m.n_ions; ++i) {
        if (cfg.ion_names[i] == "Calcium") m.ca_idx = i;
        if (cfg.ion_names[i] == "Magnesium") m.mg_idx = i;
    }
    if (d.contains("Sarcolemma"))
        for (auto& el : d.at("Sarcolemma").items())
            for (int i = 0; i < m.n_ions; ++i)
                if (cfg.ion_names[i] == el.key()) {
                    m.has_sl[i] = 1;
                    m.N1[i] = num(el.value(), "N1", "Sarcolemma");
                    m.K1[i] = num(el.value(), "K1", "Sarcolemma");
                    m.N2[i] = num(el.value(), "N2", "Sarcolemma");
                    m.K2[i] = num(el.value(), "K2", "Sarcolemma");
                }
    bool start_eq = d.contains("Start") && d.at("Start") == "Equilibrium";
    // buffers and ion-buffer pairs (ion-major, buffer-minor)
    const json& bufs = need(d, "Buffers", "Dyad");
    std::vector<std::pair<std::string, const json*>> blist;
    for (auto& el : bufs.items()) blist.push_back({el.key(), &el.value()});
    if ((int)blist.size() > CB_MAX_BUF) fail("too many dyad buffers (max 8)");
    m.n_buf = (int)blist.size();
    std::map<std::string, std::map<std::string, double>> eq;
    for (int b = 0; b < m.n_buf; ++b) {
        cfg.buf_names.push_back(blist[b].first);
        m.Ctot[b] = num(*blist[b].second, "Total Concentration", "Dyad buffer");
        eq[blist[b].first] = equilibrium(ion_cb, *blist[b].second, start_eq);
    }
    for (int i = 0; i < m.n_ions; ++i)
        for (int b = 0; b < m.n_buf; ++b) {
            const json& kin = need(*blist[b].second, "Ions", "Dyad buffer");
            if (!kin.contains(cfg.ion_names[i])) continue;
            if (m.n_pairs >= CB_MAX_PAIRS) fail("too many ion-buffer pairs (max 12)");
            int p = m.n_pairs++;
            const json& k = kin.at(cfg.ion_names[i]);
            m.pair_ion[p] = i;
            m.pair_buf[p] = b;
            m.D_pair[p] = num(k, "D", "buffer ion");
            m.kon[p] = num(k, "kon", "buffer ion");
            m.koff[p] = num(k, "koff", "buffer ion");
            m.pair_init[p] = eq[blist[b].first][cfg.ion_names[i]];
            cfg.pair_names.push_back(cfg.ion_names[i] + "-" + blist[b].first);
        }
    m.F = m.n_ions + m.n_pairs;

    // RyR channels: the first (sorted) entry of "Channels"
    const json& chs = need(d, "Channels", "Dyad");
    if (chs.empty()) fail("Dyad.Channels is empty");
    const json& ch = chs.begin().value();
    std::string model = need(ch, "Model", "Channels").get<std::string>();
    const json par = ch.contains("Parameters") ? ch.at("Parameters") : json::object();
    auto P = [&](const char* k) { return num(par, k, "Channels.Parameters"); };
    std::vector<double> cp;
    if (model == "SheepCannell") {
        m.ch_model = CB_SHEEP_CANNELL;
        cp = {P("kopen0"), P("ncaopen"), P("kopenmax"), P("kclose0"), P("ncaclose")};
    } else if (model == "TwoStateMWC") {
        m.ch_model = CB_TWO_STATE_MWC;
        cp = {P("fCa"), P("KCa"), P("fMg"), P("KMg"), P("KO0"), P("KMgI"), P("kclose")};
    } else if (model == "TwoStateaHTG") {
        m.ch_model = CB_TWO_STATE_AHTG;
        cp = {P("fCa"), P("KCa"), P("fMg"), P("KMg"), P("KO0"), P("KMgI"), P("KCL"), P("KI"), P("KOL"), P("kclose")};
    } else if (model == "TwoStateSpline") {
        m.ch_model = CB_TWO_STATE_SPLINE;
        const char* keys[2] = {"Kopen filename", "Kclose filename"};
        for (int w = 0; w < 2; ++w) {
            std::vector<double> xs, ys;
            read_table(join(base_dir, need(ch, keys[w], "Channels").get<std::string>()), xs, ys);
            natural_spline(xs, ys, cfg.sp_c[w]);
            cfg.sp_x[w] = xs;
            m.sp_n[w] = (int)xs.size();
        }
    } else if (model == "SingleSiteMWC") {
        // 60-state Q-matrix model (CaSim/SingleSiteMWC.cpp:5-37); absent names read as 0
        // like the reference's std::map lookups
        m.ch_model = CB_SINGLE_SITE_MWC;
        const char* names[MWC_NPAR] = {"fCa4I", "fCa", "KCa", "alphaCa", "konCa", "fMg", "KMg", "konMg", "alphaMg", "alphaMgI",
                                       "KO0", "alphakco", "alphakcoI", "kco", "KMgI", "konmgI", "fICa", "fIMg", "gMg", "gCa"};
        for (int k = 0; k < MWC_NPAR; ++k) cp.push_back(num_or(par, names[k], 0.0));
    } else {
        fail("gating model \"" + model + "\" is not supported by this build (SheepCannell, TwoStateMWC, TwoStateaHTG, TwoStateSpline, "
             "SingleSiteMWC)");
    }
    for (size_t k = 0; k < cp.size(); ++k) m.ch_par[k] = cp[k];
    if ((m.ch_model == CB_TWO_STATE_MWC || m.ch_model == CB_TWO_STATE_AHTG || m.ch_model == CB_SINGLE_SITE_MWC) && m.mg_idx < 0)
        fail("gating model " + model + " needs a Magnesium ion");
    if (m.ca_idx < 0) fail("gating needs a Calcium ion");
    const json& cond = need(ch, "Conductance", "Channels");
    for (int i = 0; i < m.n_ions; ++i) m.g[i] = num_or(cond, cfg.ion_names[i].c_str(), 0.0);

    // jSR pool (CaSim/SRPool.cpp:3-46)
    const json& jsr = need(j, "jSR", "Parameters");
    m.jsr_const = jsr.contains("Constant") && jsr.at("Constant").get<bool>() ? 1 : 0;
    m.CQ = num(jsr, "Total CQ (uM)", "jSR");
    m.V_jsr = num(jsr, "V jSR (nm3)", "jSR");
    const json& jions = need(jsr, "Ions", "jSR");
    for (int i = 0; i < m.n_ions; ++i) {
        if (jions.contains(cfg.ion_names[i])) {
            const json& p = jions.at(cfg.ion_names[i]);
            m.nCQ[i] = num(p, "Binding sites of CQ", "jSR ion");
            m.K_CQ[i] = num(p, "K CQ (uM)", "jSR ion");
            m.tau_refill[i] = num(p, "T refill (ms)", "jSR ion");
            m.jsr0[i] = num(p, "Concentration", "jSR ion");
        } else {
            m.nCQ[i] = 0;
            m.K_CQ[i] = 0;
            m.tau_refill[i] = 1;
            m.jsr0[i] = 0;
        }
    }
    // nSR constant pool (CaSim/NSRConstPool.cpp:3-12): values by position
    const json& nsr = need(need(j, "nSR", "Parameters"), "Ions", "nSR");
    {
        int i = 0;
        for (auto& el : nsr.items()) {
            if (i < m.n_ions) m.nsr[i] = num(el.value(), "Concentration (uM)", "nSR ion");
            ++i;
        }
        if (i < m.n_ions && !m.jsr_const) fail("nSR must list at least as many ions as the Dyad");
    }

    // cytosol (CaSim/CytosolPool.cpp:1-155); RD3D adds "Nodes" and "dx"
    const json& c = need(j, "Cytosol", "Parameters");
    std::string ctype = c.contains("Type") ? c.at("Type").get<std::string>() : "Pool";
    if (ctype == "Pool") m.cyto_type = CB_CYTO_POOL;
    else if (ctype == "RD3D") m.cyto_type = CB_CYTO_RD3D;
    else fail("Cytosol.Type \"" + ctype + "\" is not supported (Pool, RD3D)");
    double leak = num_or(c, "Leak mult", 0.0);
    if (c.contains("Ions") && !c.at("Ions").is_null() && !c.at("Ions").empty())
        fail("cytosol-only ions are not supported");
    for (int i = 0; i < m.n_ions; ++i) {
        m.c_bg[i] = m.Cb[i];
        m.c_onetau_ion[i] = leak * m.D_ion[i];
    }
    // the RD3D cytosol carries only the dyad buffers that diffuse (an
    // immobile cleft buffer such as fixed membrane sites stays in the cleft)
    std::vector<std::pair<std::string, const json*>> cbl;
    std::vector<int> cb_in_dyad;
    std::vector<int> dyad_buf_index;
    for (int b = 0; b < (int)blist.size(); ++b) {
        bool mobile = false;
        for (auto& el : need(*blist[b].second, "Ions", "Dyad buffer").items())
            if (num(el.value(), "D", "buffer ion") > 0) mobile = true;
        if (m.cyto_type == CB_CYTO_RD3D && !mobile) continue;
        cbl.push_back(blist[b]);
        cb_in_dyad.push_back(1);
        dyad_buf_index.push_back(b);
    }
    if (c.contains("Buffers"))
        for (auto& el : c.at("Buffers").items()) {
            cbl.push_back({el.key(), &el.value()});
            cb_in_dyad.push_back(0);
            dyad_buf_index.push_back(-1);
        }
    if ((int)cbl.size() > CB_MAX_CBUF) fail("too many cytosol buffers");
    m.c_n_buf = (int)cbl.size();
    for (int p = 0; p < CB_MAX_PAIRS; ++p) m.dyad_c_pair[p] = -1;
    for (int i = 0; i < m.n_ions; ++i)
        for (int b = 0; b < m.c_n_buf; ++b) {
            m.c_Ctot[b] = num(*cbl[b].second, "Total Concentration", "Cytosol buffer");
            const json& kin = need(*cbl[b].second, "Ions", "Cytosol buffer");
            if (!kin.contains(cfg.ion_names[i])) continue;
            if (m.c_n_pairs >= CB_MAX_CPAIRS) fail("too many cytosol ion-buffer pairs");
            int q = m.c_n_pairs++;
            const json& k = kin.at(cfg.ion_names[i]);
            m.c_pair_ion[q] = i;
            m.c_pair_buf[q] = b;
            m.c_kon[q] = num(k, "kon", "buffer ion");
            m.c_koff[q] = num(k, "koff", "buffer ion");
            m.c_D_pair[q] = num(k, "D", "buffer ion");
            m.c_init[q] = equilibrium(ion_cb, *cbl[b].second, start_eq)[cfg.ion_names[i]];
            m.c_onetau_pair[q] = leak * m.c_D_pair[q];
            m.c_in_dyad[q] = cb_in_dyad[b];
            m.c_dyad_pair[q] = -1;
            if (cb_in_dyad[b])
                for (int p = 0; p < m.n_pairs; ++p)
                    if (m.pair_ion[p] == i && m.pair_buf[p] == dyad_buf_index[b]) {
                        m.c_dyad_pair[q] = p;
                        m.dyad_c_pair[p] = q;
                    }
            cfg.cyto_pair_names.push_back(cfg.ion_names[i] + "-" + cbl[b].first);
        }
    if (c.contains("SERCA")) {
        int s = 0;
        for (int i = 0; i < m.n_ions; ++i)
            if (c.at("SERCA").contains(cfg.ion_names[i])) {
                const json& sp = c.at("SERCA").at(cfg.ion_names[i]);
                m.c_serca[i] = 1;
                m.c_Jmax[s] = num(sp, "Jmax", "SERCA");
                m.c_Kup[s] = num(sp, "Kup", "SERCA");
                ++s;
            }
    }
    if (m.cyto_type == CB_CYTO_RD3D) {
        m.mc = (int)num(c, "Nodes", "Cytosol");
        m.hc = num(c, "dx", "Cytosol");
        if (m.mc < 4 || m.mc > 64) fail("Cytosol.Nodes must be in [4, 64]");
        if (!(m.hc > 0)) fail("Cytosol.dx must be positive");
        m.inv_hc2 = 1.0 / (m.hc * m.hc);
        m.inv_hc3 = 1.0 / (m.hc * m.hc * m.hc);
    }

    // derived constants
    m.grad_mult = 3.0 / (4 * std::acos(-1.0) * m.R * m.R * m.R);
    if (m.dim == 2) {
        m.sx = m.dy * m.z / m.dx;
        m.sy = m.dx * m.z / m.dy;
        m.V_elem = m.dx * m.dy * m.z;
    } else {
        m.sx = m.dy * m.dz / m.dx;
        m.sy = m.dx * m.dz / m.dy;
        m.V_elem = 0.5 * m.dx * m.dy * m.dz;  // CaSim/DyadRDCPU.cpp:195-197
    }
    m.inv_dx2 = 1.0 / (m.dx * m.dx);
    m.inv_dy2 = 1.0 / (m.dy * m.dy);
    m.inv_dz2 = 1.0 / (m.dz * m.dz);

    // sites
    int nx0 = (int)(num(d, "x", "Dyad") / m.dx + 1);
    int ny0 = (int)(num(d, "y", "Dyad") / m.dy + 1);
    int nz0 = m.dim == 3 ? (int)(m.z / m.dz + 1) : 1;
    int S = tab ? tab->n_sites : cfg.num_batch;
    if (S <= 0) fail("number of sites must be positive");
    std::vector<double> fx, fy;
    bool need_file = !tab || !tab->n_channels || !tab->ch_x || !tab->ch_y;
    if (need_file) {
        std::string path = join(base_dir, need(ch, "Coordinates", "Channels").get<std::string>());
        read_table(path, fx, fy);
        if (fx.empty()) fail("no RyR coordinates in " + path);
    }
    // seeds: JSON "Seed" zero-padded to six words; an invalid seed leaves the
    // package default 12345 x 6 in place, as RngStream::SetPackageSeed does.
    uint64_t pkg[6] = {12345, 12345, 12345, 12345, 12345, 12345};
    if (d.contains("Seed")) {
        uint64_t s6[6] = {0, 0, 0, 0, 0, 0};
        int k = 0;
        for (auto& v : d.at("Seed")) {
            if (k < 6) s6[k] = v.get<uint64_t>();
            ++k;
        }
        if (cbrng::seed_ok(s6))
            for (int q = 0; q < 6; ++q) pkg[q] = s6[q];
    }
    cfg.sites.resize(S);
    long long chp = 0;
    cbrng::State stream{};
    for (int q = 0; q < 6; ++q) stream.s[q] = (uint32_t)pkg[q];
    for (int s = 0; s < S; ++s) {
        cb_site_host& h = cfg.sites[s];
        h.nx = tab && tab->nx ? tab->nx[s] : nx0;
        h.ny = tab && tab->ny ? tab->ny[s] : ny0;
        h.nz = m.dim == 3 ? (tab && tab->nz ? tab->nz[s] : nz0) : 1;
        if (h.nx < 5 || h.ny < 5) fail("each site needs at least 5 x 5 nodes");
        if (m.dim == 3 && h.nz < 2) fail("3D sites need at least 2 z layers");
        int nch = need_file ? (int)fx.size() : tab->n_channels[s];
        if (nch < 1 || nch > CB_MAX_CHANNELS) fail("RyR count per site must be in [1, 1024]");
        for (int c2 = 0; c2 < nch; ++c2) {
            double X = need_file ? fx[c2] : tab->ch_x[chp + c2];
            double Y = need_file ? fy[c2] : tab->ch_y[chp + c2];
            int gx = grid_index(X, m.dx), gy = grid_index(Y, m.dy), gz = 0;
            if (gx < 0 || gx >= h.nx || gy < 0 || gy >= h.ny)
                fail("RyR " + std::to_string(c2) + " of site " + std::to_string(s) + " lies outside the grid");
            h.ch_node_xyz.push_back(gx);
            h.ch_node_xyz.push_back(gy);
            h.ch_node_xyz.push_back(gz);
        }
        if (!need_file) chp += nch;
        if (tab && tab->seeds) {
            uint64_t s6[6];
            for (int q = 0; q < 6; ++q) s6[q] = tab->seeds[6 * s + q];
            if (!cbrng::seed_ok(s6)) fail("seed of site " + std::to_string(s) + " is not a valid MRG32k3a seed");
            for (int q = 0; q < 6; ++q) h.seed[q] = (uint32_t)s6[q];
        } else {
            // site s draws from stream s of the package seed (2^127 apart)
            for (int q = 0; q < 6; ++q) h.seed[q] = stream.s[q];
            cbrng::jump_pow2(stream, 127, 1);
        }
        for (int i = 0; i < m.n_ions; ++i) h.jsr0[i] = tab && tab->jsr_init ? tab->jsr_init[(long long)s * m.n_ions + i] : m.jsr0[i];
    }
    return cfg;
}

// Adjacency lists in the push order of CaSim/SingleSiteMWC.cpp:55-89 and the stationary
// distribution p of the full Q at (ca0, mg0): p = 1^T (S S^T)^-1 with S = [Q | 1], the
// least-squares solution of p Q = 0, sum p = 1 (CaSim/QMatrixModel.cpp:38-47).
void cb_mwc_build(const double* P, double ca0, double mg0, cb_mwc_tab& t) {
    std::memset(&t, 0, sizeof(t));
    auto push = [&](int x, int y) { t.adj[x][t.nadj[x]++] = (unsigned char)y; };
    auto in_all_blocks = [&](int x, int y) {
        push(x, y);
        push(x + 45, y + 45);
        push(x + 15, y + 15);
        push(x + 30, y + 30);
    };
    auto idx = [](int i, int j) { return 15 - (6 - j) * (5 - j) / 2 + i; };
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5 - i; ++j) {
            const int c = idx(i, j);
            if (i + j < 4) in_all_blocks(c, idx(i + 1, j));
            if (i > 0) in_all_blocks(c, idx(i - 1, j));
            if (i + j < 4) in_all_blocks(c, idx(i, j + 1));
            if (j > 0) in_all_blocks(c, idx(i, j - 1));
            push(c, c + 15);
            push(c + 15, c);
            push(c + 45, c + 30);
            push(c + 30, c + 45);
            push(c, c + 45);
            push(c + 45, c);
            push(c + 15, c + 30);
            push(c + 30, c + 15);
        }
    std::vector<std::vector<double>> Q(CB_MWC_N, std::vector<double>(CB_MWC_N, 0.0));
    for (int s = 0; s < CB_MWC_N; ++s) {
        double r = 0;
        for (int k = 0; k < t.nadj[s]; ++k) {
            const int d = t.adj[s][k];
            Q[s][d] = cb_mwc_q(P, s, d, ca0, mg0);
            r += Q[s][d];
        }
        Q[s][s] = -r;
    }
    std::vector<std::vector<double>> M(CB_MWC_N, std::vector<double>(CB_MWC_N, 0.0));
    for (int i = 0; i < CB_MWC_N; ++i)
        for (int j = 0; j < CB_MWC_N; ++j) {
            double v = 1.0;
            for (int k = 0; k < CB_MWC_N; ++k) v += Q[i][k] * Q[j][k];
            M[i][j] = v;
        }
    const std::vector<double> p = solve_pivoted(M, std::vector<double>(CB_MWC_N, 1.0));
    for (int i = 0; i < CB_MWC_N; ++i) t.p_init[i] = p[i];
}
