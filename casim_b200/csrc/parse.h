// Host-side resolution of a reference-schema Parameters.json into the device
// model and the packed site table.
#pragma once
#include <string>
#include <vector>

#include "../../include/casim_b200.h"
#include "model.h"

struct cb_site_host {
    int nx = 0, ny = 0, nz = 1;
    std::vector<int> ch_node_xyz;  // 3 grid indices per RyR (Point::GetCoordsOnGrid)
    uint32_t seed[6] = {0, 0, 0, 0, 0, 0};
    double jsr0[CB_MAX_IONS] = {0, 0, 0, 0};
};

struct cb_config {
    cb_model m{};
    std::vector<std::string> ion_names, buf_names, pair_names, cyto_pair_names;
    std::vector<cb_site_host> sites;
    // spline tables: knots x and per-interval cubic coefficients (a, b, c, d)
    std::vector<double> sp_x[2], sp_c[2];
    int num_batch = 1;
    int min_cluster = 1;  // "B200": {"MinClusterSize": C}: smallest cluster per site on the resident path
    int light_rows = 0;   // "B200": {"LightEdgeRows": true}: fewer rows on the edge and plane-0 blocks
    int generic_kernels = 0;  // "B200": {"GenericKernels": true}: the plain path's generic kernels only
};

// Throws std::runtime_error with a readable message on any schema problem.
// `sites` may be null (NumBatch identical sites from the JSON).
cb_config cb_parse_config(const std::string& json_text, const std::string& base_dir, const casim_site_table* sites);

// Largest dt*D*sum(2/h^2) over all diffusing species (explicit Euler is
// stable for values <= 1).
double cb_cfl_number(const cb_model& m);
