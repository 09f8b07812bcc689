"""Trajectory output in the reference's HDF5 dataset schema (casim_b200.output):
the datasets the reference's writer fills (CaSim/ParallelHybridSolver.cpp:234-337)
hold, at the cadence's time indices, the values the reference's own CPU classes
produced for the same run (golden fixture ref2d_sheep: snapshots after 1, 500 and
3000 steps)."""
import json
import os

import numpy as np
import pytest

import casim_b200 as cb
from casim_b200 import configs
from casim_b200.output import ScenarioOutput, first_channels, n_iterations
from tests.helpers import golden_case, load_golden, rel_err

pytestmark = pytest.mark.gpu


def _params_with_cadence(params, n_steps, every, names):
    p = json.loads(json.dumps(params))
    p["Max Time, ms"] = n_steps * float(p["dt, ns"]) * 1e-6 * (1 + 1e-12)
    for k in ("Iterations for Dyad", "Iterations for Cytosol", "Iterations for SR", "Iterations for IonChannels",
              "Iterations for IonsNearChannels"):
        p[k] = every
    p["Outputs"] = names
    p["NumScenarios"] = 1
    return p


@pytest.mark.parametrize("path", ["plain", "resident"])
def test_datasets_hold_the_reference_trajectory(cuda_device, tmp_path, path):
    z = load_golden("ref2d_sheep")
    params, sites = golden_case(z)
    d = params["Dyad"]
    names = sorted(d["Ions"]) + sorted(d["Buffers"]) + ["RyR"]
    p = _params_with_cadence(params, 3000, 500, names)
    assert n_iterations(p) == 3000
    sim = cb.ReleaseSiteBatch(p, sites, precision="fp64", path=path)
    files = ScenarioOutput(sim, p, str(tmp_path)).run()
    assert json.load(open(os.path.join(str(tmp_path), "Parameters.json"))) == p
    nx, ny = int(sites["nx"][0]), int(sites["ny"][0])
    for (group, name), f in files.items():
        a = np.load(f)
        assert a.shape[:2] == (7, 1), (group, name, a.shape)
    # fixture snapshot k after steps[k]: time index steps[k] / 500 (500 -> 1, 3000 -> 6)
    for k, t in ((1, 1), (2, 6)):
        for key in z.files:
            if key.startswith("f%d_" % k):
                sp = key.split("_", 1)[1]
                a = np.load(files[("Dyad", sp)])
                assert a.shape == (7, 1, nx, ny)
                assert rel_err(a[t, 0].reshape(-1), z[key]) <= 1e-12, key
        assert np.array_equal(np.load(files[("Channels", "RyR")])[t, 0], z["s%d" % k])
        assert rel_err(np.load(files[("IonsChannels", "Calcium")])[t, 0], z["m%d_Calcium" % k]) <= 1e-12
        n_ch = len(z["s%d" % k])
        assert rel_err(np.load(files[("SR", "Calcium")])[t, 0], z["sr%d" % k][:n_ch]) <= 1e-12
        assert rel_err(np.load(files[("Cytosol", "Calcium")])[t, :1], z["cy%d" % k][:1]) <= 1e-12


def test_batches_fill_the_scenario_axis(cuda_device, tmp_path):
    """Two batches of two sites: scenarios 0-1 then 2-3; the second batch starts from a
    reset state with the RyR of (S*batch + site) / sc_per_channel open and the site's
    RNG stream continued, as the reference's loop does."""
    params, sites = configs.config1(n_sites=2, seed0=3, nx=20, ny=24, n_ryr=4)
    p = json.loads(json.dumps(params))
    p.update({"Max Time, ms": 0.0101, "NumScenarios": 4, "Outputs": ["Calcium", "ATP", "RyR"]})
    for k in ("Iterations for Dyad", "Iterations for Cytosol", "Iterations for SR", "Iterations for IonChannels",
              "Iterations for IonsNearChannels"):
        p[k] = 50
    sim = cb.ReleaseSiteBatch(p, sites, precision="fp64", path="plain")
    files = ScenarioOutput(sim, p, str(tmp_path)).run()
    ryr = np.load(files[("Channels", "RyR")])
    assert ryr.shape == (n_iterations(p) // 50 + 1, 4, 4)
    for b in range(2):
        assert np.array_equal(ryr[0, 2 * b:2 * b + 2], np.eye(4, dtype=np.int32)[first_channels(2, 2, 4, b)])
    ca = np.load(files[("Dyad", "Calcium")])
    assert ca.shape[1:] == (4, 20, 24) and np.all(np.isfinite(ca))
    assert not np.array_equal(ca[-1, 0], ca[-1, 2])  # batch 2 is a new scenario, not a replay
    assert set(k[1] for k in files if k[0] == "Dyad") == {"Calcium", "Calcium-ATP"}
