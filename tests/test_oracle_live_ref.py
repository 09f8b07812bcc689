"""The CPU restatement against the live reference build (oracle/_ref), on
cases beyond the committed fixtures. Skipped where the reference build is
absent (it is built only where the reference tree is mounted)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle, ref
from casim_b200 import configs

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def _run_both(params, sites, steps, tmp_path):
    cpath = os.path.join(str(tmp_path), "c.txt")
    np.savetxt(cpath, np.c_[sites["ch_x"], sites["ch_y"]])
    p = json.loads(json.dumps(params))
    p["Dyad"]["Channels"]["RyR"]["Coordinates"] = cpath
    p["Dyad"]["Seed"] = [int(v) for v in sites["seeds"][0]]
    r = ref.RefSim(p, 1, 1)
    r.start([int(sites["first_channel"][0])])
    o = oracle.OracleSim(params, sites)
    o.start(sites["first_channel"])
    r.step(steps)
    o.step(steps)
    return r, o


@pytest.mark.parametrize("dim", [2, 3])
def test_config1_like_site_matches_reference(dim, tmp_path):
    params, sites = configs.config1(n_sites=1, seed0=9, nx=24, ny=28, n_ryr=6)
    if dim == 3:
        params["Dyad"]["Type"] = "CPU3D"
        params["Dyad"]["dz"] = 7.5
        sites["nz"][:] = 3
    r, o = _run_both(params, sites, 800, tmp_path)
    assert np.array_equal(r.get("dyad:Calcium"), o.field(0, 0))
    assert np.array_equal(r.states(), o.states(0))
    assert r.get("sr")[0] == o.jsr(0)[0]


def test_single_site_mwc_site_matches_reference(tmp_path):
    """60-state gating (CaSim/SingleSiteMWC.cpp): the micro-state trajectory of every RyR
    is the reference's (initial draws from the stationary distribution included) and the
    fields agree to rounding (two ions change the reference's summation order)."""
    params, sites = configs.config1(n_sites=1, seed0=9, nx=24, ny=28, n_ryr=6)
    params = configs.with_single_site_mwc(params, speed=20.0)
    r, o = _run_both(params, sites, 0, tmp_path)
    assert np.array_equal(r.states(), o.micro_states(0))
    changed = 0
    for _ in range(8):
        before = o.micro_states(0)
        r.step(200)
        o.step(200)
        assert np.array_equal(r.states(), o.micro_states(0))
        changed += int(np.sum(before != o.micro_states(0)))
        a, b = r.get("dyad:Calcium"), o.field(0, 0)
        assert np.max(np.abs(a - b)) <= 1e-11 * np.max(np.abs(b))
    assert changed >= 10  # the run does make transitions
    assert np.array_equal(o.states(0), (o.micro_states(0) >= 45).astype(np.int32))


def test_oracle_matches_reference_on_config1_geometry(tmp_path):
    """The restatement against the reference's own CPU classes on the exact config-1
    sites (64 x 64, 20 jittered RyRs, seeds [s]*6, s = 1..4; one NumBatch = 1
    reference run per site) after 2000 steps, bit for bit."""
    params, sites = configs.config1(n_sites=4, seed0=1)
    orc = oracle.OracleSim(params, sites)
    orc.start(sites["first_channel"])
    orc.step(2000, threads=4)
    off = np.concatenate([[0], np.cumsum(sites["n_ch"])])
    for s in range(4):
        q = json.loads(json.dumps(params))
        cpath = os.path.join(str(tmp_path), "c%d.txt" % s)
        np.savetxt(cpath, np.c_[sites["ch_x"][off[s]:off[s + 1]], sites["ch_y"][off[s]:off[s + 1]]], fmt="%.17g")
        q["Dyad"]["Channels"]["RyR"]["Coordinates"] = cpath
        q["Dyad"]["Seed"] = [int(v) for v in sites["seeds"][s]]
        q["Dyad"]["Type"] = "CPU2D"
        r = ref.RefSim(q, 1, 1)
        r.start([int(sites["first_channel"][s])])
        r.step(2000)
        assert np.array_equal(r.states(), orc.states(s))
        assert np.array_equal(r.get("dyad:Calcium"), orc.field(s, 0))
        assert np.array_equal(r.get("mouth:Calcium"), orc.mouth(s, 0))
        assert r.get("sr")[0] == orc.jsr(s)[0]
        r.close()
