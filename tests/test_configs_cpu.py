"""Synthetic workload builders: the large-sweep halves (tetrameric MWC and its
spline tabulation) and the precision-study sites, checked on the CPU."""
import numpy as np

from casim_b200 import configs
from oracle import oracle


def test_config5_halves(tmp_path):
    halves = configs.config5(n_sites=64, seed=1, table_dir=str(tmp_path))
    assert [p["Dyad"]["Channels"]["RyR"]["Model"] for p, _ in halves] == ["TwoStateMWC", "TwoStateSpline"]
    for p, s in halves:
        assert len(s["nx"]) == 32
        assert s["n_ch"].min() >= 10 and s["n_ch"].max() <= 150
        # every RyR lies inside the rim of its cleft
        off = np.concatenate([[0], np.cumsum(s["n_ch"])])
        for k in range(32):
            edge = (s["nx"][k] - 1) * 10.0
            x, y = s["ch_x"][off[k]:off[k + 1]], s["ch_y"][off[k]:off[k + 1]]
            assert x.min() > 0 and y.min() > 0 and x.max() < edge and y.max() < edge
        assert "Magnesium" in p["Dyad"]["Ions"]
    # the tabulated opening rate is the MWC law at its knots
    t = np.loadtxt(halves[1][0]["Dyad"]["Channels"]["RyR"]["Kopen filename"])
    assert np.allclose(t[:, 1], configs.mwc_open_rate(t[:, 0]), rtol=1e-15, atol=0)


def test_config5_spline_follows_mwc(tmp_path):
    """The natural spline through the tabulated opening rate (the oracle's
    restatement of the spline model) stays within 1 % of the analytic MWC law
    between the knots over the Ca range of a cleft (0.1 uM .. 1 mM)."""
    halves = configs.config5(n_sites=2, seed=2, side=(40, 40), table_dir=str(tmp_path))
    t = np.loadtxt(halves[1][0]["Dyad"]["Channels"]["RyR"]["Kopen filename"])
    coef, _, _ = oracle.natural_spline(t[:, 0], t[:, 1])
    ca = np.logspace(-1, 3, 400)
    i = np.searchsorted(t[:, 0], ca, side="right") - 1
    h = ca - t[i, 0]
    got = coef[i, 0] + h * (coef[i, 1] + h * (coef[i, 2] + h * coef[i, 3]))
    assert np.max(np.abs(got / configs.mwc_open_rate(ca) - 1)) < 1e-2


def test_precision_compare_lockstep_and_errors():
    """Host logic of the precision study: a site whose states or draw count
    differ leaves the error statistics; relative errors are taken per RyR
    mouth and per site."""
    from casim_b200.precision import compare
    n_ch = np.array([2, 3])
    jsr0 = np.array([1000.0, 800.0])
    b = {"states": np.array([1, 0, 0, 1, 0]), "mouth": np.array([200.0, 1.0, 2.0, 150.0, 0.5]),
         "jsr": np.array([900.0, 700.0]), "release": np.array([10.0, 20.0]), "draws": np.array([100, 200])}
    a = {k: v.copy() for k, v in b.items()}
    a["mouth"][0] *= 1.001
    a["jsr"][0] = 899.9           # depletion 100.1 against 100
    a["release"][0] = 10.002
    a["states"][3] = 0            # site 1 left lockstep
    r = compare(a, b, n_ch, jsr0)
    assert r["lockstep_sites"] == 1 and r["sites"] == 2
    assert abs(r["mouth_ca_rel_err"]["max"] - 1e-3) < 1e-12
    assert abs(r["open_mouth_ca_rel_err"]["max"] - 1e-3) < 1e-12
    assert abs(r["jsr_depletion_rel_err"]["max"] - 1e-3) < 1e-9
    assert abs(r["release_rel_err"]["max"] - 2e-4) < 1e-12


def test_subset_sites_keeps_each_sites_rows():
    _, s = configs.config2(n_sites=6, seed=4)
    sub = configs.subset_sites(s, [4, 1])
    off = np.concatenate([[0], np.cumsum(s["n_ch"])])
    assert list(sub["nx"]) == [s["nx"][4], s["nx"][1]]
    assert np.array_equal(sub["ch_x"], np.concatenate([s["ch_x"][off[4]:off[5]], s["ch_x"][off[1]:off[2]]]))
    assert np.array_equal(sub["seeds"], s["seeds"][[4, 1]])
    assert list(sub["first_channel"]) == [s["first_channel"][4], s["first_channel"][1]]


def test_sweep_split_by_side():
    """The sweep's resident/plain split: the largest sides go plain, the
    threshold is the largest side the predicate accepts, every site lands in
    exactly one part, and the predicate is probed O(log sides) times."""
    from casim_b200.sweep import split_by_side
    rng = np.random.default_rng(0)
    sides = rng.integers(40, 121, size=500)
    n_ch = rng.integers(10, 151, size=500)
    calls = []

    def fits(idx):
        calls.append(len(idx))
        return sides[idx].max() <= 108

    parts = split_by_side(sides, n_ch, fits)
    assert [p for _, p in parts] == ["resident", "plain"]
    res, pla = parts[0][0], parts[1][0]
    assert sides[res].max() <= 108 and sides[pla].min() > 108
    assert sorted(np.concatenate([res, pla]).tolist()) == list(range(500))
    assert len(calls) <= 1 + int(np.ceil(np.log2(len(np.unique(sides))))) + 1
    assert split_by_side(sides, n_ch, lambda idx: True)[0][1] == "resident"
    none = split_by_side(sides, n_ch, lambda idx: False)
    assert len(none) == 1 and none[0][1] == "plain" and len(none[0][0]) == 500
