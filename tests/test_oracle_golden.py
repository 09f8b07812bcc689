"""The CPU restatement (oracle/) against golden vectors produced by the
reference's own CPU classes (tests/golden/gen_golden.py). Bit-exact: the
restatement follows the reference's operation order."""
import numpy as np
import pytest

from oracle import oracle
from tests.helpers import example_case, golden_case, load_golden, species_index

CASES = ["ref2d_sheep", "ref2d_sheep_s3", "ref3d_sheep", "ref2d_mwc", "ref2d_ahtg", "ref2d_spline"]
# the spline coefficients are solved here by another elimination order than the
# reference's tk::spline band solver: equal to rounding, not to the bit
TOL = {"ref2d_spline": 1e-12}


def _same(a, b, tol):
    if tol == 0:
        return np.array_equal(a, b)
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.max(np.abs(a - b)) <= tol * max(np.max(np.abs(b)), 1e-300)


def test_rng_matches_rngstream():
    z = load_golden("rng")
    for k in range(3):
        got = oracle.mrg_u01d(z["seed%d" % k], 4096)
        assert np.array_equal(got, z["draws%d" % k])


def test_rng_jump_is_consistent():
    seed = [12345] * 6
    # advancing 2^3 * 5 = 40 steps by matrix powers equals 20 draws (2 steps each)
    jumped = oracle.mrg_jump(seed, 3, 5)
    d1 = oracle.mrg_u01d(jumped, 10)
    d0 = oracle.mrg_u01d(seed, 30)
    assert np.array_equal(d1, d0[20:30])


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference(name):
    z = load_golden(name)
    params, sites = golden_case(z)
    sim = oracle.OracleSim(params, sites)
    sim.start(sites["first_channel"])
    idx = species_index(params)
    tol = TOL.get(name, 0.0)
    done = 0
    for k, n in enumerate(z["steps"]):
        sim.step(int(n) - done)
        done = int(n)
        for key in z.files:
            if key.startswith("f%d_" % k):
                sp = key.split("_", 1)[1]
                assert _same(sim.field(0, idx[sp]), z[key], tol), key
        assert np.array_equal(sim.states(0), z["s%d" % k])
        assert _same(sim.mouth(0, idx["Calcium"]), z["m%d_Calcium" % k], tol)
        assert _same(sim.jsr(0)[:1], z["sr%d" % k][:1], tol)
        assert _same(sim.cyto(0)[:1], z["cy%d" % k][:1], tol)
        assert _same(sim.total_current(0)[:1], z["tc%d" % k][:1], tol)


def test_oracle_gating_trajectory():
    z = load_golden("ref2d_fastgating")
    params, sites = golden_case(z)
    sim = oracle.OracleSim(params, sites)
    sim.start(sites["first_channel"])
    every = int(z["every"])
    for k in range(len(z["states"])):
        sim.step(every)
        assert np.array_equal(sim.states(0), z["states"][k]), "step %d" % ((k + 1) * every)
        assert np.array_equal(sim.mouth(0, 0), z["mouth"][k])
    assert np.array_equal(sim.field(0, 0), z["ca_final"])


@pytest.mark.parametrize("name", ["ex_spline_gpu", "ex_iaparov_gpu"])
def test_oracle_reproduces_reference_examples(name):
    """The reference's own example configs (examples/SplineGPU: two ions, three buffers,
    spline-tabulated rates from kopen/kclose_data_v2.txt; examples/IaparovGPU: 60-state
    SingleSiteMWC gating): the restatement matches the reference's run bit for bit,
    micro-states included."""
    z = load_golden(name)
    _, _, params, sites = example_case(z)
    sim = oracle.OracleSim(params, sites)
    sim.start(sites["first_channel"])
    idx = species_index(params)
    done = 0
    for k, n in enumerate(z["steps"]):
        sim.step(int(n) - done)
        done = int(n)
        for key in z.files:
            if key.startswith("f%d_" % k):
                assert np.array_equal(sim.field(0, idx[key.split("_", 1)[1]]), z[key]), key
        states = sim.micro_states(0) if "iaparov" in name else sim.states(0)
        assert np.array_equal(states, z["s%d" % k])
        assert np.array_equal(sim.mouth(0, idx["Calcium"]), z["m%d_Calcium" % k])
        assert np.array_equal(sim.jsr(0)[:2], z["sr%d" % k][[0, 20]])
