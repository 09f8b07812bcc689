"""Quasi-stationary release sites on the CPU side: the CPU restatement's Gillespie loop
reproduces the reference's own (fixture qs_mwc: CaSim/QuasyStationaryReleaseSite.cpp run
by oracle/ref_qs.cpp, 40 scenarios on one stream) row for row; the library's
Naraghi-Neher increments (host code, a symmetric Jacobi eigen-solve) agree with the
restatement's (a general eigen-solve, as the reference's Eigen) and, without buffers,
with the free point source I / (4 pi F D r)."""
import json
import os

import numpy as np
import pytest

import casim_b200 as cb
from oracle import qs_oracle
from tests.helpers import load_golden


def _case(tmp_path):
    z = load_golden("qs_mwc")
    p = json.loads(bytes(z["params"]).decode())
    np.savetxt(os.path.join(str(tmp_path), "coords.txt"), z["coords"], fmt="%.17g")
    return z, p, str(tmp_path)


def test_restatement_reproduces_reference_gillespie(tmp_path):
    z, p, base = _case(tmp_path)
    cfg = qs_oracle.parse(p, base)
    added = np.asarray(z["increments"])
    s6 = np.full(6, 12345, np.uint32)  # one stream through all scenarios, as the reference's one thread
    off = 0
    n = len(z["coords"])
    for k, first in enumerate(z["first"]):
        t, c, st, _, s6 = qs_oracle.run(cfg, added, s6, int(first))
        rows = int(z["rows_per_scenario"][k])
        assert rows == len(t) + 1, k
        states = np.zeros(n, np.int8)
        states[first] = 1
        assert np.array_equal(z["row_states"][off], states) and z["row_t"][off] == 0.0
        for e in range(len(t)):
            states[c[e]] = st[e]
            assert np.array_equal(z["row_states"][off + 1 + e], states), (k, e)
            assert z["row_t"][off + 1 + e] == t[e], (k, e)
        off += rows
    assert off == len(z["row_t"])


def test_library_increments_match_restatement(tmp_path):
    z, p, base = _case(tmp_path)
    q = cb.QuasiStationarySites(p, 2, base_dir=base)  # no device work: the increments are host code
    got = q.increments()
    q.close()
    want = np.asarray(z["increments"])
    # the library's symmetric Jacobi solve and the restatement's general solve differ
    # by ~2e-12; both sit within 1e-10 of the same steps carried at 50 digits
    assert np.max(np.abs(got - want) / np.abs(want)) < 1e-10
    pytest.importorskip("mpmath")
    exact = qs_oracle.naraghi_neher_exact(qs_oracle.parse(p, base))
    assert np.max(np.abs(got - exact) / exact) < 1e-10
    assert np.max(np.abs(want - exact) / exact) < 1e-10
    assert np.allclose(np.diag(got), p["Calcium Release Site"]["Parameters"]["Open Concentration"])


def test_increments_without_buffers_are_the_free_point_source(tmp_path):
    z, p, base = _case(tmp_path)
    p["Calcium Release Site"]["Parameters"]["Dyadic Cleft"]["Buffers"] = {}
    q = cb.QuasiStationarySites(p, 1, base_dir=base)
    got = q.increments()
    q.close()
    xy = z["coords"]
    r = np.sqrt(((xy[:, None, :] - xy[None, :, :]) ** 2).sum(-1))
    ch = p["Calcium Release Site"]["Parameters"]
    dca = ch["Dyadic Cleft"]["Ions"]["Calcium"]["D"]
    cur = ch["Channels"]["RyR"]["Current"]
    with np.errstate(divide="ignore"):
        want = cur / (4 * np.pi * 96485.33e-6 * dca) / r * 1e-4
    off = ~np.eye(len(xy), dtype=bool)
    assert np.max(np.abs(got[off] - want[off]) / want[off]) < 1e-12


def test_invalid_quasi_stationary_configs_are_rejected(tmp_path):
    z, p, base = _case(tmp_path)
    q = json.loads(json.dumps(p))
    q["Calcium Release Site"]["Parameters"]["Channels"]["RyR"]["Model"] = "NoSuchModel"
    with pytest.raises(cb.CasimError) as e:
        cb.QuasiStationarySites(q, 1, base_dir=base)
    assert e.value.status == cb.EUNSUPPORTED
    q = json.loads(json.dumps(p))
    q["Calcium Release Site"]["Parameters"]["Dyadic Cleft"]["Buffers"]["ATP"]["D"] = 0.0
    with pytest.raises(cb.CasimError) as e:
        cb.QuasiStationarySites(q, 1, base_dir=base)
    assert e.value.status == cb.EINVAL


def test_restatement_matches_live_reference(tmp_path):
    """The reference's QuasyStationaryReleaseSite (oracle/_ref, where it was built) on a
    fresh stream: 25 scenarios from other first channels than the fixture's."""
    from oracle import ref
    if not ref.available() or not hasattr(ref.lib(), "qsref_run"):
        pytest.skip("oracle/_ref not built")
    import ctypes
    z, p, base = _case(tmp_path)
    p["Calcium Release Site"]["Parameters"]["Channels"]["RyR"]["Coordinates"] = os.path.join(base, "coords.txt")
    cfg = qs_oracle.parse(p, base)
    added = np.ascontiguousarray(z["increments"])
    L = ref.lib()
    L.qsref_set_increments.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.qsref_run.restype = ctypes.c_long
    L.qsref_run.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_ulong), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                            ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                            ctypes.c_long]
    n = len(z["coords"])
    L.qsref_set_increments(n, added.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    S, mr = 25, 100000
    first = ((np.arange(S) * 3 + 1) % n).astype(np.int32)
    rt, rs, rps = np.zeros(mr), np.zeros(mr * n, np.int32), np.zeros(S, np.int32)
    seed0 = [987654321, 123456789, 55555, 4242, 77777, 31415]
    seed = (ctypes.c_ulong * 6)(*seed0)
    tot = L.qsref_run(json.dumps(p).encode(), seed, S, first.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                      rt.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), rs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                      rps.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), mr)
    assert 0 < tot <= mr
    rs = rs[:tot * n].reshape(tot, n)
    s6 = np.asarray(seed0, np.uint32)
    off = 0
    for k in range(S):
        t, c, st, _, s6 = qs_oracle.run(cfg, added, s6, int(first[k]))
        assert rps[k] == len(t) + 1
        states = rs[off].copy()
        assert states.sum() == 1 and states[first[k]] == 1 and rt[off] == 0.0
        for e in range(len(t)):
            states[c[e]] = st[e]
            assert np.array_equal(rs[off + 1 + e], states) and rt[off + 1 + e] == t[e], (k, e)
        off += rps[k]
