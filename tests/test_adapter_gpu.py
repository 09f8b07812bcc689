"""The DyadSeries adapter driven like ParallelHybridSolver drives a dyad
(ResetSystem, InitOpening, Update, then RunRD/RunMC/Update per step; driver
oracle/adapter_driver.cpp, compiled against the reference's DyadSeries.h): after
500 steps its GetConcentrations, GetChannelsStates, GetIonsNearChannels and
GetTotalSRCurrent equal the reference's own CPU run (golden fixture ref2d_sheep),
FP64 to 1e-12."""
import ctypes
import json
import os

import numpy as np
import pytest

import casim_b200 as cb
from tests.helpers import load_golden, rel_err

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libadapter_driver.so")


@pytest.mark.skipif(not os.path.exists(LIB), reason="adapter driver not built (needs the reference tree at build time)")
@pytest.mark.parametrize("path", ["plain", "resident"])
def test_reference_shaped_loop_through_the_adapter(cuda_device, tmp_path, path):
    cb.lib()  # the library the driver links, loaded and checked
    z = load_golden("ref2d_sheep")
    params = json.loads(bytes(z["params"]).decode())
    cpath = os.path.join(str(tmp_path), "coords.txt")
    np.savetxt(cpath, z["coords"], fmt="%.17g")
    params["Dyad"]["Channels"]["RyR"]["Coordinates"] = cpath
    params["Dyad"]["Seed"] = [int(v) for v in z["seed"]]
    params["B200"] = {"Precision": "fp64", "Path": path}
    d = params["Dyad"]
    nx, ny = int(d["x"] / d["dx"] + 1), int(d["y"] / d["dy"] + 1)
    n_ch = len(z["coords"])
    n_ions = len(d["Ions"])
    L = ctypes.CDLL(LIB)
    ca = np.zeros(nx * ny)
    st = np.zeros(n_ch, np.int32)
    mo = np.zeros(n_ch)
    tc = np.zeros(n_ions)
    ef = np.zeros(n_ions)
    sc = np.zeros(8)
    err = ctypes.create_string_buffer(512)
    first = np.array([int(z["first"])], np.int32)
    P = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    rc = L.adapter_run(json.dumps(params).encode(), str(tmp_path).encode(), 1, 500, P(first, ctypes.c_int),
                       P(ca, ctypes.c_double), P(st, ctypes.c_int), P(mo, ctypes.c_double), P(tc, ctypes.c_double),
                       P(ef, ctypes.c_double), P(sc, ctypes.c_double), err, 512)
    assert rc == 0, err.value.decode()
    assert rel_err(ca, z["f1_Calcium"]) <= 1e-12
    assert np.array_equal(st, z["s1"])
    assert rel_err(mo, z["m1_Calcium"]) <= 1e-12
    assert rel_err(tc[:1], z["tc1"][:1]) <= 1e-10
    assert sc[0] == n_ch and sc[1] == 1 and sc[4] == n_ions and sc[5] == 4 and sc[6] == nx * ny and sc[7] == n_ch
    assert sc[3] == d["Radius"]
