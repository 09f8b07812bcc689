"""Shared helpers for the parity tests: turn a golden fixture into the
(params, sites) pair both the oracle and the product consume."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def golden_case(z):
    """(params, sites) of a fixture; spline-gated fixtures get their rate
    tables written to a temporary directory and referenced by absolute path."""
    params = json.loads(bytes(z["params"]).decode())
    if "sp_open" in z.files:
        import tempfile
        td = tempfile.mkdtemp(prefix="casim_tables_")
        ch = params["Dyad"]["Channels"]["RyR"]
        for key, arr in (("Kopen filename", z["sp_open"]), ("Kclose filename", z["sp_close"])):
            path = os.path.join(td, os.path.basename(ch[key]))
            np.savetxt(path, arr, fmt="%.17g")
            ch[key] = path
    coords = z["coords"]
    d = params["Dyad"]
    nx = int(d["x"] / d["dx"] + 1)
    ny = int(d["y"] / d["dy"] + 1)
    three_d = "3D" in d["Type"]
    nz = int(d["z"] / d["dz"] + 1) if three_d else 1
    sites = {
        "nx": np.array([nx], np.int32), "ny": np.array([ny], np.int32), "nz": np.array([nz], np.int32),
        "n_ch": np.array([len(coords)], np.int32), "ch_x": coords[:, 0].copy(), "ch_y": coords[:, 1].copy(),
        "seeds": np.asarray(z["seed"], np.uint32).reshape(1, 6), "jsr_init": None,
        "first_channel": np.array([int(z["first"])], np.int32),
    }
    return params, sites


def example_case(z):
    """A fixture of one of the reference's example configs: its Parameters.json text
    (unchanged), a directory holding the files it names (byte for byte), and the
    (params, sites) of the one-site run the fixture was made from, for the oracle
    (absolute file names; the package seed's first stream, as the reference falls
    back to when the config names no seed)."""
    import tempfile
    td = tempfile.mkdtemp(prefix="casim_example_")
    for k, fn in enumerate(z["file_names"]):
        with open(os.path.join(td, str(fn)), "wb") as f:
            f.write(bytes(z["file%d" % k]))
    text = bytes(z["json_text"]).decode()
    params = json.loads(text)
    ch = params["Dyad"]["Channels"]["RyR"]
    for key in ("Kopen filename", "Kclose filename"):
        if key in ch:
            ch[key] = os.path.join(td, ch[key])
    coords = np.loadtxt(os.path.join(td, ch["Coordinates"]))
    d = params["Dyad"]
    sites = {
        "nx": np.array([int(d["x"] / d["dx"] + 1)], np.int32), "ny": np.array([int(d["y"] / d["dy"] + 1)], np.int32),
        "nz": np.array([1], np.int32), "n_ch": np.array([len(coords)], np.int32),
        "ch_x": coords[:, 0].copy(), "ch_y": coords[:, 1].copy(),
        "seeds": np.full((1, 6), 12345, np.uint32), "jsr_init": None, "first_channel": np.array([0], np.int32),
    }
    return text, td, params, sites


def species_index(params):
    """name -> species index in the shared order: ions, then ion-buffer pairs (ion-major)."""
    d = params["Dyad"]
    ions = sorted(d["Ions"].keys())
    bufs = sorted(d["Buffers"].keys())
    idx = {ion: k for k, ion in enumerate(ions)}
    k = len(ions)
    for ion in ions:
        for b in bufs:
            if ion in d["Buffers"][b]["Ions"]:
                idx["%s-%s" % (ion, b)] = k
                k += 1
    return idx


def rel_err(a, b, floor=1e-300):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0
