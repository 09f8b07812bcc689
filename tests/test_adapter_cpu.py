"""The DyadSeries adapter (include/casim_b200_dyad_series.hpp) compiles against the
reference's own CaSim/DyadSeries.h: the class implements every pure virtual of the
interface (the driver instantiates it through a DyadSeries pointer). Built by
`make -C oracle adapter` where the reference tree is present; skipped elsewhere."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle")
LIB = os.path.join(ORACLE, "_ref", "libadapter_driver.so")


def _reference_present():
    r = subprocess.run(["make", "-C", ORACLE, "-s", "ref-if-present", "-n"], capture_output=True, text=True)
    return "not found" not in r.stdout


@pytest.mark.skipif(not _reference_present(), reason="reference tree not mounted here")
def test_adapter_compiles_against_the_reference_interface():
    r = subprocess.run(["make", "-C", ORACLE, "adapter"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert os.path.exists(LIB)
    import ctypes
    assert hasattr(ctypes.CDLL(LIB), "adapter_run")
