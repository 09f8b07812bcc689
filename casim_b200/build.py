"""Builds libcasim_b200.so in-tree with nvcc for sm_100a (B200).

    python -m casim_b200.build          # or: from casim_b200.build import build; build()
"""
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcasim_b200.so")
SOURCES = ["resident_f64_z3.cu", "resident_f32_z3.cu", "resident_f64_z1.cu", "resident_f32_z1.cu", "capi.cu", "plain.cu",
           "resident.cu", "noalloc.cu", "surrogate.cu", "sg_gate.cu", "analysis.cu", "qs.cu", "parse.cpp"]
HEADERS = ["model.h", "engine.h", "physics.cuh", "mrg32k3a.cuh", "parse.h", "resident_kernel.cuh", "pools.cuh", "mwc.h", "stream_kernels.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def json_include():
    p = os.path.join(sysconfig.get_paths()["purelib"], "include", "cudnn_frontend", "thirdparty")
    if os.path.exists(os.path.join(p, "nlohmann", "json.hpp")):
        return p
    raise RuntimeError("nlohmann/json.hpp not found under " + p)


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "casim_b200.h"), __file__]
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + json_include(), "-I" + os.path.join(ROOT, "include")]
    hdr_t = max(os.path.getmtime(os.path.join(CSRC, h)) for h in HEADERS)
    hdr_t = max(hdr_t, os.path.getmtime(os.path.join(ROOT, "include", "casim_b200.h")), os.path.getmtime(__file__))

    def one(src):
        obj = os.path.join(objdir, src + ".o")
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) > max(hdr_t, os.path.getmtime(os.path.join(CSRC, src)))
                and not extra and not verbose):
            return obj, ""
        cmd = [nvcc()] + ARCH + common + list(extra) + ["-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        else:
            cmd += ["-x", "cu"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
        return obj, r.stderr

    jobs = max(1, min(len(SOURCES), os.cpu_count() or 1))
    with ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(one, SOURCES))
    objs = [o for o, _ in results]
    if verbose:
        for _, err in results:
            sys.stderr.write(err)
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
