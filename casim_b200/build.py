"""Builds libcasim_b200.so in-tree with nvcc for sm_100a (B200).

    python -m casim_b200.build          # or: from casim_b200.build import build; build()
"""
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcasim_b200.so")
SOURCES = ["capi.cu", "plain.cu", "resident.cu", "noalloc.cu", "parse.cpp"]
HEADERS = ["model.h", "engine.h", "physics.cuh", "mrg32k3a.cuh", "parse.h"]
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
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmd = [nvcc()] + ARCH + common + list(extra) + ["-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        else:
            cmd += ["-x", "cu"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
