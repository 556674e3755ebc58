"""Builds libparatc_gpu.so (the CUDA hot path + C ABI) in-tree with nvcc.

sm_100a only: every .cu file is compiled with
  -gencode arch=compute_100a,code=sm_100a -lineinfo
and linked with the host C++ sources into paratc_b200/_lib/libparatc_gpu.so.
Objects go to paratc_b200/_build/; a file is recompiled when it or a header
is newer than its object.
"""
import concurrent.futures as cf
import glob
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libparatc_gpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
           "-I" + os.path.join(ROOT, "include")]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        [os.path.join(ROOT, "include", "paratc.h")]


def _included_sources(src):
    """The .cu files a translation unit includes (the FP32 storage
    instantiations include the FP64 kernel sources with a switch set)."""
    out = []
    for line in open(src):
        m = re.match(r'\s*#include\s+"([^"]+\.cu)"', line)
        if m:
            out.append(os.path.join(os.path.dirname(src), m.group(1)))
    return out


def _stale(obj, src, hdrs):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + hdrs + _included_sources(src))


def _compile(nvcc, src, obj, verbose_ptxas):
    cmd = [nvcc] + ARCH + NVFLAGS + ["-c", src, "-o", obj]
    if verbose_ptxas and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, r.stdout + r.stderr


def build(force=False, verbose_ptxas=False, quiet=True):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = _nvcc()
    hdrs = _headers()
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(o, s, hdrs):
            jobs.append((s, o))
    logs = []
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for src, rc, out in ex.map(lambda so: _compile(nvcc, so[0], so[1], verbose_ptxas), jobs):
            logs.append((src, out))
            if rc != 0:
                raise RuntimeError("nvcc failed on %s:\n%s" % (src, out))
    if force or jobs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    if not quiet:
        for src, out in logs:
            if out.strip():
                print("==", os.path.basename(src))
                print(out)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv, quiet=False)
    print(LIB)
