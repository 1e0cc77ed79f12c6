"""Builds libvt.so in-tree for sm_100a with nvcc.

Every CUDA translation unit is compiled with --fmad=false and IEEE division
and square root: the ray-casting arithmetic then rounds exactly as a host
evaluation of the reference's expressions, which the parity tests rely on.
Host C++ is compiled with -ffp-contract=off for the same reason.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libvt.so")
BUILD = os.path.join(ROOT, "_build", "vt")

CU = ["render.cu", "cache.cu", "gen.cu", "builder.cu", "mlp.cu"]
CPP = ["volume.cpp", "octree.cpp", "runtime.cpp", "h5lite.cpp"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    return r.stdout + r.stderr


def build(force=False, verbose=False):
    """Compiles csrc/ into visualtur_b200/libvt.so; returns its path."""
    srcs = [os.path.join(CSRC, f) for f in CU + CPP]
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hdrs.append(os.path.join(ROOT, "include", "vt.h"))
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(p) <= t for p in srcs + hdrs + [__file__]):
            return LIB
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    host = ["-ccbin", "/usr/bin/g++"]
    xc = "-fPIC,-fopenmp,-ffp-contract=off,-O2"
    common = host + ["-std=c++17", "-O3", "-I" + os.path.join(ROOT, "include"), "-Xcompiler", xc]
    cuflags = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "--fmad=false",
               "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
    jobs = []
    for f in CU:
        o = os.path.join(BUILD, f + ".o")
        jobs.append((o, [nvcc, "-c", os.path.join(CSRC, f), "-o", o] + common + cuflags +
                     (["-Xptxas", "-v"] if verbose else [])))
    for f in CPP:
        o = os.path.join(BUILD, f + ".o")
        jobs.append((o, [nvcc, "-x", "c++", "-c", os.path.join(CSRC, f), "-o", o] + common))
    # translation units compile independently: run them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        outs = list(ex.map(lambda j: _run(j[1]), jobs))
    if verbose:
        for out in outs:
            sys.stderr.write(out)
    objs = [o for o, _ in jobs]
    tmp = LIB + ".tmp"
    _run([nvcc, "-shared", "-o", tmp] + objs + host +
         ["-Xcompiler", "-fopenmp", "-lcudart", "-lgomp", "-gencode", "arch=compute_100a,code=sm_100a"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
