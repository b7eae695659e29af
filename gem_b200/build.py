"""Build recipe for libgem (C++ host + sm_100a CUDA), the `gem` CLI and the
CPU oracle.  Incremental: an object is rebuilt when its source or any header
of the package is newer.  Run `python -m gem_b200.build` or call build()."""
import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(PKG, "libgem.so")
CLI = os.path.join(PKG, "bin", "gem")
ORACLE_SRC = os.path.join(ROOT, "oracle", "oracle.c")
ORACLE_LIB = os.path.join(ROOT, "oracle", "_build", "liboracle.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp,-O3",
                  "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-march=x86-64-v3",
            "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include"]


def _headers():
    hs = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                hs.append(os.path.join(d, f))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose=False, ptxas_info=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    os.makedirs(os.path.dirname(ORACLE_LIB), exist_ok=True)
    hdrs = _headers()
    jobs = []
    objs = []
    for f in sorted(os.listdir(CSRC)):
        src = os.path.join(CSRC, f)
        if f == "gem_cli.cpp":
            continue
        if f.endswith(".cu"):
            o = os.path.join(OBJ, f + ".o")
            cmd = [NVCC] + NVFLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", src, "-o", o]
        elif f.endswith(".cpp"):
            o = os.path.join(OBJ, f + ".o")
            cmd = ["g++"] + CXXFLAGS + ["-c", src, "-o", o]
        else:
            continue
        objs.append(o)
        if ptxas_info or _stale(o, [src] + hdrs):
            jobs.append(cmd)
    logs = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for out in ex.map(lambda c: _run(c, verbose), jobs):
            logs.append(out)
    if jobs or not os.path.exists(LIB):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"], verbose)
    cli_src = os.path.join(CSRC, "gem_cli.cpp")
    if os.path.exists(cli_src) and _stale(CLI, [cli_src, LIB] + hdrs):
        _run(["g++"] + CXXFLAGS + [cli_src, "-o", CLI, "-L" + PKG, "-lgem",
                                   "-Wl,-rpath,$ORIGIN/..", "-L/usr/local/cuda/lib64", "-lcudart"], verbose)
    if _stale(ORACLE_LIB, [ORACLE_SRC]):
        _run(["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-shared", "-fPIC", ORACLE_SRC, "-o", ORACLE_LIB, "-lm"], verbose)
    return "\n".join(logs)


if __name__ == "__main__":
    out = build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    if "--ptxas" in sys.argv:
        print(out)
