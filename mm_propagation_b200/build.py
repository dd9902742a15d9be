"""Build libmmp_b200.so in-tree for sm_100a (nvcc, no JIT, no torch extension cache).

    python -m mm_propagation_b200.build [-j N] [--force]

Objects go to mm_propagation_b200/_build/; the shared library lands next to
this file so it travels with the source tree. kern_inst.cu is compiled once per
(precision, log2 NT) with -D switches so the unrolled FFT kernels build in
parallel. Rebuilds only what is older than its sources.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmmp_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I", CSRC, "-I", INCLUDE] + ARCH
CXX = os.environ.get("MMP_CXX", "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++")
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-I", INCLUDE]
LOGN_RANGE = range(6, 17)
# row-split variants (kernel_table.h kSplit*): log2 NT ranges per precision
SPLIT_F32 = range(12, 17)
SPLIT_F64 = range(11, 15)


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _units():
    units = []
    inst = os.path.join(CSRC, "kern_inst.cu")
    for tag, real, split in (("f32", "float", SPLIT_F32), ("f64", "double", SPLIT_F64)):
        for L in LOGN_RANGE:
            for xc in ((0, 1) if L in split else (0,)):
                obj = os.path.join(BUILD, f"kern_{tag}_{L}_x{xc}.o")
                units.append((inst, obj, [f"-DMMP_REAL={real}", f"-DMMP_LOGN={L}", f"-DMMP_TAG={tag}",
                                          f"-DMMP_XC={xc}"]))
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        if os.path.basename(src) == "kern_inst.cu":
            continue
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        units.append((src, obj, []))
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cpp"))):  # host-only units
        units.append((src, os.path.join(BUILD, os.path.basename(src)[:-4] + ".o"), []))
    return units


def _compile(unit, force: bool, verbose: bool):
    src, obj, defs = unit
    deps = [src] + _headers() + [os.path.abspath(__file__)]
    if not force and not _stale(obj, deps):
        return obj, False, ""
    if src.endswith(".cpp"):
        cmd = [CXX, "-c", src, "-o", obj] + CXX_FLAGS
    else:
        cmd = [nvcc(), "-c", src, "-o", obj] + NVCC_FLAGS + defs
    if verbose and not src.endswith(".cpp"):
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(obj)}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, True, r.stderr


def build(jobs: int | None = None, force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    units = _units()
    jobs = jobs or max(1, os.cpu_count() or 1)
    logs = {}
    rebuilt = False
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for obj, did, log in ex.map(lambda u: _compile(u, force, verbose), units):
            rebuilt |= did
            if log:
                logs[obj] = log
    objs = [u[1] for u in units]
    if rebuilt or _stale(LIB, objs):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        for obj, log in sorted(logs.items()):
            print(f"== {os.path.basename(obj)}\n{log}")
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", "--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true", help="print ptxas register/spill reports")
    a = ap.parse_args(argv)
    print(build(a.jobs, a.force, a.verbose))


if __name__ == "__main__":
    sys.exit(main())
