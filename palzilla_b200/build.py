"""Builds the sm_100a CUDA library in-tree: palzilla_b200/libpalzilla_b200.so, and the
C++ facade's driver program palzilla_b200/pk_render.

Each translation unit is compiled with nvcc for sm_100a.  Units whose results must
be bit-exact with the CPU oracle (BVH keys, traversal, photons, eye pass, the batched
solver, path cuts, the adjoint, the subdivision solve) are built with -fmad=false so
that no multiply-add pair is contracted into an FMA; the plain solver is built both ways.  Objects are rebuilt
only when a source or header is newer than the object.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpalzilla_b200.so")
PK_RENDER = os.path.join(HERE, "pk_render")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]

# object name -> (source, extra flags)
UNITS = {
    "pz_sort": ("pz_sort.cu", []),
    "pz_bvh": ("pz_bvh.cu", ["-fmad=false"]),
    "pz_trace": ("pz_trace.cu", ["-fmad=false"]),
    "pz_photon": ("pz_photon.cu", ["-fmad=false"]),
    "pz_frame": ("pz_frame.cu", ["-fmad=false"]),
    "pz_solve": ("pz_solve.cu", []),
    "pz_solve_exact": ("pz_solve.cu", ["-fmad=false", "-DPZ_SOLVE_EXACT"]),
    "pz_batched": ("pz_batched.cu", ["-fmad=false"]),
    "pz_capi": ("pz_capi.cu", []),
    "pz_capi_frame": ("pz_capi_frame.cu", []),
    "pz_sort_static": ("pz_sort_static.cu", []),
    "pz_pathcuts": ("pz_pathcuts.cu", ["-fmad=false"]),
    "pz_adjoint": ("pz_adjoint.cu", ["-fmad=false"]),
    "pz_subdiv": ("pz_subdiv.cu", ["-fmad=false"]),
    "pz_solve_device": ("pz_solve_device.cu", ["-fmad=false"]),
}


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _stamp_flags(extra) -> str:
    """A file recording the extra flags of the objects in _build/; rewritten (so that every
    object is rebuilt) when they change."""
    stamp = os.path.join(OBJ, "extra_flags.txt")
    text = " ".join(extra)
    if not os.path.exists(stamp) or open(stamp).read() != text:
        with open(stamp, "w") as f:
            f.write(text)
    return stamp


def build(verbose: bool = False, jobs: int | None = None) -> str:
    """Builds the library.  PZ_EXTRA_NVCC_FLAGS (space-separated) adds flags to every unit,
    e.g. the sort's shape: -DPZ_SORT_THREADS=256 -DPZ_SORT_ITEMS=16 -DPZ_SORT_RANK_MATCH=0
    -DPZ_SORT_EARLY_COUNTS=1 -DPZ_SORT_MIN_BLOCKS=4 (the defaults)."""
    os.makedirs(OBJ, exist_ok=True)
    extra = os.environ.get("PZ_EXTRA_NVCC_FLAGS", "").split()
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.cuh")) + \
        [_stamp_flags(extra)]
    objs, procs = [], []
    for unit, (srcname, flags) in UNITS.items():
        src = os.path.join(CSRC, srcname)
        obj = os.path.join(OBJ, unit + ".o")
        objs.append(obj)
        if _newer(obj, [src] + headers + [__file__]):
            cmd = [NVCC] + ARCH + COMMON + flags + extra + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((unit, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for unit, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append(unit)
            sys.stderr.write(out.decode())
        elif verbose and out:
            sys.stdout.write(out.decode())
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    if _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    build_pk_render(verbose)
    return LIB


def build_pk_render(verbose: bool = False) -> str:
    """The C++ facade's driver (include/palzilla_b200.hpp, cpp/pk_render.cpp)."""
    src = os.path.join(HERE, "cpp", "pk_render.cpp")
    hdrs = glob.glob(os.path.join(ROOT, "include", "*.h*"))
    if _newer(PK_RENDER, [src, LIB] + hdrs):
        cmd = ["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(CUDA_HOME, "include"),
               src, "-o", PK_RENDER, "-L" + HERE, "-lpalzilla_b200", "-L" + os.path.join(CUDA_HOME, "lib64"),
               "-lcudart", "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64")]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return PK_RENDER


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
