"""In-tree build of the native libraries.

* libstormm_b200.so        the CUDA path (csrc/*.cu) for sm_100a, C ABI in include/stormm_b200.h
* libstormm_b200_synth.so  the seeded synthetic-molecule builder (csrc/synthetic.cpp)

Run ``python -m stormm_b200.build`` (or __graft_entry__.build()).  nvcc cross-compiles without
a GPU.  Each translation unit compiles to its own object under _build/ (in parallel, one nvcc per
core); the library is linked from the objects.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJDIR = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libstormm_b200.so")
SYNTH_LIB = os.path.join(PKG, "libstormm_b200_synth.so")

CUDA_SOURCES = ["eval_fused.cu", "minimize.cu", "synthesis.cu", "transfers.cu",
                "static_scratch.cu", "server.cu", "tiled.cu", "fp64.cu", "line_search.cu", "charmm.cu", "sasa.cu",
                "exclusion_mask.cpp", "valence_units.cpp", "amber_io.cpp", "sdf_io.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-ftz=true"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.exists(cand) or cand == "nvcc"):
            return cand
    return "nvcc"


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _compile(src, headers, force, verbose):
    obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
    if not force and not _stale(obj, [src] + headers):
        return obj
    cmd = [_nvcc()] + NVCC_FLAGS + ["-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}")
    return obj


def build(force: bool = False, verbose: bool = False) -> None:
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES]
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "stormm_b200.h"))
    os.makedirs(OBJDIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as pool:
        objs = list(pool.map(lambda s: _compile(s, headers, force, verbose), srcs))
    if force or _stale(LIB, objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of libstormm_b200.so failed")
    synth_src = os.path.join(CSRC, "synthetic.cpp")
    if force or _stale(SYNTH_LIB, [synth_src]):
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", SYNTH_LIB, synth_src]
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
