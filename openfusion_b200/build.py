"""In-tree build of the native libraries.

libopenfusion_b200.so  -- the sm_100a CUDA path behind include/openfusion_b200.h
libof_synth.so         -- host C++ synthetic seeded scenes (depth renderer)

Run ``python -m openfusion_b200.build`` (or ``__graft_entry__.build()``).
Objects go to ``openfusion_b200/_build``; the shared libraries to
``openfusion_b200/lib``. nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"

CUDA_SOURCES = [
    "of_core.cu",
    "of_preprocess.cu",
    "of_integrate.cu",
    "of_raycast.cu",
    "of_icp.cu",
    "of_tracker.cu",
    "of_adapters.cu",
    "of_synth_gpu.cu",
    "of_cnn.cu",
    "of_batch.cu",
    "of_recording.cu",
    "of_mesh.cu",
    "of_filters.cu",
]
SYNTH_SOURCES = ["of_synth.cpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I" + str(ROOT / "include")]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build openfusion_b200")


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, ptxas_verbose: bool = False) -> dict[str, Path]:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    nvcc = _nvcc()
    headers = sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "openfusion_b200.h",
                                           CSRC / "of_synth.h"]
    objs = []
    jobs = []
    for src in CUDA_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_verbose:
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-c", str(s), "-o", str(o)]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(_run, jobs))
    lib = LIBDIR / "libopenfusion_b200.so"
    if _stale(lib, objs):
        _run([nvcc, *ARCH, "-shared", "-o", str(lib), *map(str, objs), "-lcudart"])
    synth = LIBDIR / "libof_synth.so"
    ssrc = [CSRC / s for s in SYNTH_SOURCES]
    if _stale(synth, ssrc + [CSRC / "of_synth.h"]):
        _run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp",
              *map(str, ssrc), "-o", str(synth)])
    if verbose:
        print("built", lib, synth)
    return {"cuda": lib, "synth": synth}


if __name__ == "__main__":
    build(verbose=True, ptxas_verbose="-v" in sys.argv)
