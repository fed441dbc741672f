"""Builds the reference's own kernel sources into oracle/_ref/.

TEST INFRASTRUCTURE ONLY. Each harness TU in this folder includes one
unmodified .cu file of gilbs10/OpenFusion from the reference tree (read in
place, never copied), compiled by nvcc for sm_100a with two empty OpenGL stub
headers (the reference pulls in GLEW/freeglut only for its display structs).
Output goes to oracle/_ref/ (git-ignored; it travels to the GPU box with the
repository snapshot). Skips quietly when the reference tree is absent.

Two libraries:
  libref_kernels.so     the reference's geometry as written in Constants.h
                        (512^3 over 1024 mm, truncation 10 mm, max weight 120);
                        the golden fixtures come from it.
  libref_kernels_c2.so  the full-size workload's geometry (512^3 over 3000 mm,
                        truncation 30 mm, max weight 128). The reference sets
                        these as compile-time constants (Constants.h:23-25,
                        52-54), so the build generates a Constants.h with the
                        new values into oracle/_ref/c2_gen/ and force-includes
                        it: it carries the reference's include guard, so the
                        reference's own Constants.h then adds nothing. The
                        raycast's march step and end margin are literals for a
                        1024 mm cube (Raycaster.cu:110, :195; 1.5 mm = 0.75
                        voxel of 2 mm); a generated copy of Raycaster.cu in the
                        same folder scales both by worldVolume / 1024, so the
                        step stays 0.75 voxel. maxSteps (850) is kept: it
                        covers the same 1.245 cube widths. Nothing generated is
                        committed.
"""
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / "_ref"
REF = Path("/root/reference/Source")
TUS = ["ref_camera.cu", "ref_volume.cu", "ref_general.cu", "ref_raycast.cu", "ref_icp.cu",
       "ref_pipeline.cu", "ref_filters.cu"]


# (reference file, pattern, replacement): each pattern must match exactly once
# (anchored at a line start, so commented-out alternatives are left alone)
C2_EDITS = [
    ("include/Constants.h", r"^const unsigned int worldVolume = 1024;",
     "const unsigned int worldVolume = 3000;"),
    ("include/Constants.h", r"^#define TRUNCATION \(10\.f\)", "#define TRUNCATION (30.f)"),
    ("include/Constants.h", r"^#define MAX_WEIGHT \(120\)", "#define MAX_WEIGHT (128)"),
    ("src/Raycaster.cu", r"const float tstep = 1\.5f;",
     "const float tstep = 1.5f * ((float)worldVolume / 1024.f);"),
    ("src/Raycaster.cu", r"if \(t > tfar - 2\.0\) break;",
     "if (t > tfar - 2.0 * ((float)worldVolume / 1024.f)) break;"),
]


def generate_c2(gen: Path) -> None:
    """Writes the full-size geometry's Constants.h and Raycaster.cu into `gen`."""
    gen.mkdir(parents=True, exist_ok=True)
    for rel in sorted({r for r, _, _ in C2_EDITS}):
        text = (REF / rel).read_text()
        for r2, pat, rep in C2_EDITS:
            if r2 != rel:
                continue
            text, n = re.subn(pat, rep, text, flags=re.M)
            if n != 1:
                raise RuntimeError(f"{rel}: pattern {pat!r} matched {n} times")
        (gen / Path(rel).name).write_text(text)


def build() -> Path | None:
    if not REF.exists():
        return None
    OUT.mkdir(exist_ok=True)
    lib = _build_variant("libref_kernels.so", OUT / "obj", [], [])
    gen = OUT / "c2_gen"
    generate_c2(gen)
    _build_variant("libref_kernels_c2.so", OUT / "obj_c2", ["-I", str(gen)],
                   ["-include", str(gen / "Constants.h")])
    return lib


def _build_variant(name: str, objdir: Path, first_inc: list[str], extra: list[str]) -> Path:
    lib = OUT / name
    srcs = [HERE / t for t in TUS]
    if lib.exists() and all(lib.stat().st_mtime >= s.stat().st_mtime
                            for s in srcs + [Path(__file__)]):
        return lib
    objdir.mkdir(parents=True, exist_ok=True)
    nvcc = "/usr/local/cuda/bin/nvcc"
    inc = first_inc + [
        "-I", str(HERE / "stubs"), "-I", str(HERE), "-I", str(REF / "include"),
        "-I", str(REF / "include" / "Utils"), "-I", str(REF / "src"),
        "-I", str(REF / "src" / "CameraSupport"), "-I", str(REF / "include" / "Eigen" / "..")]
    objs = []
    procs = []
    for s in srcs:
        o = objdir / (s.name + ".o")
        objs.append(o)
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-w",
               "-Xcompiler", "-fPIC", *extra, *inc, "-c", str(s), "-o", str(o)]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                            text=True)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("reference harness build failed:\n" + " ".join(cmd) + "\n" + out)
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(lib),
                    *map(str, objs), "-lcudart"], check=True)
    return lib


if __name__ == "__main__":
    print(build())
    sys.exit(0)
