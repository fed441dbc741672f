"""Builds oracle/_ref/libref_kernels.so from the reference's own kernel sources.

TEST INFRASTRUCTURE ONLY. Each harness TU in this folder includes one
unmodified .cu file of gilbs10/OpenFusion from the reference tree (read in
place, never copied), compiled by nvcc for sm_100a with two empty OpenGL stub
headers (the reference pulls in GLEW/freeglut only for its display structs).
Output goes to oracle/_ref/ (git-ignored; it travels to the GPU box with the
repository snapshot). Skips quietly when the reference tree is absent.
"""
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / "_ref"
REF = Path("/root/reference/Source")
TUS = ["ref_camera.cu", "ref_volume.cu", "ref_general.cu", "ref_raycast.cu", "ref_icp.cu",
       "ref_pipeline.cu", "ref_filters.cu"]


def build() -> Path | None:
    if not REF.exists():
        return None
    OUT.mkdir(exist_ok=True)
    lib = OUT / "libref_kernels.so"
    srcs = [HERE / t for t in TUS]
    if lib.exists() and all(lib.stat().st_mtime >= s.stat().st_mtime for s in srcs):
        return lib
    nvcc = "/usr/local/cuda/bin/nvcc"
    inc = ["-I", str(HERE / "stubs"), "-I", str(HERE), "-I", str(REF / "include"),
           "-I", str(REF / "include" / "Utils"), "-I", str(REF / "src"),
           "-I", str(REF / "src" / "CameraSupport"), "-I", str(REF / "include" / "Eigen" / "..")]
    objs = []
    procs = []
    for s in srcs:
        o = OUT / (s.name + ".o")
        objs.append(o)
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-w",
               "-Xcompiler", "-fPIC", *inc, "-c", str(s), "-o", str(o)]
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
