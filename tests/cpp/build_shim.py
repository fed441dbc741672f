"""Builds tests/cpp/shim_track (g++ against the in-tree shared libraries)."""
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
OUT = ROOT / "tests" / "cpp" / "_build" / "shim_track"


def build() -> Path:
    OUT.parent.mkdir(exist_ok=True)
    lib = ROOT / "openfusion_b200" / "lib"
    src = ROOT / "tests" / "cpp" / "shim_track.cpp"
    deps = [src, ROOT / "include" / "openfusion_b200.hpp", ROOT / "include" / "openfusion_b200.h"]
    if OUT.exists() and all(OUT.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return OUT
    cmd = ["g++", "-O2", "-std=c++17", str(src), "-o", str(OUT),
           "-I", str(ROOT / "include"), "-I", str(ROOT / "openfusion_b200" / "csrc"),
           "-I", "/usr/local/cuda/include", "-L", str(lib), "-lopenfusion_b200", "-lof_synth",
           "-L", "/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath,$ORIGIN/../../../openfusion_b200/lib",
           "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build())
    sys.exit(0)
