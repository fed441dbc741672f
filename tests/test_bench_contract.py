"""bench.py's reference arm on the CPU: one JSON line with the keys of the
benchmark contract, the reference tag, a CPU baseline describing the run and
an end-to-end figure with no host-device copies."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

CONTRACT_KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                 "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config"}


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "1", "--frames", "6"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert CONTRACT_KEYS <= d.keys()
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["unit"] == "frames/s" and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["steps"] >= 1 and d["warmup"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("c2_640x480_512")


def test_reference_arm_under_torchrun_prints_from_rank_0_only():
    """Two ranks launched the way the multi-GPU runs are (torchrun, one node,
    127.0.0.1): rank 0 alone measures and prints; the other exits 0."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                          "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
                          "--master-port", str(port), str(ROOT / "bench.py"), "--impl",
                          "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
                          "--frames", "6"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.lstrip().startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0].strip())
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
