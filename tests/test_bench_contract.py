"""The JSON line bench.py prints, checked on the CPU through its reference
arm (the reference's scalar kernels built for the host, or the oracle port
when that build is absent) on a small grid."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_reference_arm_line():
    d = _run("--impl", "reference", "--steps", "2", "--warmup", "1", "--nx", "32", "--ny", "16",
             "--nz", "16")
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["metric"] == "Gcell-RHS/s" and d["unit"] == "Gcell-RHS/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["steps"] == 2 and d["warmup"] == 1 and d["dtype"] == "f64"
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("reference", "port") and cb["cores"] >= 1
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 == e["d2h_bytes_per_step"]
    c = d["config"]
    assert c["grid"] == [32, 16, 16] and c["inputs_exceed_l2"] is False
    assert "workload" in c and "model" not in c
    # one reference step is one whole SSP-RK3 time step of the full grid,
    # as on the GPU arm (3 RHS evaluations per step)
    assert c["rhs_per_step"] == 3 and "SSP-RK3 time step of the 32x16x16 grid" in cb["sample"]
    assert d["dt"] > 0


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def torchrun_bench(nproc, *args, timeout=600):
    """bench.py under torch.distributed.run, one rank per process, as the
    multi-GPU runs launch it; returns (JSON lines printed, stderr)."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={nproc}", "--master-addr=127.0.0.1",
           f"--master-port={_free_port()}", os.path.join(ROOT, "bench.py"), *args]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-3000:]
    return [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")], out.stderr


def test_reference_arm_two_ranks_prints_once():
    """Under torchrun the reference arm runs on rank 0 alone; the other ranks
    exit 0 without work or output."""
    lines, _ = torchrun_bench(2, "--impl", "reference", "--gpus", "2", "--steps", "2",
                              "--warmup", "1", "--nx", "32", "--ny", "16", "--nz", "16")
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["config"]["parallelism"] == "blocks2x1x1"
