"""bench.py's reference arm (--impl reference) runs on the host cores, so its JSON line is checked here:
one line with the keys of the benchmark's contract, at one rank and under torchrun with two ranks
(rank 0 alone runs and prints; the other rank exits 0 without work), on the small configuration."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["--impl", "reference", "--config", "small", "--steps", "3", "--warmup", "3"]


def _lines(out):
    return [json.loads(x) for x in out.splitlines() if x.startswith("{")]


def _check(line, n_gpus):
    assert line["impl"] == "reference" and line["metric"] == "walker-steps/s" and line["unit"] == "walker-steps/s"
    assert line["value"] > 0 and line["ms_per_step"] > 0 and line["higher_is_better"] is True
    assert (line["n_gpus"], line["steps"], line["warmup"]) == (n_gpus, 3, 3)
    assert line["dtype"] == "f64" and line["data"] == "synthetic" and line["vs_baseline"] is None
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    cfg = line["config"]
    assert cfg["M"] == 24 and cfg["walkers_per_gpu"] == 32 and "workload" in cfg and "l2" in cfg


def test_reference_arm_line_one_rank():
    r = subprocess.run([sys.executable, "bench.py"] + ARGS, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0], 1)


def test_reference_arm_rejects_short_warmup():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--config", "small", "--warmup", "2"],
                       cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode != 0 and "warmup" in r.stderr


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_prints_one_line():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--gpus", "2"] + ARGS
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=540)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0], 2)
