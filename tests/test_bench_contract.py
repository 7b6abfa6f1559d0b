"""bench.py's output contract, checked on the CPU through its reference arm (the reference's own CPU
trainer, oracle/_ref): one JSON line with the metric, the bounded-sample description and the e2e
block; under torchrun with two ranks, rank 0 alone prints it and every rank exits 0."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
ARGS = ["--impl", "reference", "--steps", "2", "--warmup", "3", "--workload", "fast-80k"]


def _lines(out: str):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def _check(line, n_gpus):
    assert line["impl"] == "reference" and line["unit"] == "it/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 2 and line["warmup"] == 3 and line["n_gpus"] == n_gpus
    assert line["config"]["workload"] == "fast-80k"
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"] and cb["cores"] >= 1
    assert "fast-80k" in cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "it/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


@pytest.fixture(scope="module")
def reference_built(reference):
    return reference


def test_reference_arm_prints_one_line(reference_built):
    r = subprocess.run([sys.executable, "bench.py", *ARGS], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0], 1)


def test_reference_arm_under_torchrun_two_ranks(reference_built):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--gpus", "2", *ARGS],
                       cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0], 2)


def test_roofline_figures_come_from_the_committed_profiles():
    """The bench's roofline line reads the dominant kernels' DRAM traffic and pipe utilisation from the
    committed ncu summaries (profiles/*_high-300k.md)."""
    sys.path.insert(0, str(ROOT))
    import bench
    for kernel in ("compositeBackwardKernel", "compositeForwardKernel", "chainKernel"):
        traffic = bench.profiled_traffic(kernel)
        assert traffic is not None and traffic > 1e6, kernel
        for metric in ("smsp__issue_active.avg.pct_of_peak_sustained_active",
                       "sm__pipe_fma_cycles_active.avg.pct_of_peak_sustained_active",
                       "gpu__dram_throughput.avg.pct_of_peak_sustained_elapsed"):
            v = bench.profiled_metric(kernel, metric)
            assert v is not None and 0.0 <= v <= 100.0, (kernel, metric, v)
    assert bench.profiled_traffic("noSuchKernel") is None
