"""C++ programs against the reference's own types through the header-only drop-in (include/u3d_gpu.hpp),
built by tests/cpp/Makefile where the reference headers exist (the binaries travel with the repository):
tests/cpp/drop_in_test, the reference's trainer test with the trainer switched to the GPU one, and
tests/cpp/stage_test, the pipeline's training stage (Reconstructor.cpp:296-361) on the GPU trainer."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

EXE = Path(__file__).resolve().parent / "cpp" / "drop_in_test"
STAGE = Path(__file__).resolve().parent / "cpp" / "stage_test"


@pytest.mark.gpu
def test_cpp_drop_in(tmp_path):
    if not EXE.exists():
        pytest.skip("tests/cpp/drop_in_test is not built (the reference headers were absent)")
    r = subprocess.run([str(EXE)], capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "drop-in ok" in r.stdout


@pytest.mark.gpu
def test_cpp_pipeline_training_stage(tmp_path):
    if not STAGE.exists():
        pytest.skip("tests/cpp/stage_test is not built (the reference headers were absent)")
    r = subprocess.run([str(STAGE)], capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "stage ok" in r.stdout
