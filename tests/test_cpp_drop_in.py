"""The reference's own trainer test in C++ against the reference's types, training through the
header-only drop-in (include/u3d_gpu.hpp): tests/cpp/drop_in_test, built by tests/cpp/Makefile where
the reference headers exist (the binary travels with the repository)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

EXE = Path(__file__).resolve().parent / "cpp" / "drop_in_test"


@pytest.mark.gpu
def test_cpp_drop_in(tmp_path):
    if not EXE.exists():
        pytest.skip("tests/cpp/drop_in_test is not built (the reference headers were absent)")
    r = subprocess.run([str(EXE)], capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "drop-in ok" in r.stdout
