"""The deferred Clifford frame's direct rotation update against full tableau
composition (tableau.rs:180-209 composed as in tableau.rs:109-143), on the
host, compiled from the engine's own header with g++."""

import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_rotation_update_equals_full_composition(tmp_path):
    exe = tmp_path / "tableau_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe), str(HERE / "tableau_check.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr
