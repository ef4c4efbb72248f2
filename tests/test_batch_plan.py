"""The host-side planning of lrb_int2e_batch (librint_b200/csrc/batch_plan.h:
shell-index and bas-entry checks, chunking, the molecule ranges each chunk
uploads) equals a serial restatement of its rules on random batches and
corruptions: tests/batch_plan_check.cpp, built with the host compiler and
run here (no GPU)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_plan_batch_matches_serial_restatement(tmp_path):
    exe = str(tmp_path / "batch_plan_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-Wall",
                    os.path.join(HERE, "batch_plan_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok "), r.stdout
    assert int(r.stdout.split()[1]) > 5000
