"""The host-buffer pipeline's batch cut (utlpfor_b200/csrc/utl_pieces.h),
compiled with the host compiler and checked on seeded random stream tables
(tests/pieces_check.cc).  No GPU."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "utlpfor_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_cut_pieces(tmp_path):
    exe = str(tmp_path / "pieces_check")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", CSRC, os.path.join(HERE, "pieces_check.cc"), "-o", exe])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok "), out.stdout
