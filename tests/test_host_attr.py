"""Kernel attributes (dynamic shared memory above 48 KiB, carveout) are set
once per device and thread-safely (cpsfdtd_b200/csrc/attr_once.h, used by
every sweep, batch and DFT launcher): checked here with a fake device switch
and attribute call.  Host code only, compiled with g++."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "cpsfdtd_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_attributes_set_once_per_device(tmp_path):
    exe = str(tmp_path / "attr_once_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", CSRC,
                    os.path.join(HERE, "host", "attr_once_check.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("ok")
