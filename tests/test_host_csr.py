"""TF/SF table assembly (cpsfdtd_b200/csrc/tfsf_csr.h, used by cps_tfsf_init):
the multi-threaded counting sort, per-plane stable sorts and target runs give
byte for byte the arrays of a serial restatement of the same ordering, so
each TF/SF target keeps its contributions in the reference's face order
(TF_SF.cpp:988-1089, 1201-1300).  Host code only: compiled here with g++."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "cpsfdtd_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_tfsf_assembly_matches_serial_order(tmp_path):
    exe = str(tmp_path / "tfsf_csr_check")
    subprocess.run(["g++", "-O2", "-std=c++20", "-pthread", "-I", CSRC,
                    os.path.join(HERE, "host", "tfsf_csr_check.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("ok")
