"""The binary16 and bfloat16 stochastic rounding of the 16-bit storage formats
runs on the hardware's cvt.rs for pairs of planes (h16x2_enc_sr,
bf16x2_enc_sr), fed the bits that the software roundings h16_enc /
bf16_store take from the same draws.  bfloat16 must agree everywhere.  A
native check (tests/native/sr_check.cu) converts 2^21 deterministic
pseudo-random values both ways: the results must agree for normal binary16
results (the only differences sit at the overflow edge above 65504); in the
subnormal range the hardware dithers at the subnormal's last bit and the
software does not, so those are counted, not compared."""
import os
import re
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def test_hardware_stochastic_rounding_matches_software_in_the_normal_range(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("no nvcc")
    exe = tmp_path / "sr_check"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
                    "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "cfd_cavity_b200", "csrc"),
                    os.path.join(ROOT, "tests", "native", "sr_check.cu"), "-o", str(exe)],
                   check=True, capture_output=True, timeout=300)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    m = re.search(r"err (\d+)\s+mismatches \(normal range\) (\d+)\s+\(subnormal range\) (\d+)\s+of \d+\s+"
                  r"bf16 (\d+)", r.stdout)
    assert m and int(m.group(1)) == 0, r.stdout
    assert int(m.group(2)) <= 64, r.stdout  # overflow edge only (33 on a B200)
    assert int(m.group(4)) == 0, r.stdout
