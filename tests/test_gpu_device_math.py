"""Device arithmetic helpers checked against CUDA's own results on the GPU."""

import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
HERE = Path(__file__).resolve().parent


def test_fast_reciprocal_within_two_ulps(tmp_path):
    """sapb::fast_recip (Newton-Raphson from an FP32 seed, used for the LDL^T
    pivots) stays within 2 ulps of the IEEE quotient 1.0/d over 1e-35..1e35."""
    exe = tmp_path / "recip_check"
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-o", str(exe),
                    str(HERE / "cuda" / "recip_check.cu")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    worst = int(out.split("max_ulps")[1].split()[0])
    assert worst <= 2, out
