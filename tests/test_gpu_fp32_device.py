"""The fp32 forms of the seed-search filters, checked exhaustively on the device with the
very device functions the search kernels call (gpurecsplit_b200/csrc/rsb_fp32.cuh): the
full-node part index added by a rounded-down fused multiply-add for every fanout and 16-bit
hash, the integer part index of every non-full node of every leaf size, and the rotation-leaf
bit as an fp32 power of two for every leaf size (tests/cpp/fp32_device_check.cu)."""
import os
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_fp32_filters_on_the_device(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    exe = tmp_path / "fp32_device_check"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-I",
                    os.path.join(ROOT, "gpurecsplit_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "fp32_device_check.cu"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fp32 device ok" in r.stdout
