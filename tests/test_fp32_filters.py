"""The fp32 arithmetic of the seed-search filters, checked on the host: the full-node part
index added by a fused multiply-add rounded toward minus infinity (exact floor), the
rotation-leaf bit index and its fp32 power of two, and the collision test of a left-mask sum
(tests/cpp/fp32_filters.c, exhaustive over every 16-bit hash). The device kernels compute the
same IEEE-754 binary32 operations (__fmaf_rd, __fadd_rn, __float2uint_rz)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_fp32_filter_arithmetic(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = tmp_path / "fp32_filters"
    subprocess.run([cc, "-std=c99", "-O2", "-frounding-math", "-Wall",
                    os.path.join(ROOT, "tests", "cpp", "fp32_filters.c"), "-o", str(exe), "-lm"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fp32 ok" in r.stdout
