"""Layout of the INT8 FP64 matvec kernels, checked on the host: every store,
bulk copy, descriptor range and tensor-memory column of oz_digits_kernel,
oz_pack_b_kernel and oz_mma_kernel against the buffers the solver allocates,
and exact once-only coverage of the digit planes and B image for small sizes
(tests/oz_layout_check.cu, built with nvcc as host code; no GPU needed)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "fastmbcui_b200", "csrc")


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    return None


def test_int8_matvec_layout(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not available")
    exe = str(tmp_path / "oz_layout_check")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-I", CSRC,
                    os.path.join(HERE, "oz_layout_check.cu"), "-o", exe], check=True, timeout=600)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "all layout checks passed" in r.stdout
