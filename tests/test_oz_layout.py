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


def _cutlass_include():
    """A CUTLASS include tree vendored in the environment (flashinfer's), if any."""
    try:
        import importlib.util

        spec = importlib.util.find_spec("flashinfer")
    except (ImportError, ValueError):
        return None
    if spec is None or not spec.submodule_search_locations:
        return None
    for loc in spec.submodule_search_locations:
        inc = os.path.join(loc, "data", "cutlass", "include")
        if os.path.exists(os.path.join(inc, "cute", "arch", "mma_sm100_desc.hpp")):
            return inc
    return None


def test_tcgen05_descriptors_match_cutlass(tmp_path):
    """The hand-built kind::i8 / kind::tf32 instruction descriptors and the
    128-byte-swizzle shared-memory descriptor equal CUTLASS's sm100
    constructors (tests/oz_desc_check.cu)."""
    nvcc, inc = _nvcc(), _cutlass_include()
    if nvcc is None or inc is None:
        pytest.skip("nvcc or a CUTLASS include tree not available")
    exe = str(tmp_path / "oz_desc_check")
    subprocess.run([nvcc, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a", "-I", inc, "-I", CSRC,
                    os.path.join(HERE, "oz_desc_check.cu"), "-o", exe], check=True, timeout=600)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "all descriptors equal" in r.stdout
