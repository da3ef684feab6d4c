"""Host-side logic of the seam kernels' shared-memory layout, compiled with
nvcc and run on the CPU (no GPU): closed-form staging offsets against
brute-force sums, the total against seam_smem_elems, and the staged / direct
choice for the shapes the library runs (tests/host/seam_layout.cu)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _nvcc():
    home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    exe = os.path.join(home, "bin", "nvcc")
    return exe if os.path.exists(exe) else shutil.which("nvcc")


@pytest.mark.skipif(_nvcc() is None, reason="nvcc not found")
def test_seam_layout(tmp_path):
    exe = str(tmp_path / "seam_layout")
    src = os.path.join(HERE, "host", "seam_layout.cu")
    r = subprocess.run([_nvcc(), "-std=c++17", "-o", exe, src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
