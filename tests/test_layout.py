"""CPU: alignment and coverage of the stage kernel's shared-memory carve-up
and of the pair layout, checked by compiling tests/layout_check.cu (host code
only) against dm-heom_b200/csrc/heom_kernels.cuh."""
import os
import shutil
import subprocess

import pytest


def test_smem_layout_and_pair_table(tmp_path, root):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = tmp_path / "layout_check"
    subprocess.run([nvcc, "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(root, "dm-heom_b200", "csrc"),
                    "-o", str(exe), os.path.join(root, "tests", "layout_check.cu")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout[-2000:]
    assert out.stdout.strip().startswith("ok")
