"""The per-context cache of freed pool blocks (pbgpu_internal.cuh BlockCache):
best fit within want .. 2 want + 64 KiB, and its byte and block caps, checked
by a host-only program compiled against the library's header (no GPU)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="nvcc not found")
def test_block_cache_host_logic(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = str(tmp_path / "block_cache_check")
    src = os.path.join(ROOT, "tests", "native", "block_cache_check.cu")
    subprocess.run([nvcc, "-std=c++17", "-O1", "-o", exe, src], check=True, capture_output=True, timeout=300)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "block cache ok" in out.stdout
