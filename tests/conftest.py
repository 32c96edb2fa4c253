import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a path")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the native libraries once per session (no-op when up to date)."""
    from cudanextgenpb_b200 import build
    build.build_all()
    yield


def cuda_available():
    try:
        import ctypes

        from cudanextgenpb_b200 import _native as N
        lib = N.load_gpu()
        ctx = ctypes.c_void_p()
        st = lib.pbgpu_ctx_create(ctypes.byref(ctx), 0, None)
        if st == 0:
            lib.pbgpu_ctx_destroy(ctx)
            return True
    except Exception:
        pass
    return False
