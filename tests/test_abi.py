"""The C ABI libraries load and export every entry point their headers declare."""
import ctypes
import os
import re

import pytest

from cudanextgenpb_b200 import _native as N
from cudanextgenpb_b200 import parse_lis_options

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b((?:pbgpu|pbhost)_[a-z_0-9]+)\s*\(", text)))


@pytest.mark.parametrize("header,loader", [("pbgpu.h", N.load_gpu), ("pbhost.h", N.load_host)])
def test_exports_every_declared_symbol(header, loader):
    lib = loader()
    names = declared(header)
    assert len(names) > 10
    for name in names:
        assert hasattr(lib, name), name


def test_bindings_cover_header():
    assert set(declared("pbgpu.h")) == set(N.PBGPU_FUNCS)
    assert set(declared("pbhost.h")) == set(N.PBHOST_FUNCS)


def test_parse_lis_options():
    o = parse_lis_options("-i bicgstab -p jacobi -tol 1.e-8")
    assert (o.method, o.precond, o.tol) == (N.PBGPU_BICGSTAB, N.PBGPU_PRECOND_JACOBI, 1e-8)
    # the reference's default solver_options (src/pb_class.cpp:970)
    o = parse_lis_options("-p ssor -ssor_omega 0.51 -i cgs -tol 1.e-6 -print 2 -conv_cond 2 -tol_w 0")
    assert (o.method, o.precond, o.tol) == (N.PBGPU_CGS, N.PBGPU_PRECOND_BLOCK_JACOBI, 1e-6)
    assert (o.conv_cond, o.tol_w) == (2, 0.0)
    o = parse_lis_options("-i bicgstab")
    assert (o.conv_cond, o.tol_w) == (0, 1.0)
    with pytest.raises(Exception):
        parse_lis_options("-conv_cond 3")
    o = parse_lis_options("-i cg -p jacobi -tol 1e-10 -maxiter 77")
    assert (o.method, o.max_iter, o.tol) == (N.PBGPU_CG, 77, 1e-10)
    with pytest.raises(Exception):
        parse_lis_options("-tol -1")


def test_null_arguments_are_rejected():
    lib = N.load_gpu()
    assert lib.pbgpu_ctx_create(None, 0, None) == N.PBGPU_ERR_ARG
    assert lib.pbgpu_create_markers(None) == N.PBGPU_ERR_ARG
    assert lib.pbgpu_solve(None, None, None) == N.PBGPU_ERR_ARG
    assert lib.pbgpu_last_error(None) == b"null context"


def test_no_device_reports_cuda_error():
    from conftest import cuda_available
    if cuda_available():
        pytest.skip("a CUDA device is present")
    lib = N.load_gpu()
    ctx = ctypes.c_void_p()
    assert lib.pbgpu_ctx_create(ctypes.byref(ctx), 0, None) == N.PBGPU_ERR_CUDA
