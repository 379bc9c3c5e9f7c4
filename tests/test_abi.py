"""CPU tests of the C ABI library: it loads, exports every symbol the header
declares, and fails loudly (no fallback) when no GPU is present."""
import ctypes
import os
import re

import pytest

from conftest import ROOT
from tflows_b200 import native

HEADER = os.path.join(ROOT, "include", "tf_krylov.h")


def header_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tf_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(native.LIB_PATH):
        import subprocess, sys
        subprocess.run([sys.executable, os.path.join(ROOT, "t-flows_b200", "build.py"),
                        "--lib"], check=True)
    return native.load()


def test_library_exports_every_declared_symbol(lib):
    syms = header_symbols()
    assert len(syms) >= 19
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert set(native.EXPORTS) <= set(syms)


def test_status_strings(lib):
    assert lib.tf_status_string(0) == b"ok"
    assert lib.tf_status_string(64) == b"unknown native solver"
    assert lib.tf_status_string(72) == b"unknown preconditioner"
    assert lib.tf_status_string(9) == b"host-side failure"
    assert b"sm_100a" in lib.tf_version()


def test_no_silent_fallback_without_gpu(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert lib.tf_ctx_create(0, ctypes.byref(h)) == 6   # TF_ERR_NO_DEVICE
    with pytest.raises(native.TFError):
        native.Context(0)


def test_null_arguments_rejected(lib):
    assert lib.tf_ctx_create(0, None) == 3
    assert lib.tf_ctx_destroy(None) == 3
    assert lib.tf_matrix_release(None) == 3
    n = ctypes.c_int()
    r = ctypes.c_double()
    assert lib.tf_solve(None, None, 0, 1, None, None, None, 10, ctypes.byref(n), 1e-6,
                        ctypes.byref(r), None) == 3
    # batched entry points reject a missing handle before touching a device
    assert lib.tf_batch_add_many(None, 0, None, None, None, None, None, None, None, None,
                                 None, None, 0, None) == 3
    assert lib.tf_batch_run(None) == 3


def header_prototypes():
    """{name: number of parameters} of every function the header declares."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(tf_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", txt, flags=re.S):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_bindings_pass_as_many_arguments_as_the_header_declares(lib):
    """Every argtypes list set by the Python bindings has the length of the
    C prototype (a mismatch would pass garbage through the ABI)."""
    from tflows_b200 import batch, pool
    batch._lib()
    pool._lib()
    protos = header_prototypes()
    checked = 0
    for name, nargs in protos.items():
        fn = getattr(lib, name, None)
        argtypes = getattr(fn, "argtypes", None) if fn is not None else None
        if argtypes is None:
            continue
        assert len(argtypes) == nargs, (name, len(argtypes), nargs)
        checked += 1
    assert checked >= 40
