"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares (no compute calls here)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names += re.findall(r"^SG_API\s+[\w\s\*]+?\b(sg_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "sg_lde_commit" in names and "sg_ctx_create" in names
    assert len(names) >= 20


@pytest.fixture(scope="module")
def so():
    from lambda_vm_b200 import build
    path = build.build()
    return ctypes.CDLL(path)


@pytest.mark.parametrize("name", declared_symbols())
def test_library_exports(so, name):
    assert hasattr(so, name), f"{name} declared in include/ but not exported"


def test_python_prototypes_cover_header():
    from lambda_vm_b200 import native
    missing = [n for n in declared_symbols() if n not in native.PROTOTYPES]
    assert not missing, missing


def test_errors_without_gpu_are_status_codes(so):
    """Without a usable device the context call returns an error status
    (never aborts); with one it succeeds. Either way no exception escapes."""
    from lambda_vm_b200 import native
    L = native.lib()
    h = ctypes.c_void_p()
    rc = L.sg_ctx_create(0, 0, ctypes.byref(h))
    if rc == native.SG_OK:
        L.sg_ctx_destroy(h)
    else:
        assert rc in (native.SG_ERR_CUDA, native.SG_ERR_INVALID, native.SG_ERR_UNSUPPORTED)
        assert L.sg_last_error()
