"""The C-ABI library loads without a GPU and exports every function include/*.h declares."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(be_[a-z0-9_]+)\s*\(", src):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("be_create", "be_destroy", "be_label2d", "be_label3d", "be_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    import labeling_b200 as be
    lib = ctypes.CDLL(be.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_no_cpu_fallback():
    import labeling_b200 as be
    assert be.version().count(".") == 2
    h = ctypes.c_void_p()
    rc = be.lib().be_create(ctypes.byref(h), 0)
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        assert rc != 0, "be_create must fail loudly without a GPU"
    else:
        assert rc == 0
        be.lib().be_destroy(h)
