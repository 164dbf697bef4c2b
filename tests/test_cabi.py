"""The C ABI library loads without a GPU and exports every function that
include/dampm_cuda.h declares."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "dampm_cuda.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(dampm_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from amsc_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    names = declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_null_context():
    from amsc_b200 import dampm
    lib = dampm.load_library()
    assert b"sm_100a" in lib.dampm_version()
    assert lib.dampm_ctx_destroy(None) != 0
    assert lib.dampm_step(None, 1) != 0
