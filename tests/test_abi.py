"""CPU checks of the C ABI library: it loads, and it exports every entry point
that include/samos_gpu.h declares (no compute calls without a GPU)."""
import ctypes
import os
import re

import pytest

from samos_b200 import engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "samos_gpu.h")).read()
    return sorted(set(re.findall(r"\b(sg_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_abi():
    syms = declared_symbols()
    for name in ("sg_create", "sg_run", "sg_set_nlist", "sg_add_pair", "sg_add_integrator", "sg_get_pairs"):
        assert name in syms


def test_library_exports_every_declared_symbol():
    if not os.path.exists(engine.library_path()):
        pytest.fail("libsamos_gpu.so has not been built (run __graft_entry__.build())")
    lib = ctypes.CDLL(engine.library_path())
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_error_strings_without_device():
    lib = engine.load()
    assert lib.sg_error_string(0) == b"ok"
    assert lib.sg_error_string(-5) == b"neighbour capacity exceeded"
