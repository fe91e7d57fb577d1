"""The C-ABI library loads and exports every entry point include/exciting_b200.h declares."""
import ctypes
import os
import re

import pytest

from exciting_b200 import abi, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(exs_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if build.needs_build():
        build.build()
    return ctypes.CDLL(abi.LIB_PATH)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "exs_hamiltonandoverlapsetup" in names and "exs_match" in names and "exs_forcek" in names


@pytest.mark.parametrize("name", declared_symbols())
def test_symbol_exported(lib, name):
    assert hasattr(lib, name), name


def test_binding_covers_header():
    assert set(abi.SIGNATURES) == set(declared_symbols())


def test_null_arguments_rejected_without_gpu(lib):
    lib.exs_ctx_create.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.exs_ctx_create.restype = ctypes.c_int
    assert lib.exs_ctx_create(None, None) == -1
    out = ctypes.c_void_p()
    assert lib.exs_ctx_create(None, ctypes.byref(out)) == -1
