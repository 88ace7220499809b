"""The C ABI library: builds for sm_100a, loads without a GPU, and exports
every entry point declared in include/verb4d_b200.h (no compute calls here)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "verb4d_b200.h")
LIB = os.path.join(ROOT, "verb-4d_b200", "verb4d_b200", "libverb4d_b200.so")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*|void)\s+(verb_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "verb-4d_b200", "csrc")], check=True)
    return ctypes.CDLL(LIB)


def test_header_declares_the_api():
    syms = declared_symbols()
    for s in ("verb_create", "verb_step", "verb_local", "verb_radial", "verb_convection",
              "verb_diffusion_2d", "verb_convection_2d", "verb_assimilate_radial"):
        assert s in syms


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_signatures_cover_header():
    import sys

    sys.path.insert(0, os.path.join(ROOT, "verb-4d_b200"))
    from verb4d_b200 import _lib

    assert set(declared_symbols()) <= set(_lib.SIGNATURES), \
        set(declared_symbols()) - set(_lib.SIGNATURES)


def test_version_string(lib):
    lib.verb_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.verb_version()
    lib.verb_status_string.restype = ctypes.c_char_p
    assert lib.verb_status_string(3) == b"Courant number > 1"
