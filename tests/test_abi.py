"""The C-ABI library loads and exports every entry point include/hyqmom.h declares
(no compute call: this runs without a GPU)."""
import os
import re

import pytest

from hyqmom import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "hyqmom.h")).read()
    return sorted(set(re.findall(r"\b(hyq_[a-z_A-Z]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert set(declared_symbols()) == set(_lib.SYMBOLS)


@pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="library not built")
def test_library_exports_all_symbols():
    lib = _lib.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.hyq_abi_version() == 1


def test_missing_library_fails_loudly(tmp_path):
    saved = _lib._lib
    _lib._lib = None
    try:
        with pytest.raises(_lib.HyqError):
            _lib.load(str(tmp_path / "nope.so"))
    finally:
        _lib._lib = saved
