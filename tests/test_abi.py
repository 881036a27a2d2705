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
    assert lib.hyq_abi_version() == 2


def test_missing_library_fails_loudly(tmp_path):
    saved = _lib._lib
    _lib._lib = None
    try:
        with pytest.raises(_lib.HyqError):
            _lib.load(str(tmp_path / "nope.so"))
    finally:
        _lib._lib = saved


@pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="library not built")
def test_create_rejects_grids_beyond_the_list_limit():
    """hyq_create checks the grid on the host before any CUDA call, so this
    runs without a GPU: 2^29 cells and more do not fit the 32-bit entries of
    the step's cell lists."""
    import ctypes
    from hyqmom.runner import params_struct
    from hyqmom import ic
    lib = _lib.load()
    p = ic.default_params(Nx=1024, Ny=1024, Nz=512)  # exactly 2^29 cells
    h = ctypes.c_void_p()
    assert lib.hyq_create(ctypes.byref(params_struct(p)), ctypes.byref(h)) == -1
    assert "2^29" in lib.hyq_last_error(None).decode()
    p = ic.default_params(Nx=1, Ny=4, Nz=4)
    assert lib.hyq_create(ctypes.byref(params_struct(p)), ctypes.byref(h)) == -1


@pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="library not built")
def test_create_rejects_unknown_mode():
    """The eigenvalue-path mode is checked on the host before any CUDA call."""
    import ctypes
    from hyqmom.runner import params_struct
    from hyqmom import ic
    lib = _lib.load()
    hp = params_struct(ic.default_params(Nx=8, Ny=8, Nz=8))
    hp.mode = 7
    h = ctypes.c_void_p()
    assert lib.hyq_create(ctypes.byref(hp), ctypes.byref(h)) == -1
    assert "mode" in lib.hyq_last_error(None).decode()


def test_params_struct_layout_matches_header():
    """hyq_params / hyq_stats: the ctypes layouts have the C struct sizes
    (int32 x 6, int64, double x 11, int32 x 2; stats: double x 3, int64,
    int32 x 2, int64 x 2, int32 x 2, double x 3, int64, double, int64)."""
    import ctypes
    assert ctypes.sizeof(_lib.HyqParams) == 6 * 4 + 8 + 11 * 8 + 2 * 4
    assert ctypes.sizeof(_lib.HyqStats) == 3 * 8 + 8 + 2 * 4 + 2 * 8 + 2 * 4 + 3 * 8 + 8 + 8 + 8
