"""The C-ABI library loads and exports every entry point the public header declares.
No compute calls: this runs without a GPU."""
import ctypes as C

from mguso import _lib


def test_header_declares_entry_points():
    syms = _lib.header_symbols()
    assert "mguso_linear_solve" in syms and "mguso_bsr_spmv" in syms
    assert len(syms) >= 20


def test_library_exports_every_header_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [s for s in _lib.header_symbols() if not hasattr(lib, s)]
    assert not missing, f"declared in include/mguso_cuda.h but not exported: {missing}"


def test_version_and_last_error_without_gpu():
    lib = _lib.load()
    assert lib.mguso_version() >= 100
    buf = C.create_string_buffer(64)
    lib.mguso_last_error(buf, 64)  # empty on a fresh thread; must not crash


def test_invalid_arguments_are_rejected_without_gpu():
    lib = _lib.load()
    assert lib.mguso_linear_solver_create(None, 1, 32, 1, None) == 1  # INVALID_ARG
    assert "null" in _lib.last_error()
