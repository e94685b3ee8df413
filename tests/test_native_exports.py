"""The C-ABI library loads on CPU-only hosts and exports every declared symbol."""
import ctypes

from tpt_fem import _native as N


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(N.LIB_PATH)
    declared = N.declared_symbols()
    assert len(declared) >= 25
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert set(N.declared_symbols()) == set(N.SIGNATURES)


def test_version_string_without_gpu():
    lib = N.load()
    assert b"sm_100a" in lib.tptfem_version()
