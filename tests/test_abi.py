"""The C-ABI library loads and exports every symbol include/*.h declares (no GPU needed)."""
import glob
import os
import re

import accelerint_b200 as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(accelerInt_\w+)\s*\(", src))
    return names


def _lib():
    if not os.path.exists(A.library_path()):
        from accelerint_b200.build import build
        build()
    return A.load_library()


def test_header_and_binding_agree():
    assert declared_symbols() == set(A.EXPORTED_SYMBOLS)


def test_library_exports_declared_symbols():
    lib = _lib()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert b"sm_100a" in lib.accelerInt_version()


def test_setters_validate_without_a_device():
    lib = _lib()
    assert lib.accelerInt_set_solver(99) == -1
    assert lib.accelerInt_set_tolerances(-1.0, 1e-6) == -1
    assert lib.accelerInt_set_lu_precision(7) == -1
