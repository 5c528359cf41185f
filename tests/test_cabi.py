"""The C-ABI library loads on a CPU host and exports every declared symbol."""

import ctypes
import re
from pathlib import Path

from easyfsi_b200 import _native
from easyfsi_b200.build import LIB_PATH, build

HEADER = Path(__file__).resolve().parent.parent / "include" / "easyfsi_b200.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+char\*|int|uint64_t)\s+(efsi_\w+)\s*\(", text, flags=re.M)))


def test_library_builds_and_loads():
    build()
    assert LIB_PATH.exists()
    lib = ctypes.CDLL(str(LIB_PATH))
    lib.efsi_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.efsi_version()


def test_every_declared_symbol_is_exported():
    build()
    lib = ctypes.CDLL(str(LIB_PATH))
    names = declared_functions()
    assert len(names) >= 38
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_header():
    assert sorted(_native.exported_names()) == declared_functions()


def test_argument_validation_without_gpu():
    # Argument checks run before any device work, so they are callable here.
    lib = _native.load()
    status = lib.efsi_fv_plan_create(None, 0, 1, None)
    assert status == 1
    assert b"invalid plan arguments" in lib.efsi_last_error()
    assert lib.efsi_mpm_plan_create(0, 4, 4, 4, None) == 1
