"""The C-ABI library loads on a CPU host and exports every declared symbol."""

import ctypes
import re
from pathlib import Path

import pytest

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


def test_membrane_entry_points_reject_bad_arguments_without_gpu():
    # efsi_shell_*: the state checks run before any launch
    from ctypes import byref, c_float

    lib = _native.load()
    assert lib.efsi_shell_step(None, None, None, None, None) == 1
    assert b"shell state is NULL" in lib.efsi_last_error()
    st = _native.ShellState()
    st.particle_count, st.face_count, st.nx, st.ny, st.nz = 3, 1, 3, 8, 8
    assert lib.efsi_shell_update_normals(byref(st), None) == 1
    assert b"grid_nodes must be at least 4" in lib.efsi_last_error()
    st.nx = 8
    for a in range(3):
        st.dx[a] = 0.1
    assert lib.efsi_shell_add_region_area_load(byref(st), 1, (c_float * 3)(0, 0, 1), None) == 1
    assert b"buffer is NULL" in lib.efsi_last_error()


def test_ib_entry_points_reject_bad_arguments_without_gpu():
    """The IB node search, boundary-condition and row entry points check
    their arguments before any device work (hibm_mpm.py:6069-6094, 7673-7678)."""
    from ctypes import byref, c_void_p

    lib = _native.load()
    fake_plan = c_void_p(1)  # never dereferenced: every call below fails an argument check first
    prm = _native.IbSearchParams()
    out = _native.IbSearchFields()
    assert lib.efsi_ib_node_search(None, byref(prm), byref(out), None) == 1
    assert b"null argument" in lib.efsi_last_error()
    prm.nx = prm.ny = prm.nz = 2
    prm.search_radius_m = 0.0
    prm.interior_probe_distance_m = 0.1
    assert lib.efsi_ib_node_search(fake_plan, byref(prm), byref(out), None) == 1
    assert b"search_radius_m" in lib.efsi_last_error()
    prm.search_radius_m = float("inf")
    assert lib.efsi_ib_node_search(fake_plan, byref(prm), byref(out), None) == 1
    assert b"search_radius_m" in lib.efsi_last_error()
    prm.search_radius_m = 0.1
    prm.sign_tolerance_m = -1.0
    assert lib.efsi_ib_node_search(fake_plan, byref(prm), byref(out), None) == 1
    assert b"sign_tolerance_m" in lib.efsi_last_error()
    prm.sign_tolerance_m = 0.0
    prm.marker_count = 3  # marker arrays missing
    assert lib.efsi_ib_node_search(fake_plan, byref(prm), byref(out), None) == 1
    assert b"marker arrays" in lib.efsi_last_error()

    assert lib.efsi_ib_build_boundary_conditions(-1, None, None, None, None, None, None, None, 0, None, None, None,
                                                 None, None, None) == 1
    vd = _native.IbVdParams()
    vd.nx, vd.ny, vd.nz = 1, 4, 4
    fields = _native.IbVdFields()
    assert lib.efsi_ib_velocity_dirichlet_rows(fake_plan, byref(vd), byref(fields), 1, None) == 1
    assert b">= 2" in lib.efsi_last_error()
    assert lib.efsi_ib_reset_anchor_cells(None, 4, None) == 1


def test_header_compiles_as_c99_and_cxx_and_links(tmp_path):
    """include/easyfsi_b200.h is a plain C header: a C99 and a C++17
    translation unit that include it compile warning-free and link against
    the library; the C program runs (no device work)."""
    import shutil
    import subprocess

    build()
    src_c = tmp_path / "use.c"
    src_c.write_text(
        '#include <stdio.h>\n#include <string.h>\n#include "easyfsi_b200.h"\n'
        "int main(void) {\n"
        '  if (strstr(efsi_version(), "sm_100a") == NULL) return 1;\n'
        "  if (efsi_mpm_plan_create(0, 4, 4, 4, NULL) != EFSI_ERR_ARG) return 2;\n"
        '  printf("%s\\n", efsi_last_error());\n'
        "  return 0;\n}\n"
    )
    src_cpp = tmp_path / "use.cpp"
    src_cpp.write_text('#include "easyfsi_b200.h"\nint probe() { return EFSI_OK; }\n')
    gcc, gxx = shutil.which("gcc"), shutil.which("g++")
    if gcc is None or gxx is None:
        pytest.skip("no host C/C++ compiler")
    inc = str(HEADER.parent)
    exe = tmp_path / "use"
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", inc, str(src_c), "-o", str(exe),
                    str(LIB_PATH), f"-Wl,-rpath,{LIB_PATH.parent}"], check=True, capture_output=True)
    subprocess.run([gxx, "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", inc, "-c", str(src_cpp), "-o",
                    str(tmp_path / "use_cpp.o")], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True)
    assert out.stdout.strip()
