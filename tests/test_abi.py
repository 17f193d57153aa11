"""CPU checks of the C-ABI boundary: the library loads without a GPU and
exports every function include/dcm.h declares (no compute calls here)."""
import ctypes
import os
import re

from conftest import ROOT, load_dcm

HEADER = os.path.join(ROOT, "include", "dcm.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dcm_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared()
    for n in ("dcm_create", "dcm_bicgstab", "dcm_mpdata_3d", "dcm_sources",
              "dcm_advance_momentum", "dcm_step"):
        assert n in names


def test_library_exports_every_declared_symbol():
    dcm = load_dcm()
    lib = ctypes.CDLL(dcm.LIBPATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_exports():
    dcm = load_dcm()
    assert set(declared()) == set(dcm.EXPORTS)


def test_status_strings_and_decomposition_without_gpu():
    dcm = load_dcm()
    lib = dcm.library()
    assert lib.dcm_status_string(0) == b"ok"
    assert lib.dcm_status_string(1) == b"convergence failure"
    dcm.check_decomposition((1, 1, 1))
    try:
        dcm.check_decomposition((2, 1, 1))
    except dcm.DCMError as e:
        assert e.status == dcm.DCM_E_DECOMP
    else:
        raise AssertionError("a 2x1x1 process grid must be rejected")


def test_create_rejects_bad_grid_before_touching_the_device():
    dcm = load_dcm()
    lib = dcm.library()
    g = dcm._Grid()
    g.ip, g.jp, g.kp = 8, 8, 1  # kp < 3
    h = ctypes.c_void_p()
    assert lib.dcm_create(ctypes.byref(g), 0, ctypes.byref(h)) == dcm.DCM_E_ARG


def declared_arity():
    """Number of parameters of every function include/dcm.h declares."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(dcm_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", text):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_binding_signatures_match_the_header():
    dcm = load_dcm()
    lib = dcm.library()
    arity = declared_arity()
    bad = {n: (len(getattr(lib, n).argtypes), k) for n, k in arity.items()
           if len(getattr(lib, n).argtypes or ()) != k}
    assert not bad, bad


def test_header_compiles_as_c_and_links(tmp_path):
    """A C99 translation unit includes include/dcm.h, takes the address of
    every declared function and links against the library as a C host (the
    layer under the Fortran ISO_C_BINDING interface) would; the program runs
    without a GPU."""
    import shutil
    import subprocess

    import pytest

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    dcm = load_dcm()
    names = declared()
    src = tmp_path / "abi.c"
    src.write_text(
        "#include <stdio.h>\n#include <string.h>\n#include \"dcm.h\"\n"
        "int main(void) {\n"
        "    void (*fns[])(void) = {\n" +
        "".join("        (void (*)(void))%s,\n" % n for n in names) +
        "    };\n"
        "    if (strcmp(dcm_status_string(0), \"ok\") != 0) return 1;\n"
        "    printf(\"%d\\n\", (int)(sizeof fns / sizeof fns[0]));\n"
        "    return 0;\n}\n")
    exe = tmp_path / "abi"
    libdir = os.path.dirname(dcm.LIBPATH)
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
                    "-I" + os.path.join(ROOT, "include"), str(src), dcm.LIBPATH,
                    "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    assert int(out) == len(names)


def test_column_transport_checks_arguments_before_the_device():
    """dcm_mpdata_vec_1d validates its arguments on the host: bad halo
    widths or options return DCM_E_ARG and zero columns return DCM_OK,
    without touching a device."""
    dcm = load_dcm()
    lib = dcm.library()
    call = lambda *a: lib.dcm_mpdata_vec_1d(*a)  # noqa: E731
    none = [None] * 4
    assert call(3, 10, 1, 0, 1, None, None, *none, 0, None, None, 1, 0, 0) == dcm.DCM_E_ARG
    assert call(3, 10, 1, 1, 0, None, None, *none, 0, None, None, 1, 0, 0) == dcm.DCM_E_ARG
    assert call(3, 10, 1, 1, 1, None, None, *none, 0, None, None, 1, 0, 3) == dcm.DCM_E_ARG
    assert call(3, 10, 1, 1, 1, None, None, *none, 7, None, None, 1, 0, 0) == dcm.DCM_E_ARG
    assert call(3, 10, 1, 1, 1, None, None, *none, 0, None, None, 1, 0, 0) == dcm.DCM_E_ARG
    assert call(0, 10, 1, 1, 1, None, None, *none, 0, None, None, 1, 0, 0) == dcm.DCM_OK
