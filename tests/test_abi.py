"""The C ABI without a GPU: the header compiles as C, the in-tree library loads and exports
every function include/gear_b200.h declares, and calls that need no device (sizes, error
reporting) behave; gear_dag_create without a device fails with a status, not a crash."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gear_b200.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w]+\s*\**\s*(gear_\w+)\s*\(", src, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    from gear_b200 import build
    if not os.path.exists(build.LIB):
        build.build()
    return ctypes.CDLL(build.LIB)


def test_header_compiles_as_c(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    f = tmp_path / "use.c"
    f.write_text('#include "gear_b200.h"\nint main(void) { return gear_last_launch_count(); }\n')
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.dirname(HEADER), str(f)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_every_declared_function_is_exported(lib):
    names = _declared()
    assert "gear_crown_lower" in names and "gear_bab_split" in names and len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    from gear_b200 import _lib
    assert sorted(_lib.EXPORTED) == names     # the Python binding covers the same set


def test_calls_that_need_no_device(lib):
    lib.gear_bab_workspace_bytes.restype = ctypes.c_int64
    lib.gear_bab_workspace_bytes.argtypes = [ctypes.c_int64]
    assert lib.gear_bab_workspace_bytes(100000) > 0
    lib.gear_crown_static_scratch_bytes.restype = ctypes.c_int64
    assert lib.gear_crown_static_scratch_bytes() == 64 << 20
    lib.gear_crown_workspace_bytes.restype = ctypes.c_int64
    lib.gear_crown_workspace_bytes.argtypes = [ctypes.c_void_p, ctypes.c_int64]
    assert lib.gear_crown_workspace_bytes(None, 10) == -1       # no handle: -1, no crash


def test_dag_create_rejects_bad_arguments(lib):
    lib.gear_last_error.restype = ctypes.c_char_p
    h = ctypes.c_void_p()
    hdr = (ctypes.c_int32 * 3)(0, 0, 0)
    st = lib.gear_dag_create(hdr, ctypes.c_int64(3), None, ctypes.c_int64(0), None, ctypes.c_int64(0), None,
                             ctypes.c_int64(0), None, ctypes.c_int64(0), None, ctypes.c_int64(0), None,
                             ctypes.c_int64(0), ctypes.byref(h))
    assert st == -1 and not h.value
    assert b"bad arguments" in lib.gear_last_error()


def test_multi_and_plain_sizes_reject_bad_arguments(lib):
    lib.gear_crown_multi_workspace_bytes.restype = ctypes.c_int64
    lib.gear_crown_multi_workspace_bytes.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    assert lib.gear_crown_multi_workspace_bytes(None, -1) == -1
    assert lib.gear_crown_multi_workspace_bytes(None, 0) == 0        # nothing to launch
    lib.gear_crown_plain_workspace_bytes.restype = ctypes.c_int64
    lib.gear_crown_plain_workspace_bytes.argtypes = [ctypes.c_void_p, ctypes.c_int64]
    assert lib.gear_crown_plain_workspace_bytes(None, 1) == -1
    lib.gear_crown_cuts_workspace_bytes.restype = ctypes.c_int64
    lib.gear_crown_cuts_workspace_bytes.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32]
    assert lib.gear_crown_cuts_workspace_bytes(None, 1, 4) == -1
