"""The C-ABI library loads and exports every entry point include/autorift_gpu.h declares.

No compute call is made here; on a machine without a GPU, context creation must fail with a
status code rather than crash.
"""

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "autorift_gpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\s*\*)\s+(ar_\w+)\s*\(", text, re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for n in ("ar_ctx_create", "ar_ctx_destroy", "ar_pair_upload", "ar_track",
              "ar_track_device", "ar_correlate", "ar_refine_patches", "ar_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(ar):
    import __graft_entry__ as ge

    ge._load_build_ext().build()
    lib = ctypes.CDLL(str(ar._lib.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # Every declared function has a ctypes signature in the binding.
    assert set(declared_functions()) <= set(ar._lib.SIGNATURES)


def test_no_gpu_fails_cleanly(ar):
    lib = ar._lib.load()
    count = ctypes.c_int(0)
    try:
        cudart = ctypes.CDLL("libcudart.so.12")
        has_gpu = cudart.cudaGetDeviceCount(ctypes.byref(count)) == 0 and count.value > 0
    except OSError:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present; covered by the gpu tests")
    h = ctypes.c_void_p()
    assert lib.ar_ctx_create(0, ctypes.byref(h)) != 0
    assert lib.ar_version() >= 100
    # Null-argument handling never touches the device.
    assert lib.ar_ctx_destroy(None) == ar._lib.AR_ERR_ARG
    assert lib.ar_pair_destroy(None) == ar._lib.AR_ERR_ARG


def test_struct_layouts_match_the_header(ar, tmp_path):
    """ctypes mirrors of the header's structs have the C sizes and field offsets."""
    import ctypes
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    from pathlib import Path
    inc = Path(__file__).resolve().parents[1] / "include"
    src = tmp_path / "sz.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "autorift_gpu.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu\\n\", sizeof(ar_points),"
        " sizeof(ar_prepare_opts), sizeof(ar_multichip_params), sizeof(ar_request),"
        " offsetof(ar_request, prepare), offsetof(ar_request, params), offsetof(ar_request, grid));"
        "return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run([cc, f"-I{inc}", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    L = ar._lib
    want = [ctypes.sizeof(L.ArPoints), ctypes.sizeof(L.ArPrepareOpts),
            ctypes.sizeof(L.ArMultichipParams), ctypes.sizeof(L.ArRequest),
            L.ArRequest.prepare.offset, L.ArRequest.params.offset, L.ArRequest.grid.offset]
    assert got == want
