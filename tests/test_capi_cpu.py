"""The C-ABI library on a machine without a GPU: it loads, exports exactly the
entry points the public headers declare, and its device-free entry points
behave like the reference's (pyrowave_c.cpp)."""
import ctypes
import os
import re
import subprocess

import pytest

from pyrowave_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("pyrowave.h", "pyrowave_cuda.h")]


def declared_symbols():
    names = set()
    for path in HEADERS:
        text = open(path).read()
        for m in re.finditer(r"PYROWAVE_PUBLIC_API\s+[\w\s\*]+?\b(pyrowave_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def exported_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", capi.library_path()], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_loads():
    assert os.path.exists(capi.library_path())
    capi.lib()


def test_exports_match_headers():
    declared = declared_symbols()
    assert len(declared) >= 40
    exported = exported_symbols()
    assert declared == exported, (declared - exported, exported - declared)
    assert set(capi.API_SYMBOLS) <= declared


def test_api_version():
    assert capi.api_version() == (0, 4, 0)


def test_no_device_without_cuda():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    L = capi.lib()
    h = ctypes.c_void_p()
    assert L.pyrowave_create_default_device(ctypes.byref(h)) == capi.PYROWAVE_ERROR_NO_VULKAN
    assert not h.value


def test_null_arguments_are_rejected():
    L = capi.lib()
    h = ctypes.c_void_p()
    info = capi.EncoderCreateInfo(None, 64, 64, capi.CHROMA_420)
    assert L.pyrowave_encoder_create(ctypes.byref(info), ctypes.byref(h)) == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    dinfo = capi.DecoderCreateInfo(None, 64, 64, capi.CHROMA_420, False)
    assert L.pyrowave_decoder_create(ctypes.byref(dinfo), ctypes.byref(h)) == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    assert L.pyrowave_encoder_create(None, ctypes.byref(h)) == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    n = ctypes.c_size_t()
    assert L.pyrowave_encoder_compute_num_packets(None, 1024, ctypes.byref(n)) == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    assert L.pyrowave_decoder_push_packet(None, None, 0) == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    assert not L.pyrowave_decoder_decode_is_ready(None, True)
    # Destroying NULL handles is a no-op, as in the reference.
    L.pyrowave_encoder_destroy(None)
    L.pyrowave_decoder_destroy(None)
    L.pyrowave_device_destroy(None)


def test_vulkan_only_entry_points_report_not_implemented():
    L = capi.lib()
    L.pyrowave_encoder_encode_gpu_synchronous.argtypes = [ctypes.c_void_p] * 5
    L.pyrowave_decoder_decode_gpu_buffer.argtypes = [ctypes.c_void_p] * 4
    L.pyrowave_sync_object_cpu_signal.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
    L.pyrowave_create_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    ni = capi.PYROWAVE_ERROR_NOT_IMPLEMENTED
    assert L.pyrowave_encoder_encode_gpu_synchronous(None, None, None, None, None) == ni
    assert L.pyrowave_decoder_decode_gpu_buffer(None, None, None, None) == ni
    assert L.pyrowave_sync_object_cpu_signal(None, 0) == ni
    # Importing an application's Vulkan device is impossible without Vulkan.
    h = ctypes.c_void_p()
    assert L.pyrowave_create_device(None, ctypes.byref(h)) == capi.PYROWAVE_ERROR_NO_VULKAN
    assert not L.pyrowave_device_confirm_interop_support(None)
    assert not L.pyrowave_decoder_device_prefers_fragment_path(None)


@pytest.mark.parametrize("lang, std", [("c", "c99"), ("c++", "c++11")])
def test_public_headers_compile_and_link_for_c_and_cpp_callers(tmp_path, lang, std):
    """A caller of the reference's C header keeps its source: both headers build
    as pedantic C99 and C++11 and the program links against the library."""
    src = tmp_path / "caller.c"
    src.write_text('#include "pyrowave.h"\n#include "pyrowave_cuda.h"\n'
                   "int main(void)\n{\n\tpyrowave_device d;\n\tuint32_t a, b, c;\n"
                   "\tpyrowave_get_api_version(&a, &b, &c);\n"
                   "\treturn pyrowave_create_default_device(&d) != PYROWAVE_SUCCESS;\n}\n")
    compiler = "gcc" if lang == "c" else "g++"
    r = subprocess.run([compiler, "-x", lang, f"-std={std}", "-Wall", "-Wextra", "-pedantic", "-Werror",
                        "-I", os.path.join(ROOT, "include"), str(src), "-o", str(tmp_path / "caller"),
                        "-L", os.path.dirname(capi.library_path()), "-l:libpyrowave-shared.so.0"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
