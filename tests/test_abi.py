"""The C-ABI library loads without a GPU and exports every symbol that
include/gpustark.h declares (no compute calls here)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gpustark.h")
LIB = os.path.join(ROOT, "nitroozk-stwo_b200", "gpustark", "libgpustark.so")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gs_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    assert "gs_ctx_create" in names and "gs_commit_on_layer" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        import subprocess
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "nitroozk-stwo_b200"), "-j8"])
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_declares_only_exported_symbols():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "nitroozk-stwo_b200"))
    import gpustark
    lib = ctypes.CDLL(LIB)
    for n in gpustark.declared_symbols():
        assert hasattr(lib, n), n
    assert set(gpustark.declared_symbols()) <= set(declared())


def test_fft_tuning_setter_validates_without_gpu():
    """gs_fft_set_tuning / gs_fft_get_tuning are host-only: bad splits are
    refused with ERR_INVALID, good ones read back per (log size, extension),
    and the default 13 / 4 is put back."""
    lib = ctypes.CDLL(LIB)
    ALL = 0xFFFFFFFF
    t, c = ctypes.c_uint32(), ctypes.c_uint32()

    def get(log, ext):
        assert lib.gs_fft_get_tuning(log, ext, ctypes.byref(t), ctypes.byref(c)) == 0
        return t.value, c.value

    assert get(20, 0) == (13, 4) and get(20, 2) == (13, 4)
    for bad in [(20, ALL, 14, 4), (20, ALL, 5, 0), (20, 0, 13, 6), (20, 1, 9, 5), (32, ALL, 13, 4)]:
        assert lib.gs_fft_set_tuning(*bad) == 1, bad
    try:
        assert lib.gs_fft_set_tuning(20, ALL, 11, 3) == 0
        assert get(20, 0) == (11, 3) and get(20, 3) == (11, 3) and get(20, 7) == (11, 3)
        assert lib.gs_fft_set_tuning(20, 2, 12, 5) == 0
        assert get(20, 2) == (12, 5) and get(20, 1) == (11, 3)
        assert get(21, 0) == (13, 4)
    finally:
        assert lib.gs_fft_set_tuning(0, ALL, 13, 4) == 0
