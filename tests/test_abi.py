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


def test_poseidon252_host_channel_matches_oracle():
    """gs_poseidon252_channel_op (the library's host Poseidon252Channel, used
    by the Poseidon252 proofs) against the oracle's restatement: the
    reference's mix_u64 known answer, then a script of every operation."""
    import json
    import numpy as np
    import poseidon252 as PS
    lib = ctypes.CDLL(LIB)
    golden = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_vectors.json")))

    def op(digest, nd, code, data=b"", value=0, words=(), n=0):
        d = (ctypes.c_uint8 * 32).from_buffer_copy(digest)
        b = (ctypes.c_uint8 * 32).from_buffer_copy(data.ljust(32, b"\0")[:32])
        w = (ctypes.c_uint32 * max(1, len(words)))(*words)
        out = (ctypes.c_uint32 * max(1, 7 * n))()
        dout = (ctypes.c_uint8 * 32)()
        nd_out = ctypes.c_uint32()
        count = len(words) // 4 if code == 3 else n
        assert lib.gs_poseidon252_channel_op(d, nd, code, b, ctypes.c_uint64(value), w, ctypes.c_size_t(count), out,
                                             dout, ctypes.byref(nd_out)) == 0
        return bytes(dout), nd_out.value, list(out)

    zero = bytes(32)
    d, nd, _ = op(zero, 0, 1, value=golden["poseidon252_channel_mix_u64"]["value"])
    assert int.from_bytes(d, "big") == int(golden["poseidon252_channel_mix_u64"]["digest"], 16)
    rng = np.random.default_rng(5)
    ch, d, nd = PS.Channel(), zero, 0
    for step in ["mix_root", "draw_secure_felts", "mix_felts", "draw_u32s", "mix_u64", "draw_secure_felts",
                 "mix_felts", "draw_u32s", "draw_secure_felts", "mix_root"]:
        if step == "mix_root":
            r = int.from_bytes(rng.bytes(32), "big") % PS.P
            d, nd, _ = op(d, nd, 0, data=r.to_bytes(32, "big"))
            ch.mix_root(r)
        elif step == "mix_u64":
            v = int(rng.integers(0, 2 ** 63))
            d, nd, _ = op(d, nd, 1, value=v)
            ch.mix_u64(v)
        elif step == "mix_felts":
            f = [tuple(int(x) for x in rng.integers(0, PS.M31, 4)) for _ in range(int(rng.integers(1, 6)))]
            d, nd, _ = op(d, nd, 3, words=[x for q in f for x in q])
            ch.mix_felts(f)
        elif step == "draw_secure_felts":
            d, nd, out = op(d, nd, 4, n=3)
            assert out[:12] == [x for q in ch.draw_secure_felts(3) for x in q]
        else:
            d, nd, out = op(d, nd, 5, n=2)
            assert out[:14] == ch.draw_u32s() + ch.draw_u32s()
        assert int.from_bytes(d, "big") == ch.digest and nd == ch.n_draws, step
    # operation 2 (mix_u32s) is not part of the prover's path and is refused
    assert lib.gs_poseidon252_channel_op((ctypes.c_uint8 * 32)(), 0, 2, None, ctypes.c_uint64(0), None,
                                         ctypes.c_size_t(0), None, (ctypes.c_uint8 * 32)(),
                                         ctypes.byref(ctypes.c_uint32())) != 0
