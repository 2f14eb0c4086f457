"""The library's kernels against the reference's own CUDA kernels, built for
sm_100a from the reference sources by oracle/Makefile.refcuda into
oracle/_ref/libstwo_cuda_ref.so (skipped when that library is absent): the
circle FFT (ntt_n2b_columns / ntt_b2n_column), the Blake2s leaf layer
(commit_on_first_layer), the FRI folds (fold_line, fold_circle_into_line),
the OODS evaluation (batch_eval_at_points) and the proof of work
(grind_blake2s) and the Poseidon252 Merkle layers (poseidon252_commit_on_
first_layer / _with_previous) must give identical outputs on the same inputs.
With -s, the timing test prints both implementations' device times."""
import ctypes as C
import os

import numpy as np
import pytest

import pyoracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
P = O.P
REF_LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "libstwo_cuda_ref.so")


class QM31(C.Structure):
    """CudaSecureField (bindings.rs:9-15), passed by value."""
    _fields_ = [("a", C.c_uint32), ("b", C.c_uint32), ("c", C.c_uint32), ("d", C.c_uint32)]


@pytest.fixture(scope="module")
def ref():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(REF_LIB):
        pytest.skip("reference CUDA library not built (oracle/Makefile.refcuda)")
    lib = C.CDLL(REF_LIB)
    VP = C.c_void_p
    # bindings.rs:503-519, 262-275
    lib.ntt_n2b_columns.argtypes = [C.POINTER(VP), C.c_uint, C.c_uint, VP, C.c_uint, C.c_uint]
    lib.ntt_b2n_column.argtypes = [C.POINTER(VP), C.c_uint32, C.c_uint32, VP, C.c_uint32, C.c_uint32]
    lib.commit_on_first_layer.argtypes = [C.c_uint32, C.c_uint32, VP, VP]
    # fold_line.cu: void fold_line(m31*, uint32_t offset, uint32_t n, m31** eval, qm31 alpha, m31** folded)
    lib.fold_line.argtypes = [VP, C.c_uint32, C.c_uint32, C.POINTER(VP), QM31, C.POINTER(VP)]
    lib.fold_circle_into_line.argtypes = [VP, C.c_uint32, C.c_uint32, C.POINTER(VP), QM31, C.POINTER(VP)]
    lib.batch_eval_at_points.argtypes = [VP, C.c_int, C.c_int, QM31, QM31, C.POINTER(QM31)]
    lib.grind_blake2s.argtypes = [C.POINTER(C.c_uint32), C.c_uint32]
    lib.grind_blake2s.restype = C.c_uint64
    lib.poseidon252_commit_on_first_layer.argtypes = [C.c_size_t, C.c_size_t, VP, VP]
    lib.poseidon252_commit_on_layer_with_previous.argtypes = [C.c_size_t, C.c_size_t, VP, VP, VP]
    for f in (lib.ntt_n2b_columns, lib.ntt_b2n_column, lib.commit_on_first_layer, lib.fold_line,
              lib.fold_circle_into_line, lib.batch_eval_at_points, lib.poseidon252_commit_on_first_layer,
              lib.poseidon252_commit_on_layer_with_previous):
        f.restype = None
    return lib


@pytest.fixture(scope="module")
def B():
    from gpustark.backend import GpuBackend
    return GpuBackend


def ref_fold_line(ref, planes, log, alpha, tw, out):
    tw_len = 1 << tw.root_log
    ref.fold_line(tw.itwiddles.data_ptr(), tw_len - (1 << log), 1 << log, ptrs(planes), QM31(*alpha), ptrs(out))


def ptrs(tensors):
    return (C.c_void_p * len(tensors))(*[t.data_ptr() for t in tensors])


def ref_evaluate(ref, cols, log, tw):
    arr = ptrs(cols)
    ref.ntt_n2b_columns(arr, log, len(cols), tw.twiddles.data_ptr(), 1 << (log - 1), 1 << (log - 1))


def ref_interpolate(ref, cols, log, tw):
    arr = ptrs(cols)
    ref.ntt_b2n_column(arr, log, len(cols), tw.itwiddles.data_ptr(), 1 << (log - 1), 1 << (log - 1))


@pytest.mark.parametrize("log,n_cols", [(13, 3), (16, 2), (19, 1), (20, 4), (24, 1), (25, 1), (26, 1)])
def test_fft_matches_reference_cuda(ref, B, log, n_cols):
    from gpustark.backend import to_device
    rng = np.random.default_rng(log)
    tw = B.precompute_twiddles(log - 1)
    coeffs = [to_device(rng.integers(0, P, 1 << log, dtype=np.int64).astype(np.uint32)) for _ in range(n_cols)]
    ours = B.evaluate_polynomials(coeffs, log, tw)
    theirs = [c.clone() for c in coeffs]
    ref_evaluate(ref, theirs, log, tw)
    torch.cuda.synchronize()
    for a, b in zip(ours, theirs):
        assert torch.equal(a, b)
    back = [t.clone() for t in theirs]
    ref_interpolate(ref, back, log, tw)
    B.interpolate_columns(theirs, log, tw)
    torch.cuda.synchronize()
    for a, b, c in zip(back, theirs, coeffs):
        assert torch.equal(a, b) and torch.equal(b, c)


@pytest.mark.parametrize("log,n_cols", [(10, 1), (14, 7), (16, 64)])
def test_merkle_leaves_match_reference_cuda(ref, B, log, n_cols):
    from gpustark.backend import to_device
    rng = np.random.default_rng(100 + n_cols)
    cols = [to_device(rng.integers(0, P, 1 << log, dtype=np.int64).astype(np.uint32)) for _ in range(n_cols)]
    ours = B.commit_on_layer(log, None, cols)
    table = torch.tensor([c.data_ptr() for c in cols], dtype=torch.int64, device="cuda")
    theirs = torch.empty_like(ours)
    ref.commit_on_first_layer(1 << log, n_cols, table.data_ptr(), theirs.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(ours, theirs)


@pytest.mark.parametrize("log", [3, 12, 22])
def test_fold_line_matches_reference_cuda(ref, B, log):
    from gpustark.backend import to_device
    rng = np.random.default_rng(200 + log)
    tw = B.precompute_twiddles(log + 1)
    planes = [to_device(rng.integers(0, P, 1 << log, dtype=np.int64).astype(np.uint32)) for _ in range(4)]
    alpha = [int(v) for v in rng.integers(0, P, 4)]
    ours = B.fold_line(planes, log, alpha, tw)
    theirs = [torch.empty_like(o) for o in ours]
    ref_fold_line(ref, planes, log, alpha, tw, theirs)
    torch.cuda.synchronize()
    for a, b in zip(ours, theirs):
        assert torch.equal(a, b)


@pytest.mark.parametrize("log", [4, 13, 21, 23])
def test_fold_circle_into_line_matches_reference_cuda(ref, B, log):
    from gpustark.backend import to_device
    rng = np.random.default_rng(300 + log)
    tw = B.precompute_twiddles(log - 1)
    src = [to_device(rng.integers(0, P, 1 << log, dtype=np.int64).astype(np.uint32)) for _ in range(4)]
    dst0 = [rng.integers(0, P, 1 << (log - 1), dtype=np.int64).astype(np.uint32) for _ in range(4)]
    alpha = [int(v) for v in rng.integers(0, P, 4)]
    ours = [to_device(d) for d in dst0]
    B.fold_circle_into_line(ours, src, log, alpha, tw)
    theirs = [to_device(d) for d in dst0]
    ref.fold_circle_into_line(tw.itwiddles.data_ptr(), (1 << tw.root_log) - (1 << (log - 1)), 1 << log, ptrs(src),
                              QM31(*alpha), ptrs(theirs))
    torch.cuda.synchronize()
    for a, b in zip(ours, theirs):
        assert torch.equal(a, b)


@pytest.mark.parametrize("log,n_polys", [(8, 3), (16, 20), (18, 5)])
def test_batch_eval_at_point_matches_reference_cuda(ref, B, log, n_polys):
    from gpustark.backend import to_device
    rng = np.random.default_rng(400 + log)
    polys = [to_device(rng.integers(0, P, 1 << log, dtype=np.int64).astype(np.uint32)) for _ in range(n_polys)]
    point = [int(v) for v in rng.integers(0, P, 8)]
    ours = B.batch_eval_at_point(polys, point)
    table = torch.tensor([p.data_ptr() for p in polys], dtype=torch.int64, device="cuda")
    res = (QM31 * n_polys)()
    ref.batch_eval_at_points(table.data_ptr(), 1 << log, n_polys, QM31(*point[:4]), QM31(*point[4:]), res)
    assert [[r.a, r.b, r.c, r.d] for r in res] == [[int(v) for v in o] for o in ours]


@pytest.mark.parametrize("pow_bits", [1, 10, 18])
def test_grind_matches_reference_cuda(ref, B, pow_bits):
    import hashlib
    import struct
    from gpustark import _lib as L
    from gpustark.backend import default_context
    digest = hashlib.blake2s(b"grind %d" % pow_bits).digest()
    pre = hashlib.blake2s(struct.pack("<I", 0x12345678) + bytes(12) + digest + struct.pack("<I", pow_bits)).digest()
    words = (C.c_uint32 * 8)(*struct.unpack("<8I", pre))
    nonce = C.c_uint64()
    L.check(L.lib().gs_grind_blake2s(default_context().handle, words, pow_bits, C.byref(nonce)), "grind")
    assert ref.grind_blake2s(words, pow_bits) == nonce.value


def _ref_poseidon252(ref, log, cols, prev, out):
    table = torch.tensor([c.data_ptr() for c in cols] or [0], dtype=torch.int64, device="cuda")
    if prev is None:
        ref.poseidon252_commit_on_first_layer(1 << log, len(cols), table.data_ptr(), out.data_ptr())
    else:
        ref.poseidon252_commit_on_layer_with_previous(1 << log, len(cols), table.data_ptr(), prev.data_ptr(),
                                                      out.data_ptr())
    return table


@pytest.mark.parametrize("log,n_cols,with_prev", [(10, 1, False), (12, 8, False), (12, 9, True), (13, 0, True),
                                                  (14, 20, False), (15, 3, True)])
def test_poseidon252_layer_matches_reference_cuda(ref, B, log, n_cols, with_prev):
    from gpustark.backend import to_device
    rng = np.random.default_rng(500 + log + n_cols)
    cols = [to_device(rng.integers(0, P, 1 << log, dtype=np.int64).astype(np.uint32)) for _ in range(n_cols)]
    prev = None
    if with_prev:  # a valid previous layer: hashes of random leaves
        leaf_cols = [to_device(rng.integers(0, P, 1 << (log + 1), dtype=np.int64).astype(np.uint32)) for _ in range(2)]
        prev = B.poseidon252_commit_on_layer(log + 1, None, leaf_cols)
    ours = B.poseidon252_commit_on_layer(log, prev, cols)
    theirs = torch.empty_like(ours)
    _ref_poseidon252(ref, log, cols, prev, theirs)
    torch.cuda.synchronize()
    assert torch.equal(ours, theirs)


def _time(fn, reps=5):
    fn()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    b.synchronize()
    return a.elapsed_time(b) / reps


def test_timing_against_reference_cuda(ref, B):
    """Device time of the same work through both libraries (printed with -s);
    asserts only that both ran."""
    from gpustark.backend import to_device
    rng = np.random.default_rng(1)
    rows = []
    for log in (20, 24, 26):
        tw = B.precompute_twiddles(log - 1)
        x = to_device(rng.integers(0, P, 1 << log, dtype=np.int64).astype(np.uint32))
        y = torch.empty_like(x)
        ours = _time(lambda: (B.evaluate_polynomials([x], log, tw, out=[y]), B.interpolate_columns([y], log, tw)))
        z = x.clone()
        theirs = _time(lambda: (ref_evaluate(ref, [z], log, tw), ref_interpolate(ref, [z], log, tw)))
        rows.append(("fft%d eval+interp" % log, ours, theirs))
    cols = [to_device(rng.integers(0, P, 1 << 20, dtype=np.int64).astype(np.uint32)) for _ in range(64)]
    out = torch.empty((1 << 20) * 8, dtype=torch.int32, device="cuda")
    table = torch.tensor([c.data_ptr() for c in cols], dtype=torch.int64, device="cuda")
    ours = _time(lambda: B.commit_on_layer(20, None, cols, out=out))
    theirs = _time(lambda: ref.commit_on_first_layer(1 << 20, 64, table.data_ptr(), out.data_ptr()))
    rows.append(("merkle leaves 64x2^20", ours, theirs))
    tw = B.precompute_twiddles(23)
    planes = [to_device(rng.integers(0, P, 1 << 22, dtype=np.int64).astype(np.uint32)) for _ in range(4)]
    folded = [torch.empty(1 << 21, dtype=torch.int32, device="cuda") for _ in range(4)]
    ours = _time(lambda: B.fold_line(planes, 22, [1, 2, 3, 4], tw))
    theirs = _time(lambda: ref_fold_line(ref, planes, 22, [1, 2, 3, 4], tw, folded))
    rows.append(("fold_line 2^22", ours, theirs))
    epolys = [to_device(rng.integers(0, P, 1 << 18, dtype=np.int64).astype(np.uint32)) for _ in range(160)]
    epoint = [int(v) for v in rng.integers(0, P, 8)]
    etable = torch.tensor([p.data_ptr() for p in epolys], dtype=torch.int64, device="cuda")
    eres = (QM31 * 160)()
    ours = _time(lambda: B.batch_eval_at_point(epolys, epoint), reps=3)
    theirs = _time(lambda: ref.batch_eval_at_points(etable.data_ptr(), 1 << 18, 160, QM31(*epoint[:4]),
                                                   QM31(*epoint[4:]), eres), reps=3)
    rows.append(("OODS 160 polys x 2^18", ours, theirs))
    pcols = [to_device(rng.integers(0, P, 1 << 18, dtype=np.int64).astype(np.uint32)) for _ in range(8)]
    pout = torch.empty((1 << 18) * 32, dtype=torch.uint8, device="cuda")
    ours = _time(lambda: B.poseidon252_commit_on_layer(18, None, pcols, out=pout), reps=3)
    theirs = _time(lambda: _ref_poseidon252(ref, 18, pcols, None, pout), reps=3)
    rows.append(("poseidon252 leaves 8x2^18", ours, theirs))
    pnode = torch.empty((1 << 17) * 32, dtype=torch.uint8, device="cuda")
    ours = _time(lambda: B.poseidon252_commit_on_layer(17, pout, [], out=pnode), reps=3)
    theirs = _time(lambda: _ref_poseidon252(ref, 17, [], pout, pnode), reps=3)
    rows.append(("poseidon252 nodes 2^17", ours, theirs))
    print()
    for name, o, t in rows:
        print("%-24s gpustark %8.3f ms   reference CUDA %8.3f ms   %5.1fx" % (name, o, t, t / o))
    assert all(o > 0 and t > 0 for _, o, t in rows)
