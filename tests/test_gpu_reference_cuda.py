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
    # bindings.rs:268-274, 214, 354-381, 141-158, 426-449, 469-490 (the AIR kernels called directly,
    # without the component dispatcher)
    lib.commit_on_layer_with_previous.argtypes = [C.c_uint32, C.c_uint32, VP, VP, VP]
    lib.accumulate.argtypes = [C.c_int, C.POINTER(VP), C.POINTER(VP)]
    lib.accumulate_numerators_batch.argtypes = [C.c_int, VP, C.POINTER(QM31), C.POINTER(QM31),
                                                C.POINTER(C.c_uint32), C.c_int, VP, VP, VP, VP]
    lib.compute_quotients_and_combine.argtypes = [C.c_int, C.c_int, C.c_uint32, C.c_uint32, C.c_int,
                                                  C.POINTER(VP), C.POINTER(C.c_int), C.POINTER(QM31),
                                                  C.POINTER(QM31), VP, VP, VP, VP]
    lib.barycentric_weights_cuda.argtypes = [C.c_uint32, C.c_uint32, C.c_int, C.c_int, QM31, QM31, QM31,
                                             C.c_uint32, VP]
    lib.barycentric_eval_at_point_cuda.argtypes = [VP, VP, C.c_int, C.POINTER(QM31)]
    lib.generate_wide_fibonacci_trace.argtypes = [VP, VP, C.c_uint32, C.POINTER(VP), C.c_uint32, C.c_uint32]
    lib.generate_poseidon_traces.argtypes = [C.POINTER(VP), C.POINTER(VP), C.POINTER(VP), C.c_uint32]
    lib.generate_poseidon_interaction_traces.argtypes = [VP, C.POINTER(VP), C.POINTER(VP), C.c_uint32,
                                                         C.POINTER(VP), VP]
    lib.evaluate_wide_fibonacci_constraint_quotients_on_domain.argtypes = [
        VP, VP, VP, VP, C.POINTER(VP), C.c_uint32, C.POINTER(VP), C.c_uint32, VP, VP, C.c_uint32, C.c_uint32,
        C.c_uint32, C.c_uint32]
    lib.evaluate_poseidon_constraint_quotients_on_domain.argtypes = [
        VP, VP, VP, VP, C.POINTER(VP), C.c_uint32, C.POINTER(VP), C.c_uint32, C.POINTER(VP), C.c_uint32, VP, VP,
        C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, VP, QM31, C.c_bool, C.c_bool, VP]
    for f in (lib.ntt_n2b_columns, lib.ntt_b2n_column, lib.commit_on_first_layer, lib.fold_line,
              lib.fold_circle_into_line, lib.batch_eval_at_points, lib.poseidon252_commit_on_first_layer,
              lib.poseidon252_commit_on_layer_with_previous, lib.commit_on_layer_with_previous, lib.accumulate,
              lib.accumulate_numerators_batch, lib.compute_quotients_and_combine, lib.barycentric_weights_cuda,
              lib.barycentric_eval_at_point_cuda, lib.generate_wide_fibonacci_trace, lib.generate_poseidon_traces,
              lib.generate_poseidon_interaction_traces, lib.evaluate_wide_fibonacci_constraint_quotients_on_domain,
              lib.evaluate_poseidon_constraint_quotients_on_domain):
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


def dtable(tensors):
    """A device array of column pointers (what the reference's kernels index directly)."""
    return torch.tensor([t.data_ptr() for t in tensors] or [0], dtype=torch.int64, device="cuda")


def rnd(rng, n):
    from gpustark.backend import to_device
    return to_device(rng.integers(0, P, n, dtype=np.int64).astype(np.uint32))


def qm_aos(planes):
    """4 planes -> the reference's array of QM31 structs (n x 4 words) on the device."""
    return torch.stack(planes, dim=1).contiguous()


@pytest.mark.parametrize("log,n_cols", [(10, 0), (12, 4), (16, 1), (20, 0)])
def test_merkle_node_layer_matches_reference_cuda(ref, B, log, n_cols):
    """commit_on_layer_with_previous (blake2s.cu:473-485): node hashes of the
    layer below, with columns of this size injected."""
    rng = np.random.default_rng(700 + log)
    leaves = [rnd(rng, 1 << (log + 1)) for _ in range(2)]
    prev = B.commit_on_layer(log + 1, None, leaves)
    cols = [rnd(rng, 1 << log) for _ in range(n_cols)]
    ours = B.commit_on_layer(log, prev, cols)
    theirs = torch.empty_like(ours)
    table = dtable(cols)
    ref.commit_on_layer_with_previous(1 << log, n_cols, table.data_ptr(), prev.data_ptr(), theirs.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(ours, theirs)


def _line_coeffs(rng, n):
    return [[int(v) for v in rng.integers(0, P, 4)] for _ in range(n)]


@pytest.mark.parametrize("log,n_cols,n_coeffs", [(10, 3, 5), (17, 108, 108), (19, 164, 164)])
def test_accumulate_numerators_matches_reference_cuda(ref, B, log, n_cols, n_coeffs):
    """accumulate_numerators_batch (quotients.cu:206-238)."""
    rng = np.random.default_rng(800 + log)
    cols = [rnd(rng, 1 << log) for _ in range(n_cols)]
    idx = [int(i) for i in rng.integers(0, n_cols, n_coeffs)]
    b, c = _line_coeffs(rng, n_coeffs), _line_coeffs(rng, n_coeffs)
    ours = B.accumulate_numerators(cols, log, idx, b, c)
    theirs = [torch.empty(1 << log, dtype=torch.int32, device="cuda") for _ in range(4)]
    table = dtable(cols)
    ref.accumulate_numerators_batch(1 << log, table.data_ptr(), (QM31 * n_coeffs)(*[QM31(*x) for x in b]),
                                    (QM31 * n_coeffs)(*[QM31(*x) for x in c]), (C.c_uint32 * n_coeffs)(*idx),
                                    n_coeffs, *[t.data_ptr() for t in theirs])
    torch.cuda.synchronize()
    for a, t in zip(ours, theirs):
        assert torch.equal(a, t)


def _ref_quotients(ref, accs, lift, out):
    n = len(accs)
    partial = (C.c_void_p * (4 * n))(*[p.data_ptr() for a in accs for p in a[0]])
    logs = (C.c_int * n)(*[a[1] for a in accs])
    flt = (QM31 * n)(*[QM31(*a[2]) for a in accs])
    pts = (QM31 * (2 * n))(*[QM31(*a[3][k * 4:(k + 1) * 4]) for a in accs for k in range(2)])
    init, step = 1 << (31 - (lift + 1)), 1 << (31 - (lift - 1))  # half coset of CanonicCoset(lift)
    ref.compute_quotients_and_combine(1 << lift, lift, init, step, n, partial, logs, flt, pts,
                                      *[t.data_ptr() for t in out])


@pytest.mark.parametrize("lift,logs", [(8, [8]), (17, [17, 16]), (20, [20, 20, 19])])
def test_compute_quotients_and_combine_matches_reference_cuda(ref, B, lift, logs):
    """compute_quotients_and_combine (quotients.cu:240-326), lifted partial numerators."""
    from test_gpu_trait_ops import secure_point
    rng = np.random.default_rng(900 + lift)
    accs = [([rnd(rng, 1 << l) for _ in range(4)], l, [int(v) for v in rng.integers(0, P, 4)],
             [int(v) for v in secure_point(12345 + 7 * k)]) for k, l in enumerate(logs)]
    ours = B.compute_quotients_and_combine(accs, lift)
    theirs = [torch.empty(1 << lift, dtype=torch.int32, device="cuda") for _ in range(4)]
    _ref_quotients(ref, accs, lift, theirs)
    torch.cuda.synchronize()
    for a, t in zip(ours, theirs):
        assert torch.equal(a, t)


def test_accumulate_matches_reference_cuda(ref, B):
    """accumulate (accumulate.cu:5-27): a += b."""
    rng = np.random.default_rng(950)
    a0 = [rnd(rng, 1 << 18) for _ in range(4)]
    b = [rnd(rng, 1 << 18) for _ in range(4)]
    ours = [t.clone() for t in a0]
    B.accumulate(ours, b)
    theirs = [t.clone() for t in a0]
    ref.accumulate(1 << 18, (C.c_void_p * 4)(*[t.data_ptr() for t in theirs]),
                   (C.c_void_p * 4)(*[t.data_ptr() for t in b]))
    torch.cuda.synchronize()
    for x, y in zip(ours, theirs):
        assert torch.equal(x, y)


@pytest.mark.parametrize("log", [6, 12, 17])
def test_barycentric_matches_reference_cuda(ref, B, log):
    """barycentric_weights_cuda / barycentric_eval_at_point_cuda (barycentric.cu:142-262)."""
    from test_gpu_trait_ops import secure_point
    from gpustark.backend import _qm_mul
    rng = np.random.default_rng(960 + log)
    pt = [int(v) for v in secure_point(424242 + log)]
    ours = B.barycentric_weights(log, pt)
    # the reference's caller computes V(p) and 4^(log-1) on the host (prover/backend/cuda/poly.rs:351-391)
    vn = pt[:4]
    for _ in range(log - 1):
        s = _qm_mul(vn, vn)
        vn = [(2 * s[0] - 1) % P, 2 * s[1] % P, 2 * s[2] % P, 2 * s[3] % P]
    theirs = torch.empty((1 << log) * 4, dtype=torch.int32, device="cuda")
    ref.barycentric_weights_cuda(1 << (31 - (log + 1)), 1 << (31 - (log - 1)), 1 << log, log, QM31(*vn),
                                 QM31(*pt[:4]), QM31(*pt[4:]), pow(4, log - 1, P), theirs.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(qm_aos(ours).reshape(-1), theirs)
    ev = rnd(rng, 1 << log)
    res = QM31()
    ref.barycentric_eval_at_point_cuda(ev.data_ptr(), theirs.data_ptr(), 1 << log, C.byref(res))
    assert [res.a, res.b, res.c, res.d] == list(B.barycentric_eval_at_point(ev, ours))


@pytest.mark.parametrize("log,n_cols", [(8, 8), (16, 100)])
def test_wide_fibonacci_trace_matches_reference_cuda(ref, B, log, n_cols):
    """generate_wide_fibonacci_trace (evaluate_wide_fibonacci.cu:146-179)."""
    rng = np.random.default_rng(970 + log)
    a, b = rnd(rng, 1 << log), rnd(rng, 1 << log)
    ours = B.generate_wide_fibonacci_trace(a, b, n_cols)
    theirs = [torch.empty(1 << log, dtype=torch.int32, device="cuda") for _ in range(n_cols)]
    ref.generate_wide_fibonacci_trace(a.data_ptr(), b.data_ptr(), 1 << log,
                                      (C.c_void_p * n_cols)(*[t.data_ptr() for t in theirs]), n_cols, n_cols)
    torch.cuda.synchronize()
    for x, y in zip(ours, theirs):
        assert torch.equal(x, y)


def _ref_poseidon_traces(ref, log):
    mk = lambda k: [torch.zeros(1 << log, dtype=torch.int32, device="cuda") for _ in range(k)]
    trace, init, fin = mk(158), mk(16), mk(16)
    arr = lambda ts: (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])
    ref.generate_poseidon_traces(arr(trace), arr(init), arr(fin), log)
    return trace, init, fin


@pytest.mark.parametrize("log", [4, 12, 18])
def test_poseidon_traces_match_reference_cuda(ref, B, log):
    """generate_poseidon_traces and generate_poseidon_interaction_traces
    (evaluate_poseidon_constraint.cu:270-640): trace, lookup states, the
    interaction column and the claimed sum."""
    rng = np.random.default_rng(980 + log)
    trace, init, fin = B.generate_poseidon_traces(log)
    rt, ri, rf = _ref_poseidon_traces(ref, log)
    torch.cuda.synchronize()
    for x, y in zip(trace + init + fin, rt + ri + rf):
        assert torch.equal(x, y)
    z, alpha = ([int(v) for v in rng.integers(0, P, 4)] for _ in range(2))
    inter, cs = B.generate_poseidon_interaction_traces(z, alpha, init, fin)
    from gpustark.backend import _qm_mul
    powers, cur = [], [1, 0, 0, 0]
    for _ in range(16):
        powers.append(cur)
        cur = _qm_mul(cur, alpha)
    le = (C.c_uint32 * 72)(*(z + alpha + [w for p in powers for w in p]))
    rinter = [torch.empty(1 << log, dtype=torch.int32, device="cuda") for _ in range(4)]
    rsum = torch.zeros(4, dtype=torch.int32, device="cuda")  # accumulated atomically: must start at zero
    arr = lambda ts: (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])
    ref.generate_poseidon_interaction_traces(C.cast(le, C.c_void_p), arr(ri), arr(rf), log, arr(rinter),
                                             rsum.data_ptr())
    torch.cuda.synchronize()
    assert [int(v) for v in rsum.cpu().numpy().view(np.uint32)] == cs
    for x, y in zip(inter, rinter):
        assert torch.equal(x, y)


def _denoms(trace_log, eval_log):
    from test_gpu_trait_ops import _denoms as d
    return d(trace_log, eval_log)


@pytest.mark.parametrize("trace_log,n_cols", [(6, 10), (16, 100)])
def test_wide_fibonacci_constraints_match_reference_cuda(ref, B, trace_log, n_cols):
    """evaluate_wide_fibonacci_constraint_quotients_on_domain
    (evaluate_wide_fibonacci.cu:64-125), called directly (eval id
    "fibonacci_example")."""
    from gpustark.backend import eval_blob_wide_fibonacci
    rng = np.random.default_rng(990 + trace_log)
    E = trace_log + 1
    trace = [rnd(rng, 1 << E) for _ in range(n_cols)]
    nc = n_cols - 2
    powers = _line_coeffs(rng, nc)
    den = _denoms(trace_log, E)
    ours = [torch.zeros(1 << E, dtype=torch.int32, device="cuda") for _ in range(4)]
    B.evaluate_constraint_quotients_on_domain(ours, [], trace, [], powers, den, trace_log, E, nc,
                                              eval_blob_wide_fibonacci(trace_log), should_accumulate=False)
    theirs = [torch.zeros(1 << E, dtype=torch.int32, device="cuda") for _ in range(4)]
    pw = torch.tensor(np.array(powers, np.uint32).view(np.int32).reshape(-1), device="cuda")
    dn = torch.tensor(np.array(den, np.uint32).view(np.int32), device="cuda")
    none = (C.c_void_p * 1)(0)
    ref.evaluate_wide_fibonacci_constraint_quotients_on_domain(
        *[t.data_ptr() for t in theirs], none, 0, (C.c_void_p * n_cols)(*[t.data_ptr() for t in trace]), n_cols,
        pw.data_ptr(), dn.data_ptr(), trace_log, E, nc, 0)
    torch.cuda.synchronize()
    for a, t in zip(ours, theirs):
        assert torch.equal(a, t)


def _ref_poseidon_eval(log_n, z, alpha, claimed):
    """The PoseidonEval struct as the reference's kernel reads it
    (evaluate_poseidon_constraint.cuh:91-96): eval_id, log_n_rows, z, alpha,
    alpha_powers[16], claimed_sum."""
    from gpustark.backend import _qm_mul, fnv1a_eval_id
    powers, cur = [], [1, 0, 0, 0]
    for _ in range(16):
        powers.append(cur)
        cur = _qm_mul(cur, alpha)
    words = [fnv1a_eval_id("poseidon_example"), log_n] + list(z) + list(alpha) + \
        [w for p in powers for w in p] + list(claimed)
    return (C.c_uint32 * len(words))(*[int(w) for w in words])


@pytest.mark.parametrize("trace_log", [5, 18])
def test_poseidon_constraints_match_reference_cuda(ref, B, trace_log):
    """evaluate_poseidon_constraint_quotients_on_domain
    (evaluate_poseidon_constraint.cu:144-265) with its logup post kernel
    (evaluate_common.cuh:47-120), called directly: two logup fractions per
    row, accumulating into zeroed quotients."""
    from gpustark.backend import eval_blob_poseidon
    rng = np.random.default_rng(1100 + trace_log)
    E = trace_log + 2
    trace = [rnd(rng, 1 << E) for _ in range(158)]
    inter = [rnd(rng, 1 << E) for _ in range(4)]
    z, alpha, cs, shift = ([int(v) for v in rng.integers(0, P, 4)] for _ in range(4))
    powers = _line_coeffs(rng, 143)
    den = _denoms(trace_log, E)
    ours = [torch.zeros(1 << E, dtype=torch.int32, device="cuda") for _ in range(4)]
    B.evaluate_constraint_quotients_on_domain(ours, [], trace, inter, powers, den, trace_log, E, 143,
                                              eval_blob_poseidon(trace_log, z, alpha, cs), cumsum_shift=shift,
                                              should_accumulate=True)
    theirs = [torch.zeros(1 << E, dtype=torch.int32, device="cuda") for _ in range(4)]
    pw = torch.tensor(np.array(powers, np.uint32).view(np.int32).reshape(-1), device="cuda")
    dn = torch.tensor(np.array(den, np.uint32).view(np.int32), device="cuda")
    ev = _ref_poseidon_eval(trace_log, z, alpha, cs)
    none = (C.c_void_p * 1)(0)
    ref.evaluate_poseidon_constraint_quotients_on_domain(
        *[t.data_ptr() for t in theirs], none, 0, (C.c_void_p * 158)(*[t.data_ptr() for t in trace]), 158,
        (C.c_void_p * 4)(*[t.data_ptr() for t in inter]), 4, pw.data_ptr(), dn.data_ptr(), trace_log, E, 143, 2,
        C.cast(ev, C.c_void_p), QM31(*shift), True, False, None)
    torch.cuda.synchronize()
    for a, t in zip(ours, theirs):
        assert torch.equal(a, t)


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


def test_timing_more_against_reference_cuda(ref, B):
    """Device time of the rest of the path through both libraries at the
    benchmark shapes (printed with -s): Merkle node layer, quotient
    numerators and combination, accumulation, barycentric weights, the two
    AIRs' constraint quotients and the Poseidon2 trace / interaction."""
    from gpustark.backend import eval_blob_poseidon, eval_blob_wide_fibonacci
    from test_gpu_trait_ops import secure_point
    rng = np.random.default_rng(2)
    rows = []
    # Merkle node layer 2^20 from 2^21 children
    prev = B.commit_on_layer(21, None, [rnd(rng, 1 << 21)])
    out = torch.empty((1 << 20) * 8, dtype=torch.int32, device="cuda")
    t0 = dtable([])
    rows.append(("merkle node layer 2^20", _time(lambda: B.commit_on_layer(20, prev, [], out=out)),
                 _time(lambda: ref.commit_on_layer_with_previous(1 << 20, 0, t0.data_ptr(), prev.data_ptr(),
                                                                 out.data_ptr()))))
    # numerators: 164 columns x 2^19 (Poseidon2 trace + interaction at the lifting size)
    cols = [rnd(rng, 1 << 19) for _ in range(164)]
    idx = list(range(164))
    b, c = _line_coeffs(rng, 164), _line_coeffs(rng, 164)
    res = [torch.empty(1 << 19, dtype=torch.int32, device="cuda") for _ in range(4)]
    tab = dtable(cols)
    bb, cc, ii = (QM31 * 164)(*[QM31(*x) for x in b]), (QM31 * 164)(*[QM31(*x) for x in c]), (C.c_uint32 * 164)(*idx)
    rows.append(("numerators 164 x 2^19", _time(lambda: B.accumulate_numerators(cols, 19, idx, b, c), reps=3),
                 _time(lambda: ref.accumulate_numerators_batch(1 << 19, tab.data_ptr(), bb, cc, ii, 164,
                                                               *[t.data_ptr() for t in res]), reps=3)))
    # quotient combination on 2^20 with 2 sample points
    accs = [([rnd(rng, 1 << 20) for _ in range(4)], 20, [int(v) for v in rng.integers(0, P, 4)],
             [int(v) for v in secure_point(99 + k)]) for k in range(2)]
    qout = [torch.empty(1 << 20, dtype=torch.int32, device="cuda") for _ in range(4)]
    rows.append(("quotients 2 points x 2^20", _time(lambda: B.compute_quotients_and_combine(accs, 20)),
                 _time(lambda: _ref_quotients(ref, accs, 20, qout))))
    # accumulate 2^20
    a = [rnd(rng, 1 << 20) for _ in range(4)]
    bq = [rnd(rng, 1 << 20) for _ in range(4)]
    ap, bp = (C.c_void_p * 4)(*[t.data_ptr() for t in a]), (C.c_void_p * 4)(*[t.data_ptr() for t in bq])
    rows.append(("accumulate 2^20", _time(lambda: B.accumulate(a, bq)), _time(lambda: ref.accumulate(1 << 20, ap, bp))))
    # barycentric weights 2^17
    pt = [int(v) for v in secure_point(31337)]
    wbuf = torch.empty((1 << 17) * 4, dtype=torch.int32, device="cuda")
    rows.append(("barycentric weights 2^17", _time(lambda: B.barycentric_weights(17, pt)),
                 _time(lambda: ref.barycentric_weights_cuda(1 << 13, 1 << 15, 1 << 17, 17, QM31(1, 2, 3, 4),
                                                            QM31(*pt[:4]), QM31(*pt[4:]), pow(4, 16, P),
                                                            wbuf.data_ptr()))))
    # Wide-Fibonacci constraints 100 columns on 2^17
    E = 17
    trace = [rnd(rng, 1 << E) for _ in range(100)]
    powers, den = _line_coeffs(rng, 98), _denoms(16, E)
    q = [torch.zeros(1 << E, dtype=torch.int32, device="cuda") for _ in range(4)]
    pw = torch.tensor(np.array(powers, np.uint32).view(np.int32).reshape(-1), device="cuda")
    dn = torch.tensor(np.array(den, np.uint32).view(np.int32), device="cuda")
    none = (C.c_void_p * 1)(0)
    tr = (C.c_void_p * 100)(*[t.data_ptr() for t in trace])
    rows.append(("WF constraints 100 x 2^17",
                 _time(lambda: B.evaluate_constraint_quotients_on_domain(q, [], trace, [], powers, den, 16, E, 98,
                                                                         eval_blob_wide_fibonacci(16),
                                                                         should_accumulate=False)),
                 _time(lambda: ref.evaluate_wide_fibonacci_constraint_quotients_on_domain(
                     *[t.data_ptr() for t in q], none, 0, tr, 100, pw.data_ptr(), dn.data_ptr(), 16, E, 98, 0))))
    # Poseidon2 constraints on 2^20 (2^18 rows, LOG_EXPAND 2)
    E = 20
    ptrace = [rnd(rng, 1 << E) for _ in range(158)]
    pinter = [rnd(rng, 1 << E) for _ in range(4)]
    z, alpha, cs, shift = ([int(v) for v in rng.integers(0, P, 4)] for _ in range(4))
    ppow, pden = _line_coeffs(rng, 143), _denoms(18, E)
    pq = [torch.zeros(1 << E, dtype=torch.int32, device="cuda") for _ in range(4)]
    ppw = torch.tensor(np.array(ppow, np.uint32).view(np.int32).reshape(-1), device="cuda")
    pdn = torch.tensor(np.array(pden, np.uint32).view(np.int32), device="cuda")
    ev = _ref_poseidon_eval(18, z, alpha, cs)
    ptr = (C.c_void_p * 158)(*[t.data_ptr() for t in ptrace])
    pin = (C.c_void_p * 4)(*[t.data_ptr() for t in pinter])
    blob = eval_blob_poseidon(18, z, alpha, cs)
    rows.append(("Poseidon2 constraints 2^20",
                 _time(lambda: B.evaluate_constraint_quotients_on_domain(pq, [], ptrace, pinter, ppow, pden, 18, E,
                                                                         143, blob, cumsum_shift=shift), reps=3),
                 _time(lambda: ref.evaluate_poseidon_constraint_quotients_on_domain(
                     *[t.data_ptr() for t in pq], none, 0, ptr, 158, pin, 4, ppw.data_ptr(), pdn.data_ptr(), 18, E,
                     143, 2, C.cast(ev, C.c_void_p), QM31(*shift), True, False, None), reps=3)))
    # Poseidon2 trace and interaction, 2^18 rows
    rows.append(("Poseidon2 trace 2^18", _time(lambda: B.generate_poseidon_traces(18), reps=3),
                 _time(lambda: _ref_poseidon_traces(ref, 18), reps=3)))
    _, init, fin = B.generate_poseidon_traces(18)
    from gpustark.backend import _qm_mul
    le_pw, cur = [], [1, 0, 0, 0]
    for _ in range(16):
        le_pw.append(cur)
        cur = _qm_mul(cur, alpha)
    le = (C.c_uint32 * 72)(*(z + alpha + [w for p in le_pw for w in p]))
    rinter = [torch.empty(1 << 18, dtype=torch.int32, device="cuda") for _ in range(4)]
    rsum = torch.zeros(4, dtype=torch.int32, device="cuda")
    arr = lambda ts: (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])
    ia, fa, ra = arr(init), arr(fin), arr(rinter)
    rows.append(("Poseidon2 interaction 2^18", _time(lambda: B.generate_poseidon_interaction_traces(z, alpha, init, fin),
                                                     reps=3),
                 _time(lambda: ref.generate_poseidon_interaction_traces(C.cast(le, C.c_void_p), ia, fa, 18, ra,
                                                                        rsum.data_ptr()), reps=3)))
    print()
    for name, o, t in rows:
        print("%-28s gpustark %8.3f ms   reference CUDA %8.3f ms   %5.1fx" % (name, o, t, t / o))
    assert all(o > 0 and t > 0 for _, o, t in rows)
