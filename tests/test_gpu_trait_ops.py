"""The per-trait entry points a drop-in backend needs besides the kernels of
test_gpu_kernels.py, through the C ABI, against the oracle:
Column::batch_at_multi / hash gathers (cuda_batch_gather_multi_uint32,
cuda_batch_get_blake_2s_hash), PolyOps::barycentric_weights /
barycentric_eval_at_point, AccumulationOps::generate_secure_powers, and
ComponentProver::evaluate_constraint_quotients_on_domain for the two example
components (eval id + #[repr(C)] Eval bytes)."""
import numpy as np
import pytest

import pyoracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
P = O.P


@pytest.fixture(scope="module")
def B():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpustark.backend import GpuBackend
    return GpuBackend


def dev(a):
    from gpustark.backend import to_device
    return to_device(a)


def host(t):
    from gpustark.backend import to_host
    return to_host(t)


def rand(rng, n):
    return rng.integers(0, P, n, dtype=np.int64).astype(np.uint32)


def secure_point(k):
    """CirclePoint::<SecureField>::get_point(k): the secure-field generator times k."""
    out = np.zeros(8, np.uint32)
    O.lib().oracle_secure_gen_mul(k, 0, out.ctypes.data_as(O.U32P))
    return out


# ----------------------------------------------------------------- gathers
@pytest.mark.parametrize("n_cols,log,n_idx", [(1, 4, 3), (7, 10, 70), (100, 17, 140)])
def test_batch_at_multi(B, n_cols, log, n_idx):
    rng = np.random.default_rng(n_cols)
    cols = [rand(rng, 1 << log) for _ in range(n_cols)]
    idx = rng.integers(0, 1 << log, n_idx)
    got = B.batch_at_multi([dev(c) for c in cols], idx)
    want = np.array([[c[i] for c in cols] for i in idx], np.uint32).reshape(-1)
    assert np.array_equal(got, want)


def test_batch_at_multi_rejects_out_of_range(B):
    from gpustark import GpuStarkError
    c = dev(np.arange(16, dtype=np.uint32))
    with pytest.raises(GpuStarkError, match="out of range"):
        B.batch_at_multi([c], [3, 16])


def test_batch_get_hashes(B):
    rng = np.random.default_rng(5)
    cols = [rand(rng, 1 << 9) for _ in range(3)]
    layer = B.commit_on_layer(9, None, [dev(c) for c in cols])
    idx = [0, 511, 17, 17, 300]
    got = B.batch_get_hashes(layer, idx)
    all_h = host(layer).view(np.uint8).reshape(-1, 32)
    assert np.array_equal(got, all_h[idx])


# ------------------------------------------------------------- barycentric
@pytest.mark.parametrize("log", [2, 5, 10, 16])
def test_barycentric_weights_match_oracle(B, log):
    pt = secure_point(1000003 * log + 7)
    got = [host(t) for t in B.barycentric_weights(log, pt)]
    want = O.barycentric_weights(log, pt)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_barycentric_known_answer(B):
    """The reference's test_cpu_barycentric_evaluation (prover/backend/cpu/
    circle.rs:525-560): an 8-coefficient polynomial on CanonicCoset(10),
    barycentric evaluation at get_point(348), (9736524), (13), (346752) equals
    the direct evaluation."""
    coeffs = np.zeros(1 << 10, np.uint32)
    coeffs[:8] = [691, 805673, 5, 435684, 4832, 23876431, 197, 897346068]
    tw = B.precompute_twiddles(10)
    ev = B.evaluate_polynomials([dev(coeffs)], 10, tw)[0]
    for k in (348, 9736524, 13, 346752):
        pt = secure_point(k)
        w = B.barycentric_weights(10, pt)
        got = B.barycentric_eval_at_point(ev, w)
        assert list(got) == list(O.eval_at_point(coeffs, pt))
        assert list(got) == list(O.barycentric_eval(host(ev), [host(t) for t in w]))


@pytest.mark.parametrize("log", [8, 17, 20])
def test_barycentric_eval_matches_coefficient_eval(B, log):
    rng = np.random.default_rng(log)
    c = rand(rng, 1 << log)
    tw = B.precompute_twiddles(log)
    ev = B.evaluate_polynomials([dev(c)], log, tw)[0]
    pt = secure_point(987654321 + log)
    w = B.barycentric_weights(log, pt)
    assert B.barycentric_eval_at_point(ev, w) == B.batch_eval_at_point([dev(c)], pt)[0]


# ----------------------------------------------------------- secure powers
@pytest.mark.parametrize("n", [1, 2, 143, 10000])
def test_generate_secure_powers(B, n):
    felt = np.array([12345, 678, 91011, 1213], np.uint32)
    got = [host(t) for t in B.generate_secure_powers(felt, n)]
    for g, w in zip(got, O.secure_powers(felt, n)):
        assert np.array_equal(g, w)


# ------------------------------------------------------ constraint quotients
def _powers(rng, n):
    return [[int(x) for x in rng.integers(0, P, 4)] for _ in range(n)]


def _denoms(trace_log, eval_log):
    """1 / coset_vanishing(CanonicCoset(trace_log), eval_domain.at(i)), bit-reversed
    (component_prover.rs:304-310), from the oracle's circle helpers."""
    from test_gpu_kernels import canonic_domain_point, bit_reverse_index
    k = eval_log - trace_log
    vals = []
    for i in range(1 << k):
        x, _ = canonic_domain_point(eval_log, i)
        for _ in range(trace_log - 1):  # vanishing of CanonicCoset(t) at a point = pi^(t-1)(x)
            x = (2 * x * x - 1) % P
        vals.append(O.lib().oracle_m31_inv(x))
    return [vals[bit_reverse_index(i, k)] for i in range(1 << k)]


@pytest.mark.parametrize("trace_log,n_cols", [(4, 3), (6, 10), (10, 100)])
def test_wide_fibonacci_constraint_quotients(B, trace_log, n_cols):
    from gpustark.backend import eval_blob_wide_fibonacci
    rng = np.random.default_rng(trace_log)
    E = trace_log + 1
    trace = [rand(rng, 1 << E) for _ in range(n_cols)]
    nc = n_cols - 2
    powers, den = _powers(rng, nc), _denoms(trace_log, E)
    out = [torch.zeros(1 << E, dtype=torch.int32, device="cuda") for _ in range(4)]
    B.evaluate_constraint_quotients_on_domain(out, [], [dev(c) for c in trace], [], powers, den, trace_log, E, nc,
                                              eval_blob_wide_fibonacci(trace_log))
    want = O.constraint_quotients("wide_fibonacci", trace, [], trace_log, E, powers, den)
    for g, w in zip(out, want):
        assert np.array_equal(host(g), w)
    # should_accumulate: a second call adds the same values
    B.evaluate_constraint_quotients_on_domain(out, [], [dev(c) for c in trace], [], powers, den, trace_log, E, nc,
                                              eval_blob_wide_fibonacci(trace_log), should_accumulate=True)
    for g, w in zip(out, want):
        assert np.array_equal(host(g), (2 * w.astype(np.int64) % P).astype(np.uint32))


@pytest.mark.parametrize("trace_log", [4, 7])
def test_poseidon_constraint_quotients(B, trace_log):
    from gpustark.backend import eval_blob_poseidon
    rng = np.random.default_rng(100 + trace_log)
    E = trace_log + 2
    trace = [rand(rng, 1 << E) for _ in range(158)]
    inter = [rand(rng, 1 << E) for _ in range(4)]
    z, alpha, cs, shift = (rng.integers(0, P, 4).astype(np.uint32) for _ in range(4))
    powers, den = _powers(rng, 143), _denoms(trace_log, E)
    out = [torch.zeros(1 << E, dtype=torch.int32, device="cuda") for _ in range(4)]
    B.evaluate_constraint_quotients_on_domain(out, [], [dev(c) for c in trace], [dev(c) for c in inter], powers, den,
                                              trace_log, E, 143, eval_blob_poseidon(trace_log, z, alpha, cs),
                                              cumsum_shift=shift, should_accumulate=False)
    want = O.constraint_quotients("poseidon", trace, inter, trace_log, E, powers, den, z=z, alpha=alpha, shift=shift)
    for g, w in zip(out, want):
        assert np.array_equal(host(g), w)


def test_unknown_component_is_unsupported(B):
    """No CPU fallback: an eval id without a device kernel is an error."""
    import struct
    from gpustark import GpuStarkError
    out = [torch.zeros(32, dtype=torch.int32, device="cuda") for _ in range(4)]
    cols = [torch.zeros(32, dtype=torch.int32, device="cuda") for _ in range(3)]
    with pytest.raises(GpuStarkError, match="status 4"):
        B.evaluate_constraint_quotients_on_domain(out, [], cols, [], [[1, 0, 0, 0]], [1], 4, 5, 1,
                                                  struct.pack("<3I", 0x12345678, 0, 4))
