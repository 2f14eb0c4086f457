"""DEEP-quotient, lifted-accumulation and out-of-domain-evaluation kernels vs
the CPU oracle (bit-exact) on seeded inputs."""
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


def rand(rng, *shape):
    return rng.integers(0, P, shape, dtype=np.int64).astype(np.uint32)


def qmul(a, b):
    out = np.zeros(4, np.uint32)
    O.lib().oracle_qm31_mul(O.u32(a)[1], O.u32(b)[1], out.ctypes.data_as(O.U32P))
    return out


def conj(q):
    return np.array([q[0], q[1], (P - q[2]) % P, (P - q[3]) % P], np.uint32)


def qsub(a, b):
    return np.array([(int(x) - int(y)) % P for x, y in zip(a, b)], np.uint32)


def line_coeffs(point8, value4, alpha4):
    """complex_conjugate_line_coeffs (core/constraints.rs:119-134), restated
    here to feed the GPU entry point; the oracle computes its own."""
    py = point8[4:]
    a = qsub(conj(value4), value4)
    c = qsub(conj(py), py)
    b = qsub(qmul(value4, c), qmul(a, py))
    return qmul(alpha4, a), qmul(alpha4, b), qmul(alpha4, c)


@pytest.mark.parametrize("log_size,n_cols,n_entries", [(3, 2, 2), (8, 5, 7), (10, 3, 4), (10, 6, 6), (11, 7, 7),
                                                       (12, 17, 17), (16, 100, 108)])
def test_accumulate_numerators(B, log_size, n_cols, n_entries):
    rng = np.random.default_rng(log_size * 1000 + n_cols)
    cols = [rand(rng, 1 << log_size) for _ in range(n_cols)]
    point = rand(rng, 8)
    idx = rng.integers(0, n_cols, n_entries).astype(np.uint32)
    vals = rand(rng, n_entries, 4)
    rnd = rand(rng, n_entries, 4)
    exp_partial, exp_flt = O.accumulate_numerators(cols, log_size, point, idx, vals, rnd)
    coeffs = [line_coeffs(point, vals[k], rnd[k]) for k in range(n_entries)]
    got = B.accumulate_numerators([dev(c) for c in cols], log_size, idx, [c[1] for c in coeffs],
                                  [c[2] for c in coeffs])
    assert np.array_equal(np.stack([host(t) for t in got], 1), exp_partial)
    flt = np.zeros(4, np.uint32)
    for c in coeffs:
        flt = np.array([(int(x) + int(y)) % P for x, y in zip(flt, c[0])], np.uint32)
    assert np.array_equal(flt, exp_flt)


@pytest.mark.parametrize("lift,sizes", [(4, [4]), (8, [8, 6]), (12, [12, 12, 9]), (17, [17, 16, 17, 12, 17])])
def test_compute_quotients_and_combine(B, lift, sizes):
    rng = np.random.default_rng(lift)
    partials = [rand(rng, 1 << s, 4) for s in sizes]
    flts = rand(rng, len(sizes), 4)
    points = rand(rng, len(sizes), 8)
    exp = O.compute_quotients_and_combine(partials, flts, points, lift)
    accs = [([dev(p[:, i].copy()) for i in range(4)], s, flts[a], points[a])
            for a, (p, s) in enumerate(zip(partials, sizes))]
    got = B.compute_quotients_and_combine(accs, lift)
    assert np.array_equal(np.stack([host(t) for t in got], 1), exp)


@pytest.mark.parametrize("sizes", [[1], [2, 5], [3, 3, 7, 9], [10, 12, 16]])
def test_lift_and_accumulate(B, sizes):
    rng = np.random.default_rng(sum(sizes))
    cols = [rand(rng, 1 << s, 4) for s in sizes]
    exp = O.lift_and_accumulate(cols)
    got = B.lift_and_accumulate([[dev(c[:, i].copy()) for i in range(4)] for c in cols])
    assert np.array_equal(np.stack([host(t) for t in got], 1), exp)


@pytest.mark.parametrize("log_n,n_polys", [(0, 2), (1, 3), (5, 4), (10, 3), (11, 2), (12, 4), (13, 9), (18, 5)])
def test_batch_eval_at_point(B, log_n, n_polys):
    rng = np.random.default_rng(log_n * 7 + n_polys)
    polys = [rand(rng, 1 << log_n) for _ in range(n_polys)]
    point = rand(rng, 8)
    got = B.batch_eval_at_point([dev(p) for p in polys], point)
    for p, g in zip(polys, got):
        assert list(O.eval_at_point(p, point)) == [int(x) for x in g]
