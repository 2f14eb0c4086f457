"""Kernel parity: each CUDA op through the C ABI vs the CPU oracle, bit-exact,
on seeded inputs; at the sweep's full sizes, size-independent properties."""
import hashlib

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


def rand_m31(rng, *shape):
    return rng.integers(0, P, shape, dtype=np.int64).astype(np.uint32)


def test_twiddles_match_reference_literals(B):
    """The device twiddle tree of half_odds(6) against the literal values in
    the reference CUDA backend's interpolation test."""
    import json, os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")))
    g = g["cuda_interpolate_twiddle_tree"]
    t = B.precompute_twiddles(g["root_log_size"])
    assert [int(v) for v in host(t.twiddles)] == g["twiddles"]
    assert [int(v) for v in host(t.itwiddles)] == g["itwiddles"]


@pytest.mark.parametrize("root_log", [1, 2, 3, 5, 8, 13, 17])
def test_twiddles(B, root_log):
    t = B.precompute_twiddles(root_log)
    tw, itw = O.twiddles_half_odds(root_log)
    assert np.array_equal(host(t.twiddles), tw)
    assert np.array_equal(host(t.itwiddles), itw)


@pytest.mark.parametrize("log_n", [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 20, 21, 22])
def test_interpolate_matches_oracle(B, log_n):
    rng = np.random.default_rng(100 + log_n)
    n_cols = 1 if log_n > 20 else (3 if log_n > 14 else 5)
    cols = [rand_m31(rng, 1 << log_n) for _ in range(n_cols)]
    root = max(log_n - 1, 1) + (1 if log_n % 2 else 0)  # also exercise a larger tree
    tw = B.precompute_twiddles(root)
    d = [dev(c) for c in cols]
    B.interpolate_columns(d, log_n, tw)
    expect = O.interpolate_columns(cols, log_n, root_log=root)
    for g, e in zip(d, expect):
        assert np.array_equal(host(g), e)


@pytest.mark.parametrize("coeff_log,log_n", [(1, 1), (1, 2), (2, 2), (1, 3), (3, 3), (4, 5), (8, 9), (10, 12), (12, 12),
                                              (13, 14), (15, 16), (16, 17), (18, 19), (19, 20), (5, 18), (20, 22), (22, 22),
                                              (23, 24)])
def test_evaluate_matches_oracle(B, coeff_log, log_n):
    rng = np.random.default_rng(200 + coeff_log * 31 + log_n)
    cols = [rand_m31(rng, 1 << coeff_log) for _ in range(1 if log_n > 20 else 3)]
    tw = B.precompute_twiddles(max(log_n - 1, 1))
    out = B.evaluate_polynomials([dev(c) for c in cols], log_n, tw)
    expect = O.evaluate_columns(cols, log_n, root_log=max(log_n - 1, 1))
    for g, e in zip(out, expect):
        assert np.array_equal(host(g), e)


def test_bit_reverse(B):
    rng = np.random.default_rng(7)
    for log_n in (0, 1, 5, 16):
        a = rand_m31(rng, 1 << log_n)
        d = dev(a)
        B.bit_reverse_column(d)
        assert np.array_equal(host(d), O.bit_reverse(a))


@pytest.mark.parametrize("n_cols", [0, 1, 4, 15, 16, 17, 100, 158])
@pytest.mark.parametrize("with_prev", [False, True])
def test_commit_on_layer(B, n_cols, with_prev):
    rng = np.random.default_rng(300 + n_cols * 2 + with_prev)
    log_size = 9
    cols = [rand_m31(rng, 1 << log_size) for _ in range(n_cols)]
    prev = rng.integers(0, 256, (1 << (log_size + 1)) * 32, dtype=np.uint8) if with_prev else None
    prev_d = dev(prev.view(np.uint32)) if with_prev else None
    out = B.commit_on_layer(log_size, prev_d, [dev(c) for c in cols])
    expect = O.commit_on_layer(log_size, prev, cols)
    assert np.array_equal(host(out).view(np.uint8).reshape(-1, 32), expect)


def test_merkle_root_of_mixed_sizes(B):
    """Full commit with columns injected at their own layer (prover/vcs/prover.rs:22-48)."""
    rng = np.random.default_rng(9)
    sizes = [10, 10, 9, 7, 7, 7, 3, 1]
    cols = [rand_m31(rng, 1 << s) for s in sizes]
    prev = None
    for ls in range(max(sizes), -1, -1):
        layer_cols = [dev(c) for c, s in zip(cols, sizes) if s == ls]
        prev = B.commit_on_layer(ls, prev, layer_cols)
    root = host(prev).view(np.uint8).tobytes()
    assert root == O.merkle_root(cols)


def qm_rand(rng, n):
    return rand_m31(rng, n, 4)


@pytest.mark.parametrize("log_n", [1, 2, 3, 6, 12, 16])
def test_fold_line(B, log_n):
    rng = np.random.default_rng(400 + log_n)
    ev = qm_rand(rng, 1 << log_n)
    alpha = rand_m31(rng, 4)
    tw = B.precompute_twiddles(log_n + 1)
    leaves = __import__("torch").empty((1 << (log_n - 1)) * 8, dtype=__import__("torch").int32, device="cuda")
    out = B.fold_line([dev(ev[:, i].copy()) for i in range(4)], log_n, alpha, tw, leaf_hashes=leaves)
    got = np.stack([host(t) for t in out], axis=1)
    expect = O.fold_line(ev, log_n, alpha)
    assert np.array_equal(got, expect)
    # fused leaf hashes = Merkle leaf layer of the folded planes
    exp_leaves = O.commit_on_layer(log_n - 1, None, [expect[:, i].copy() for i in range(4)])
    assert np.array_equal(host(leaves).view(np.uint8).reshape(-1, 32), exp_leaves)


@pytest.mark.parametrize("log_n", [1, 2, 3, 4, 7, 13, 17])
def test_fold_circle_into_line(B, log_n):
    rng = np.random.default_rng(500 + log_n)
    src = qm_rand(rng, 1 << log_n)
    dst = qm_rand(rng, 1 << (log_n - 1))
    alpha = rand_m31(rng, 4)
    tw = B.precompute_twiddles(max(log_n - 1, 1))
    d = [dev(dst[:, i].copy()) for i in range(4)]
    B.fold_circle_into_line(d, [dev(src[:, i].copy()) for i in range(4)], log_n, alpha, tw)
    got = np.stack([host(t) for t in d], axis=1)
    expect = O.fold_circle_into_line(dst, src, log_n, alpha)
    assert np.array_equal(got, expect)


@pytest.mark.parametrize("pow_bits,salt", [(0, 0), (1, 0), (5, 0), (10, 0), (10, 1), (10, 2), (10, 3), (14, 0),
                                           (18, 0), (21, 0)])
def test_grind(B, pow_bits, salt):
    """The smallest passing nonce (the early-exit grid skips only steps above
    a recorded hit). The device searches low words below 2^20 under high word
    0, 1, ... (simd/grind.rs, the reference CUDA grind); the oracle searches
    0, 1, 2, ... (cpu/grind.rs). They meet whenever a hit lies below 2^20;
    otherwise the device's nonce has a higher word and passes the check."""
    digest = hashlib.blake2s(b"channel-%d-%d" % (pow_bits, salt), digest_size=32).digest()
    got = B.grind(digest, pow_bits)
    want = O.grind(digest, pow_bits)
    if want < (1 << 20):
        assert got == want
    else:
        assert got >> 32 >= 1 and (got & 0xFFFFFFFF) < (1 << 20)
        assert O.verify_pow(digest, pow_bits, got)


# ---------------------------------------------------------------- full sizes
def bit_reverse_index(i, log_n):
    return int(format(i, f"0{log_n}b")[::-1], 2) if log_n else i


def canonic_domain_point(log_n, i):
    """CanonicCoset(log_n).circle_domain().at(i) (core/poly/circle/domain.rs:
    57-68) as an M31 point: the half coset half_odds(log_n - 1) then its
    conjugate."""
    half = 1 << (log_n - 1)
    init, step = 1 << (31 - (log_n + 1)), 1 << (31 - (log_n - 1))
    idx = (init + step * (i % half)) % (1 << 31)
    if i >= half:
        idx = (-idx) % (1 << 31)
    xy = np.zeros(2, np.uint32)
    O.lib().oracle_index_to_point(idx, xy.ctypes.data_as(O.U32P))
    return int(xy[0]), int(xy[1])


@pytest.mark.parametrize("log_n,n_points", [(22, 4), (24, 3), (26, 2)])
def test_fft_full_size_against_oracle_points(B, log_n, n_points):
    """The kernel sweep's top sizes: evaluate on CanonicCoset(n) and check
    sampled rows against the oracle's direct evaluation of the coefficient
    polynomial at those domain points (fold over the circle FFT basis,
    independent of any twiddle table), then interpolate back and require the
    original coefficients. The reference's own CUDA FFT is compared at the
    same sizes in test_gpu_reference_cuda.py."""
    rng = np.random.default_rng(600 + log_n)
    c = rand_m31(rng, 1 << log_n)
    tw = B.precompute_twiddles(log_n)
    ev = B.evaluate_polynomials([dev(c)], log_n, tw)[0]
    ev_h = host(ev)
    for j in rng.integers(0, 1 << log_n, n_points):
        x, y = canonic_domain_point(log_n, bit_reverse_index(int(j), log_n))
        want = O.eval_at_point(c, np.array([x, 0, 0, 0, y, 0, 0, 0], np.uint32))
        assert list(want) == [int(ev_h[j]), 0, 0, 0], f"row {j}"
    B.interpolate_columns([ev], log_n, tw)
    assert np.array_equal(host(ev), c)


def test_merkle_64x2p20_root(B):
    rng = np.random.default_rng(700)
    cols = [rand_m31(rng, 1 << 20) for _ in range(64)]
    prev = B.commit_on_layer(20, None, [dev(x) for x in cols])
    for ls in range(19, -1, -1):
        prev = B.commit_on_layer(ls, prev, [])
    assert host(prev).view(np.uint8).tobytes() == O.merkle_root(cols)


@pytest.mark.parametrize("top", [1, 5, 9, 10, 11, 12, 15, 18, 19, 20])
def test_commit_node_layers_fused(B, top):
    """The one-launch tree (512-child units, the last block of each group
    going on to the next stage) equals per-layer oracle commit_on_layer
    calls, across the unit boundaries (9/10 and 18/19/20 leaves-log)."""
    rng = np.random.default_rng(900 + top)
    leaves = rng.integers(0, 256, (1 << top) * 32, dtype=np.uint8)
    layers = [__import__("torch").empty((1 << L) * 8, dtype=__import__("torch").int32, device="cuda")
              for L in range(top + 1)]
    layers[top].copy_(dev(leaves.view(np.uint32)))
    B.commit_node_layers(layers)
    prev = leaves
    for L in range(top - 1, -1, -1):
        prev = O.commit_on_layer(L, prev.reshape(-1), [])
        assert np.array_equal(host(layers[L]).view(np.uint8).reshape(-1, 32), prev), L


def test_commit_node_layers_repeated_launches(B):
    """The ticket counters wrap back to zero: trees of different sizes
    launched back to back on one context keep giving the oracle's roots."""
    import torch
    rng = np.random.default_rng(950)
    for top in (19, 12, 20, 10, 19, 3, 19):
        leaves = rng.integers(0, 256, (1 << top) * 32, dtype=np.uint8)
        layers = [torch.empty((1 << L) * 8, dtype=torch.int32, device="cuda") for L in range(top + 1)]
        layers[top].copy_(dev(leaves.view(np.uint32)))
        B.commit_node_layers(layers)
        prev = leaves
        for L in range(top - 1, -1, -1):
            prev = O.commit_on_layer(L, prev.reshape(-1), [])
        assert np.array_equal(host(layers[0]).view(np.uint8).reshape(-1, 32), prev), top


def test_fold_line_2p22(B):
    rng = np.random.default_rng(800)
    ev = qm_rand(rng, 1 << 22)
    alpha = rand_m31(rng, 4)
    tw = B.precompute_twiddles(23)
    out = B.fold_line([dev(ev[:, i].copy()) for i in range(4)], 22, alpha, tw)
    got = np.stack([host(t) for t in out], axis=1)
    assert np.array_equal(got, O.fold_line(ev, 22, alpha))
