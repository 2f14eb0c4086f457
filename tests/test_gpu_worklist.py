"""Work-lists of uneven sizes. FFTs (gs_fft_worklist): every item equals the
oracle's interpolation or evaluation on the same twiddle tree, and the
per-size entries gs_interpolate_columns / gs_evaluate_columns, bit for bit;
items inside the work-list range (log 3..13, one launch) and outside it
(the per-size path) mixed in one call; in-place interpolations; errors for
bad items. Merkle trees (gs_merkle_worklist): every layer of every tree
equals gs_commit_on_layer + gs_commit_node_layers and the oracle's layers,
trees of log 0..10 in one launch and larger ones on the per-tree path."""
import ctypes as C

import numpy as np
import pytest

import pyoracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
ROOT_LOG = 14  # one twiddle tree for domains up to 2^15


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


def rand_m31(rng, n):
    return rng.integers(0, O.P, n, dtype=np.int64).astype(np.uint32)


def make_items(rng, n_items, logs):
    """(kind, host source, coeff/domain logs, in place) per item."""
    out = []
    for _ in range(n_items):
        log = int(rng.choice(logs))
        if rng.random() < 0.5:
            out.append(("interpolate", rand_m31(rng, 1 << log), log, log, bool(rng.random() < 0.5)))
        else:
            m = int(rng.integers(1, log + 1))
            out.append(("evaluate", rand_m31(rng, 1 << m), m, log, False))
    return out


def run(B, tw, spec):
    items = []
    for kind, src, m, log, in_place in spec:
        s = dev(src)
        d = s if in_place else torch.empty(1 << log, dtype=torch.int32, device="cuda")
        items.append((kind, s, d))
    outs = B.fft_worklist(items, tw)
    torch.cuda.synchronize()
    return [host(o) for o in outs]


@pytest.mark.parametrize("seed,n_items,logs", [(1, 40, list(range(1, 16))), (2, 300, list(range(3, 14))),
                                               (3, 7, [13]), (4, 9, [1, 2, 14, 15])])
def test_worklist_matches_oracle_and_per_size_entries(B, seed, n_items, logs):
    rng = np.random.default_rng(seed)
    tw = B.precompute_twiddles(ROOT_LOG)
    spec = make_items(rng, n_items, logs)
    got = run(B, tw, spec)
    for (kind, src, m, log, _), g in zip(spec, got):
        if kind == "interpolate":
            d = dev(src)
            B.interpolate_columns([d], log, tw)
            ref = host(d)
            if log <= 10:
                assert np.array_equal(ref, O.interpolate(src, log, root_log=ROOT_LOG))
        else:
            ref = host(B.evaluate_polynomials([dev(src)], log, tw)[0])
            if log <= 10:
                assert np.array_equal(ref, O.evaluate(src, log, root_log=ROOT_LOG))
        assert np.array_equal(g, ref), (kind, m, log)


def test_worklist_repeated_calls_and_empty(B):
    rng = np.random.default_rng(9)
    tw = B.precompute_twiddles(ROOT_LOG)
    spec = make_items(rng, 50, list(range(3, 14)))
    assert all(np.array_equal(a, b) for a, b in zip(run(B, tw, spec), run(B, tw, spec)))
    assert B.fft_worklist([], tw) == []


def test_worklist_rejects_bad_items(B):
    from gpustark import GpuStarkError
    tw = B.precompute_twiddles(6)
    x = torch.zeros(1 << 5, dtype=torch.int32, device="cuda")
    with pytest.raises(GpuStarkError, match="distinct"):
        B.fft_worklist([("evaluate", x, x)], tw)
    big = torch.zeros(1 << 9, dtype=torch.int32, device="cuda")
    with pytest.raises(GpuStarkError, match="size out of range"):
        B.fft_worklist([("interpolate", big, big)], tw)


def test_worklist_longer_than_the_staging_ring(B):
    """70,000 items (2.2 MB of descriptors, more than the staging ring takes
    at once): the list gets a device buffer of its own; sampled items equal
    the oracle."""
    rng = np.random.default_rng(12)
    tw = B.precompute_twiddles(ROOT_LOG)
    n, log = 70000, 3
    data = rng.integers(0, O.P, (n, 1 << log), dtype=np.int64).astype(np.uint32)
    flat = dev(data.reshape(-1))
    cols = [flat[k << log:(k + 1) << log] for k in range(n)]
    B.fft_worklist([("interpolate", c, c) for c in cols], tw)
    got = host(flat).reshape(n, 1 << log)
    for k in rng.choice(n, 60, replace=False):
        assert np.array_equal(got[k], O.interpolate(data[k], log, root_log=ROOT_LOG))


# ----------------------------------------------------------- Merkle trees
def tree_reference(B, cols):
    """The per-tree path: gs_commit_on_layer for the leaves, then
    gs_commit_node_layers."""
    log = cols[0].numel().bit_length() - 1
    layers = [torch.empty((1 << lg) * 8, dtype=torch.int32, device="cuda") for lg in range(log + 1)]
    B.commit_on_layer(log, None, cols, out=layers[log])
    if log:
        B.commit_node_layers(layers)
    return layers


@pytest.mark.parametrize("seed,n_trees,logs,max_cols", [(5, 30, list(range(0, 13)), 40), (6, 200, list(range(2, 11)), 20),
                                                         (7, 3, [11, 12], 17)])
def test_merkle_worklist_matches_oracle_and_per_tree_path(B, seed, n_trees, logs, max_cols):
    rng = np.random.default_rng(seed)
    host_trees, trees = [], []
    for _ in range(n_trees):
        log, k = int(rng.choice(logs)), int(rng.integers(1, max_cols + 1))
        h = [rand_m31(rng, 1 << log) for _ in range(k)]
        host_trees.append(h)
        trees.append([dev(c) for c in h])
    got = B.merkle_worklist(trees)
    torch.cuda.synchronize()
    for h, cols, layers in zip(host_trees, trees, got):
        ref = tree_reference(B, cols)
        for a, b in zip(layers, ref):
            assert np.array_equal(host(a), host(b))
        log = len(layers) - 1
        if log <= 8:  # the oracle, layer by layer
            exp = O.commit_on_layer(log, None, h)
            assert np.array_equal(host(layers[log]).view(np.uint8), exp.reshape(-1))
            for lg in range(log - 1, -1, -1):
                exp = O.commit_on_layer(lg, exp, [])
                assert np.array_equal(host(layers[lg]).view(np.uint8), exp.reshape(-1))


def test_merkle_worklist_rejects_bad_trees(B):
    """A tree without columns, and a misaligned layer, are refused before any launch."""
    from gpustark import GpuStarkError
    from gpustark import _lib as L
    from gpustark.backend import default_context
    ctx = default_context()
    col = torch.zeros(1 << 4, dtype=torch.int32, device="cuda")
    layers = [torch.zeros(((1 << lg) * 8) + 4, dtype=torch.int32, device="cuda") for lg in range(5)]
    cp, kc = L.ptr_array([col.data_ptr()])
    item = L.MerkleItem()
    lp, kl = L.ptr_array([t.data_ptr() for t in layers])
    item.cols, item.n_cols, item.log_size, item.layers = cp, 0, 4, lp
    assert L.lib().gs_merkle_worklist(ctx.handle, C.byref(item), 1) != 0
    assert b"columns and layers" in L.lib().gs_last_error()
    lp2, kl2 = L.ptr_array([t.data_ptr() + (4 if lg == 2 else 0) for lg, t in enumerate(layers)])
    item.n_cols, item.layers = 1, lp2
    assert L.lib().gs_merkle_worklist(ctx.handle, C.byref(item), 1) != 0
    assert b"16-byte aligned" in L.lib().gs_last_error()
