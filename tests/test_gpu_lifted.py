"""Lifted Merkle commitment (MerkleOpsLifted) on the GPU against the oracle:
leaves for mixed sizes, more than one message block, lifting above the
largest column, no columns; the full tree through the node layers."""
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


def host_hashes(t):
    return t.cpu().numpy().view(np.uint8).reshape(-1, 32)


@pytest.mark.parametrize("logs,lift", [([3], 3), ([1, 4, 2, 4], 4), ([5] * 17 + [2] * 3, 6), ([10, 3, 7], 12),
                                       ([1], 1), (list(range(1, 15)), 16)])
def test_lifted_leaves(B, logs, lift):
    from gpustark.backend import to_device
    rng = np.random.default_rng(len(logs) * 100 + lift)
    cols = [rng.integers(0, P, 1 << lg, dtype=np.int64).astype(np.uint32) for lg in logs]
    got = host_hashes(B.build_leaves_lifted([to_device(c) for c in cols], lift))
    assert np.array_equal(got, O.lifted_leaves(cols, lift))


def test_lifted_no_columns(B):
    assert np.array_equal(host_hashes(B.build_leaves_lifted([], 7)), O.lifted_leaves([], 7))


def test_lifted_tree_root(B):
    """MerkleProverLifted::commit: leaves, then build_next_layer down to the root."""
    from gpustark.backend import to_device
    rng = np.random.default_rng(9)
    logs, lift = [8, 3, 12, 12, 5], 13
    cols = [rng.integers(0, P, 1 << lg, dtype=np.int64).astype(np.uint32) for lg in logs]
    layers = [torch.empty((1 << L) * 8, dtype=torch.int32, device="cuda") for L in range(lift + 1)]
    B.build_leaves_lifted([to_device(c) for c in cols], lift, out=layers[lift])
    B.commit_node_layers(layers)
    prev = O.lifted_leaves(cols, lift)
    for L in range(lift - 1, -1, -1):
        prev = O.commit_on_layer(L, prev, [])
    assert np.array_equal(host_hashes(layers[0]), prev)
