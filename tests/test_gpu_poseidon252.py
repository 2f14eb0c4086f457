"""Poseidon252 Merkle hashing on the GPU (gs_poseidon252_commit_on_layer,
gs_poseidon252_permute) against the oracle's restatement of Starknet's
Poseidon and the reference's own hash_node known answers."""
import json
import os

import numpy as np
import pytest

import poseidon252 as PS

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")))


@pytest.fixture(scope="module")
def B():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpustark.backend import GpuBackend
    return GpuBackend


def felts_to_dev(values):
    return torch.tensor(np.frombuffer(b"".join(PS.to_bytes_be(v) for v in values), dtype=np.uint8).copy(),
                        device="cuda")


def dev_to_felts(t):
    b = t.cpu().numpy().tobytes()
    return [int.from_bytes(b[32 * i:32 * i + 32], "big") for i in range(len(b) // 32)]


def col(values):
    return torch.tensor(np.array(values, dtype=np.uint32).view(np.int32), device="cuda")


def test_permutation_matches_oracle(B):
    rng = np.random.default_rng(1)
    states = [[0, 0, 0], [PS.P - 1, PS.P - 1, PS.P - 1], [1, 2, 3], [0, 0, 2]]
    for _ in range(60):
        states.append([int.from_bytes(rng.bytes(32), "big") % PS.P for _ in range(3)])
    got = dev_to_felts(B.poseidon252_permute(felts_to_dev([v for s in states for v in s])))
    for k, s in enumerate(states):
        assert got[3 * k:3 * k + 3] == PS.permute(s), k


def test_hash_node_known_answers(B):
    a, b = GOLDEN["poseidon252_hash_node"]
    # hash_node(None, [0, 1]): one node, two columns of one row
    out = B.poseidon252_commit_on_layer(0, None, [col([v]) for v in a["columns"]])
    assert dev_to_felts(out) == [int(a["hash"])]
    # hash_node(Some((1, 2)), [3])
    prev = felts_to_dev(b["children"])
    out = B.poseidon252_commit_on_layer(0, prev, [col([v]) for v in b["columns"]])
    assert dev_to_felts(out) == [int(b["hash"])]


@pytest.mark.parametrize("n_cols", [0, 1, 7, 8, 9, 16, 17])
@pytest.mark.parametrize("with_prev", [False, True])
def test_layer_matches_oracle(B, n_cols, with_prev):
    rng = np.random.default_rng(10 * n_cols + with_prev)
    log_size = 4
    n = 1 << log_size
    cols = [rng.integers(0, PS.M31, n, dtype=np.int64).astype(np.uint32) for _ in range(n_cols)]
    prev = [int.from_bytes(rng.bytes(32), "big") % PS.P for _ in range(2 * n)] if with_prev else None
    got = B.poseidon252_commit_on_layer(log_size, felts_to_dev(prev) if prev else None, [col(c) for c in cols])
    want = PS.commit_on_layer(log_size, prev, cols)
    assert dev_to_felts(got) == want


def test_tree_root_matches_oracle(B):
    """Leaves of 2^6 rows x 20 columns (columns equal to M31 edge values
    included), then node layers to the root."""
    rng = np.random.default_rng(7)
    n_log = 6
    cols = [rng.integers(0, PS.M31, 1 << n_log, dtype=np.int64).astype(np.uint32) for _ in range(19)]
    cols.append(np.full(1 << n_log, PS.M31 - 1, dtype=np.uint32))
    layer = B.poseidon252_commit_on_layer(n_log, None, [col(c) for c in cols])
    want = PS.commit_on_layer(n_log, None, cols)
    assert dev_to_felts(layer) == want
    for L in range(n_log - 1, -1, -1):
        layer = B.poseidon252_commit_on_layer(L, layer, [])
        want = PS.commit_on_layer(L, want, [])
        assert dev_to_felts(layer) == want, L
    assert len(want) == 1


@pytest.mark.parametrize("pow_bits,salt", [(0, 0), (1, 0), (6, 0), (10, 0), (10, 1), (12, 0)])
def test_grind_matches_oracle(B, pow_bits, salt):
    """GrindOps<Poseidon252Channel>: the same smallest nonce as the oracle's
    sequential search, and the nonce passes the channel's check."""
    ch = PS.Channel()
    ch.mix_u64(0x1111222233334444 + 7 * salt + pow_bits)
    got = B.poseidon252_grind(ch.digest, pow_bits)
    assert got == ch.grind(pow_bits)
    assert ch.verify_pow_nonce(pow_bits, got)


def test_large_layers_and_batches_match_the_oracle(B):
    """Layers of 2^13..2^15 nodes (leaves with an all-(P-1) column, node-only
    layers, two felts per leaf) and permutation batches of 300 and 20000
    states (grid-stride loops) against the C++ oracle."""
    import pyoracle as O
    rng = np.random.default_rng(21)
    for log_size, n_cols in [(13, 8), (14, 0), (15, 9)]:
        n = 1 << log_size
        cols = [rng.integers(0, PS.M31, n, dtype=np.int64).astype(np.uint32) for _ in range(n_cols)]
        cols[-1:] = [np.full(n, PS.M31 - 1, np.uint32)] if n_cols else []
        prev = None
        if n_cols == 0:
            prev = np.frombuffer(b"".join(PS.to_bytes_be(int.from_bytes(rng.bytes(32), "big") % PS.P)
                                          for _ in range(2 * n)), np.uint8)
        got = B.poseidon252_commit_on_layer(log_size, torch.tensor(prev, device="cuda") if prev is not None else None,
                                            [col(c) for c in cols])
        want = O.p252_commit_on_layer(log_size, prev, cols)
        assert np.array_equal(got.cpu().numpy().reshape(-1, 32), want), (log_size, n_cols)
    for n in [300, 20000]:
        raw = b"".join(PS.to_bytes_be(int.from_bytes(rng.bytes(32), "big") % PS.P) for _ in range(3 * n))
        got = B.poseidon252_permute(torch.tensor(np.frombuffer(raw, np.uint8).copy(), device="cuda"))
        assert bytes(got.cpu().numpy()) == O.p252_permute(raw), n
