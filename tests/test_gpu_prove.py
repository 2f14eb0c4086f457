"""End-to-end parity: the GPU prover's serialised proof is byte-identical to
the CPU oracle's for the same AIR, inputs and PcsConfig."""
import numpy as np
import pytest

import pyoracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def G():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpustark import prove
    return prove


@pytest.mark.parametrize("log_n,n_cols,mode", [(4, 8, 0), (6, 16, 1), (8, 100, 0), (10, 100, 1), (12, 37, 1)])
def test_wide_fibonacci_proof_bytes(G, log_n, n_cols, mode):
    got = G.prove_wide_fibonacci(log_n, n_cols, seed=11, input_mode=mode)
    exp = O.prove("wide_fibonacci", log_n, n_cols=n_cols, seed=11, input_mode=mode)
    assert got == exp


@pytest.mark.parametrize("log_n,mode", [(4, 0), (6, 0), (8, 1), (10, 0), (12, 1)])
def test_poseidon_proof_bytes(G, log_n, mode):
    got = G.prove_poseidon(log_n, seed=5, input_mode=mode)
    exp = O.prove("poseidon", log_n, seed=5, input_mode=mode)
    assert got == exp


def test_poseidon_reference_split_is_rejected_like_the_reference(G):
    """With the reference's fixed composition split the lifted protocol cannot
    prove a LOG_EXPAND = 2 component: both provers report ConstraintsNotSatisfied."""
    with pytest.raises(G.ConstraintsNotSatisfied):
        G.prove_poseidon(6, composition_log_split=1)
    with pytest.raises(O.ConstraintsNotSatisfied):
        O.prove("poseidon", 6, split_log=1)


# last layers of 2^(last + blowup) values: up to 2^5 with a degree bound of at
# most 2^3 take the device's last-layer step (one to three Blake2s blocks in
# its mix), larger ones the host's
@pytest.mark.parametrize("blowup,queries,pow_bits,last", [(2, 20, 4, 0), (1, 3, 10, 0), (3, 9, 0, 1), (1, 5, 8, 3),
                                                          (2, 7, 3, 4), (1, 6, 5, 4)])
def test_pcs_configs(G, blowup, queries, pow_bits, last):
    cfg = G.pcs_config(pow_bits=pow_bits, log_blowup=blowup, n_queries=queries, log_last_layer=last)
    got = G.prove_wide_fibonacci(9, 20, seed=3, input_mode=1, config=cfg)
    exp = O.prove("wide_fibonacci", 9, n_cols=20, seed=3, input_mode=1, pow_bits=pow_bits, n_queries=queries,
                  log_blowup=blowup, log_last_layer=last)
    assert got == exp


def test_host_inputs_match_seeded(G):
    log_n = 8
    st = np.array([[O.seeded_m31(9, i, r) for r in range(1 << log_n)] for i in range(16)], np.uint32)
    got = G.prove_poseidon(log_n, input_mode=G.INPUT_HOST, host_inputs=st)
    assert got == G.prove_poseidon(log_n, seed=9, input_mode=G.INPUT_SEEDED)
    ab = st[:2]
    assert G.prove_wide_fibonacci(log_n, 30, input_mode=G.INPUT_HOST, host_inputs=ab) == \
        G.prove_wide_fibonacci(log_n, 30, seed=9, input_mode=G.INPUT_SEEDED)


@pytest.mark.slow
def test_wide_fibonacci_config_size(G):
    """Wide-Fibonacci 2^16 rows x 100 columns, seeded inputs (the benchmark configuration)."""
    assert G.prove_wide_fibonacci(16, 100, seed=0, input_mode=1) == \
        O.prove("wide_fibonacci", 16, n_cols=100, seed=0, input_mode=1)


@pytest.mark.slow
def test_poseidon_config_size(G):
    """Poseidon2 2^18 instances, seeded inputs (the benchmark configuration)."""
    assert G.prove_poseidon(18, seed=0, input_mode=1) == O.prove("poseidon", 18, seed=0, input_mode=1)


# ---------------------------------------------- Poseidon252MerkleChannel proofs
@pytest.mark.parametrize("log_n,n_cols,mode", [(4, 8, 0), (7, 9, 1), (10, 100, 1)])
def test_wide_fibonacci_poseidon252_proof_bytes(G, log_n, n_cols, mode):
    """cuda_prove_wide_fibonacci_poseidon: every tree, the channel and the
    proof of work over Poseidon252, byte-identical to the oracle."""
    got = G.prove_wide_fibonacci(log_n, n_cols, seed=4, input_mode=mode, merkle_channel="poseidon252")
    exp = O.prove("wide_fibonacci", log_n, n_cols=n_cols, seed=4, input_mode=mode, merkle_channel="poseidon252")
    assert got == exp
    assert got != G.prove_wide_fibonacci(log_n, n_cols, seed=4, input_mode=mode)


@pytest.mark.parametrize("log_n,mode", [(4, 0), (8, 1)])
def test_poseidon_poseidon252_proof_bytes(G, log_n, mode):
    got = G.prove_poseidon(log_n, seed=6, input_mode=mode, merkle_channel="poseidon252")
    exp = O.prove("poseidon", log_n, seed=6, input_mode=mode, merkle_channel="poseidon252")
    assert got == exp


def test_poseidon252_pcs_config(G):
    cfg = G.pcs_config(pow_bits=6, log_blowup=2, log_last_layer=1, n_queries=11)
    got = G.prove_wide_fibonacci(8, 12, seed=2, input_mode=1, config=cfg, merkle_channel="poseidon252")
    exp = O.prove("wide_fibonacci", 8, n_cols=12, seed=2, input_mode=1, pow_bits=6, n_queries=11, log_blowup=2,
                  log_last_layer=1, merkle_channel="poseidon252")
    assert got == exp


@pytest.mark.slow
def test_wide_fibonacci_poseidon252_config_size(G):
    """The Wide-Fibonacci 2^16 x 100 benchmark proof over the Poseidon252
    channel, byte-identical to the oracle's."""
    assert G.prove_wide_fibonacci(16, 100, seed=0, input_mode=1, merkle_channel="poseidon252") == \
        O.prove("wide_fibonacci", 16, n_cols=100, seed=0, input_mode=1, merkle_channel="poseidon252")


@pytest.mark.slow
def test_poseidon_poseidon252_2e14(G):
    assert G.prove_poseidon(14, seed=3, input_mode=1, merkle_channel="poseidon252") == \
        O.prove("poseidon", 14, seed=3, input_mode=1, merkle_channel="poseidon252")


def test_context_stream_restored_after_proof(G):
    """A proof runs on the context's own prioritised streams and hands the
    caller's stream back when it returns, also when that stream is the legacy
    default stream (a null handle): work the caller then enqueues on its
    stream and passes to the library stays ordered. Pattern: a proof (Poseidon2,
    which uses the side stream), then torch clones of an evaluation consumed
    at once by an in-place interpolation on the same context."""
    import torch
    from gpustark.backend import GpuBackend as B, to_device
    assert G.prove_poseidon(6, seed=3, input_mode=G.INPUT_SEEDED)
    rng = np.random.default_rng(77)
    log, blowup = 17, 2
    tw = B.precompute_twiddles(log + blowup - 1)
    coeffs = [to_device(rng.integers(0, O.P, 1 << log, dtype=np.int64).astype(np.uint32)) for _ in range(2)]
    for _ in range(3):
        ev = B.evaluate_polynomials(coeffs, log + blowup, tw)
        back = [e.clone() for e in ev]
        B.interpolate_columns(back, log + blowup, tw)
        torch.cuda.synchronize()
        for b, c in zip(back, coeffs):
            assert torch.equal(b[: c.numel()], c) and not torch.any(b[c.numel():])
