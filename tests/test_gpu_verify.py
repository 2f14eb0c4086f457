"""Acceptance of the GPU prover's proofs by the verifier (oracle/verifier.h,
restating the reference's verification rule: core/verifier.rs,
core/pcs/verifier.rs, core/fri.rs, core/vcs/verifier.rs): Wide-Fibonacci
proofs with the reference's composition split of 2, Poseidon2 proofs with
the split of 4 the prover uses for this component, both Merkle channels, the
PcsConfigs the prover supports, and the benchmark sizes. A GPU proof with one
flipped bit in any section is rejected."""
import numpy as np
import pytest

import pyoracle as O
from proof_layout import flip, sections

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def G():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpustark import prove
    return prove


@pytest.mark.parametrize("log_n,n_cols,mode", [(4, 3, 0), (6, 16, 1), (8, 100, 0), (10, 100, 1), (12, 37, 1)])
def test_wide_fibonacci_gpu_proofs_accepted(G, log_n, n_cols, mode):
    p = G.prove_wide_fibonacci(log_n, n_cols, seed=11, input_mode=mode)
    assert O.verify(p, "wide_fibonacci", log_n, n_cols=n_cols, split_log=1, config=(10, 1, 0, 70, 1))


@pytest.mark.parametrize("log_n,mode", [(4, 0), (6, 1), (8, 1), (10, 0), (12, 1)])
def test_poseidon_gpu_proofs_accepted(G, log_n, mode):
    p = G.prove_poseidon(log_n, seed=5, input_mode=mode)
    cs = O.poseidon_claimed_sum(p, log_n, seed=5, input_mode=mode)
    assert O.verify(p, "poseidon", log_n, split_log=2, claimed_sum=cs, config=(10, 1, 0, 70, 1))


@pytest.mark.parametrize("blowup,queries,pow_bits,last", [(2, 20, 4, 0), (1, 3, 10, 0), (3, 9, 0, 1), (1, 30, 2, 2)])
def test_pcs_configs_gpu_proofs_accepted(G, blowup, queries, pow_bits, last):
    cfg = G.pcs_config(pow_bits=pow_bits, log_blowup=blowup, n_queries=queries, log_last_layer=last)
    p = G.prove_wide_fibonacci(9, 20, seed=3, input_mode=1, config=cfg)
    assert O.verify(p, "wide_fibonacci", 9, n_cols=20, config=(pow_bits, blowup, last, queries, 1))
    p = G.prove_poseidon(7, seed=3, input_mode=1, config=cfg)
    cs = O.poseidon_claimed_sum(p, 7, seed=3, input_mode=1)
    assert O.verify(p, "poseidon", 7, claimed_sum=cs, config=(pow_bits, blowup, last, queries, 1))


def test_host_input_gpu_proofs_accepted(G):
    log_n = 8
    rng = np.random.default_rng(21)
    st = rng.integers(0, O.P, (16, 1 << log_n), dtype=np.int64).astype(np.uint32)
    p = G.prove_poseidon(log_n, input_mode=G.INPUT_HOST, host_inputs=st)
    cs = O.poseidon_claimed_sum(p, log_n, input_mode=2, host_inputs=st)
    assert O.verify(p, "poseidon", log_n, claimed_sum=cs)
    p = G.prove_wide_fibonacci(log_n, 30, input_mode=G.INPUT_HOST, host_inputs=st[:2])
    assert O.verify(p, "wide_fibonacci", log_n, n_cols=30)


@pytest.mark.parametrize("air,log_n", [("wide_fibonacci", 7), ("poseidon", 6)])
def test_poseidon252_channel_gpu_proofs_accepted(G, air, log_n):
    if air == "poseidon":
        p = G.prove_poseidon(log_n, seed=6, input_mode=1, merkle_channel="poseidon252")
        cs = O.poseidon_claimed_sum(p, log_n, seed=6, input_mode=1, merkle_channel="poseidon252")
    else:
        p = G.prove_wide_fibonacci(log_n, 9, seed=6, input_mode=1, merkle_channel="poseidon252")
        cs = None
    assert O.verify(p, air, log_n, n_cols=9, claimed_sum=cs, merkle_channel="poseidon252")


def test_wide_fibonacci_benchmark_gpu_proof_accepted(G):
    """Wide-Fibonacci 2^16 rows x 100 columns, seeded: the reference's
    protocol unchanged, accepted by its verification rule."""
    p = G.prove_wide_fibonacci(16, 100, seed=0, input_mode=1)
    assert O.verify(p, "wide_fibonacci", 16, n_cols=100, split_log=1, config=(10, 1, 0, 70, 1))


@pytest.mark.slow
def test_poseidon_benchmark_gpu_proof_accepted_and_tamper_rejected(G):
    """The benchmarked Poseidon2 2^18 proof is accepted; flipping one bit in
    any of its sections makes the verifier reject it."""
    log_n = 18
    p = G.prove_poseidon(log_n, seed=0, input_mode=1)
    cs = O.poseidon_claimed_sum(p, log_n, seed=0, input_mode=1)
    kw = dict(split_log=2, claimed_sum=cs, config=(10, 1, 0, 70, 1))
    assert O.verify(p, "poseidon", log_n, **kw)
    n = 0
    for name, s, e in sections(p):
        if name.startswith("config"):
            continue
        for off in (s, s + ((e - s) // 2) // 4 * 4, e - 4):
            with pytest.raises(O.VerificationError):
                O.verify(flip(p, off), "poseidon", log_n, **kw)
            n += 1
    assert n >= 60


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_high_pow_bits_gpu_proofs_accepted(G, seed):
    """pow_bits 22: the device's first chunk of nonces (below 2^20, searched
    right after the FRI layers) holds a hit with probability about 0.22, so
    these seeds take both the device nonce and the host-driven search of the
    next chunks. Either way the proof is accepted; a nonce below 2^20 is the
    smallest passing one, so the whole proof equals the oracle's."""
    cfg = G.pcs_config(pow_bits=22, n_queries=5)
    p = G.prove_wide_fibonacci(7, 12, seed=seed, input_mode=1, config=cfg)
    assert O.verify(p, "wide_fibonacci", 7, n_cols=12, config=(22, 1, 0, 5, 1))
    (s, _), = [(s, e) for name, s, e in sections(p) if name == "proof_of_work"]
    nonce = int.from_bytes(p[s:s + 8], "little")
    if nonce < (1 << 20):
        assert p == O.prove("wide_fibonacci", 7, n_cols=12, seed=seed, input_mode=1, pow_bits=22, n_queries=5)
    else:
        assert nonce >> 32 >= 1 and (nonce & 0xFFFFFFFF) < (1 << 20)
