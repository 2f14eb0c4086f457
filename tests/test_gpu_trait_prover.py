"""A whole Wide-Fibonacci proof through the per-trait C-ABI entry points only
(tests/trait_prover.py: the reference's generic prover on the host, each
device step one backend-trait call) equals the fused prover's bytes
(gs_prove_wide_fibonacci) on the same inputs and PcsConfig, and the verifier
accepts it. With -s the test prints both provers' wall times."""
import time

import numpy as np
import pytest

import pyoracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def env():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpustark import prove as G
    from gpustark.backend import GpuBackend
    from trait_prover import TraitProver
    return G, TraitProver(GpuBackend)


CASES = [
    (4, 3, (10, 1, 0, 70)),
    (6, 16, (10, 1, 0, 70)),
    (8, 100, (4, 2, 0, 20)),
    (9, 20, (0, 3, 1, 9)),
    (10, 100, (10, 1, 0, 70)),
    (12, 37, (2, 1, 2, 30)),
    (16, 100, (10, 1, 0, 70)),
]


@pytest.mark.parametrize("log_n,n_cols,cfg", CASES)
def test_trait_driven_proof_equals_fused_prover(env, log_n, n_cols, cfg):
    G, T = env
    pow_bits, blowup, last, queries = cfg
    rng = np.random.default_rng(1000 + log_n)
    a, b = (rng.integers(0, O.P, 1 << log_n, dtype=np.int64).astype(np.uint32) for _ in range(2))
    got = T.prove_wide_fibonacci(a, b, n_cols, pow_bits=pow_bits, log_blowup=blowup, log_last_layer=last,
                                 n_queries=queries)
    conf = G.pcs_config(pow_bits=pow_bits, log_blowup=blowup, log_last_layer=last, n_queries=queries)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    want = G.prove_wide_fibonacci(log_n, n_cols, input_mode=G.INPUT_HOST, host_inputs=np.stack([a, b]), config=conf)
    fused_s = time.perf_counter() - t0
    assert got == want
    assert O.verify(got, "wide_fibonacci", log_n, n_cols=n_cols, config=(pow_bits, blowup, last, queries, 1))
    print(f"\n2^{log_n} x {n_cols}: trait-driven {T.elapsed_s * 1e3:.1f} ms ({T.calls} trait calls so far), "
          f"fused {fused_s * 1e3:.2f} ms")
