"""The verifier (oracle/verifier.h, a restatement of the reference's
core/verifier.rs, core/pcs/verifier.rs, core/fri.rs and core/vcs/verifier.rs)
on the CPU oracle's proofs: honest proofs are accepted, and a proof with one
flipped bit in any section, a truncated or extended proof, or a proof checked
against another statement is rejected. The GPU prover's proofs go through
the same verifier in test_gpu_verify.py."""
import numpy as np
import pytest

import pyoracle as O
from proof_layout import flip, sections


def wf(log_n, n_cols=8, **kw):
    return O.prove("wide_fibonacci", log_n, n_cols=n_cols, **kw)


@pytest.mark.parametrize("log_n,n_cols,mode", [(4, 3, 0), (5, 8, 1), (8, 100, 0), (10, 37, 1)])
def test_wide_fibonacci_proofs_accepted(log_n, n_cols, mode):
    """COMPOSITION_LOG_SPLIT = 1, the reference's verifier unchanged."""
    p = wf(log_n, n_cols, seed=7, input_mode=mode)
    assert O.verify(p, "wide_fibonacci", log_n, n_cols=n_cols, split_log=1, config=(10, 1, 0, 70, 1))


@pytest.mark.parametrize("blowup,queries,pow_bits,last", [(2, 20, 4, 0), (1, 3, 10, 0), (3, 9, 0, 1), (1, 30, 2, 2)])
def test_pcs_configs_accepted(blowup, queries, pow_bits, last):
    p = wf(9, 20, seed=3, input_mode=1, pow_bits=pow_bits, n_queries=queries, log_blowup=blowup,
           log_last_layer=last)
    assert O.verify(p, "wide_fibonacci", 9, n_cols=20, config=(pow_bits, blowup, last, queries, 1))


@pytest.mark.parametrize("log_n,mode", [(4, 0), (6, 1), (8, 0)])
def test_poseidon_proofs_accepted(log_n, mode):
    """Composition split 2 (4 parts): the verifier generalised in the split only."""
    p = O.prove("poseidon", log_n, seed=5, input_mode=mode)
    cs = O.poseidon_claimed_sum(p, log_n, seed=5, input_mode=mode)
    assert O.verify(p, "poseidon", log_n, split_log=2, claimed_sum=cs)


@pytest.mark.parametrize("air,log_n", [("wide_fibonacci", 5), ("poseidon", 5)])
def test_poseidon252_channel_proofs_accepted(air, log_n):
    p = O.prove(air, log_n, n_cols=12, seed=2, input_mode=1, merkle_channel="poseidon252")
    cs = O.poseidon_claimed_sum(p, log_n, seed=2, input_mode=1, merkle_channel="poseidon252") \
        if air == "poseidon" else None
    assert O.verify(p, air, log_n, n_cols=12, claimed_sum=cs, merkle_channel="poseidon252")
    with pytest.raises(O.VerificationError):  # the same bytes read as a Blake2s-channel proof
        O.verify(p, air, log_n, n_cols=12, claimed_sum=cs)


def test_wide_fibonacci_benchmark_size_accepted():
    """2^16 rows x 100 columns, seeded inputs: the benchmark configuration."""
    p = wf(16, 100, seed=0, input_mode=1)
    assert O.verify(p, "wide_fibonacci", 16, n_cols=100, config=(10, 1, 0, 70, 1))


def _tamper_cases(proof):
    """One flipped bit in the middle of every section (the low bit of a
    field word, so values stay canonical in almost every case)."""
    for name, s, e in sections(proof):
        if name.startswith("config"):
            continue  # the verifier takes its PcsConfig from the caller, as the reference does
        mid = s + ((e - s) // 2) // 4 * 4
        yield name, flip(proof, mid)


@pytest.mark.parametrize("air,channel", [("wide_fibonacci", "blake2s"), ("poseidon", "blake2s"),
                                         ("wide_fibonacci", "poseidon252")])
def test_tampered_sections_rejected(air, channel):
    log_n = 6
    p = O.prove(air, log_n, n_cols=10, seed=9, input_mode=1, merkle_channel=channel, log_last_layer=1,
                n_queries=20)
    cs = O.poseidon_claimed_sum(p, log_n, seed=9, input_mode=1, merkle_channel=channel) if air == "poseidon" else None
    kw = dict(n_cols=10, claimed_sum=cs, merkle_channel=channel, config=(10, 1, 1, 20, 1))
    assert O.verify(p, air, log_n, **kw)
    names = [n for n, _, _ in sections(p)]
    for required in ("commitments", "sampled_values[1]", "decommitments[1].hash_witness", "queried_values[1]",
                     "proof_of_work", "fri.first.fri_witness", "fri.first.decommitment.hash_witness",
                     "fri.first.commitment", "fri.inner[0].commitment", "fri.last_layer_poly"):
        assert required in names, required
    n_cases = 0
    for name, bad in _tamper_cases(p):
        with pytest.raises(O.VerificationError):
            O.verify(bad, air, log_n, **kw)
        n_cases += 1
    assert n_cases >= 15


def test_every_byte_of_a_small_proof():
    """Every bit-0 flip of a small proof's payload is rejected."""
    log_n = 4
    p = wf(log_n, 4, seed=1, input_mode=1, n_queries=4, pow_bits=2)
    kw = dict(n_cols=4, config=(2, 1, 0, 4, 1))
    assert O.verify(p, "wide_fibonacci", log_n, **kw)
    checked = 0
    for name, s, e in sections(p):
        if name.startswith("config"):
            continue
        for off in range(s, e):
            with pytest.raises(O.VerificationError):
                O.verify(flip(p, off), "wide_fibonacci", log_n, **kw)
            checked += 1
    assert checked > 1000


def test_structure_errors():
    p = wf(5, 6, seed=2)
    kw = dict(n_cols=6, config=(10, 1, 0, 70, 1))
    assert O.verify(p, "wide_fibonacci", 5, **kw)
    for bad in (p[:-1], p + b"\0", p[: len(p) // 2], b""):
        with pytest.raises(O.VerificationError) as e:
            O.verify(bad, "wide_fibonacci", 5, **kw)
        assert e.value.kind == "InvalidStructure"


def test_wrong_statement_rejected():
    p = wf(6, 10, seed=4, input_mode=1)
    assert O.verify(p, "wide_fibonacci", 6, n_cols=10)
    for kw in (dict(n_cols=11), dict(n_cols=9), dict(n_cols=10, split_log=2)):
        with pytest.raises(O.VerificationError):
            O.verify(p, "wide_fibonacci", 6, **kw)
    with pytest.raises(O.VerificationError):
        O.verify(p, "wide_fibonacci", 7, n_cols=10)
    with pytest.raises(O.VerificationError):  # another PcsConfig
        O.verify(p, "wide_fibonacci", 6, n_cols=10, config=(10, 1, 0, 69, 1))


def test_wrong_claimed_sum_rejected():
    log_n = 5
    p = O.prove("poseidon", log_n, seed=8, input_mode=1)
    cs = O.poseidon_claimed_sum(p, log_n, seed=8, input_mode=1)
    assert O.verify(p, "poseidon", log_n, claimed_sum=cs)
    bad = cs.copy()
    bad[0] = (int(bad[0]) + 1) % O.P
    with pytest.raises(O.VerificationError) as e:
        O.verify(p, "poseidon", log_n, claimed_sum=bad)
    assert e.value.kind == "OodsNotMatching"
    # the claimed sum of another trace (the reference's input rule)
    other = O.poseidon_claimed_sum(p, log_n, input_mode=0)
    with pytest.raises(O.VerificationError):
        O.verify(p, "poseidon", log_n, claimed_sum=other)


def test_proof_from_another_seed_rejected():
    a = wf(6, 10, seed=1, input_mode=1)
    b = wf(6, 10, seed=2, input_mode=1)
    # splice b's queried values into a: the roots no longer match
    sa, sb = dict((n, (s, e)) for n, s, e in sections(a)), dict((n, (s, e)) for n, s, e in sections(b))
    s1, e1 = sa["queried_values[1]"]
    s2, e2 = sb["queried_values[1]"]
    k = min(e1 - s1, e2 - s2, 40)  # the two proofs query different rows: splice an equal-length prefix
    spliced = a[:s1] + b[s2:s2 + k] + a[s1 + k:]
    with pytest.raises(O.VerificationError) as e:
        O.verify(spliced, "wide_fibonacci", 6, n_cols=10)
    assert e.value.kind == "Merkle"
