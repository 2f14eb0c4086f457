"""Served/batched proving: every job's proof is identical alone and in the mix,
under a tight HBM budget (admission control) and with several workers."""
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def mods():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpustark import prove, serve
    return prove, serve


JOBS = [(0, 10, 100, 1), (1, 8, 0, 2), (0, 12, 40, 3), (1, 10, 0, 4), (0, 9, 16, 5), (1, 12, 0, 6),
        (0, 14, 100, 7), (1, 6, 0, 8)]


def alone(prove, air, log_n, cols, seed):
    if air == 0:
        return prove.prove_wide_fibonacci(log_n, cols, seed=seed, input_mode=prove.INPUT_SEEDED)
    return prove.prove_poseidon(log_n, seed=seed, input_mode=prove.INPUT_SEEDED)


@pytest.mark.parametrize("workers,budget", [(4, 64 << 30), (3, 1 << 20)])
def test_served_results_match_single_proofs(mods, workers, budget):
    prove, serve = mods
    with serve.ProofServer(workers, budget) as sv:
        ids = [sv.submit(a, n, c or 100, s) for a, n, c, s in JOBS]
        got = [sv.wait(i) for i in ids]
    for (a, n, c, s), (proof, lat) in zip(JOBS, got):
        assert proof == alone(prove, a, n, c or 100, s)
        assert lat > 0


def test_server_reports_errors(mods):
    prove, serve = mods
    with serve.ProofServer(2) as sv:
        bad = sv.submit(serve.POSEIDON, 6, composition_log_split=1)
        good = sv.submit(serve.WIDE_FIBONACCI, 6, 10, 1)
        with pytest.raises(prove.ConstraintsNotSatisfied):
            sv.wait(bad)
        assert sv.wait(good)[0] == alone(prove, 0, 6, 10, 1)


def test_served_poseidon252_jobs_match_single_proofs(mods):
    """Poseidon252-channel jobs mixed with Blake2s ones: each job's proof is
    the one proved alone over its channel."""
    prove, serve = mods
    jobs = [(0, 8, 20, 1, "poseidon252"), (1, 6, 0, 2, "poseidon252"), (0, 9, 30, 3, "blake2s"),
            (0, 10, 100, 4, "poseidon252")]
    with serve.ProofServer(3) as sv:
        ids = [sv.submit(a, n, c or 100, s, merkle_channel=mc) for a, n, c, s, mc in jobs]
        got = [sv.wait(i)[0] for i in ids]
    for (a, n, c, s, mc), proof in zip(jobs, got):
        if a == 0:
            want = prove.prove_wide_fibonacci(n, c, seed=s, input_mode=prove.INPUT_SEEDED, merkle_channel=mc)
        else:
            want = prove.prove_poseidon(n, seed=s, input_mode=prove.INPUT_SEEDED, merkle_channel=mc)
        assert proof == want


@pytest.mark.parametrize("threads,fibers,budget", [(1, 8, 64 << 30), (2, 6, 64 << 30), (2, 4, 1 << 20)])
def test_fiber_server_results_match_single_proofs(mods, threads, fibers, budget):
    """Fiber mode: several proofs per host thread, each waiting by yielding
    to the others; every proof is the one proved alone, also when the
    budget admits one job at a time."""
    prove, serve = mods
    with serve.ProofServer(threads, budget, fibers_per_worker=fibers) as sv:
        ids = [sv.submit(a, n, c or 100, s) for a, n, c, s in JOBS * 2]
        got = [sv.wait(i) for i in ids]
    for (a, n, c, s), (proof, lat) in zip(JOBS * 2, got):
        assert proof == alone(prove, a, n, c or 100, s)
        assert lat > 0


def test_fiber_server_mixed_channels_and_errors(mods):
    prove, serve = mods
    with serve.ProofServer(1, fibers_per_worker=4) as sv:
        bad = sv.submit(serve.POSEIDON, 6, composition_log_split=1)
        ids = [sv.submit(0, 8, 20, 1, merkle_channel="poseidon252"), sv.submit(1, 6, 0, 2),
               sv.submit(0, 9, 30, 3, merkle_channel="poseidon252")]
        with pytest.raises(prove.ConstraintsNotSatisfied):
            sv.wait(bad)
        got = [sv.wait(i)[0] for i in ids]
    assert got[0] == prove.prove_wide_fibonacci(8, 20, seed=1, input_mode=prove.INPUT_SEEDED,
                                                merkle_channel="poseidon252")
    assert got[1] == alone(prove, 1, 6, 0, 2)
    assert got[2] == prove.prove_wide_fibonacci(9, 30, seed=3, input_mode=prove.INPUT_SEEDED,
                                                merkle_channel="poseidon252")
