"""Multi-GPU mode is independent replicas (every rank proves its own proof; no
collective on the data path). This checks, with 2 gloo ranks on the CPU, the
host-side plumbing bench.py uses for N > 1: rendezvous, barrier, max-over-ranks
timing, and that per-rank work is independent (ranks with the same seed
produce identical proofs, different seeds different ones)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import bench
    import pyoracle as O
    import torch.distributed as dist

    class A:
        pass

    w, r, _ = bench.dist_setup(A(), "gloo")
    assert (w, r) == (world, rank)
    bench.barrier(w)
    proof_same = O.prove("wide_fibonacci", 6, n_cols=12, seed=7, input_mode=1)
    proof_own = O.prove("wide_fibonacci", 6, n_cols=12, seed=100 + rank, input_mode=1)
    t = bench.max_over_ranks(float(rank + 1), w)
    gathered = [None] * world
    dist.all_gather_object(gathered, (proof_same, proof_own))
    if rank == 0:
        out.put((t, gathered))
    bench.barrier(w)
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    t, gathered = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert t == 2.0  # max over ranks
    (s0, o0), (s1, o1) = gathered
    assert s0 == s1 and o0 != o1
