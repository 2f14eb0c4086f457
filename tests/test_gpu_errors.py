"""Error paths reached from the host, none of which faults the GPU: a device
allocation the pool cannot satisfy maps to GS_ERR_OOM and leaves the context
usable; the proof-of-work search bound maps to GS_ERR_TIMEOUT (the bound set
low with the GS_GRIND_MAX_HI switch, in a child process); proof-server jobs
are validated at submission like direct proofs; a server destroyed with
queued jobs drains them within its HBM budget; the legacy Merkle path (in a
child process) gives the oracle's proofs."""
import ctypes as C
import hashlib
import os
import subprocess
import sys

import pytest

import pyoracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GS_ERR_INVALID, GS_ERR_OOM, GS_ERR_TIMEOUT = 1, 3, 6  # include/gpustark.h


@pytest.fixture(scope="module")
def G():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpustark import prove
    return prove


def test_oversized_allocation_is_oom_and_context_survives(G):
    from gpustark import _lib as L
    from gpustark.backend import default_context
    ctx = default_context()
    p = C.c_void_p()
    assert L.lib().gs_malloc(ctx.handle, 1 << 50, C.byref(p)) == GS_ERR_OOM
    assert b"alloc" in L.lib().gs_last_error().lower()
    # the same context proves afterwards, byte-identical to the oracle
    assert G.prove_wide_fibonacci(6, 10, seed=2, input_mode=1) == \
        O.prove("wide_fibonacci", 6, n_cols=10, seed=2, input_mode=1)


CHILD = r"""
import sys, hashlib
sys.path[:0] = [{pkg!r}]
from gpustark.backend import GpuBackend as B
from gpustark import GpuStarkError
digest = hashlib.blake2s(b"no-nonce-0", digest_size=32).digest()
try:
    B.grind(digest, 32)
    print("no error")
except GpuStarkError as e:
    print("error:", e)
print("after:", B.grind(digest, 4))
"""


def test_grind_search_bound_is_timeout():
    """With one high word searched, a 32-bit proof of work whose first 2^20
    nonces hold no hit (checked on the host for this digest) ends with
    GS_ERR_TIMEOUT; the next grind on the same context succeeds."""
    digest = hashlib.blake2s(b"no-nonce-0", digest_size=32).digest()
    env = dict(os.environ, GS_GRIND_MAX_HI="1")
    out = subprocess.run([sys.executable, "-c", CHILD.format(pkg=os.path.join(ROOT, "nitroozk-stwo_b200"))],
                         env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert f"status {GS_ERR_TIMEOUT}" in out.stdout and "search bound" in out.stdout, out.stdout
    nonce = int(out.stdout.split("after:")[1])
    assert O.verify_pow(digest, 4, nonce)


LEGACY_CHILD = r"""
import sys
sys.path[:0] = [{pkg!r}, {oracle!r}]
from gpustark import prove as G
import pyoracle as O
ok = all(G.prove_wide_fibonacci(n, 9, seed=4, input_mode=1) == O.prove("wide_fibonacci", n, n_cols=9, seed=4,
                                                                        input_mode=1) for n in (5, 9))
print("match" if ok else "differ")
"""


def test_legacy_merkle_path_proofs_match():
    """GS_MERKLE_LEGACY=1 (per-layer launches and a cluster tail instead of
    the one-launch tree kernel; read once per process, hence a child): the
    roots reach the host by a copy into the mailbox, and the proofs equal
    the oracle's."""
    env = dict(os.environ, GS_MERKLE_LEGACY="1")
    code = LEGACY_CHILD.format(pkg=os.path.join(ROOT, "nitroozk-stwo_b200"), oracle=os.path.join(ROOT, "oracle"))
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "match" in out.stdout, out.stdout


def test_server_validates_jobs_at_submission(G):
    from gpustark import GpuStarkError
    from gpustark.serve import POSEIDON, WIDE_FIBONACCI, ProofServer
    with ProofServer(n_workers=2) as s:
        bad = [
            dict(air=WIDE_FIBONACCI, log_n=6, n_columns=2),
            dict(air=WIDE_FIBONACCI, log_n=6, n_columns=161),
            dict(air=2, log_n=6),
            dict(air=WIDE_FIBONACCI, log_n=6, config=G.pcs_config(pow_bits=40)),
            dict(air=WIDE_FIBONACCI, log_n=6, config=G.pcs_config(n_queries=0)),
            dict(air=POSEIDON, log_n=6, config=G.pcs_config(log_last_layer=11)),
            dict(air=POSEIDON, log_n=6, config=G.pcs_config(pow_bits=100), merkle_channel="poseidon252"),
        ]
        for kw in bad:
            with pytest.raises(GpuStarkError, match=f"status {GS_ERR_INVALID}"):
                s.submit(**kw)
        j = s.submit(WIDE_FIBONACCI, 6, n_columns=10, seed=2)
        proof, _ = s.wait(j)
        assert proof == O.prove("wide_fibonacci", 6, n_cols=10, seed=2, input_mode=1)


def test_server_drains_queue_within_budget_at_shutdown():
    """Jobs still queued when the server is destroyed are proven one
    footprint at a time (a 1-byte budget admits a job only when nothing else
    is in flight) and the destroy returns."""
    from gpustark.serve import POSEIDON, WIDE_FIBONACCI, ProofServer
    s = ProofServer(n_workers=4, hbm_budget_bytes=1)
    for i in range(6):
        s.submit(WIDE_FIBONACCI if i % 2 else POSEIDON, 8, n_columns=20, seed=i)
    s.close()
