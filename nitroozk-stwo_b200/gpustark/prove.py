"""Full proofs of the two benchmark components on the GPU prover (C ABI
gs_prove_wide_fibonacci / gs_prove_poseidon, and their Poseidon252MerkleChannel
forms gs_prove_wide_fibonacci_poseidon252 / gs_prove_poseidon_poseidon252).

Mirrors the reference's example drivers cuda_prove_wide_fibonacci
(crates/examples/src/wide_fibonacci/mod.rs:140-184), cuda_prove_poseidon
(crates/examples/src/poseidon/mod.rs:617-700), cuda_prove_wide_fibonacci_poseidon
(wide_fibonacci/mod.rs:335-379) and cuda_prove_poseidon_poseidon
(poseidon/mod.rs:702-785), which build the trace and call the generic
prove(); the result is the serialised StarkProof.
"""
import ctypes as C
import threading

import numpy as np

from . import _lib as L
from .backend import default_context

INPUT_REFERENCE, INPUT_SEEDED, INPUT_HOST = 0, 1, 2
GS_ERR_PROOF = 5
MERKLE_CHANNELS = ("blake2s", "poseidon252")


class ConstraintsNotSatisfied(L.GpuStarkError):
    """prove_ex's composition sanity check failed (ProvingError::ConstraintsNotSatisfied)."""


def pcs_config(pow_bits=10, log_blowup=1, log_last_layer=0, n_queries=70, line_fold_step=1):
    """PcsConfig { pow_bits, FriConfig::new(log_last_layer, log_blowup, n_queries, line_fold_step) }."""
    return L.PcsConfig(pow_bits, log_blowup, log_last_layer, n_queries, line_fold_step)


_DEFAULT_CONFIG = pcs_config()  # read-only for the prover; shared by calls without a config


_tls = threading.local()


def _buffer(capacity):
    """Per-thread output buffer, reused across proofs (a fresh multi-MB buffer
    per call would cost its page faults every time), with its address."""
    buf = getattr(_tls, "buf", None)
    if buf is None or len(buf) < capacity:
        buf = (C.c_uint8 * capacity)()
        _tls.buf = buf
        _tls.addr = C.addressof(buf)
    return buf, _tls.addr


def _run(fn, args, ctx, capacity):
    n = C.c_size_t()
    buf, addr = _buffer(capacity)
    capacity = len(buf)
    st = fn(*args, addr, capacity, C.byref(n))
    if st == 1 and n.value > capacity:  # retry with the exact size
        buf, addr = _buffer(n.value)
        st = fn(*args, addr, len(buf), C.byref(n))
    if st == GS_ERR_PROOF:
        raise ConstraintsNotSatisfied(L.lib().gs_last_error().decode())
    L.check(st, fn.__name__)
    return C.string_at(buf, n.value)


def _inputs(host_inputs):
    if host_inputs is None:
        return None, None
    a = np.ascontiguousarray(host_inputs, dtype=np.uint32)
    return a, a.ctypes.data_as(L.U32P)


def _entry(name, merkle_channel):
    if merkle_channel not in MERKLE_CHANNELS:
        raise ValueError(f"merkle_channel must be one of {MERKLE_CHANNELS}")
    return getattr(L.lib(), name + ("_poseidon252" if merkle_channel == "poseidon252" else ""))


def prove_wide_fibonacci(log_n_rows, n_columns=100, seed=0, input_mode=INPUT_REFERENCE, host_inputs=None,
                         config=None, ctx=None, capacity=1 << 21, merkle_channel="blake2s"):
    """host_inputs (INPUT_HOST): array (2, 2^log_n_rows) of columns 0 and 1.
    merkle_channel: 'blake2s' (Blake2sMerkleChannel) or 'poseidon252'."""
    ctx = ctx or default_context()
    keep, ptr = _inputs(host_inputs)
    cfg = config or _DEFAULT_CONFIG
    return _run(_entry("gs_prove_wide_fibonacci", merkle_channel),
                (ctx.handle, log_n_rows, n_columns, seed, input_mode, ptr, C.byref(cfg)), ctx, capacity)


def prove_poseidon(log_n_instances, seed=0, input_mode=INPUT_REFERENCE, host_inputs=None, composition_log_split=2,
                   config=None, ctx=None, capacity=1 << 21, merkle_channel="blake2s"):
    """host_inputs (INPUT_HOST): array (16, 2^log_n_instances) of initial states.
    merkle_channel: 'blake2s' (Blake2sMerkleChannel) or 'poseidon252'."""
    ctx = ctx or default_context()
    keep, ptr = _inputs(host_inputs)
    cfg = config or _DEFAULT_CONFIG
    return _run(_entry("gs_prove_poseidon", merkle_channel),
                (ctx.handle, log_n_instances, seed, input_mode, ptr, composition_log_split, C.byref(cfg)), ctx,
                capacity)
