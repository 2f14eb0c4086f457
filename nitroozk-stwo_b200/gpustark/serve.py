"""Continuous-batching proof server over the C ABI (gs_server_*).

Jobs of different sizes are submitted as they arrive; worker threads (one
CUDA stream each) prove them concurrently, admitting a job when the device
footprint of the jobs in flight plus its own fits the HBM budget. A job's
proof is the same bytes as proving it alone (gpustark.prove).
"""
import ctypes as C

from . import _lib as L
from .prove import ConstraintsNotSatisfied, GS_ERR_PROOF, pcs_config

WIDE_FIBONACCI, POSEIDON = 0, 1


class ProofServer:
    def __init__(self, n_workers=4, hbm_budget_bytes=64 << 30, fibers_per_worker=1):
        """n_workers host threads; fibers_per_worker > 1 runs that many proofs
        per thread as cooperative fibers (gs_server_create_fibers)."""
        h = C.c_void_p()
        L.check(L.lib().gs_server_create_fibers(n_workers, fibers_per_worker, hbm_budget_bytes, C.byref(h)),
                "gs_server_create_fibers")
        self.handle = h

    def submit(self, air, log_n, n_columns=100, seed=0, composition_log_split=None, config=None,
               merkle_channel="blake2s"):
        """air: WIDE_FIBONACCI or POSEIDON; merkle_channel: 'blake2s' or
        'poseidon252'; returns a job id."""
        if composition_log_split is None:
            composition_log_split = 1 if air == WIDE_FIBONACCI else 2
        if merkle_channel not in ("blake2s", "poseidon252"):
            raise ValueError("merkle_channel must be 'blake2s' or 'poseidon252'")
        fn = L.lib().gs_server_submit_poseidon252 if merkle_channel == "poseidon252" else L.lib().gs_server_submit
        cfg = config or pcs_config()
        jid = C.c_uint64()
        L.check(fn(self.handle, air, log_n, n_columns, seed, composition_log_split, C.byref(cfg), C.byref(jid)),
                fn.__name__)
        return jid.value

    def wait(self, job_id, capacity=1 << 20):
        """Blocks until the job is done; returns (proof bytes, submit-to-done latency in ms)."""
        n = C.c_size_t()
        lat = C.c_double()
        buf = (C.c_uint8 * capacity)()
        st = L.lib().gs_server_wait(self.handle, job_id, C.cast(buf, C.c_void_p), capacity, C.byref(n), C.byref(lat))
        if st == 1 and n.value > capacity:
            buf = (C.c_uint8 * n.value)()
            st = L.lib().gs_server_wait(self.handle, job_id, C.cast(buf, C.c_void_p), n.value, C.byref(n),
                                        C.byref(lat))
        if st == GS_ERR_PROOF:
            raise ConstraintsNotSatisfied(L.lib().gs_last_error().decode())
        L.check(st, "gs_server_wait")
        return C.string_at(buf, n.value), lat.value

    def close(self):
        if self.handle:
            L.lib().gs_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
