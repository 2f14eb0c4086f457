"""ORACLE — test infrastructure only.

ctypes binding of the CPU restatement in this folder (``_build/liboracle.so``).
Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
it; the product path never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

P = (1 << 31) - 1


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE, "-j8"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


U32P = C.POINTER(C.c_uint32)
U8P = C.POINTER(C.c_uint8)
PP = C.POINTER(U32P)


def _declare(L):
    def f(name, res, *args):
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = list(args)

    f("oracle_set_threads", None, C.c_int)
    f("oracle_barycentric_weights", None, C.c_uint32, U32P, PP)
    f("oracle_barycentric_eval", None, U32P, PP, C.c_uint32, U32P)
    f("oracle_secure_powers", None, U32P, C.c_size_t, PP)
    f("oracle_constraint_quotients", None, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, PP, PP, U32P, C.c_uint32,
      U32P, U32P, U32P, U32P, PP)
    f("oracle_verify", C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, U32P, C.c_uint32, U32P, U8P,
      C.c_size_t, C.c_char_p, C.c_size_t)
    f("oracle_verify_lookup_elements", C.c_int, C.c_uint32, U8P, C.c_size_t, U32P, U32P)
    f("oracle_poseidon_claimed_sum", None, C.c_uint32, C.c_uint64, C.c_uint32, U32P, U32P, U32P, U32P)
    f("oracle_max_threads", C.c_int)
    f("oracle_m31_reduce", C.c_uint32, C.c_uint64)
    f("oracle_m31_partial_reduce", C.c_uint32, C.c_uint32)
    f("oracle_m31_mul", C.c_uint32, C.c_uint32, C.c_uint32)
    f("oracle_m31_inv", C.c_uint32, C.c_uint32)
    f("oracle_qm31_mul", None, U32P, U32P, U32P)
    f("oracle_qm31_inv", None, U32P, U32P)
    f("oracle_index_to_point", None, C.c_uint64, U32P)
    f("oracle_secure_gen_mul", None, C.c_uint64, C.c_uint64, U32P)
    f("oracle_blake2s", None, U8P, C.c_size_t, U8P)
    f("oracle_twiddles_half_odds", None, C.c_uint32, U32P, U32P)
    f("oracle_interpolate", None, U32P, C.c_uint32, C.c_uint32)
    f("oracle_interpolate_columns", None, PP, C.c_uint32, C.c_uint32, C.c_uint32)
    f("oracle_evaluate", None, U32P, C.c_size_t, C.c_uint32, C.c_uint32, U32P)
    f("oracle_evaluate_columns", None, PP, C.c_uint32, C.c_size_t, C.c_uint32, C.c_uint32, PP)
    f("oracle_bit_reverse", None, U32P, C.c_uint32)
    f("oracle_commit_on_layer", None, C.c_uint32, U8P, C.c_uint32, PP, U8P)
    f("oracle_merkle_root", None, C.c_uint32, PP, U32P, U8P)
    f("oracle_lifted_leaves", None, C.c_uint32, PP, U32P, C.c_uint32, U8P)
    f("oracle_channel_mix_u32s", None, U32P, C.c_size_t, U8P)
    f("oracle_channel_mix_u64", None, C.c_uint64, U8P)
    f("oracle_channel_draw_secure_felts", C.c_uint32, U8P, C.c_size_t, U32P)
    f("oracle_grind", C.c_uint64, U8P, C.c_uint32)
    f("oracle_verify_pow", C.c_int, U8P, C.c_uint32, C.c_uint64)
    f("oracle_fold_line", None, PP, C.c_uint32, U32P, PP)
    f("oracle_fold_circle_into_line", None, PP, PP, C.c_uint32, U32P)
    f("oracle_accumulate_numerators", None, C.c_uint32, C.c_uint32, PP, U32P, C.c_uint32, U32P, U32P, U32P, PP, U32P)
    f("oracle_compute_quotients_and_combine", None, C.c_uint32, PP, U32P, U32P, U32P, C.c_uint32, PP)
    f("oracle_lift_and_accumulate", None, C.c_uint32, PP, U32P, PP)
    f("oracle_eval_at_point", None, U32P, C.c_uint32, U32P, U32P)
    f("oracle_prove", C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32,
      C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t))
    f("oracle_p252_commit_on_layer", None, C.c_uint32, U8P, C.c_uint32, PP, U8P)
    f("oracle_p252_permute", None, U8P, C.c_size_t, U8P)
    f("oracle_p252_channel_op", C.c_uint32, U8P, C.c_uint32, C.c_uint32, U8P, C.c_uint64, U32P, C.c_size_t, U32P,
      U8P)
    f("oracle_p252_grind", C.c_uint64, U8P, C.c_uint32)
    f("oracle_p252_verify_pow", C.c_int, U8P, C.c_uint32, C.c_uint64)
    f("oracle_seeded_m31", C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64)


# ---------------------------------------------------------------- helpers
def u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(U32P)


def ptr_array(arrays):
    arr = (U32P * len(arrays))(*[a.ctypes.data_as(U32P) for a in arrays])
    return C.cast(arr, PP), arr


def planes(q):
    """(n,4) uint32 array -> list of 4 contiguous planes."""
    return [np.ascontiguousarray(q[:, i]) for i in range(4)]


def unplanes(ps):
    return np.stack(ps, axis=1)


def set_threads(n):
    lib().oracle_set_threads(n)


def max_threads():
    return lib().oracle_max_threads()


def blake2s(data: bytes) -> bytes:
    buf = (C.c_uint8 * max(len(data), 1)).from_buffer_copy(data or b"\0")
    out = (C.c_uint8 * 32)()
    lib().oracle_blake2s(buf, len(data), out)
    return bytes(out)


def twiddles_half_odds(log_size):
    n = 1 << log_size
    tw = np.zeros(n, np.uint32)
    itw = np.zeros(n, np.uint32)
    lib().oracle_twiddles_half_odds(log_size, tw.ctypes.data_as(U32P), itw.ctypes.data_as(U32P))
    return tw, itw


def interpolate(values, log_n, root_log=None):
    v = np.array(values, dtype=np.uint32)
    lib().oracle_interpolate(v.ctypes.data_as(U32P), log_n, root_log if root_log is not None else max(log_n - 1, 1))
    return v


def interpolate_columns(cols, log_n, root_log=None):
    cols = [np.array(c, dtype=np.uint32) for c in cols]
    pp, keep = ptr_array(cols)
    lib().oracle_interpolate_columns(pp, len(cols), log_n, root_log if root_log is not None else max(log_n - 1, 1))
    return cols


def evaluate(coeffs, log_n, root_log=None):
    c, cp = u32(coeffs)
    out = np.zeros(1 << log_n, np.uint32)
    lib().oracle_evaluate(cp, len(c), log_n, root_log if root_log is not None else max(log_n - 1, 1), out.ctypes.data_as(U32P))
    return out


def evaluate_columns(cols, log_n, root_log=None):
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    outs = [np.zeros(1 << log_n, np.uint32) for _ in cols]
    ip, k1 = ptr_array(cols)
    op, k2 = ptr_array(outs)
    lib().oracle_evaluate_columns(ip, len(cols), len(cols[0]), log_n,
                                  root_log if root_log is not None else max(log_n - 1, 1), op)
    return outs


def bit_reverse(values):
    v = np.array(values, dtype=np.uint32)
    lib().oracle_bit_reverse(v.ctypes.data_as(U32P), int(len(v)).bit_length() - 1)
    return v


def commit_on_layer(log_size, prev, cols):
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    out = np.zeros((1 << log_size) * 32, np.uint8)
    pp, keep = ptr_array(cols) if cols else (C.cast(None, PP), None)
    prev_p = None
    if prev is not None:
        prev = np.ascontiguousarray(prev, dtype=np.uint8)
        prev_p = prev.ctypes.data_as(U8P)
    lib().oracle_commit_on_layer(log_size, prev_p, len(cols), pp, out.ctypes.data_as(U8P))
    return out.reshape(-1, 32)


def merkle_root(cols):
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    logs = np.array([int(len(c)).bit_length() - 1 for c in cols], np.uint32)
    pp, keep = ptr_array(cols) if cols else (C.cast(None, PP), None)
    out = (C.c_uint8 * 32)()
    lib().oracle_merkle_root(len(cols), pp, logs.ctypes.data_as(U32P), out)
    return bytes(out)


def lifted_leaves(cols, lift):
    """MerkleOpsLifted::build_leaves: (2^lift, 32) leaf hashes ((1, 32) for no columns)."""
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    logs = np.array([int(len(c)).bit_length() - 1 for c in cols] or [0], np.uint32)
    pp, keep = ptr_array(cols) if cols else (C.cast(None, PP), None)
    n = (1 << lift) if cols else 1
    out = np.zeros(n * 32, np.uint8)
    lib().oracle_lifted_leaves(len(cols), pp, logs.ctypes.data_as(U32P), lift, out.ctypes.data_as(U8P))
    return out.reshape(-1, 32)


def channel_mix_u32s(words):
    w, wp = u32(words)
    out = (C.c_uint8 * 32)()
    lib().oracle_channel_mix_u32s(wp, len(w), out)
    return bytes(out)


def channel_mix_u64(v):
    out = (C.c_uint8 * 32)()
    lib().oracle_channel_mix_u64(v, out)
    return bytes(out)


def grind(digest: bytes, pow_bits):
    d = (C.c_uint8 * 32).from_buffer_copy(digest)
    return lib().oracle_grind(d, pow_bits)


def verify_pow(digest: bytes, pow_bits, nonce):
    d = (C.c_uint8 * 32).from_buffer_copy(digest)
    return bool(lib().oracle_verify_pow(d, pow_bits, nonce))


# ---- Poseidon252 (felt252 values as 32 big-endian bytes)
def p252_commit_on_layer(log_size, prev, cols):
    """MerkleOps<Poseidon252MerkleHasher>::commit_on_layer: (2^log_size, 32) bytes."""
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    out = np.zeros((1 << log_size) * 32, np.uint8)
    pp, keep = ptr_array(cols) if cols else (C.cast(None, PP), None)
    prev_p = None
    if prev is not None:
        prev = np.ascontiguousarray(prev, dtype=np.uint8)
        prev_p = prev.ctypes.data_as(U8P)
    lib().oracle_p252_commit_on_layer(log_size, prev_p, len(cols), pp, out.ctypes.data_as(U8P))
    return out.reshape(-1, 32)


def p252_permute(states_bytes: bytes):
    n = len(states_bytes) // 96
    src = (C.c_uint8 * len(states_bytes)).from_buffer_copy(states_bytes)
    out = (C.c_uint8 * (96 * n))()
    lib().oracle_p252_permute(src, n, out)
    return bytes(out)


P252_OPS = {"mix_root": 0, "mix_u64": 1, "mix_u32s": 2, "mix_felts": 3, "draw_secure_felts": 4, "draw_u32s": 5}


def p252_channel_op(digest: bytes, n_draws, op, data=b"", v=0, words=(), n=0):
    """One Poseidon252Channel operation from (digest, n_draws): returns
    (new digest bytes, new n_draws, output words)."""
    d = (C.c_uint8 * 32).from_buffer_copy(digest)
    b = (C.c_uint8 * 32).from_buffer_copy(data.ljust(32, b"\0")[:32])
    w, wp = u32(list(words) or [0])
    count = n if op in ("draw_secure_felts", "draw_u32s") else (len(words) // 4 if op == "mix_felts" else len(words))
    out = np.zeros(max(1, 7 * n, 4 * n), np.uint32)
    dout = (C.c_uint8 * 32)()
    nd = lib().oracle_p252_channel_op(d, n_draws, P252_OPS[op], b, v, wp, count, out.ctypes.data_as(U32P), dout)
    used = 4 * n if op == "draw_secure_felts" else (7 * n if op == "draw_u32s" else 0)
    return bytes(dout), nd, [int(x) for x in out[:used]]


def p252_grind(digest: bytes, pow_bits):
    d = (C.c_uint8 * 32).from_buffer_copy(digest)
    return lib().oracle_p252_grind(d, pow_bits)


def p252_verify_pow(digest: bytes, pow_bits, nonce):
    d = (C.c_uint8 * 32).from_buffer_copy(digest)
    return bool(lib().oracle_p252_verify_pow(d, pow_bits, nonce))


def fold_line(eval_q, log_n, alpha):
    ps = planes(eval_q)
    outs = [np.zeros(1 << (log_n - 1), np.uint32) for _ in range(4)]
    ip, k1 = ptr_array(ps)
    op, k2 = ptr_array(outs)
    a, ap = u32(alpha)
    lib().oracle_fold_line(ip, log_n, ap, op)
    return unplanes(outs)


def fold_circle_into_line(dst_q, src_q, log_n, alpha):
    dps = planes(dst_q)
    sps = planes(src_q)
    dp, k1 = ptr_array(dps)
    sp, k2 = ptr_array(sps)
    a, ap = u32(alpha)
    lib().oracle_fold_circle_into_line(dp, sp, log_n, ap)
    return unplanes(dps)


def accumulate_numerators(cols, log_size, point8, col_idx, values4, rand4):
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    pp, keep = ptr_array(cols)
    outs = [np.zeros(1 << log_size, np.uint32) for _ in range(4)]
    op, k2 = ptr_array(outs)
    flt = np.zeros(4, np.uint32)
    pt, ptp = u32(point8)
    ci, cip = u32(col_idx)
    v, vp = u32(np.asarray(values4).reshape(-1))
    r, rp = u32(np.asarray(rand4).reshape(-1))
    lib().oracle_accumulate_numerators(log_size, len(cols), pp, ptp, len(ci), cip, vp, rp, op, flt.ctypes.data_as(U32P))
    return unplanes(outs), flt


def compute_quotients_and_combine(partials, first_linear4, points8, lifting_log_size):
    all_planes = []
    logs = []
    for p in partials:
        all_planes += planes(p)
        logs.append(int(len(p)).bit_length() - 1)
    pp, keep = ptr_array(all_planes)
    lg, lgp = u32(logs)
    fl, flp = u32(np.asarray(first_linear4).reshape(-1))
    pt, ptp = u32(np.asarray(points8).reshape(-1))
    outs = [np.zeros(1 << lifting_log_size, np.uint32) for _ in range(4)]
    op, k2 = ptr_array(outs)
    lib().oracle_compute_quotients_and_combine(len(partials), pp, lgp, flp, ptp, lifting_log_size, op)
    return unplanes(outs)


def lift_and_accumulate(cols_q):
    all_planes = []
    logs = []
    for p in cols_q:
        all_planes += planes(p)
        logs.append(int(len(p)).bit_length() - 1)
    pp, keep = ptr_array(all_planes)
    lg, lgp = u32(logs)
    outs = [np.zeros(len(cols_q[-1]), np.uint32) for _ in range(4)]
    op, k2 = ptr_array(outs)
    lib().oracle_lift_and_accumulate(len(cols_q), pp, lgp, op)
    return unplanes(outs)


def eval_at_point(coeffs, point8):
    c, cp = u32(coeffs)
    pt, ptp = u32(point8)
    out = np.zeros(4, np.uint32)
    lib().oracle_eval_at_point(cp, int(len(c)).bit_length() - 1, ptp, out.ctypes.data_as(U32P))
    return out


class ConstraintsNotSatisfied(RuntimeError):
    """prove_ex's composition sanity check failed (the reference's ProvingError)."""


def default_split(air):
    """Composition split: 1 for wide fibonacci (the reference's), 2 = LOG_EXPAND for poseidon."""
    return 1 if air == "wide_fibonacci" else 2


def prove(air, log_n, n_cols=100, seed=0, input_mode=0, pow_bits=10, n_queries=70, log_blowup=1, split_log=None,
          log_last_layer=0, merkle_channel="blake2s"):
    """Full proof bytes from the CPU restatement; air: 'wide_fibonacci' | 'poseidon';
    merkle_channel: 'blake2s' | 'poseidon252'."""
    if split_log is None:
        split_log = default_split(air)
    L = lib()
    cap = 1 << 26
    buf = (C.c_uint8 * cap)()
    n = C.c_size_t()
    st = L.oracle_prove(0 if air == "wide_fibonacci" else 1, log_n, n_cols, seed, input_mode, pow_bits, n_queries,
                        log_blowup, log_last_layer, split_log, 1 if merkle_channel == "poseidon252" else 0,
                        C.cast(buf, C.c_void_p), cap, C.byref(n))
    if st == 1:
        raise ConstraintsNotSatisfied("composition OODS value does not match the constraints")
    if st != 0:
        raise RuntimeError(f"oracle prove failed with status {st}")
    return bytes(buf[: n.value])


def seeded_m31(seed, col, row):
    return lib().oracle_seeded_m31(seed, col, row)


# ------------------------------------------------------------------ verifier
VERIFY_ERRORS = {1: "InvalidStructure", 2: "Merkle", 3: "OodsNotMatching", 4: "Fri", 5: "ProofOfWork"}


class VerificationError(RuntimeError):
    """The verifier rejected the proof; ``kind`` is the reference's
    VerificationError variant (core/verifier.rs:124-139)."""

    def __init__(self, code, msg):
        self.kind = VERIFY_ERRORS.get(code, str(code))
        super().__init__(f"{self.kind}: {msg}")


def _bytes_ptr(data):
    buf = (C.c_uint8 * max(1, len(data))).from_buffer_copy(data if data else b"\0")
    return buf, C.cast(buf, U8P)


def poseidon_claimed_sum(proof, log_n, seed=0, input_mode=0, host_inputs=None, merkle_channel="blake2s"):
    """The logup claimed sum of the Poseidon2 trace the proof was made for
    (the statement the prover reports beside the proof): lookup elements
    drawn from the proof's first two commitments, then the sum over rows of
    1/combine(initial) - 1/combine(final)."""
    L = lib()
    buf, bp = _bytes_ptr(proof)
    z = np.zeros(4, np.uint32)
    a = np.zeros(4, np.uint32)
    if L.oracle_verify_lookup_elements(1 if merkle_channel == "poseidon252" else 0, bp, len(proof),
                                       z.ctypes.data_as(U32P), a.ctypes.data_as(U32P)):
        raise VerificationError(1, "proof bytes do not parse")
    out = np.zeros(4, np.uint32)
    hp = None
    if host_inputs is not None:
        h = np.ascontiguousarray(host_inputs, dtype=np.uint32)
        hp = h.ctypes.data_as(U32P)
    L.oracle_poseidon_claimed_sum(log_n, seed, input_mode, hp, z.ctypes.data_as(U32P), a.ctypes.data_as(U32P),
                                  out.ctypes.data_as(U32P))
    return out


def verify(proof, air, log_n, n_cols=100, split_log=None, claimed_sum=None, merkle_channel="blake2s", config=None):
    """Runs the verifier (verifier.h) on serialised proof bytes; returns True
    or raises VerificationError. Poseidon2 needs the claimed sum. config: the
    verifier's PcsConfig as (pow_bits, log_blowup, log_last_layer, n_queries,
    line_fold_step), or None to use the one serialised in the proof."""
    if split_log is None:
        split_log = default_split(air)
    L = lib()
    buf, bp = _bytes_ptr(proof)
    cs = None
    if claimed_sum is not None:
        c = np.ascontiguousarray(claimed_sum, dtype=np.uint32)
        cs = c.ctypes.data_as(U32P)
    cfg = None
    if config is not None:
        cw = np.array(config, np.uint32)
        cfg = cw.ctypes.data_as(U32P)
    msg = C.create_string_buffer(256)
    code = L.oracle_verify(0 if air == "wide_fibonacci" else 1, log_n, n_cols, split_log, cs,
                           1 if merkle_channel == "poseidon252" else 0, cfg, bp, len(proof), msg, 256)
    if code:
        raise VerificationError(code, msg.value.decode())
    return True


# ------------------------------------------------------- per-trait operations
def barycentric_weights(log_size, point8):
    """PolyOps::barycentric_weights(CanonicCoset(log_size), p): 4 planes."""
    out = [np.zeros(1 << log_size, np.uint32) for _ in range(4)]
    pt, ptp = u32(point8)
    pp, keep = ptr_array(out)
    lib().oracle_barycentric_weights(log_size, ptp, pp)
    return out


def barycentric_eval(evals, weights):
    e, ep = u32(evals)
    wp, keep = ptr_array([np.ascontiguousarray(w, np.uint32) for w in weights])
    out = np.zeros(4, np.uint32)
    lib().oracle_barycentric_eval(ep, wp, int(len(e)).bit_length() - 1, out.ctypes.data_as(U32P))
    return out


def secure_powers(felt4, n):
    out = [np.zeros(max(n, 1), np.uint32) for _ in range(4)]
    f, fp = u32(felt4)
    pp, keep = ptr_array(out)
    lib().oracle_secure_powers(fp, n, pp)
    return [o[:n] for o in out]


def constraint_quotients(air, trace, inter, trace_log, eval_log, powers, denom_inv, z=None, alpha=None, shift=None,
                         n_cols=None):
    """Constraint quotients over the evaluation domain (component_prover.rs:177-245):
    row_res * denom_inv[row >> trace_log]; powers: (n_constraints, 4) words."""
    n = 1 << eval_log
    out = [np.zeros(n, np.uint32) for _ in range(4)]
    tp, keep_t = ptr_array([np.ascontiguousarray(c, np.uint32) for c in trace])
    ip, keep_i = ptr_array([np.ascontiguousarray(c, np.uint32) for c in inter] or [np.zeros(1, np.uint32)])
    pw = np.ascontiguousarray(powers, np.uint32).reshape(-1)
    dn = np.ascontiguousarray(denom_inv, np.uint32)
    zz = np.ascontiguousarray(z if z is not None else np.zeros(4), np.uint32)
    aa = np.ascontiguousarray(alpha if alpha is not None else np.zeros(4), np.uint32)
    sh = np.ascontiguousarray(shift if shift is not None else np.zeros(4), np.uint32)
    op, keep_o = ptr_array(out)
    lib().oracle_constraint_quotients(0 if air == "wide_fibonacci" else 1, n_cols or len(trace), trace_log, eval_log,
                                      tp, ip, pw.ctypes.data_as(U32P), len(pw) // 4, dn.ctypes.data_as(U32P),
                                      zz.ctypes.data_as(U32P), aa.ctypes.data_as(U32P), sh.ctypes.data_as(U32P), op)
    return out
