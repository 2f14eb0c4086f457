"""ctypes loader for libgpustark.so (the C ABI declared in include/gpustark.h).

The shared library is built in-tree (``make -C nitroozk-stwo_b200``). There
is no fallback: if the library or a CUDA device is missing, the calls raise.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgpustark.so")

U32P = C.POINTER(C.c_uint32)
VPP = C.POINTER(C.c_void_p)


class QM31(C.Structure):
    _fields_ = [("a", C.c_uint32), ("b", C.c_uint32), ("c", C.c_uint32), ("d", C.c_uint32)]


class PointQM31(C.Structure):
    _fields_ = [("x", QM31), ("y", QM31)]


class QuotientAcc(C.Structure):
    _fields_ = [("partial", C.c_void_p * 4), ("log_size", C.c_uint32), ("first_linear_term", QM31),
                ("sample_point", PointQM31)]


class PcsConfig(C.Structure):
    _fields_ = [("pow_bits", C.c_uint32), ("log_blowup_factor", C.c_uint32),
                ("log_last_layer_degree_bound", C.c_uint32), ("n_queries", C.c_uint32),
                ("line_fold_step", C.c_uint32)]


class FftItem(C.Structure):
    """gs_fft_item: one FFT of a work-list (include/gpustark.h)."""
    _fields_ = [("src", C.c_void_p), ("dst", C.c_void_p), ("log_size", C.c_uint32), ("coeffs_log_size", C.c_uint32),
                ("inverse", C.c_uint32), ("reserved", C.c_uint32)]


class MerkleItem(C.Structure):
    """gs_merkle_item: one tree of a Merkle work-list (include/gpustark.h)."""
    _fields_ = [("cols", VPP), ("n_cols", C.c_uint32), ("log_size", C.c_uint32), ("layers", VPP)]


class GpuStarkError(RuntimeError):
    pass


_lib = None

# (name, argtypes); every function returns an int status unless listed in _RESTYPE.
_PROTOS = {
    "gs_ctx_create": [C.c_void_p, C.POINTER(C.c_void_p)],
    "gs_ctx_destroy": [C.c_void_p],
    "gs_ctx_synchronize": [C.c_void_p],
    "gs_malloc": [C.c_void_p, C.c_size_t, C.POINTER(C.c_void_p)],
    "gs_free": [C.c_void_p, C.c_void_p],
    "gs_memset_zero": [C.c_void_p, C.c_void_p, C.c_size_t],
    "gs_memcpy_h2d": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t],
    "gs_memcpy_d2h": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t],
    "gs_memcpy_d2d": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t],
    "gs_bit_reverse_base_field": [C.c_void_p, C.c_void_p, C.c_uint32],
    "gs_bit_reverse_secure_field": [C.c_void_p, VPP, C.c_uint32],
    "gs_batch_inverse_base_field": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t],
    "gs_precompute_twiddles": [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p],
    "gs_interpolate_columns": [C.c_void_p, VPP, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32],
    "gs_evaluate_columns": [C.c_void_p, VPP, C.c_uint32, VPP, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32],
    "gs_fft_worklist": [C.c_void_p, C.POINTER(FftItem), C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32],
    "gs_fft_autotune": [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, U32P, U32P],
    "gs_fft_set_tuning": [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32],
    "gs_fft_get_tuning": [C.c_uint32, C.c_uint32, U32P, U32P],
    "gs_commit_on_layer": [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, VPP, C.c_void_p],
    "gs_commit_node_layers": [C.c_void_p, C.c_uint32, VPP],
    "gs_merkle_worklist": [C.c_void_p, C.POINTER(MerkleItem), C.c_uint32],
    "gs_poseidon252_commit_on_layer": [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, VPP, C.c_void_p],
    "gs_poseidon252_permute": [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p],
    "gs_poseidon252_grind": [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint64)],
    "gs_fold_line": [C.c_void_p, VPP, C.c_uint32, QM31, VPP, C.c_void_p, C.c_uint32, C.c_void_p],
    "gs_fold_circle_into_line": [C.c_void_p, VPP, C.c_uint32, QM31, VPP, C.c_void_p, C.c_uint32, C.c_void_p],
    "gs_grind_blake2s": [C.c_void_p, U32P, C.c_uint32, C.POINTER(C.c_uint64)],
    "gs_accumulate_numerators": [C.c_void_p, C.c_uint32, VPP, C.c_uint32, U32P, C.c_void_p, C.c_void_p, C.c_uint32,
                                 VPP],
    "gs_compute_quotients_and_combine": [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, VPP],
    "gs_lift_and_accumulate": [C.c_void_p, VPP, U32P, C.c_uint32, VPP, C.c_uint32],
    "gs_accumulate": [C.c_void_p, VPP, VPP, C.c_size_t],
    "gs_batch_eval_at_point": [C.c_void_p, VPP, C.c_uint32, C.c_uint32, PointQM31, C.c_void_p],
    "gs_batch_eval_at_point_noalloc": [C.c_void_p, VPP, C.c_uint32, C.c_uint32, PointQM31, C.c_void_p],
    "gs_prove_wide_fibonacci": [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, U32P,
                                C.POINTER(PcsConfig), C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)],
    "gs_server_create": [C.c_uint32, C.c_size_t, C.POINTER(C.c_void_p)],
    "gs_server_create_fibers": [C.c_uint32, C.c_uint32, C.c_size_t, C.POINTER(C.c_void_p)],
    "gs_server_submit": [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32,
                         C.POINTER(PcsConfig), C.POINTER(C.c_uint64)],
    "gs_server_submit_poseidon252": [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32,
                                     C.POINTER(PcsConfig), C.POINTER(C.c_uint64)],
    "gs_server_wait": [C.c_void_p, C.c_uint64, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t),
                       C.POINTER(C.c_double)],
    "gs_server_destroy": [C.c_void_p],
    "gs_lifted_build_leaves": [C.c_void_p, VPP, U32P, C.c_uint32, C.c_uint32, C.c_void_p],
    "gs_commit_plan_create": [C.c_void_p, U32P, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_void_p)],
    "gs_commit_plan_run": [C.c_void_p, VPP, U32P],
    "gs_commit_plan_extended": [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)],
    "gs_commit_plan_layer": [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)],
    "gs_commit_plan_destroy": [C.c_void_p],
    "gs_prove_poseidon": [C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint32, U32P, C.c_uint32, C.POINTER(PcsConfig),
                          C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)],
    "gs_prove_wide_fibonacci_poseidon252": [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, U32P,
                                            C.POINTER(PcsConfig), C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)],
    "gs_prove_poseidon_poseidon252": [C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint32, U32P, C.c_uint32,
                                      C.POINTER(PcsConfig), C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)],
    "gs_batch_gather_multi_uint32": [C.c_void_p, VPP, C.c_uint32, C.c_size_t, U32P, C.c_uint32, U32P],
    "gs_batch_get_blake2s_hash": [C.c_void_p, C.c_void_p, C.c_size_t, U32P, C.c_uint32, U32P],
    "gs_barycentric_weights": [C.c_void_p, C.c_uint32, PointQM31, VPP],
    "gs_barycentric_eval_at_point": [C.c_void_p, C.c_void_p, VPP, C.c_uint32, C.POINTER(QM31)],
    "gs_generate_secure_powers": [C.c_void_p, QM31, C.c_size_t, VPP],
    "gs_evaluate_constraint_quotients_on_domain": [C.c_void_p, VPP, VPP, C.c_uint32, VPP, C.c_uint32, VPP, C.c_uint32,
                                                   C.c_void_p, U32P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                                   C.c_void_p, C.c_size_t, QM31, C.c_int],
    "gs_generate_wide_fibonacci_trace": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, VPP, C.c_uint32],
    "gs_generate_poseidon_traces": [C.c_void_p, VPP, VPP, VPP, C.c_uint32],
    "gs_generate_poseidon_interaction_traces": [C.c_void_p, C.c_void_p, VPP, VPP, C.c_uint32, VPP, U32P],
    "gs_poseidon252_channel_op": [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint64, U32P, C.c_size_t,
                                  U32P, C.c_void_p, C.POINTER(C.c_uint32)],
}
_RESTYPE = {"gs_last_error": C.c_char_p, "gs_ctx_stream": C.c_void_p, "gs_launch_count": C.c_ulonglong}
_OPTIONAL = set()


def declared_symbols():
    return sorted(set(_PROTOS) | set(_RESTYPE))


def register(name, argtypes, optional=False):
    _PROTOS[name] = argtypes
    if optional:
        _OPTIONAL.add(name)
    if _lib is not None:
        _bind(_lib, name)


def _bind(lib, name):
    if name in _RESTYPE:
        fn = getattr(lib, name)
        fn.restype = _RESTYPE[name]
        fn.argtypes = [C.c_void_p] if name == "gs_ctx_stream" else []
        return
    if not hasattr(lib, name):
        if name in _OPTIONAL:
            return
        raise GpuStarkError(f"libgpustark.so lacks symbol {name}")
    fn = getattr(lib, name)
    fn.restype = C.c_int
    fn.argtypes = _PROTOS[name]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GpuStarkError(f"{LIB_PATH} is not built; run `make -C nitroozk-stwo_b200`")
        L = C.CDLL(LIB_PATH)
        for name in list(_PROTOS) + list(_RESTYPE):
            _bind(L, name)
        _lib = L
    return _lib


def check(status, what=""):
    if status != 0:
        msg = lib().gs_last_error()
        raise GpuStarkError(f"{what or 'gpustark'} failed (status {status}): {msg.decode() if msg else ''}")


def ptr_array(ptrs):
    arr = (C.c_void_p * max(len(ptrs), 1))(*[int(p) for p in ptrs])
    return C.cast(arr, VPP), arr
