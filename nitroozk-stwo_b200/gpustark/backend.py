"""GpuBackend: the reference's backend traits over the gpustark C ABI.

Method names and argument meaning follow the reference's traits
(crates/stwo/src/prover/backend/mod.rs:20-92, prover/poly/circle/ops.rs,
prover/vcs/ops.rs, prover/fri.rs:28-49, core/proof_of_work.rs) so that a
caller of those traits finds the same operations here. Device columns are
torch CUDA tensors of dtype int32 holding M31 words bit-for-bit; QM31 columns
are lists of 4 such tensors (coordinate planes); a hash layer is an int32
tensor of 8 words per node. Every call enqueues on the context's stream,
which is torch's current stream unless another is given.
"""
import ctypes as C
import hashlib
import struct
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L

P = (1 << 31) - 1
POW_PREFIX = 0x12345678


class Context:
    """One gs_ctx bound to a CUDA stream (default: torch's current stream)."""

    def __init__(self, stream=None):
        if not torch.cuda.is_available():
            raise L.GpuStarkError("gpustark needs a CUDA device")
        if stream is None:
            stream = torch.cuda.current_stream()
        self.stream = stream
        h = C.c_void_p()
        L.check(L.lib().gs_ctx_create(C.c_void_p(stream.cuda_stream), C.byref(h)), "gs_ctx_create")
        self.handle = h

    def synchronize(self):
        L.check(L.lib().gs_ctx_synchronize(self.handle), "gs_ctx_synchronize")

    def close(self):
        if self.handle:
            L.lib().gs_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def default_context():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context()
    return _default_ctx


def to_device(a, device="cuda"):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return torch.from_numpy(a.view(np.int32)).to(device)


def to_host(t):
    return t.detach().cpu().numpy().view(np.uint32)


def qm31(v):
    v = [int(x) for x in v]
    return L.QM31(*v)


@dataclass
class TwiddleTree:
    """PolyOps::Twiddles for the coset half_odds(root_log) (prover/poly/twiddles.rs:9-14)."""
    root_log: int
    twiddles: torch.Tensor
    itwiddles: torch.Tensor


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class GpuBackend:
    """Static operations mirroring ColumnOps / PolyOps / MerkleOps / FriOps / GrindOps."""

    # ------------------------------------------------------------ ColumnOps
    @staticmethod
    def bit_reverse_column(col, ctx=None):
        ctx = ctx or default_context()
        n = col.numel()
        L.check(L.lib().gs_bit_reverse_base_field(ctx.handle, _p(col), n.bit_length() - 1), "bit_reverse_column")

    # -------------------------------------------------------------- PolyOps
    @staticmethod
    def precompute_twiddles(root_log, ctx=None) -> TwiddleTree:
        """Twiddle tree of Coset::half_odds(root_log) (ops.rs:123)."""
        ctx = ctx or default_context()
        n = 1 << root_log
        tw = torch.empty(n, dtype=torch.int32, device="cuda")
        itw = torch.empty(n, dtype=torch.int32, device="cuda")
        initial = 1 << (31 - (root_log + 2))
        step = 1 << (31 - root_log)
        L.check(L.lib().gs_precompute_twiddles(ctx.handle, initial, step, root_log, _p(tw), _p(itw)),
                "precompute_twiddles")
        return TwiddleTree(root_log, tw, itw)

    @staticmethod
    def interpolate_columns(columns, log_size, twiddles: TwiddleTree, ctx=None):
        """In place: bit-reversed evaluations on CanonicCoset(log_size) -> coefficients (ops.rs:28-39)."""
        ctx = ctx or default_context()
        pp, keep = L.ptr_array([c.data_ptr() for c in columns])
        L.check(L.lib().gs_interpolate_columns(ctx.handle, pp, len(columns), log_size, _p(twiddles.itwiddles),
                                               twiddles.root_log), "interpolate_columns")
        return columns

    @staticmethod
    def evaluate_polynomials(coeffs, log_size, twiddles: TwiddleTree, out=None, ctx=None):
        """Coefficients -> bit-reversed evaluations on CanonicCoset(log_size) (ops.rs:88-120)."""
        ctx = ctx or default_context()
        if out is None:
            out = [torch.empty(1 << log_size, dtype=torch.int32, device="cuda") for _ in coeffs]
        coeff_log = coeffs[0].numel().bit_length() - 1
        sp, k1 = L.ptr_array([c.data_ptr() for c in coeffs])
        dp, k2 = L.ptr_array([c.data_ptr() for c in out])
        L.check(L.lib().gs_evaluate_columns(ctx.handle, sp, coeff_log, dp, len(coeffs), log_size,
                                            _p(twiddles.twiddles), twiddles.root_log), "evaluate_polynomials")
        return out

    @staticmethod
    def fft_worklist(items, twiddles: TwiddleTree, ctx=None):
        """Many FFTs of uneven sizes in one launch (gs_fft_worklist). items:
        tuples ("interpolate", src, dst) with src and dst 2^log-word tensors
        (src is dst: in place) or ("evaluate", coeffs, dst) with dst of
        2^log words; returns the dst tensors."""
        ctx = ctx or default_context()
        arr = (L.FftItem * max(len(items), 1))()
        for k, (kind, src, dst) in enumerate(items):
            if kind not in ("interpolate", "evaluate"):
                raise ValueError(f"unknown work-list item kind {kind!r}")
            arr[k].src, arr[k].dst = src.data_ptr(), dst.data_ptr()
            arr[k].log_size = dst.numel().bit_length() - 1
            arr[k].coeffs_log_size = src.numel().bit_length() - 1
            arr[k].inverse = 1 if kind == "interpolate" else 0
        L.check(L.lib().gs_fft_worklist(ctx.handle, arr, len(items), _p(twiddles.twiddles), _p(twiddles.itwiddles),
                                        twiddles.root_log), "fft_worklist")
        return [dst for _, _, dst in items]

    ALL_EXTENSIONS = 0xFFFFFFFF

    @staticmethod
    def fft_autotune(min_log, max_log, max_extension=2, ctx=None):
        """Times the FFT pass splits for every log size in [min_log, max_log]
        and extension (LDE blowup log) in [0, max_extension] and installs the
        fastest (process-wide); returns {(log, extension): (tile_log,
        coalesce_bits)}. The split changes speed, never the values."""
        ctx = ctx or default_context()
        n = (max_log - min_log + 1) * (max_extension + 1)
        tiles, coal = (C.c_uint32 * n)(), (C.c_uint32 * n)()
        L.check(L.lib().gs_fft_autotune(ctx.handle, min_log, max_log, max_extension, tiles, coal), "fft_autotune")
        return {(min_log + i // (max_extension + 1), i % (max_extension + 1)): (tiles[i], coal[i]) for i in range(n)}

    @staticmethod
    def fft_set_tuning(log_size, tile_log, coalesce_bits, extension=ALL_EXTENSIONS):
        """Installs one FFT pass split for log_size (0: every size) and
        extension (default: every extension)."""
        L.check(L.lib().gs_fft_set_tuning(log_size, extension, tile_log, coalesce_bits), "fft_set_tuning")

    @staticmethod
    def fft_get_tuning(log_size, extension=0):
        t, c = C.c_uint32(), C.c_uint32()
        L.check(L.lib().gs_fft_get_tuning(log_size, extension, C.byref(t), C.byref(c)), "fft_get_tuning")
        return t.value, c.value

    # ------------------------------------------------------------ MerkleOps
    @staticmethod
    def commit_on_layer(log_size, prev_layer, columns, ctx=None, out=None):
        """One Blake2s Merkle layer (prover/vcs/ops.rs:24-28); returns 2^log_size x 8 words."""
        ctx = ctx or default_context()
        if out is None:
            out = torch.empty((1 << log_size) * 8, dtype=torch.int32, device="cuda")
        pp, keep = L.ptr_array([c.data_ptr() for c in columns])
        L.check(L.lib().gs_commit_on_layer(ctx.handle, log_size, _p(prev_layer), len(columns), pp, _p(out)),
                "commit_on_layer")
        return out

    @staticmethod
    def build_leaves_lifted(columns, lifting_log_size, ctx=None, out=None):
        """MerkleOpsLifted::build_leaves (prover/vcs_lifted/ops.rs:8-18): leaf hashes of a lifted
        commitment, 8 words per leaf (one leaf, the hash of nothing, for no columns)."""
        ctx = ctx or default_context()
        n = (1 << lifting_log_size) if columns else 1
        if out is None:
            out = torch.empty(n * 8, dtype=torch.int32, device="cuda")
        logs = (C.c_uint32 * max(len(columns), 1))(*[c.numel().bit_length() - 1 for c in columns])
        pp, keep = L.ptr_array([c.data_ptr() for c in columns])
        L.check(L.lib().gs_lifted_build_leaves(ctx.handle, pp, logs, len(columns), lifting_log_size, _p(out)),
                "build_leaves_lifted")
        return out

    @staticmethod
    def commit_node_layers(layers, ctx=None):
        """Fills layers[L] (2^L hashes) for L < len(layers)-1 from the top layer (node-only layers)."""
        ctx = ctx or default_context()
        pp, keep = L.ptr_array([t.data_ptr() for t in layers])
        L.check(L.lib().gs_commit_node_layers(ctx.handle, len(layers) - 1, pp), "commit_node_layers")
        return layers

    @staticmethod
    def merkle_worklist(trees, ctx=None):
        """Whole Blake2s Merkle trees of uneven sizes at once (gs_merkle_worklist).
        trees: lists of columns (tensors of 2^log words each, at least one per
        tree); returns per tree its layers, layers[L] of 2^L x 8 words."""
        ctx = ctx or default_context()
        arr = (L.MerkleItem * max(len(trees), 1))()
        keep, out = [], []
        for k, cols in enumerate(trees):
            log = cols[0].numel().bit_length() - 1
            layers = [torch.empty((1 << lg) * 8, dtype=torch.int32, device="cuda") for lg in range(log + 1)]
            cp, kc = L.ptr_array([c.data_ptr() for c in cols])
            lp, kl = L.ptr_array([t.data_ptr() for t in layers])
            keep += [kc, kl]
            arr[k].cols, arr[k].n_cols, arr[k].log_size, arr[k].layers = cp, len(cols), log, lp
            out.append(layers)
        L.check(L.lib().gs_merkle_worklist(ctx.handle, arr, len(trees)), "merkle_worklist")
        return out

    @staticmethod
    def poseidon252_commit_on_layer(log_size, prev_layer, columns, ctx=None, out=None):
        """MerkleOps<Poseidon252MerkleHasher>::commit_on_layer (prover/backend/
        cuda/poseidon252.rs:21-42): 2^log_size felt252 hashes as a uint8 tensor
        of 32 big-endian bytes each."""
        ctx = ctx or default_context()
        if out is None:
            out = torch.empty((1 << log_size) * 32, dtype=torch.uint8, device="cuda")
        pp, keep = L.ptr_array([c.data_ptr() for c in columns]) if columns else (None, None)
        L.check(L.lib().gs_poseidon252_commit_on_layer(ctx.handle, log_size, _p(prev_layer), len(columns), pp,
                                                      _p(out)), "poseidon252_commit_on_layer")
        return out

    @staticmethod
    def poseidon252_grind(digest, pow_bits, ctx=None):
        """GrindOps<Poseidon252Channel>::grind; digest: int (felt252) or 32
        big-endian bytes."""
        ctx = ctx or default_context()
        if isinstance(digest, int):
            digest = digest.to_bytes(32, "big")
        buf = (C.c_uint8 * 32).from_buffer_copy(digest)
        nonce = C.c_uint64()
        L.check(L.lib().gs_poseidon252_grind(ctx.handle, buf, pow_bits, C.byref(nonce)), "poseidon252_grind")
        return nonce.value

    @staticmethod
    def poseidon252_permute(states, ctx=None):
        """Hades permutations of n states (uint8 tensor of n x 96 big-endian bytes)."""
        ctx = ctx or default_context()
        n = states.numel() // 96
        out = torch.empty_like(states)
        L.check(L.lib().gs_poseidon252_permute(ctx.handle, _p(states), n, _p(out)), "poseidon252_permute")
        return out

    # --------------------------------------------------------------- FriOps
    @staticmethod
    def fold_line(eval_planes, log_size, alpha, twiddles: TwiddleTree, ctx=None, leaf_hashes=None):
        """FriOps::fold_line with fold_step 1 (prover/fri.rs:39-44)."""
        ctx = ctx or default_context()
        out = [torch.empty(1 << (log_size - 1), dtype=torch.int32, device="cuda") for _ in range(4)]
        sp, k1 = L.ptr_array([t.data_ptr() for t in eval_planes])
        dp, k2 = L.ptr_array([t.data_ptr() for t in out])
        L.check(L.lib().gs_fold_line(ctx.handle, sp, log_size, qm31(alpha), dp, _p(twiddles.itwiddles),
                                     twiddles.root_log, _p(leaf_hashes)), "fold_line")
        return out

    @staticmethod
    def fold_circle_into_line(dst_planes, src_planes, log_size, alpha, twiddles: TwiddleTree, ctx=None,
                              leaf_hashes=None):
        """FriOps::fold_circle_into_line (prover/fri.rs:61-66); dst updated in place."""
        ctx = ctx or default_context()
        sp, k1 = L.ptr_array([t.data_ptr() for t in src_planes])
        dp, k2 = L.ptr_array([t.data_ptr() for t in dst_planes])
        L.check(L.lib().gs_fold_circle_into_line(ctx.handle, sp, log_size, qm31(alpha), dp, _p(twiddles.itwiddles),
                                                 twiddles.root_log, _p(leaf_hashes)), "fold_circle_into_line")
        return dst_planes

    # ---------------------------------------------------------- QuotientOps
    @staticmethod
    def accumulate_numerators(columns, log_size, column_indices, line_coeffs_b, line_coeffs_c, ctx=None):
        """QuotientOps::accumulate_numerators for one sample batch (quotient_ops.rs:27-31).
        line_coeffs_*: sequences of QM31 (4 ints). Returns 4 planes of 2^log_size."""
        ctx = ctx or default_context()
        out = [torch.empty(1 << log_size, dtype=torch.int32, device="cuda") for _ in range(4)]
        cp, k1 = L.ptr_array([c.data_ptr() for c in columns])
        n = len(column_indices)
        idx = (C.c_uint32 * max(n, 1))(*[int(i) for i in column_indices])
        bs = (L.QM31 * max(n, 1))(*[qm31(b) for b in line_coeffs_b])
        cs = (L.QM31 * max(n, 1))(*[qm31(c) for c in line_coeffs_c])
        op, k2 = L.ptr_array([t.data_ptr() for t in out])
        L.check(L.lib().gs_accumulate_numerators(ctx.handle, log_size, cp, len(columns), idx, bs, cs, n, op),
                "accumulate_numerators")
        return out

    @staticmethod
    def compute_quotients_and_combine(accs, lifting_log_size, ctx=None):
        """accs: list of (partial_planes, log_size, first_linear_term(4), point(8)) (quotient_ops.rs:39-42)."""
        ctx = ctx or default_context()
        arr = (L.QuotientAcc * max(len(accs), 1))()
        for a, (planes_, log_size, flt, pt) in enumerate(accs):
            for i in range(4):
                arr[a].partial[i] = planes_[i].data_ptr()
            arr[a].log_size = log_size
            arr[a].first_linear_term = qm31(flt)
            arr[a].sample_point = L.PointQM31(qm31(pt[:4]), qm31(pt[4:]))
        out = [torch.empty(1 << lifting_log_size, dtype=torch.int32, device="cuda") for _ in range(4)]
        op, k = L.ptr_array([t.data_ptr() for t in out])
        L.check(L.lib().gs_compute_quotients_and_combine(ctx.handle, arr, len(accs), lifting_log_size, op),
                "compute_quotients_and_combine")
        return out

    # ------------------------------------------------------ AccumulationOps
    @staticmethod
    def lift_and_accumulate(cols, ctx=None):
        """cols: list of 4-plane QM31 columns in increasing size (accumulation.rs:127-145)."""
        ctx = ctx or default_context()
        logs = [c[0].numel().bit_length() - 1 for c in cols]
        out_log = max(logs)
        out = [torch.empty(1 << out_log, dtype=torch.int32, device="cuda") for _ in range(4)]
        pp, k1 = L.ptr_array([t.data_ptr() for c in cols for t in c])
        ls = (C.c_uint32 * len(logs))(*logs)
        op, k2 = L.ptr_array([t.data_ptr() for t in out])
        L.check(L.lib().gs_lift_and_accumulate(ctx.handle, pp, ls, len(cols), op, out_log), "lift_and_accumulate")
        return out

    @staticmethod
    def accumulate(a_planes, b_planes, ctx=None):
        """AccumulationOps::accumulate: a += b coordinate-wise (4 planes each), in place."""
        ctx = ctx or default_context()
        ap, k1 = L.ptr_array([t.data_ptr() for t in a_planes])
        bp, k2 = L.ptr_array([t.data_ptr() for t in b_planes])
        L.check(L.lib().gs_accumulate(ctx.handle, ap, bp, a_planes[0].numel()), "accumulate")
        return a_planes

    @staticmethod
    def batch_eval_at_point(polys, point, ctx=None):
        """Values of coefficient polynomials at a QM31 circle point (ops.rs:51-59)."""
        ctx = ctx or default_context()
        log_size = polys[0].numel().bit_length() - 1
        pp, k = L.ptr_array([p.data_ptr() for p in polys])
        out = (L.QM31 * len(polys))()
        pt = L.PointQM31(qm31(point[:4]), qm31(point[4:]))
        L.check(L.lib().gs_batch_eval_at_point(ctx.handle, pp, len(polys), log_size, pt, out), "batch_eval_at_point")
        return [[o.a, o.b, o.c, o.d] for o in out]

    @staticmethod
    def batch_eval_at_point_noalloc(polys, point, log_size=None, stream=None):
        """batch_eval_at_point with no allocation (static device scratch; at
        most 256 polynomials and 256 * 2^10 coefficients per polynomial at
        that count). Runs on `stream` (torch's current stream by default)."""
        if stream is None:
            stream = torch.cuda.current_stream()
        if log_size is None:
            log_size = polys[0].numel().bit_length() - 1 if polys else 0
        for p in polys:
            if not (p.is_cuda and p.dtype == torch.int32 and p.is_contiguous() and p.numel() == 1 << log_size):
                raise ValueError(f"every polynomial must be a contiguous int32 CUDA tensor of 2^{log_size} words")
        pp, k = L.ptr_array([p.data_ptr() for p in polys])
        out = (L.QM31 * max(len(polys), 1))()
        pt = L.PointQM31(qm31(point[:4]), qm31(point[4:]))
        handle = getattr(stream, "cuda_stream", stream)
        L.check(L.lib().gs_batch_eval_at_point_noalloc(handle, pp, len(polys), log_size, pt, out),
                "batch_eval_at_point_noalloc")
        return [[o.a, o.b, o.c, o.d] for o in out[:len(polys)]]

    # ------------------------------------------------------- Column gathers
    @staticmethod
    def batch_at_multi(columns, indices, ctx=None):
        """Column::batch_at_multi (prover/backend/mod.rs:73-89): values of every
        column at every index, row-major (index-major), as a uint32 array of
        len(indices) * len(columns)."""
        ctx = ctx or default_context()
        idx = np.ascontiguousarray(indices, dtype=np.uint32)
        out = np.zeros(max(len(idx) * len(columns), 1), np.uint32)
        col_len = min(c.numel() for c in columns) if columns else 0
        pp, k = L.ptr_array([c.data_ptr() for c in columns])
        L.check(L.lib().gs_batch_gather_multi_uint32(ctx.handle, pp, len(columns), col_len,
                                                     idx.ctypes.data_as(L.U32P), len(idx),
                                                     out.ctypes.data_as(L.U32P)), "batch_at_multi")
        return out[: len(idx) * len(columns)]

    @staticmethod
    def batch_get_hashes(layer, indices, ctx=None):
        """Column<Blake2sHash>::batch_at: the hashes of one Merkle layer at the
        indices, as (len(indices), 32) bytes."""
        ctx = ctx or default_context()
        idx = np.ascontiguousarray(indices, dtype=np.uint32)
        out = np.zeros(max(8 * len(idx), 8), np.uint32)
        L.check(L.lib().gs_batch_get_blake2s_hash(ctx.handle, _p(layer), layer.numel() // 8,
                                                  idx.ctypes.data_as(L.U32P), len(idx),
                                                  out.ctypes.data_as(L.U32P)), "batch_get_hashes")
        return out[: 8 * len(idx)].view(np.uint8).reshape(-1, 32)

    # ----------------------------------------------------- barycentric OODS
    @staticmethod
    def barycentric_weights(log_size, point, ctx=None):
        """PolyOps::barycentric_weights(CanonicCoset(log_size), p) (ops.rs:64-68): 4 planes."""
        ctx = ctx or default_context()
        out = [torch.empty(1 << log_size, dtype=torch.int32, device="cuda") for _ in range(4)]
        op, k = L.ptr_array([t.data_ptr() for t in out])
        pt = L.PointQM31(qm31(point[:4]), qm31(point[4:]))
        L.check(L.lib().gs_barycentric_weights(ctx.handle, log_size, pt, op), "barycentric_weights")
        return out

    @staticmethod
    def barycentric_eval_at_point(evals, weights, ctx=None):
        """PolyOps::barycentric_eval_at_point (ops.rs:73-77): sum_i evals[i] * weights[i]."""
        ctx = ctx or default_context()
        wp, k = L.ptr_array([t.data_ptr() for t in weights])
        out = L.QM31()
        L.check(L.lib().gs_barycentric_eval_at_point(ctx.handle, _p(evals), wp, evals.numel().bit_length() - 1,
                                                     C.byref(out)), "barycentric_eval_at_point")
        return [out.a, out.b, out.c, out.d]

    # ------------------------------------------------- constraint evaluation
    @staticmethod
    def generate_secure_powers(felt, n, ctx=None):
        """AccumulationOps::generate_secure_powers: felt^i for i < n, 4 planes."""
        ctx = ctx or default_context()
        out = [torch.empty(max(n, 1), dtype=torch.int32, device="cuda") for _ in range(4)]
        op, k = L.ptr_array([t.data_ptr() for t in out])
        L.check(L.lib().gs_generate_secure_powers(ctx.handle, qm31(felt), n, op), "generate_secure_powers")
        return [t[:n] for t in out]

    @staticmethod
    def evaluate_constraint_quotients_on_domain(quotients, trace0, trace1, trace2, random_coeff_powers,
                                                denominator_inverses, domain_log_size, eval_domain_log_size,
                                                n_constraints, eval_bytes, cumsum_shift=(0, 0, 0, 0),
                                                should_accumulate=True, logup_counts=0, ctx=None):
        """ComponentProver<CudaBackend>::evaluate_constraint_quotients_on_domain's
        FFI call (component_prover.rs:447-470): eval_bytes is eval_id followed
        by the component's #[repr(C)] Eval struct (eval_blob_* below)."""
        ctx = ctx or default_context()
        qp, k0 = L.ptr_array([t.data_ptr() for t in quotients])
        t0, k1 = L.ptr_array([t.data_ptr() for t in trace0])
        t1, k2 = L.ptr_array([t.data_ptr() for t in trace1])
        t2, k3 = L.ptr_array([t.data_ptr() for t in trace2])
        pw = (L.QM31 * max(len(random_coeff_powers), 1))(*[qm31(p) for p in random_coeff_powers])
        dn = np.ascontiguousarray(denominator_inverses, dtype=np.uint32)
        eb = (C.c_uint8 * len(eval_bytes)).from_buffer_copy(eval_bytes)
        L.check(L.lib().gs_evaluate_constraint_quotients_on_domain(
            ctx.handle, qp, t0, len(trace0), t1, len(trace1), t2, len(trace2), pw, dn.ctypes.data_as(L.U32P),
            domain_log_size, eval_domain_log_size, n_constraints, logup_counts, eb, len(eval_bytes),
            qm31(cumsum_shift), 1 if should_accumulate else 0), "evaluate_constraint_quotients_on_domain")
        return quotients

    # ----------------------------------------------- example trace generation
    @staticmethod
    def generate_wide_fibonacci_trace(input_a, input_b, n_columns, ctx=None):
        """generate_wide_fibonacci_trace: n_columns device columns from inputs a, b."""
        ctx = ctx or default_context()
        n = input_a.numel()
        cols = [torch.empty(n, dtype=torch.int32, device="cuda") for _ in range(n_columns)]
        cp, k = L.ptr_array([c.data_ptr() for c in cols])
        L.check(L.lib().gs_generate_wide_fibonacci_trace(ctx.handle, _p(input_a), _p(input_b), n.bit_length() - 1, cp,
                                                         n_columns), "generate_wide_fibonacci_trace")
        return cols

    @staticmethod
    def generate_poseidon_traces(log_size, ctx=None):
        """generate_poseidon_traces: (158 trace columns, 16 initial-state, 16 final-state columns)."""
        ctx = ctx or default_context()
        mk = lambda k: [torch.empty(1 << log_size, dtype=torch.int32, device="cuda") for _ in range(k)]
        trace, init, fin = mk(158), mk(16), mk(16)
        tp, k1 = L.ptr_array([c.data_ptr() for c in trace])
        ip, k2 = L.ptr_array([c.data_ptr() for c in init])
        fp, k3 = L.ptr_array([c.data_ptr() for c in fin])
        L.check(L.lib().gs_generate_poseidon_traces(ctx.handle, tp, ip, fp, log_size), "generate_poseidon_traces")
        return trace, init, fin

    @staticmethod
    def generate_poseidon_interaction_traces(z, alpha, init, fin, ctx=None):
        """generate_poseidon_interaction_traces: (4 interaction planes, claimed sum)."""
        ctx = ctx or default_context()
        log_size = init[0].numel().bit_length() - 1
        powers, cur = [], [1, 0, 0, 0]
        for _ in range(16):
            powers.append(cur)
            cur = _qm_mul(cur, alpha)
        words = list(z) + list(alpha) + [w for p in powers for w in p]
        le = (C.c_uint32 * len(words))(*[int(w) for w in words])
        out = [torch.empty(1 << log_size, dtype=torch.int32, device="cuda") for _ in range(4)]
        ip, k1 = L.ptr_array([c.data_ptr() for c in init])
        fp, k2 = L.ptr_array([c.data_ptr() for c in fin])
        op, k3 = L.ptr_array([c.data_ptr() for c in out])
        cs = (C.c_uint32 * 4)()
        L.check(L.lib().gs_generate_poseidon_interaction_traces(ctx.handle, le, ip, fp, log_size, op, cs),
                "generate_poseidon_interaction_traces")
        return out, list(cs)

    # ------------------------------------------------------------- GrindOps
    @staticmethod
    def grind(digest: bytes, pow_bits, ctx=None):
        """GrindOps<Blake2sChannel>::grind: smallest nonce for the channel digest."""
        ctx = ctx or default_context()
        pre = hashlib.blake2s(struct.pack("<I", POW_PREFIX) + bytes(12) + digest + struct.pack("<I", pow_bits),
                              digest_size=32).digest()
        words = (C.c_uint32 * 8)(*struct.unpack("<8I", pre))
        nonce = C.c_uint64()
        L.check(L.lib().gs_grind_blake2s(ctx.handle, words, pow_bits, C.byref(nonce)), "grind")
        return nonce.value


class CommitPlan:
    """Batched TreeBuilder::extend_evals + commit for columns of mixed sizes
    (gs_commit_plan_*): interpolation and extension batched per size group,
    one Merkle tree over all columns; optionally replayed from a CUDA graph."""

    def __init__(self, log_sizes, log_blowup=1, use_graph=True, ctx=None):
        self.ctx = ctx or default_context()
        self.log_sizes = [int(v) for v in log_sizes]
        self.log_blowup = log_blowup
        logs = (C.c_uint32 * len(self.log_sizes))(*self.log_sizes)
        h = C.c_void_p()
        L.check(L.lib().gs_commit_plan_create(self.ctx.handle, logs, len(self.log_sizes), log_blowup,
                                              1 if use_graph else 0, C.byref(h)), "gs_commit_plan_create")
        self.handle = h

    def run(self, columns):
        """columns: device tensors (bit-reversed evaluations); returns the 32-byte root."""
        pp, keep = L.ptr_array([c.data_ptr() for c in columns])
        root = (C.c_uint32 * 8)()
        L.check(L.lib().gs_commit_plan_run(self.handle, pp, root), "gs_commit_plan_run")
        return struct.pack("<8I", *root)

    def _read(self, ptr, words):
        out = np.zeros(words, np.uint32)
        L.check(L.lib().gs_memcpy_d2h(self.ctx.handle, out.ctypes.data_as(C.c_void_p), ptr, 4 * words), "d2h")
        return out

    def extended(self, i):
        """Host copy of column i on CanonicCoset(log + log_blowup)."""
        p = C.c_void_p()
        L.check(L.lib().gs_commit_plan_extended(self.handle, i, C.byref(p)), "gs_commit_plan_extended")
        return self._read(p, 1 << (self.log_sizes[i] + self.log_blowup))

    def layer(self, log_size):
        """Host copy of Merkle layer log_size as (2^log_size, 32) bytes."""
        p = C.c_void_p()
        L.check(L.lib().gs_commit_plan_layer(self.handle, log_size, C.byref(p)), "gs_commit_plan_layer")
        return self._read(p, 8 << log_size).view(np.uint8).reshape(-1, 32)

    def close(self):
        if getattr(self, "handle", None):
            L.lib().gs_commit_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fnv1a_eval_id(name: str) -> int:
    """fnv1a_eval_id_gen (crates/constraint-framework/src/lib.rs:353-363)."""
    h = 0x811C9DC5
    for b in name.encode():
        h = ((h ^ b) * 0x01000193) & 0xFFFFFFFF
    return h


def eval_blob_wide_fibonacci(log_n_rows):
    """The bytes ComponentProver passes for WideFibonacciEval: eval_id, then
    #[repr(C)] WideFibonacciEval { eval_id, log_n_rows }
    (crates/examples/src/wide_fibonacci/mod.rs:32-37)."""
    i = fnv1a_eval_id("fibonacci_example")
    return struct.pack("<3I", i, i, log_n_rows)


def eval_blob_poseidon(log_n_rows, z, alpha, claimed_sum):
    """The bytes for PoseidonEval: eval_id, then #[repr(C)] PoseidonEval {
    eval_id, log_n_rows, lookup_elements { z, alpha, alpha_powers[16] },
    claimed_sum } (crates/examples/src/poseidon/mod.rs:57-64), QM31 as 4 words."""
    def mul(a, b):  # QM31 product on the host
        return _qm_mul(a, b)
    i = fnv1a_eval_id("poseidon_example")
    powers, cur = [], [1, 0, 0, 0]
    for _ in range(16):
        powers.append(cur)
        cur = mul(cur, alpha)
    words = [i, i, log_n_rows] + list(z) + list(alpha) + [w for p in powers for w in p] + list(claimed_sum)
    return struct.pack(f"<{len(words)}I", *[int(w) for w in words])


def _cm_mul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def _qm_mul(p, q):
    """QM31 (a + b i) + (c + d i) u with u^2 = 2 + i (core/fields/qm31.rs), on Python ints."""
    p, q = [int(x) for x in p], [int(x) for x in q]
    x0, y0, x1, y1 = (p[0], p[1]), (p[2], p[3]), (q[0], q[1]), (q[2], q[3])
    xx, yy = _cm_mul(x0, x1), _cm_mul(y0, y1)
    r_yy = _cm_mul((2, 1), yy)
    re = ((xx[0] + r_yy[0]) % P, (xx[1] + r_yy[1]) % P)
    a, b = _cm_mul(x0, y1), _cm_mul(y0, x1)
    return [re[0], re[1], (a[0] + b[0]) % P, (a[1] + b[1]) % P]
