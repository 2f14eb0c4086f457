"""A Wide-Fibonacci prover driven through the per-trait C-ABI entry points
only: the host side restates the reference's generic prover (the code that
stays unchanged above a drop-in backend) and every device operation is one
call of a backend-trait method of include/gpustark.h, in the order the
reference calls them:

  crates/examples/src/wide_fibonacci/mod.rs:140-184   (the example driver)
  crates/stwo/src/prover/mod.rs:37-150                (prove_ex)
  crates/stwo/src/prover/pcs/mod.rs:150-494           (CommitmentSchemeProver, TreeBuilder,
                                                        prove_values with barycentric OODS
                                                        weights, CommitmentTreeProver::decommit)
  crates/stwo/src/prover/pcs/quotient_ops.rs:73-145   (compute_fri_quotients)
  crates/stwo/src/core/pcs/quotients.rs:80-330        (ColumnSampleBatch, line coefficients)
  crates/stwo/src/prover/fri.rs:85-413                (FriProver commit / decommit)
  crates/stwo/src/prover/vcs/prover.rs:39-222         (MerkleProver commit / decommit)
  crates/stwo/src/prover/air/accumulation.rs:21-125   (DomainEvaluationAccumulator)
  crates/constraint-framework/src/prover/component_prover.rs:249-498 (the CUDA component prover)
  crates/stwo/src/core/channel/blake2s.rs:20-140      (Blake2sChannel), core/queries.rs:11-60
  crates/stwo/src/prover/line.rs:54-99                (last-layer interpolation)

Device operations used (GpuBackend over the C ABI): precompute_twiddles,
interpolate_columns, evaluate_polynomials, commit_on_layer,
generate_secure_powers, evaluate_constraint_quotients_on_domain,
barycentric_weights, barycentric_eval_at_point, accumulate_numerators,
compute_quotients_and_combine, fold_circle_into_line, fold_line, grind,
batch_at_multi and batch_get_hashes. The fused prover (gs_prove_wide_fibonacci)
must produce the same bytes. Test infrastructure: the library's product path
is the fused prover; this module exists to show that the trait boundary alone
carries a whole proof.
"""
import hashlib
import struct
import time

import numpy as np
import torch

P = (1 << 31) - 1


# ------------------------------------------------------------- host fields
def m_inv(a):
    return pow(a, P - 2, P)


def cm_mul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def q_add(p, q):
    return tuple((x + y) % P for x, y in zip(p, q))


def q_sub(p, q):
    return tuple((x - y) % P for x, y in zip(p, q))


def q_mul(p, q):
    x0, y0, x1, y1 = (p[0], p[1]), (p[2], p[3]), (q[0], q[1]), (q[2], q[3])
    xx, yy = cm_mul(x0, x1), cm_mul(y0, y1)
    r = cm_mul((2, 1), yy)
    a, b = cm_mul(x0, y1), cm_mul(y0, x1)
    return ((xx[0] + r[0]) % P, (xx[1] + r[1]) % P, (a[0] + b[0]) % P, (a[1] + b[1]) % P)


def q_scale(p, s):
    return tuple(x * s % P for x in p)


def q_conj(p):
    return (p[0], p[1], (-p[2]) % P, (-p[3]) % P)


def q_inv(p):
    """QM31 inverse (core/fields/qm31.rs): (a + b u)^-1 = (a - b u) / (a^2 - (2 + i) b^2)."""
    a, b = (p[0], p[1]), (p[2], p[3])
    b2 = cm_mul(b, b)
    d = ((cm_mul(a, a)[0] - cm_mul((2, 1), b2)[0]) % P, (cm_mul(a, a)[1] - cm_mul((2, 1), b2)[1]) % P)
    n = m_inv((d[0] * d[0] + d[1] * d[1]) % P)
    di = (d[0] * n % P, (-d[1]) * n % P)
    x, y = cm_mul(a, di), cm_mul(b, di)
    return (x[0], x[1], (-y[0]) % P, (-y[1]) % P)


ONE = (1, 0, 0, 0)


def pt_add_m31(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


GEN = (2, 1268011823)  # M31_CIRCLE_GEN (core/circle.rs)


def index_point(idx):
    """CirclePointIndex(idx).to_point(): the generator times idx."""
    r, cur = (1, 0), GEN
    idx %= 1 << 31
    while idx:
        if idx & 1:
            r = pt_add_m31(r, cur)
        cur = pt_add_m31(cur, cur)
        idx >>= 1
    return r


def double_x(x):
    return (2 * x * x - 1) % P


def bitrev(i, log):
    return int(format(i, f"0{log}b")[::-1], 2) if log else i


# ------------------------------------------------------------------ channel
class Blake2sChannel:
    """Blake2sChannel (core/channel/blake2s.rs:20-140)."""

    def __init__(self):
        self.digest = bytes(32)
        self.n_draws = 0

    def _update(self, data):
        self.digest = hashlib.blake2s(self.digest + data, digest_size=32).digest()
        self.n_draws = 0

    def mix_root(self, root):
        self._update(root)

    def mix_felts(self, felts):
        self._update(b"".join(struct.pack("<4I", *f) for f in felts))

    def mix_u64(self, v):
        self._update(struct.pack("<2I", v & 0xFFFFFFFF, v >> 32))

    def draw_u32s(self):
        h = hashlib.blake2s(self.digest + struct.pack("<I", self.n_draws) + b"\0", digest_size=32).digest()
        self.n_draws += 1
        return struct.unpack("<8I", h)

    def draw_base_felts(self):
        while True:
            u = self.draw_u32s()
            if all(x < 2 * P for x in u):
                return [x % P for x in u]

    def draw_secure_felt(self):
        return tuple(self.draw_base_felts()[:4])

    def random_point(self):
        """CirclePoint::get_random_point (core/circle.rs:169-181)."""
        t = self.draw_secure_felt()
        t2 = q_mul(t, t)
        i = q_inv(q_add(t2, ONE))
        return q_mul(q_sub(ONE, t2), i), q_mul(q_add(t, t), i)

    def draw_queries(self, log_size, n):
        """draw_queries (core/queries.rs:11-28)."""
        raw = []
        while len(raw) < n:
            for w in self.draw_u32s():
                raw.append(w & ((1 << log_size) - 1))
                if len(raw) == n:
                    break
        return raw


# --------------------------------------------------------------- serialise
class Writer:
    """The proof bytes (bincode-1.x style, the serde field order of
    core/pcs/quotients.rs:29-38, core/fri.rs:363-398, core/vcs/verifier.rs:13-22)."""

    def __init__(self):
        self.b = bytearray()

    def u8(self, v):
        self.b += struct.pack("<B", v)

    def u32(self, v):
        self.b += struct.pack("<I", v)

    def u64(self, v):
        self.b += struct.pack("<Q", v)

    def qm(self, q):
        self.b += struct.pack("<4I", *q)

    def decommitment(self, hashes, column_witness):
        self.u64(len(hashes))
        for h in hashes:
            self.b += h
        self.u64(len(column_witness))
        for v in column_witness:
            self.u32(int(v))

    def fri_layer(self, layer):
        witness, hashes, colw, root = layer
        self.u64(len(witness))
        for q in witness:
            self.qm(q)
        self.decommitment(hashes, colw)
        self.b += root


# ------------------------------------------------------------------- prover
class TraitProver:
    def __init__(self, backend, ctx=None):
        self.B = backend
        self.ctx = ctx
        self.calls = 0

    def _call(self, name, *a, **k):
        self.calls += 1
        return getattr(self.B, name)(*a, ctx=self.ctx, **k)

    # MerkleProver::commit (prover/vcs/prover.rs:39-62), columns of one size
    def merkle_commit(self, columns):
        log = columns[0].numel().bit_length() - 1
        layers = [self._call("commit_on_layer", log, None, columns)]
        for ls in range(log - 1, -1, -1):
            layers.append(self._call("commit_on_layer", ls, layers[-1], []))
        layers.reverse()  # layers[L] has 2^L hashes
        return layers

    def root(self, layers):
        return self._call("batch_get_hashes", layers[0], [0])[0].tobytes()

    # MerkleProver::decommit (prover/vcs/prover.rs:84-217), columns of one size
    def merkle_decommit(self, layers, queries_per_log, columns):
        col_log = columns[0].numel().bit_length() - 1 if columns else -1
        queried, hash_witness, column_witness = [], [], []
        last = []
        for L in range(len(layers) - 1, -1, -1):
            has_prev = L + 1 < len(layers)
            prev = set(last)
            colq = set(queries_per_log.get(L, []))
            merged = sorted({q // 2 for q in last} | colq)
            if has_prev and merged:
                children = [c for n in merged for c in (2 * n, 2 * n + 1)]
                got = self._call("batch_get_hashes", layers[L + 1], children)
                for i, n in enumerate(merged):
                    for j in (0, 1):
                        if 2 * n + j not in prev:
                            hash_witness.append(got[2 * i + j].tobytes())
            qn = [n for n in merged if n in colq]
            wn = [n for n in merged if n not in colq]
            if L == col_log and qn:
                queried.extend(self._call("batch_at_multi", columns, qn).tolist())
            if L == col_log and wn:
                column_witness.extend(self._call("batch_at_multi", columns, wn).tolist())
            last = merged
        return queried, hash_witness, column_witness

    def prove_wide_fibonacci(self, a, b, n_cols, pow_bits=10, log_blowup=1, log_last_layer=0, n_queries=70):
        """Columns 0 and 1 from the caller (host), col[k+2] = col[k]^2 + col[k+1]^2."""
        from gpustark.backend import eval_blob_wide_fibonacci, to_device
        t0 = time.perf_counter()
        B = self.B
        log_n = int(len(a)).bit_length() - 1
        lift = log_n + log_blowup
        E = log_n + 1
        # trace (wide_fibonacci/mod.rs gen_trace), on the host
        cols = [np.asarray(a, np.uint64), np.asarray(b, np.uint64)]
        for _ in range(2, n_cols):
            cols.append((cols[-2] * cols[-2] + cols[-1] * cols[-1]) % P)
        trace = [to_device(c.astype(np.uint32)) for c in cols]
        tw = self._call("precompute_twiddles", lift)
        ch = Blake2sChannel()
        # preprocessed tree: no columns (MerkleProver::commit of nothing)
        roots = [hashlib.blake2s(b"", digest_size=32).digest()]
        ch.mix_root(roots[0])
        # trace tree: interpolate, extend, commit (TreeBuilder::extend_evals + commit)
        self._call("interpolate_columns", trace, log_n, tw)
        lde = self._call("evaluate_polynomials", trace, lift, tw)
        trace_layers = self.merkle_commit(lde)
        roots.append(self.root(trace_layers))
        ch.mix_root(roots[1])
        # prove_ex: composition polynomial (DomainEvaluationAccumulator + component prover)
        random_coeff = ch.draw_secure_felt()
        nc = n_cols - 2
        pw = [t.cpu().numpy().view(np.uint32) for t in self._call("generate_secure_powers", random_coeff, nc)]
        powers = [tuple(int(pw[c][k]) for c in range(4)) for k in range(nc)][::-1]
        on_domain = lde if lift == E else self._call("evaluate_polynomials", trace, E, tw)
        trace_coset_log = log_n
        den = []
        for i in range(1 << (E - trace_coset_log)):
            # coset_vanishing(CanonicCoset(log_n), eval_domain.at(i)) = pi^(log_n - 1)(x)
            x, _ = index_point((1 << (31 - (E + 1))) + i * (1 << (31 - (E - 1))))
            for _ in range(trace_coset_log - 1):
                x = double_x(x)
            den.append(m_inv(x))
        den = [den[bitrev(i, E - trace_coset_log)] for i in range(len(den))]
        acc = [torch.zeros(1 << E, dtype=torch.int32, device="cuda") for _ in range(4)]
        self._call("evaluate_constraint_quotients_on_domain", acc, [], on_domain, [], powers, den, log_n, E, nc,
                   eval_blob_wide_fibonacci(log_n), should_accumulate=True)
        self._call("interpolate_columns", acc, E, tw)  # finalize: one size, lift is the identity
        half = 1 << (E - 1)
        parts = [c[:half].clone() for c in acc] + [c[half:].clone() for c in acc]  # split_at_mid
        comp_lde = self._call("evaluate_polynomials", parts, E - 1 + log_blowup, tw)
        comp_layers = self.merkle_commit(comp_lde)
        roots.append(self.root(comp_layers))
        ch.mix_root(roots[2])
        oods = ch.random_point()
        oods8 = list(oods[0]) + list(oods[1])
        # prove_values: barycentric OODS evaluation (store_polynomials_coefficients off)
        weights = self._call("barycentric_weights", lift, oods8)
        sampled = [[], [[tuple(self._call("barycentric_eval_at_point", c, weights))] for c in lde],
                   [[tuple(self._call("barycentric_eval_at_point", c, weights))] for c in comp_lde]]
        ch.mix_felts([v for tree in sampled for col in tree for v in col])
        quot_coeff = ch.draw_secure_felt()
        # compute_fri_quotients: one size, one sample point -> one batch
        columns = list(lde) + list(comp_lde)
        values = [col[0] for tree in sampled for col in tree]
        rand, cur = [], ONE
        for _ in values:
            rand.append(cur)
            cur = q_mul(cur, quot_coeff)
        py = oods[1]
        c_line = q_sub(q_conj(py), py)
        aa, bb, cc = [], [], []
        for v, r in zip(values, rand):
            a_ = q_sub(q_conj(v), v)
            b_ = q_sub(q_mul(v, c_line), q_mul(a_, py))
            aa.append(q_mul(r, a_))
            bb.append(q_mul(r, b_))
            cc.append(q_mul(r, c_line))
        partial = self._call("accumulate_numerators", columns, lift, list(range(len(columns))), bb, cc)
        first_linear = (0, 0, 0, 0)
        for x in aa:
            first_linear = q_add(first_linear, x)
        quot = self._call("compute_quotients_and_combine", [(partial, lift, first_linear, oods8)], lift)
        # FriProver::commit
        first_layers = self.merkle_commit(quot)
        fri_roots = [self.root(first_layers)]
        ch.mix_root(fri_roots[0])
        alpha = ch.draw_secure_felt()
        line = [torch.zeros(1 << (lift - 1), dtype=torch.int32, device="cuda") for _ in range(4)]
        self._call("fold_circle_into_line", line, quot, lift, alpha, tw)
        last_log = log_last_layer + log_blowup
        inner = []  # (planes, layers, log)
        cur_log = lift - 1
        while cur_log > last_log:
            layers = self.merkle_commit(line)
            r = self.root(layers)
            ch.mix_root(r)
            alpha = ch.draw_secure_felt()
            inner.append((line, layers, cur_log, r))
            line = self._call("fold_line", line, cur_log, alpha, tw)
            cur_log -= 1
        # last layer: interpolate on the host (LineEvaluation::interpolate)
        lv = [c.cpu().numpy().view(np.uint32) for c in line]
        n_last = 1 << last_log
        vals = [tuple(int(lv[k][i]) for k in range(4)) for i in range(n_last)]
        vals = [vals[bitrev(i, last_log)] for i in range(n_last)]
        size, l = n_last, last_log
        while size > 1:  # line_ifft on half_odds(l), doubling each round
            for c0 in range(0, n_last, size):
                for i in range(size // 2):
                    x, _ = index_point((1 << (31 - (l + 2))) + i * (1 << (31 - l)))
                    xi = m_inv(x)
                    u, v = vals[c0 + i], vals[c0 + size // 2 + i]
                    vals[c0 + i] = q_add(u, v)
                    vals[c0 + size // 2 + i] = q_scale(q_sub(u, v), xi)
            size //= 2
            l -= 1
        ninv = m_inv(n_last)
        coeffs = [q_scale(v, ninv) for v in vals]  # bit-reversed order
        ordered = [coeffs[bitrev(i, last_log)] for i in range(n_last)]
        keep = 1 << log_last_layer
        assert all(v == (0, 0, 0, 0) for v in ordered[keep:]), "invalid degree"
        last_poly = [ordered[:keep][bitrev(i, log_last_layer)] for i in range(keep)]
        ch.mix_felts(last_poly)
        # proof of work, queries
        nonce = self._call("grind", ch.digest, pow_bits)
        ch.mix_u64(nonce)
        queries = sorted(set(ch.draw_queries(lift, n_queries)))

        # FriProver::decommit
        def fri_layer_decommit(planes, layers, log, qs, root):
            pos, witness = [], []
            i = 0
            while i < len(qs):
                start = (qs[i] >> 1) << 1
                for p in (start, start + 1):
                    pos.append(p)
                    if i < len(qs) and qs[i] == p:
                        i += 1
                    else:
                        witness.append(p)
            wv = self._call("batch_at_multi", planes, witness) if witness else np.zeros(0, np.uint32)
            wq = [tuple(int(x) for x in wv[4 * k: 4 * k + 4]) for k in range(len(witness))]
            _, hw, cw = self.merkle_decommit(layers, {log: pos}, planes)
            return (wq, hw, cw, root)

        fri_first = fri_layer_decommit(quot, first_layers, lift, queries, fri_roots[0])
        fri_inner = []
        qs = sorted({q >> 1 for q in queries})
        for planes, layers, log, r in inner:
            fri_inner.append(fri_layer_decommit(planes, layers, log, qs, r))
            qs = sorted({q >> 1 for q in qs})
        # tree decommitments (tree 0 has no columns: nothing to decommit)
        tree_dec = [([], [], [])]
        for layers, cols_ in ((trace_layers, lde), (comp_layers, comp_lde)):
            tree_dec.append(self.merkle_decommit(layers, {lift: queries}, list(cols_)))
        t1 = time.perf_counter()
        # serialise
        w = Writer()
        w.u32(pow_bits)
        w.u32(log_blowup)
        w.u32(log_last_layer)
        w.u64(n_queries)
        w.u32(1)
        w.u8(0)
        w.u64(3)
        for r in roots:
            w.b += r
        w.u64(3)
        for tree in sampled:
            w.u64(len(tree))
            for col in tree:
                w.u64(len(col))
                for v in col:
                    w.qm(v)
        w.u64(3)
        for q, hw, cw in tree_dec:
            w.decommitment(hw, cw)
        w.u64(3)
        for q, hw, cw in tree_dec:
            w.u64(len(q))
            for v in q:
                w.u32(int(v))
        w.u64(nonce)
        w.fri_layer(fri_first)
        w.u64(len(fri_inner))
        for L in fri_inner:
            w.fri_layer(L)
        w.u64(len(last_poly))
        for q in last_poly:
            w.qm(q)
        w.u32(log_last_layer)
        self.elapsed_s = t1 - t0
        return bytes(w.b)
