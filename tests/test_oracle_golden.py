"""Pins the CPU oracle against the reference's known-answer vectors and against
independent definitions (hashlib's Blake2s, the circle-polynomial basis)."""
import hashlib
import json
import os

import numpy as np
import pytest

import pyoracle as O

P = O.P
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")))


def test_blake2s_known_answer():
    # crates/stwo/src/core/vcs/blake2_hash.rs single_hash_test
    assert O.blake2s(b"a").hex() == GOLDEN["blake2s_a"]


@pytest.mark.parametrize("n", [0, 1, 3, 31, 32, 33, 63, 64, 65, 100, 127, 128, 129, 400, 632, 1000])
def test_blake2s_matches_rfc7693(n):
    rng = np.random.default_rng(n)
    data = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
    assert O.blake2s(data) == hashlib.blake2s(data, digest_size=32).digest()


def test_channel_known_answers():
    # crates/stwo/src/core/channel/blake2s.rs test_mix_u64 / test_mix_u32s
    g = GOLDEN["channel_mix_u64"]
    assert O.channel_mix_u64(g["value"]) == bytes(g["digest"])
    assert O.channel_mix_u32s(g["u32s"]) == bytes(g["digest"])
    g = GOLDEN["channel_mix_u32s"]
    assert O.channel_mix_u32s(g["words"]) == bytes(g["digest"])


def test_m31_doc_vectors():
    L = O.lib()
    assert GOLDEN["m31_partial_reduce"]["found"] and GOLDEN["m31_reduce"]["found"]
    assert L.oracle_m31_partial_reduce(2 * P - 19) == P - 19
    assert L.oracle_m31_reduce(P * P - 19) == P - 19
    rng = np.random.default_rng(1)
    for _ in range(200):
        a, b = (int(x) for x in rng.integers(0, P, 2))
        assert L.oracle_m31_mul(a, b) == a * b % P
        if a:
            assert L.oracle_m31_mul(L.oracle_m31_inv(a), a) == 1


def test_qm31_inverse():
    rng = np.random.default_rng(2)
    for _ in range(50):
        a = rng.integers(0, P, 4).astype(np.uint32)
        ai = np.zeros(4, np.uint32)
        O.lib().oracle_qm31_inv(O.u32(a)[1], ai.ctypes.data_as(O.U32P))
        r = np.zeros(4, np.uint32)
        O.lib().oracle_qm31_mul(O.u32(a)[1], O.u32(ai)[1], r.ctypes.data_as(O.U32P))
        assert list(r) == [1, 0, 0, 0]


def test_circle_generators():
    # crates/stwo/src/core/circle.rs: M31_CIRCLE_GEN has order 2^31.
    xy = np.zeros(2, np.uint32)
    O.lib().oracle_index_to_point(1, xy.ctypes.data_as(O.U32P))
    assert list(xy) == GOLDEN["m31_circle_gen"]
    O.lib().oracle_index_to_point(1 << 30, xy.ctypes.data_as(O.U32P))
    assert list(xy) == [P - 1, 0]
    # test_secure_field_circle_gen: GEN^(P^4-1) = identity, GEN^((P^4-1)/p) != identity.
    order = P ** 4 - 1
    prod = 1
    for p, e in GOLDEN["secure_circle_order_factors"]:
        prod *= p ** e
    assert prod == order
    out = np.zeros(8, np.uint32)

    def gen_mul(s):
        O.lib().oracle_secure_gen_mul(s & (2 ** 64 - 1), s >> 64, out.ctypes.data_as(O.U32P))
        return list(out)

    assert gen_mul(1) == GOLDEN["secure_circle_gen"][0] + GOLDEN["secure_circle_gen"][1]
    assert gen_mul(order) == [1, 0, 0, 0, 0, 0, 0, 0]
    for p, _ in GOLDEN["secure_circle_order_factors"]:
        assert gen_mul(order // p) != [1, 0, 0, 0, 0, 0, 0, 0]


def _domain_points(log_n):
    """Canonic circle domain points in natural order, by index arithmetic."""
    pts = []
    half = 1 << (log_n - 1)
    init = 1 << (31 - (log_n + 1))       # half_odds(log_n - 1).initial_index
    step = 1 << (31 - (log_n - 1))
    xy = np.zeros(2, np.uint32)
    for i in range(1 << log_n):
        idx = (init + step * i) % (1 << 31) if i < half else (-(init + step * (i - half))) % (1 << 31)
        O.lib().oracle_index_to_point(idx, xy.ctypes.data_as(O.U32P))
        pts.append((int(xy[0]), int(xy[1])))
    return pts


def _bitrev(i, n):
    return int(format(i, "0{}b".format(n))[::-1], 2) if n else i


@pytest.mark.parametrize("log_n", [1, 2, 3, 4, 5, 7])
def test_fft_matches_basis_definition(log_n):
    """evaluate() at bit-reversed position i equals the coefficient polynomial
    folded at domain point i (the circle-FFT basis, cpu/circle.rs:82-98)."""
    rng = np.random.default_rng(log_n)
    coeffs = rng.integers(0, P, 1 << log_n).astype(np.uint32)
    evals = O.evaluate(coeffs, log_n)
    pts = _domain_points(log_n)
    for i in range(1 << log_n):
        x, y = pts[i]
        v = O.eval_at_point(coeffs, [x, 0, 0, 0, y, 0, 0, 0])
        assert list(v) == [int(evals[_bitrev(i, log_n)]), 0, 0, 0]
    back = O.interpolate(evals, log_n)
    assert np.array_equal(back, coeffs)


@pytest.mark.parametrize("log_n", [8, 12, 16])
def test_fft_roundtrip_and_lde(log_n):
    rng = np.random.default_rng(log_n)
    coeffs = rng.integers(0, P, 1 << log_n).astype(np.uint32)
    ev = O.evaluate(coeffs, log_n, root_log=log_n + 1)
    assert np.array_equal(O.interpolate(ev, log_n, root_log=log_n + 1), coeffs)
    lde = O.evaluate(coeffs, log_n + 1, root_log=log_n + 1)
    back = O.interpolate(lde, log_n + 1, root_log=log_n + 1)
    assert np.array_equal(back[: 1 << log_n], coeffs) and not back[1 << log_n:].any()


def test_merkle_layer_is_blake2s_of_bytes():
    rng = np.random.default_rng(3)
    cols = [rng.integers(0, P, 8).astype(np.uint32) for _ in range(5)]
    leaves = O.commit_on_layer(3, None, cols)
    for i in range(8):
        data = b"".join(int(c[i]).to_bytes(4, "little") for c in cols)
        assert bytes(leaves[i]) == hashlib.blake2s(data, digest_size=32).digest()
    nodes = O.commit_on_layer(2, leaves.reshape(-1), cols[:2])
    for i in range(4):
        data = bytes(leaves[2 * i]) + bytes(leaves[2 * i + 1]) + b"".join(int(c[i]).to_bytes(4, "little") for c in cols[:2])
        assert bytes(nodes[i]) == hashlib.blake2s(data, digest_size=32).digest()
    # an empty tree is the hash of the empty string (prover.rs:23-27)
    assert O.merkle_root([]) == hashlib.blake2s(b"", digest_size=32).digest()


def test_grind_is_smallest_nonce():
    digest = hashlib.blake2s(b"grind", digest_size=32).digest()
    nonce = O.grind(digest, 8)
    assert O.verify_pow(digest, 8, nonce)
    assert not any(O.verify_pow(digest, 8, n) for n in range(nonce))


def _qm(a):
    return [int(v) for v in a]


def test_fold_line_formula():
    """fold_line: f0,f1 = ibutterfly(f(x), f(-x), 1/x); out = f0 + alpha f1."""
    rng = np.random.default_rng(4)
    log_n = 4
    ev = rng.integers(0, P, (1 << log_n, 4)).astype(np.uint32)
    alpha = rng.integers(0, P, 4).astype(np.uint32)
    out = O.fold_line(ev, log_n, alpha)
    # LineDomain(half_odds(4)): x of coset points; bit-reversed pair index.
    init = 1 << (31 - (log_n + 2))
    step = 1 << (31 - log_n)
    xy = np.zeros(2, np.uint32)
    L = O.lib()
    for i in range(1 << (log_n - 1)):
        j = _bitrev(i << 1, log_n)
        L.oracle_index_to_point((init + step * j) % (1 << 31), xy.ctypes.data_as(O.U32P))
        xinv = L.oracle_m31_inv(int(xy[0]))
        f0 = [(int(a) + int(b)) % P for a, b in zip(ev[2 * i], ev[2 * i + 1])]
        f1 = [((int(a) - int(b)) % P) * xinv % P for a, b in zip(ev[2 * i], ev[2 * i + 1])]
        r = np.zeros(4, np.uint32)
        L.oracle_qm31_mul(O.u32(alpha)[1], O.u32(np.array(f1, np.uint32))[1], r.ctypes.data_as(O.U32P))
        expect = [(a + int(b)) % P for a, b in zip(f0, r)]
        assert _qm(out[i]) == expect


def test_twiddle_tree_matches_reference_literals():
    """Twiddles and itwiddles of Coset::half_odds(6), as written out in the
    reference CUDA backend's interpolation test: pins the twiddle-tree layout
    (per-level x coordinates, bit-reversed, padded) and its inverses."""
    g = GOLDEN["cuda_interpolate_twiddle_tree"]
    log = g["root_log_size"]
    assert g["root_initial_index"] == 1 << (31 - log - 2) and g["root_step_index"] == 1 << (31 - log)
    tw, itw = O.twiddles_half_odds(log)
    assert [int(v) for v in tw] == g["twiddles"]
    assert [int(v) for v in itw] == g["itwiddles"]


def test_lifted_leaves_follow_the_reference_lifting_table():
    """The lifting example of the reference's lifted build_leaves doc comment
    (cpu/merkle_lifted.rs): a size-8 column in bit-reversed order
    a e c g b f d h, lifted to 16 leaves, reads a e a e c g c g b f b f d h d h."""
    col = np.arange(10, 18, dtype=np.uint32)  # a..h = 10..17 in natural order
    a, b, c, d, e, f, g, h = [int(v) for v in col]
    bitrev = [a, e, c, g, b, f, d, h]
    lifted = [a, e, a, e, c, g, c, g, b, f, b, f, d, h, d, h]
    leaves = O.lifted_leaves([np.array(bitrev, np.uint32)], 4)
    for i, v in enumerate(lifted):
        assert bytes(leaves[i]) == hashlib.blake2s(int(v).to_bytes(4, "little")).digest()


def test_lifted_leaves_order_and_empty():
    """Columns are hashed in increasing size order (stable); no columns give one
    leaf, the hash of nothing."""
    rng = np.random.default_rng(5)
    c3 = rng.integers(0, P, 8, dtype=np.int64).astype(np.uint32)
    c1 = rng.integers(0, P, 2, dtype=np.int64).astype(np.uint32)
    c3b = rng.integers(0, P, 8, dtype=np.int64).astype(np.uint32)
    leaves = O.lifted_leaves([c3, c1, c3b], 3)
    for i in range(8):
        j1 = ((i >> 3) << 1) + (i & 1)
        msg = b"".join(int(v).to_bytes(4, "little") for v in (c1[j1], c3[i], c3b[i]))
        assert bytes(leaves[i]) == hashlib.blake2s(msg).digest()
    assert bytes(O.lifted_leaves([], 5)[0]) == hashlib.blake2s(b"").digest()


# ------------------------------------------------------------ Poseidon252
def test_poseidon252_hash_node_known_answers():
    """The Poseidon252 restatement (starknet-crypto 0.6.2's Starknet Poseidon)
    reproduces the reference's hash_node vectors."""
    import poseidon252 as PS
    for case in GOLDEN["poseidon252_hash_node"]:
        ch = tuple(case["children"]) if case["children"] is not None else None
        assert PS.hash_node(ch, case["columns"]) == int(case["hash"])


def test_poseidon252_channel_known_answers():
    import poseidon252 as PS
    c = PS.Channel()
    c.mix_u64(GOLDEN["poseidon252_channel_mix_u64"]["value"])
    assert c.digest == int(GOLDEN["poseidon252_channel_mix_u64"]["digest"], 16)
    c = PS.Channel()
    c.mix_u32s(GOLDEN["poseidon252_channel_mix_u32s"]["words"])
    assert c.digest == int(GOLDEN["poseidon252_channel_mix_u32s"]["digest"], 16)


def test_poseidon252_channel_draw_counts_and_ranges():
    """The draw bookkeeping of the reference's test_channel_draws, and the
    ranges of drawn values."""
    import poseidon252 as PS
    c = PS.Channel()
    w = c.draw_u32s()
    assert c.n_draws == 1 and len(w) == 7 and all(0 <= x < 2 ** 32 for x in w)
    f = c.draw_secure_felts(9)
    assert c.n_draws == 6 and len(f) == 9 and len(set(f)) == 9
    assert all(0 <= v < PS.M31 for q in f for v in q)
    c.mix_felts(f[:3])
    assert c.n_draws == 0


def test_poseidon252_permutation_is_a_bijection_sample():
    """Distinct inputs give distinct outputs and the state stays in the field."""
    import poseidon252 as PS
    outs = {tuple(PS.permute([i, 2 * i + 1, 3])) for i in range(32)}
    assert len(outs) == 32
    assert all(0 <= v < PS.P for o in outs for v in o)


# ---------------------------------------- Poseidon252 in the C++ oracle prover
def _felt_bytes(v):
    return int(v).to_bytes(32, "big")


def test_cpp_poseidon252_known_answers():
    """The C++ restatement used by the oracle prover reproduces the
    reference's hash_node and channel vectors."""
    for case in GOLDEN["poseidon252_hash_node"]:
        cols = [np.array([v], np.uint32) for v in case["columns"]]
        prev = None
        if case["children"] is not None:
            prev = np.frombuffer(b"".join(_felt_bytes(c) for c in case["children"]), np.uint8)
        got = O.p252_commit_on_layer(0, prev, cols)
        assert int.from_bytes(bytes(got[0]), "big") == int(case["hash"])
    zero = _felt_bytes(0)
    d, nd, _ = O.p252_channel_op(zero, 0, "mix_u64", v=GOLDEN["poseidon252_channel_mix_u64"]["value"])
    assert int.from_bytes(d, "big") == int(GOLDEN["poseidon252_channel_mix_u64"]["digest"], 16) and nd == 0
    d, nd, _ = O.p252_channel_op(zero, 0, "mix_u32s", words=GOLDEN["poseidon252_channel_mix_u32s"]["words"])
    assert int.from_bytes(d, "big") == int(GOLDEN["poseidon252_channel_mix_u32s"]["digest"], 16)


def test_cpp_poseidon252_matches_python_restatement():
    """Permutations, Merkle layers (0..17 columns, with and without children)
    and a random script of channel operations agree with the pure-Python
    restatement."""
    import poseidon252 as PS
    rng = np.random.default_rng(3)
    states = [[0, 0, 0], [PS.P - 1] * 3] + [[int.from_bytes(rng.bytes(32), "big") % PS.P for _ in range(3)]
                                            for _ in range(6)]
    out = O.p252_permute(b"".join(_felt_bytes(v) for s in states for v in s))
    assert [int.from_bytes(out[32 * i:32 * i + 32], "big") for i in range(3 * len(states))] == \
        [v for s in states for v in PS.permute(s)]
    for n_cols in [0, 1, 7, 8, 9, 17]:
        for with_prev in [False, True]:
            n = 8
            cols = [rng.integers(0, PS.M31, n, dtype=np.int64).astype(np.uint32) for _ in range(n_cols)]
            prev = [int.from_bytes(rng.bytes(32), "big") % PS.P for _ in range(2 * n)] if with_prev else None
            pb = np.frombuffer(b"".join(_felt_bytes(v) for v in prev), np.uint8) if prev else None
            if n_cols == 0 and not with_prev:
                got = O.p252_commit_on_layer(0, None, [])
                assert int.from_bytes(bytes(got[0]), "big") == PS.hash_node(None, [])
                continue
            got = O.p252_commit_on_layer(3, pb, cols)
            assert [int.from_bytes(bytes(r), "big") for r in got] == PS.commit_on_layer(3, prev, cols)
    ch, d, nd = PS.Channel(), _felt_bytes(0), 0
    script = ["mix_root", "draw_secure_felts", "mix_felts", "draw_u32s", "mix_u64", "draw_secure_felts",
              "mix_u32s", "draw_u32s", "draw_secure_felts"]
    for op in script:
        if op == "mix_root":
            r = int.from_bytes(rng.bytes(32), "big") % PS.P
            d, nd, _ = O.p252_channel_op(d, nd, op, data=_felt_bytes(r))
            ch.mix_root(r)
        elif op == "mix_u64":
            v = int(rng.integers(0, 2 ** 63))
            d, nd, _ = O.p252_channel_op(d, nd, op, v=v)
            ch.mix_u64(v)
        elif op == "mix_u32s":
            w = [int(x) for x in rng.integers(0, 2 ** 32, 11, dtype=np.uint64)]
            d, nd, _ = O.p252_channel_op(d, nd, op, words=w)
            ch.mix_u32s(w)
        elif op == "mix_felts":
            f = [tuple(int(x) for x in rng.integers(0, PS.M31, 4)) for _ in range(5)]
            d, nd, _ = O.p252_channel_op(d, nd, op, words=[x for q in f for x in q])
            ch.mix_felts(f)
        elif op == "draw_secure_felts":
            d, nd, got = O.p252_channel_op(d, nd, op, n=3)
            assert got == [x for q in ch.draw_secure_felts(3) for x in q]
        else:
            d, nd, got = O.p252_channel_op(d, nd, op, n=2)
            assert got == ch.draw_u32s() + ch.draw_u32s()
        assert int.from_bytes(d, "big") == ch.digest and nd == ch.n_draws, op
    for bits in [0, 3, 8]:
        nonce = O.p252_grind(d, bits)
        assert nonce == PS.Channel(int.from_bytes(d, "big")).grind(bits)
        assert O.p252_verify_pow(d, bits, nonce)


def test_cpp_oracle_proves_with_poseidon252_channel():
    """The oracle prover runs with Poseidon252MerkleChannel; the proof differs
    from the Blake2s one and is deterministic."""
    a = O.prove("wide_fibonacci", 6, n_cols=8, merkle_channel="poseidon252")
    b = O.prove("wide_fibonacci", 6, n_cols=8, merkle_channel="poseidon252")
    c = O.prove("wide_fibonacci", 6, n_cols=8)
    assert a == b and a != c
