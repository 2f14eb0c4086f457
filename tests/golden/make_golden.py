"""Extracts the reference's known-answer vectors for the prover hot path into
``reference_vectors.json``.

The reference is a Rust crate that cannot be built in this container, so its
own test files are read as text and the literal expected values are copied
out. Run from the repository root, in the container that holds the reference:

    python tests/golden/make_golden.py <reference checkout>

Sources (paths inside the reference checkout):
  crates/stwo/src/core/vcs/blake2_hash.rs      single_hash_test   (Blake2s of b"a")
  crates/stwo/src/core/channel/blake2s.rs      test_mix_u64, test_mix_u32s (channel digests)
  crates/stwo/src/core/fields/m31.rs           doc-tests of partial_reduce / reduce
  crates/stwo/src/core/circle.rs               M31_CIRCLE_GEN, SECURE_FIELD_CIRCLE_GEN,
                                               test_secure_field_circle_gen prime factors
  crates/stwo/src/prover/backend/cuda/poly.rs  test_interpolate_from_fib (twiddle tree literals)
  crates/stwo/src/core/vcs/poseidon252_merkle.rs  test_vector (Poseidon252 hash_node)
  crates/stwo/src/core/channel/poseidon252.rs     test_mix_u64, test_mix_u32s (Poseidon252 channel)
"""
import json
import os
import re
import sys


def _read(root, rel):
    with open(os.path.join(root, rel)) as f:
        return f.read()


def _byte_array_after(text, marker):
    # the expected digest is the first bracketed list of hex bytes after `marker`
    i = text.index(marker)
    m = re.search(r"\[\s*0x", text[i:])
    j = i + m.start()
    block = text[j:text.index("]", j) + 1]
    return [int(x, 16) for x in re.findall(r"0x([0-9a-fA-F]+)", block)]


def main(root):
    out = {}
    bh = _read(root, "crates/stwo/src/core/vcs/blake2_hash.rs")
    m = re.search(r'Blake2sHasher::hash\(b"a"\);\s*assert_eq!\(\s*hash_a\.to_string\(\),\s*"([0-9a-f]{64})"', bh)
    out["blake2s_a"] = m.group(1)

    ch = _read(root, "crates/stwo/src/core/channel/blake2s.rs")
    out["channel_mix_u64"] = {
        "value": int(re.search(r"mix_u64\((0x[0-9a-fA-F]+)\)", ch).group(1), 16),
        "digest": _byte_array_after(ch, "let digest_bytes: [u8; 32] = digest_64.into();"),
        "u32s": [int(x, 16) for x in re.search(r"mix_u32s\(&\[(0x[0-9a-fA-F]+),\s*(0x[0-9a-fA-F]+)\]\)", ch).groups()],
    }
    m = re.search(r"pub fn test_mix_u32s.*?mix_u32s\(&\[([0-9,\s]+)\]\)", ch, re.S)
    out["channel_mix_u32s"] = {
        "words": [int(x) for x in m.group(1).split(",") if x.strip()],
        "digest": _byte_array_after(ch, "pub fn test_mix_u32s"),
    }

    m31 = _read(root, "crates/stwo/src/core/fields/m31.rs")
    out["m31_partial_reduce"] = {"input_expr": "2*P-19", "expected_expr": "P-19",
                                 "found": "let val = 2 * P - 19;" in m31}
    out["m31_reduce"] = {"input_expr": "P^2-19", "expected_expr": "P-19",
                         "found": "let val = (P as u64).pow(2) - 19;" in m31}

    circ = _read(root, "crates/stwo/src/core/circle.rs")
    g = re.search(r"M31_CIRCLE_GEN: CirclePoint<M31> = CirclePoint \{\s*x: M31::from_u32_unchecked\((\d+)\),\s*y: M31::from_u32_unchecked\((\d+)\)", circ)
    out["m31_circle_gen"] = [int(g.group(1)), int(g.group(2))]
    sg = re.search(r"SECURE_FIELD_CIRCLE_GEN: CirclePoint<SecureField> = CirclePoint \{\s*x: SecureField::from_u32_unchecked\(([\d,\s]+)\),\s*y: SecureField::from_u32_unchecked\(([\d,\s]+)\)", circ)
    out["secure_circle_gen"] = [[int(v) for v in sg.group(1).split(",")], [int(v) for v in sg.group(2).split(",")]]
    pf = re.search(r"let prime_factors = \[(.*?)\];", circ, re.S).group(1)
    out["secure_circle_order_factors"] = [[int(a), int(b)] for a, b in re.findall(r"\((\d+),\s*(\d+)\)", pf)]

    # Twiddle tree literals of the CUDA backend's interpolation test
    # (cuda/poly.rs, test_interpolate_from_fib): twiddles and itwiddles of
    # the root coset, which pin the twiddle-tree layout.
    poly = _read(root, "crates/stwo/src/prover/backend/cuda/poly.rs")
    body = poly[poly.index("fn test_interpolate_from_fib"):]
    def vec_of(name):
        block = re.search(r"let %s = vec!\[(.*?)\];" % name, body, re.S).group(1)
        return [int(v) for v in re.findall(r"BaseField::from\((\d+)\)", block)]
    rc = body[body.index("let root_coset"):]
    out["cuda_interpolate_twiddle_tree"] = {
        "root_initial_index": int(re.search(r"initial_index: CirclePointIndex\((\d+)\)", rc).group(1)),
        "root_step_index": int(re.search(r"step_size: CirclePointIndex\((\d+)\)", rc).group(1)),
        "root_log_size": int(re.search(r"log_size: (\d+)", rc).group(1)),
        "twiddles": vec_of("twiddles"),
        "itwiddles": vec_of("itwiddles"),
    }

    # Poseidon252 Merkle hasher: hash_node(None, [0, 1]) and
    # hash_node(Some((1, 2)), [3]) as decimal felt252 strings
    pm = _read(root, "crates/stwo/src/core/vcs/poseidon252_merkle.rs")
    tv = pm[pm.index("fn test_vector"):]
    decs = re.findall(r'from_dec_str\(\s*"(\d+)"', tv)[:2]
    m1 = re.search(r"hash_node\(None, &\[m31!\((\d+)\), m31!\((\d+)\)\]\)", tv)
    m2 = re.search(r"FieldElement252::from\((\d+)u32\), FieldElement252::from\((\d+)u32\)\)\),\s*&\[m31!\((\d+)\)\]", tv)
    out["poseidon252_hash_node"] = [
        {"children": None, "columns": [int(m1.group(1)), int(m1.group(2))], "hash": decs[0]},
        {"children": [int(m2.group(1)), int(m2.group(2))], "columns": [int(m2.group(3))], "hash": decs[1]},
    ]
    # Poseidon252 channel: digest after mix_u64 / mix_u32s from the default channel
    pc = _read(root, "crates/stwo/src/core/channel/poseidon252.rs")
    t64 = pc[pc.index("fn test_mix_u64"):]
    t32 = pc[pc.index("fn test_mix_u32s"):]
    out["poseidon252_channel_mix_u64"] = {
        "value": int(re.search(r"mix_u64\((0x[0-9a-fA-F]+)\)", t64).group(1), 16),
        "digest": re.search(r'from_hex_be\(\s*"(0x[0-9a-fA-F]+)"', t64).group(1),
    }
    out["poseidon252_channel_mix_u32s"] = {
        "words": [int(x) for x in re.search(r"mix_u32s\(&\[([0-9,\s]+)\]\)", t32).group(1).split(",") if x.strip()],
        "digest": re.search(r'from_hex_be\(\s*"(0x[0-9a-fA-F]+)"', t32).group(1),
    }

    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <reference checkout>")
    main(sys.argv[1])
