"""Byte ranges of the sections of a serialised StarkProof, for tamper tests.

The layout is the one both provers write (bincode-1.x style: little-endian
fixed-width integers, u64 sequence lengths, a hash as 32 raw bytes, M31 as
u32, QM31 as 4 x u32) in the field order of the reference's serde structs:
CommitmentSchemeProof (crates/stwo/src/core/pcs/quotients.rs:29-38), FriProof
and FriLayerProof (core/fri.rs:363-398), MerkleDecommitment
(core/vcs/verifier.rs:13-22) and LinePoly (core/poly/line.rs:96-101).
"""
import struct


class _R:
    def __init__(self, b):
        self.b, self.o = b, 0

    def u32(self):
        v = struct.unpack_from("<I", self.b, self.o)[0]
        self.o += 4
        return v

    def u64(self):
        v = struct.unpack_from("<Q", self.b, self.o)[0]
        self.o += 8
        return v

    def skip(self, n):
        s = self.o
        self.o += n
        return (s, self.o)


def sections(proof: bytes):
    """[(name, start, end)] of every payload section (lengths excluded)."""
    r = _R(proof)
    out = []

    def add(name, rng):
        if rng[1] > rng[0]:
            out.append((name, rng[0], rng[1]))

    add("config", r.skip(24))  # pow_bits, log_blowup, log_last_layer, n_queries (u64), fold_step
    if proof[r.o]:
        add("config.lifting", r.skip(5))
    else:
        r.skip(1)
    n = r.u64()
    add("commitments", r.skip(32 * n))
    for t in range(r.u64()):
        s = r.o
        for c in range(r.u64()):
            r.skip(16 * r.u64())
        add(f"sampled_values[{t}]", (s, r.o))

    def decommitment(name):
        add(name + ".hash_witness", r.skip(32 * r.u64()))
        add(name + ".column_witness", r.skip(4 * r.u64()))

    for t in range(r.u64()):
        decommitment(f"decommitments[{t}]")
    for t in range(r.u64()):
        add(f"queried_values[{t}]", r.skip(4 * r.u64()))
    add("proof_of_work", r.skip(8))

    def layer(name):
        add(name + ".fri_witness", r.skip(16 * r.u64()))
        decommitment(name + ".decommitment")
        add(name + ".commitment", r.skip(32))

    layer("fri.first")
    for i in range(r.u64()):
        layer(f"fri.inner[{i}]")
    add("fri.last_layer_poly", r.skip(16 * r.u64()))
    r.skip(4)
    assert r.o == len(proof), "trailing bytes"
    return out


def flip(proof: bytes, offset: int, bit: int = 0) -> bytes:
    b = bytearray(proof)
    b[offset] ^= 1 << bit
    return bytes(b)
