"""Test infrastructure (oracle): a pure-Python restatement of the Poseidon252
Merkle hasher and channel of the reference, used only by tests/ to check the
library's GPU kernels. Nothing in the library imports it.

The reference takes the hash itself from a third-party crate that is not in
its tree: ``starknet-crypto = 0.6.2`` (``poseidon_hash``,
``poseidon_hash_many``, ``poseidon_permute_comp``; crates/stwo/Cargo.toml:42).
Restated here is that crate's published algorithm, Starknet's Poseidon: the
Hades permutation over the STARK field p = 2^251 + 17·2^192 + 1 with state
width 3, S-box x^3, 4 full rounds, 83 partial rounds (S-box on the last
element only) and 4 full rounds, the MDS matrix [[3, 1, 1], [1, -1, 1],
[1, 1, -2]], and round constants SHA-256("Hades" || decimal index) mod p
for index 3·round + element. (``poseidon_permute_comp`` is the same
permutation with its partial-round constants folded; the results are equal.)

Pinned by the reference's own known answers (tests/golden/reference_vectors.json,
extracted from crates/stwo/src/core/vcs/poseidon252_merkle.rs test_vector and
crates/stwo/src/core/channel/poseidon252.rs test_mix_u64 / test_mix_u32s).
"""
import hashlib

P = 2 ** 251 + 17 * 2 ** 192 + 1
WIDTH = 3
FULL_ROUNDS = 8
PARTIAL_ROUNDS = 83
N_ROUNDS = FULL_ROUNDS + PARTIAL_ROUNDS
M31 = (1 << 31) - 1


def round_constant(index):
    return int.from_bytes(hashlib.sha256(b"Hades%d" % index).digest(), "big") % P


ROUND_CONSTANTS = [[round_constant(WIDTH * r + j) for j in range(WIDTH)] for r in range(N_ROUNDS)]


def _round(s, r, full):
    s = [(x + c) % P for x, c in zip(s, ROUND_CONSTANTS[r])]
    if full:
        s = [pow(x, 3, P) for x in s]
    else:
        s[2] = pow(s[2], 3, P)
    t = (s[0] + s[1] + s[2]) % P
    return [(t + 2 * s[0]) % P, (t - 2 * s[1]) % P, (t - 3 * s[2]) % P]


def permute(state):
    """Hades permutation of a 3-element state (poseidon_permute_comp)."""
    s = [x % P for x in state]
    r = 0
    for _ in range(FULL_ROUNDS // 2):
        s = _round(s, r, True)
        r += 1
    for _ in range(PARTIAL_ROUNDS):
        s = _round(s, r, False)
        r += 1
    for _ in range(FULL_ROUNDS // 2):
        s = _round(s, r, True)
        r += 1
    return s


def hash2(x, y):
    """poseidon_hash(x, y): capacity element 2."""
    return permute([x, y, 2])[0]


def hash_many(values):
    """poseidon_hash_many: absorb pairs, then 1 after the data (the element
    after a lone last value, or the first element after an even count)."""
    s = [0, 0, 0]
    i = 0
    while i + 2 <= len(values):
        s[0] = (s[0] + values[i]) % P
        s[1] = (s[1] + values[i + 1]) % P
        s = permute(s)
        i += 2
    rem = len(values) - i
    if rem == 1:
        s[0] = (s[0] + values[i]) % P
    s[rem] = (s[rem] + 1) % P
    return permute(s)[0]


def length_padding(felt, n):
    """add_length_padding (crates/stwo/src/core/vcs/utils.rs:32-35): + n·2^248."""
    return (felt + n * 2 ** 248) % P


def felt_from_m31s(word):
    """construct_felt252_from_m31s (core/vcs/poseidon252_merkle.rs:44-72): up to
    8 values, each shifted in by 31 bits; a shorter word gets its length at
    bit 248."""
    f = 0
    for v in word:
        f = (f << 31) | int(v)
    if len(word) < 8:
        f = length_padding(f, len(word))
    return f % P


def hash_node(children, column_values):
    """Poseidon252MerkleHasher::hash_node (core/vcs/poseidon252_merkle.rs:18-40)."""
    values = []
    if children is not None:
        if len(column_values) == 0:
            return hash2(children[0], children[1])
        values += [children[0], children[1]]
    for i in range(0, len(column_values), 8):
        values.append(felt_from_m31s(column_values[i:i + 8]))
    return hash_many(values)


def commit_on_layer(log_size, prev, cols):
    """MerkleOps<Poseidon252MerkleHasher>::commit_on_layer (CPU backend
    prover/backend/cpu/poseidon252.rs): node i from children 2i, 2i+1 of `prev`
    (or none) and every column's value at row i."""
    n = 1 << log_size
    out = []
    for i in range(n):
        ch = (prev[2 * i], prev[2 * i + 1]) if prev is not None else None
        out.append(hash_node(ch, [int(c[i]) for c in cols]))
    return out


def to_bytes_be(felt):
    """The reference's device layout of one hash (32 bytes, big-endian)."""
    return int(felt).to_bytes(32, "big")


class Channel:
    """Poseidon252Channel (core/channel/poseidon252.rs:18-155)."""

    POW_PREFIX = 0x12345678

    def __init__(self, digest=0):
        self.digest = digest
        self.n_draws = 0

    def update_digest(self, d):
        self.digest = d % P
        self.n_draws = 0

    def mix_root(self, root):  # Poseidon252MerkleChannel::mix_root (core/vcs/poseidon252_merkle.rs:83-87)
        self.update_digest(hash2(self.digest, root))

    def mix_u64(self, v):
        self.update_digest(hash2(self.digest, v))

    def mix_u32s(self, data):
        padding_len = 6 - ((len(data) + 6) % 7)
        d = list(data) + [0] * padding_len
        felts = []
        for i in range(0, len(d), 7):
            f = 0
            for y in d[i:i + 7]:
                f = (f * 2 ** 32 + y) % P
            felts.append(f)
        if padding_len:
            felts[-1] = length_padding(felts[-1], 7 - padding_len)
        self.update_digest(hash_many([self.digest] + felts))

    def mix_felts(self, felts):
        """felts: QM31 values as 4-tuples of M31; two per felt252, leading 1."""
        res = [self.digest]
        for i in range(0, len(felts), 2):
            cur = 1
            for q in felts[i:i + 2]:
                for y in q:
                    cur = (cur * 2 ** 31 + int(y)) % P
            res.append(cur)
        self.update_digest(hash_many(res))

    def draw_felt252(self):
        s = permute([self.digest, self.n_draws, 3])
        self.n_draws += 1
        return s[0]

    def draw_base_felts(self):
        cur = self.draw_felt252()
        out = []
        for _ in range(8):
            cur, r = divmod(cur, 2 ** 31)
            out.append(r % M31)  # BaseField::reduce of a 31-bit value
        return out

    def draw_secure_felt(self):
        return tuple(self.draw_base_felts()[:4])

    def draw_secure_felts(self, n):
        flat = []
        out = []
        while len(out) < n:
            if len(flat) < 4:
                flat += self.draw_base_felts()
            out.append(tuple(flat[:4]))
            flat = flat[4:]
        return out

    def draw_u32s(self):
        cur = self.draw_felt252()
        out = []
        for _ in range(7):
            cur, r = divmod(cur, 2 ** 32)
            out.append(r)
        return out

    GRIND_LOW_BITS = 14  # prover/backend/simd/grind.rs:150

    def grind(self, pow_bits):
        """GrindOps<Poseidon252Channel>::grind (prover/backend/simd/grind.rs:
        152-190): the smallest (hi << 32) | low, low < 2^14, hi = 0, 1, ..."""
        pre = hash_many([self.POW_PREFIX, self.digest, pow_bits])
        hi = 0
        while True:
            for low in range(1 << self.GRIND_LOW_BITS):
                nonce = (hi << 32) | low
                h = hash2(pre, nonce) & ((1 << 128) - 1)
                tz = (h & -h).bit_length() - 1 if h else 128
                if tz >= pow_bits:
                    return nonce
            hi += 1

    def verify_pow_nonce(self, n_bits, nonce):
        pre = hash_many([self.POW_PREFIX, self.digest, n_bits])
        h = hash2(pre, nonce)
        low = h & ((1 << 128) - 1)
        tz = (low & -low).bit_length() - 1 if low else 128
        return tz >= n_bits
