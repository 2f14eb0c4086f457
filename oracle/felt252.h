// ORACLE — test infrastructure only (see fields.h).
// Starknet's Poseidon hash over the STARK field, the Poseidon252 Merkle hasher
// and the Poseidon252 Fiat-Shamir channel.
//
// The reference takes the hash from a crate outside its tree,
// starknet-crypto 0.6.2 (crates/stwo/Cargo.toml:42: poseidon_hash,
// poseidon_hash_many, poseidon_permute_comp). Restated here from its published
// algorithm: the Hades permutation over p = 2^251 + 17·2^192 + 1, state width
// 3, S-box x^3, 4 full + 83 partial + 4 full rounds, MDS [[3,1,1],[1,-1,1],
// [1,1,-2]], round constant of (round r, element j) = SHA-256("Hades" ||
// decimal(3r + j)) read big-endian, mod p. The textbook (uncompressed) round
// form is used; SHA-256 is restated from FIPS 180-4 with its constants
// derived from the primes at start-up.
//
// Call sites followed:
//   crates/stwo/src/core/vcs/poseidon252_merkle.rs:18-87 (hash_node,
//       construct_felt252_from_m31s, mix_root)
//   crates/stwo/src/core/vcs/utils.rs:32-35              (add_length_padding)
//   crates/stwo/src/core/channel/poseidon252.rs:18-155   (channel)
//   crates/stwo/src/prover/backend/simd/grind.rs:148-190 (grind: smallest
//       (hi << 32) | low, low < 2^14)
// Pinned by the reference's known answers (poseidon252_merkle.rs test_vector,
// channel/poseidon252.rs test_mix_u64 / test_mix_u32s) through the tests.
#pragma once
#include <array>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include "fields.h"

namespace orc {
namespace p252 {

// 256-bit unsigned integer, little-endian 64-bit limbs.
struct U256 {
  uint64_t w[4] = {0, 0, 0, 0};
  bool operator==(const U256& o) const { return memcmp(w, o.w, sizeof w) == 0; }
};
using u128 = unsigned __int128;

inline const U256& prime() {
  static const U256 p = {{1ull, 0ull, 0ull, 0x0800000000000011ull}};
  return p;
}

inline bool geq(const U256& a, const U256& b) {
  for (int i = 3; i >= 0; i--)
    if (a.w[i] != b.w[i]) return a.w[i] > b.w[i];
  return true;
}
inline U256 add_raw(const U256& a, const U256& b, uint64_t& carry) {
  U256 r;
  u128 c = 0;
  for (int i = 0; i < 4; i++) {
    c += (u128)a.w[i] + b.w[i];
    r.w[i] = (uint64_t)c;
    c >>= 64;
  }
  carry = (uint64_t)c;
  return r;
}
inline U256 sub_raw(const U256& a, const U256& b, uint64_t& borrow) {
  U256 r;
  uint64_t br = 0;
  for (int i = 0; i < 4; i++) {
    u128 d = (u128)a.w[i] - b.w[i] - br;
    r.w[i] = (uint64_t)d;
    br = (uint64_t)(d >> 64) & 1;
  }
  borrow = br;
  return r;
}

// Field element in Montgomery form (R = 2^256), always below p.
struct Fe {
  U256 m;
  bool operator==(const Fe& o) const { return m == o.m; }
};

inline Fe fadd(const Fe& a, const Fe& b) {
  uint64_t c, br;
  U256 r = add_raw(a.m, b.m, c);
  if (c || geq(r, prime())) r = sub_raw(r, prime(), br);
  return {r};
}
inline Fe fsub(const Fe& a, const Fe& b) {
  uint64_t br, c;
  U256 r = sub_raw(a.m, b.m, br);
  if (br) r = add_raw(r, prime(), c);
  return {r};
}

// Montgomery product a·b·2^-256 mod p (operand-scanning form with one
// reduction step per limb; -p^-1 mod 2^64 = 2^64 - 1 since p = 1 mod 2^64).
inline Fe fmul(const Fe& a, const Fe& b) {
  const U256& p = prime();
  uint64_t t[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 4; i++) {
    u128 c = 0;
    for (int j = 0; j < 4; j++) {
      c += (u128)a.m.w[j] * b.m.w[i] + t[j];
      t[j] = (uint64_t)c;
      c >>= 64;
    }
    c += t[4];
    t[4] = (uint64_t)c;
    t[5] = (uint64_t)(c >> 64);
    uint64_t m = t[0] * 0xffffffffffffffffull;
    c = (u128)m * p.w[0] + t[0];
    c >>= 64;
    for (int j = 1; j < 4; j++) {
      c += (u128)m * p.w[j] + t[j];
      t[j - 1] = (uint64_t)c;
      c >>= 64;
    }
    c += t[4];
    t[3] = (uint64_t)c;
    t[4] = t[5] + (uint64_t)(c >> 64);
    t[5] = 0;
  }
  U256 r = {{t[0], t[1], t[2], t[3]}};
  uint64_t br;
  if (t[4] || geq(r, prime())) r = sub_raw(r, prime(), br);
  return {r};
}

// 2^512 mod p by doubling (the factor that brings an integer into Montgomery form).
inline const Fe& r2() {
  static const Fe v = [] {
    Fe x;
    x.m.w[0] = 1;
    for (int i = 0; i < 512; i++) x = fadd(x, x);
    return x;
  }();
  return v;
}
// An integer below p into the field.
inline Fe from_int(const U256& v) { return fmul(Fe{v}, r2()); }
inline Fe from_u64(uint64_t v) { U256 u; u.w[0] = v; return from_int(u); }
// The canonical integer of a field element.
inline U256 to_int(const Fe& a) {
  Fe one;
  one.m.w[0] = 1;
  return fmul(a, one).m;
}

inline U256 from_be_bytes(const uint8_t* b) {
  U256 r;
  for (int i = 0; i < 32; i++) r.w[3 - i / 8] |= (uint64_t)b[i] << (8 * (7 - i % 8));
  return r;
}
inline std::array<uint8_t, 32> to_be_bytes(const U256& v) {
  std::array<uint8_t, 32> b;
  for (int i = 0; i < 32; i++) b[i] = (uint8_t)(v.w[3 - i / 8] >> (8 * (7 - i % 8)));
  return b;
}
// Bytes as a big-endian integer, reduced mod p by subtraction (values below 2^256).
inline U256 reduce_be(const uint8_t* b) {
  U256 v = from_be_bytes(b);
  uint64_t br;
  while (geq(v, prime())) v = sub_raw(v, prime(), br);
  return v;
}

// ------------------------------------------------------------- SHA-256
// FIPS 180-4. The round constants are the first 32 bits of the fractional
// parts of the cube roots of the first 64 primes, the initial state those of
// the square roots of the first 8: computed here by exact integer roots.
struct Sha256 {
  static const std::array<uint32_t, 64>& K() {
    static const std::array<uint32_t, 64> k = [] {
      std::array<uint32_t, 64> out{};
      int n = 0;
      for (uint64_t q = 2; n < 64; q++) {
        bool prime = true;
        for (uint64_t d = 2; d * d <= q; d++)
          if (q % d == 0) prime = false;
        if (!prime) continue;
        // floor(cbrt(q · 2^96)) = floor(cbrt(q) · 2^32)
        u128 x = (u128)q << 96;
        uint64_t lo = 0, hi = 1ull << 40;
        while (lo + 1 < hi) {
          uint64_t mid = (lo + hi) / 2;
          if ((u128)mid * mid * mid <= x) lo = mid;
          else hi = mid;
        }
        out[n++] = (uint32_t)lo;
      }
      return out;
    }();
    return k;
  }
  static std::array<uint32_t, 8> H0() {
    std::array<uint32_t, 8> out{};
    int n = 0;
    for (uint64_t q = 2; n < 8; q++) {
      bool prime = true;
      for (uint64_t d = 2; d * d <= q; d++)
        if (q % d == 0) prime = false;
      if (!prime) continue;
      u128 x = (u128)q << 64;  // floor(sqrt(q · 2^64)) = floor(sqrt(q) · 2^32)
      uint64_t lo = 0, hi = 1ull << 36;
      while (lo + 1 < hi) {
        uint64_t mid = (lo + hi) / 2;
        if ((u128)mid * mid <= x) lo = mid;
        else hi = mid;
      }
      out[n++] = (uint32_t)lo;
    }
    return out;
  }
  static uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
  static std::array<uint8_t, 32> hash(const uint8_t* data, size_t len) {
    std::vector<uint8_t> m(data, data + len);
    m.push_back(0x80);
    while (m.size() % 64 != 56) m.push_back(0);
    uint64_t bits = (uint64_t)len * 8;
    for (int i = 7; i >= 0; i--) m.push_back((uint8_t)(bits >> (8 * i)));
    std::array<uint32_t, 8> h = H0();
    const auto& k = K();
    for (size_t off = 0; off < m.size(); off += 64) {
      uint32_t w[64];
      for (int i = 0; i < 16; i++)
        w[i] = ((uint32_t)m[off + 4 * i] << 24) | ((uint32_t)m[off + 4 * i + 1] << 16) |
               ((uint32_t)m[off + 4 * i + 2] << 8) | m[off + 4 * i + 3];
      for (int i = 16; i < 64; i++) {
        uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
        uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
        w[i] = w[i - 16] + s0 + w[i - 7] + s1;
      }
      uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
      for (int i = 0; i < 64; i++) {
        uint32_t S1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25);
        uint32_t ch = (e & f) ^ (~e & g);
        uint32_t t1 = hh + S1 + ch + k[i] + w[i];
        uint32_t S0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);
        uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
        uint32_t t2 = S0 + mj;
        hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
      }
      h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
    }
    std::array<uint8_t, 32> out;
    for (int i = 0; i < 8; i++)
      for (int j = 0; j < 4; j++) out[4 * i + j] = (uint8_t)(h[i] >> (24 - 8 * j));
    return out;
  }
};

// ------------------------------------------------------------- Poseidon
constexpr int N_FULL_HALF = 4, N_PARTIAL = 83, N_ROUNDS = 2 * N_FULL_HALF + N_PARTIAL;

inline const std::vector<std::array<Fe, 3>>& round_constants() {
  static const std::vector<std::array<Fe, 3>> rc = [] {
    std::vector<std::array<Fe, 3>> out(N_ROUNDS);
    for (int r = 0; r < N_ROUNDS; r++)
      for (int j = 0; j < 3; j++) {
        std::string s = "Hades" + std::to_string(3 * r + j);
        auto d = Sha256::hash((const uint8_t*)s.data(), s.size());
        out[r][j] = from_int(reduce_be(d.data()));
      }
    return out;
  }();
  return rc;
}

inline Fe cube(const Fe& x) { return fmul(fmul(x, x), x); }

// The Hades permutation (poseidon_permute_comp), textbook round form.
inline void permute(std::array<Fe, 3>& s) {
  const auto& rc = round_constants();
  for (int r = 0; r < N_ROUNDS; r++) {
    for (int j = 0; j < 3; j++) s[j] = fadd(s[j], rc[r][j]);
    const bool full = r < N_FULL_HALF || r >= N_FULL_HALF + N_PARTIAL;
    if (full)
      for (int j = 0; j < 3; j++) s[j] = cube(s[j]);
    else
      s[2] = cube(s[2]);
    // [[3,1,1],[1,-1,1],[1,1,-2]]
    Fe t = fadd(fadd(s[0], s[1]), s[2]);
    Fe s0 = fadd(t, fadd(s[0], s[0]));
    Fe s1 = fsub(t, fadd(s[1], s[1]));
    Fe s2 = fsub(t, fadd(fadd(s[2], s[2]), s[2]));
    s = {s0, s1, s2};
  }
}

// poseidon_hash(x, y): capacity element 2.
inline Fe hash2(const Fe& x, const Fe& y) {
  std::array<Fe, 3> s = {x, y, from_u64(2)};
  permute(s);
  return s[0];
}

// poseidon_hash_many: pairs absorbed into elements 0 and 1, then a 1 after
// the data (element 1 after a lone last value, element 0 after an even count).
inline Fe hash_many(const std::vector<Fe>& v) {
  std::array<Fe, 3> s = {Fe{}, Fe{}, Fe{}};
  size_t i = 0;
  for (; i + 2 <= v.size(); i += 2) {
    s[0] = fadd(s[0], v[i]);
    s[1] = fadd(s[1], v[i + 1]);
    permute(s);
  }
  const Fe one = from_u64(1);
  if (v.size() - i == 1) {
    s[0] = fadd(s[0], v[i]);
    s[1] = fadd(s[1], one);
  } else {
    s[0] = fadd(s[0], one);
  }
  permute(s);
  return s[0];
}

// add_length_padding: + n · 2^248.
inline Fe length_padding(const Fe& f, uint64_t n) {
  U256 v;
  v.w[3] = n << 56;
  return fadd(f, from_int(v));
}

// construct_felt252_from_m31s: up to 8 values shifted in by 31 bits each; a
// shorter word gets its length at bit 248.
inline Fe felt_from_m31s(const M31* vals, size_t n) {
  U256 v;
  for (size_t k = 0; k < n; k++) {
    for (int i = 3; i > 0; i--) v.w[i] = (v.w[i] << 31) | (v.w[i - 1] >> 33);
    v.w[0] = (v.w[0] << 31) | vals[k].v;
  }
  Fe f = from_int(v);
  return n < 8 ? length_padding(f, n) : f;
}

inline Fe from_hash(const uint8_t* be) { return from_int(from_be_bytes(be)); }
inline std::array<uint8_t, 32> to_hash(const Fe& f) { return to_be_bytes(to_int(f)); }

// Poseidon252MerkleHasher::hash_node; hashes as 32 big-endian bytes.
inline std::array<uint8_t, 32> hash_node(const uint8_t* left, const uint8_t* right, const M31* vals, size_t n) {
  std::vector<Fe> values;
  if (left) {
    if (n == 0) return to_hash(hash2(from_hash(left), from_hash(right)));
    values.push_back(from_hash(left));
    values.push_back(from_hash(right));
  }
  for (size_t i = 0; i < n; i += 8) values.push_back(felt_from_m31s(vals + i, n - i < 8 ? n - i : 8));
  return to_hash(hash_many(values));
}

// ------------------------------------------------------------- channel
struct Channel {
  Fe digest;  // default: zero
  uint32_t n_draws = 0;
  static constexpr uint32_t POW_PREFIX = 0x12345678u;
  static constexpr uint32_t GRIND_LOW_BITS = 14;

  void update_digest(const Fe& d) { digest = d; n_draws = 0; }
  void mix_root(const uint8_t* root) { update_digest(hash2(digest, from_hash(root))); }
  void mix_u64(uint64_t v) { update_digest(hash2(digest, from_u64(v))); }
  // QM31 values two per felt252: 1, then each M31 coordinate shifted in by 31 bits.
  void mix_felts(const std::vector<std::array<uint32_t, 4>>& felts) {
    std::vector<Fe> res = {digest};
    const Fe shift = from_u64(1ull << 31);
    for (size_t i = 0; i < felts.size(); i += 2) {
      Fe cur = from_u64(1);
      for (size_t k = i; k < i + 2 && k < felts.size(); k++)
        for (int c = 0; c < 4; c++) cur = fadd(fmul(cur, shift), from_u64(felts[k][c]));
      res.push_back(cur);
    }
    update_digest(hash_many(res));
  }
  // u32 words seven per felt252, big-endian; a short last chunk padded with
  // zeros and given its length at bit 248.
  void mix_u32s(const std::vector<uint32_t>& data) {
    size_t padding = 6 - ((data.size() + 6) % 7);
    std::vector<uint32_t> d(data);
    d.resize(data.size() + padding, 0);
    std::vector<Fe> felts = {digest};
    const Fe shift = from_u64(1ull << 32);
    for (size_t i = 0; i < d.size(); i += 7) {
      Fe cur;
      for (size_t k = i; k < i + 7; k++) cur = fadd(fmul(cur, shift), from_u64(d[k]));
      felts.push_back(cur);
    }
    if (padding) felts.back() = length_padding(felts.back(), 7 - padding);
    update_digest(hash_many(felts));
  }
  U256 draw_felt252() {
    std::array<Fe, 3> s = {digest, from_u64(n_draws), from_u64(3)};
    permute(s);
    n_draws++;
    return to_int(s[0]);
  }
  static uint64_t take_bits(U256& v, int bits) {
    uint64_t r = v.w[0] & ((1ull << bits) - 1);
    for (int i = 0; i < 3; i++) v.w[i] = (v.w[i] >> bits) | (v.w[i + 1] << (64 - bits));
    v.w[3] >>= bits;
    return r;
  }
  // eight 31-bit chunks, low first, each reduced mod 2^31 - 1
  std::array<uint32_t, 8> draw_base_felts() {
    U256 cur = draw_felt252();
    std::array<uint32_t, 8> r;
    for (int i = 0; i < 8; i++) r[i] = (uint32_t)(take_bits(cur, 31) % P);
    return r;
  }
  std::vector<uint32_t> draw_u32s() {
    U256 cur = draw_felt252();
    std::vector<uint32_t> r(7);
    for (int i = 0; i < 7; i++) r[i] = (uint32_t)take_bits(cur, 32);
    return r;
  }
  Fe pow_prefixed(uint32_t n_bits) const {
    return hash_many({from_u64(POW_PREFIX), digest, from_u64(n_bits)});
  }
  static bool check_nonce(const Fe& prefixed, uint32_t n_bits, uint64_t nonce) {
    U256 h = to_int(hash2(prefixed, from_u64(nonce)));
    uint32_t tz = 0;
    for (uint32_t i = 0; i < 2 && tz == 64 * i; i++) tz += h.w[i] ? (uint32_t)__builtin_ctzll(h.w[i]) : 64;
    return tz >= n_bits;
  }
  bool verify_pow_nonce(uint32_t n_bits, uint64_t nonce) const { return check_nonce(pow_prefixed(n_bits), n_bits, nonce); }
  uint64_t grind(uint32_t n_bits) const {
    Fe pre = pow_prefixed(n_bits);
    for (uint64_t hi = 0;; hi++)
      for (uint64_t low = 0; low < (1ull << GRIND_LOW_BITS); low++)
        if (check_nonce(pre, n_bits, (hi << 32) | low)) return (hi << 32) | low;
  }
};

}  // namespace p252
}  // namespace orc
