// ORACLE — test infrastructure only (see fields.h).
// Fiat-Shamir channel (Blake2s, or Poseidon252 when `kind` says so: the
// MerkleChannel pairs each hasher with its channel), query drawing and
// proof-of-work.
// Follows:
//   crates/stwo/src/core/channel/blake2s.rs:20-140   (digest, n_draws, mix/draw, verify_pow_nonce)
//   crates/stwo/src/core/vcs/blake2_merkle.rs:53-58  (mix_root = H(digest || root))
//   crates/stwo/src/core/queries.rs:11-28            (draw_queries)
//   crates/stwo/src/prover/backend/cpu/grind.rs:5-16 (smallest nonce by linear search)
#pragma once
#include "blake2s.h"
#include "felt252.h"
#include "fields.h"

namespace orc {

// Blake2sMerkleChannel or Poseidon252MerkleChannel (the hasher of every
// Merkle tree and the channel of the proof).
enum class MerkleHash { Blake2s, Poseidon252 };

struct Channel {
  MerkleHash kind = MerkleHash::Blake2s;
  Hash32 digest{};
  uint32_t n_draws = 0;
  p252::Channel pc;  // the Poseidon252 channel's state
  static constexpr uint32_t POW_PREFIX = 0x12345678u;

  Channel() = default;
  explicit Channel(MerkleHash k) : kind(k) {}
  bool p252() const { return kind == MerkleHash::Poseidon252; }

  void update_digest(const Hash32& d) { digest = d; n_draws = 0; }
  void mix_root(const Hash32& root) {
    if (p252()) return pc.mix_root(root.data());
    Blake2s s; s.update(digest.data(), 32); s.update(root.data(), 32);
    update_digest(s.finalize());
  }
  void mix_felts(const std::vector<QM31>& felts) {
    if (p252()) {
      std::vector<std::array<uint32_t, 4>> v;
      for (auto& f : felts) v.push_back({f.coord(0), f.coord(1), f.coord(2), f.coord(3)});
      return pc.mix_felts(v);
    }
    Blake2s s; s.update(digest.data(), 32);
    for (auto& f : felts) for (int i = 0; i < 4; i++) s.update_u32(f.coord(i));
    update_digest(s.finalize());
  }
  void mix_u32s(const std::vector<uint32_t>& data) {
    if (p252()) return pc.mix_u32s(data);
    Blake2s s; s.update(digest.data(), 32);
    for (uint32_t w : data) s.update_u32(w);
    update_digest(s.finalize());
  }
  void mix_u64(uint64_t v) {
    if (p252()) return pc.mix_u64(v);
    mix_u32s({(uint32_t)v, (uint32_t)(v >> 32)});
  }
  // 8 words (Blake2s) or 7 (Poseidon252)
  std::vector<uint32_t> draw_u32s() {
    if (p252()) return pc.draw_u32s();
    uint8_t in[37];
    memcpy(in, digest.data(), 32);
    for (int i = 0; i < 4; i++) in[32 + i] = (uint8_t)(n_draws >> (8 * i));
    in[36] = 0;
    n_draws++;
    Hash32 h = Blake2s::hash(in, 37);
    std::vector<uint32_t> r(8);
    for (int i = 0; i < 8; i++) r[i] = hash_word(h, i);
    return r;
  }
  std::array<M31, 8> draw_base_felts() {
    if (p252()) {
      auto u = pc.draw_base_felts();
      std::array<M31, 8> r;
      for (int i = 0; i < 8; i++) r[i] = M31(u[i]);
      return r;
    }
    for (;;) {
      auto u = draw_u32s();
      bool ok = true;
      for (auto x : u) if (x >= 2 * P) ok = false;
      if (ok) {
        std::array<M31, 8> r;
        for (int i = 0; i < 8; i++) r[i] = M31(reduce64(u[i]));
        return r;
      }
    }
  }
  QM31 draw_secure_felt() {
    auto f = draw_base_felts();
    return QM31::from_m31(f[0], f[1], f[2], f[3]);
  }
  std::vector<QM31> draw_secure_felts(size_t n) {
    std::vector<QM31> r;
    while (r.size() < n) {
      auto f = draw_base_felts();
      r.push_back(QM31::from_m31(f[0], f[1], f[2], f[3]));
      if (r.size() < n) r.push_back(QM31::from_m31(f[4], f[5], f[6], f[7]));
    }
    return r;
  }
  Hash32 pow_prefixed_digest(uint32_t n_bits) const {
    Blake2s s;
    s.update_u32(POW_PREFIX);
    uint8_t z[12] = {0};
    s.update(z, 12);
    s.update(digest.data(), 32);
    s.update_u32(n_bits);
    return s.finalize();
  }
  static bool check_nonce(const Hash32& prefixed, uint32_t n_bits, uint64_t nonce) {
    Blake2s s;
    s.update(prefixed.data(), 32);
    uint8_t nb[8];
    for (int i = 0; i < 8; i++) nb[i] = (uint8_t)(nonce >> (8 * i));
    s.update(nb, 8);
    Hash32 r = s.finalize();
    // trailing zeros of the first 16 bytes read as a little-endian u128
    uint32_t tz = 0;
    for (int i = 0; i < 16; i++) {
      uint8_t b = r[i];
      if (b == 0) { tz += 8; continue; }
      while (!(b & 1)) { tz++; b >>= 1; }
      break;
    }
    return tz >= n_bits;
  }
  bool verify_pow_nonce(uint32_t n_bits, uint64_t nonce) const {
    if (p252()) return pc.verify_pow_nonce(n_bits, nonce);
    return check_nonce(pow_prefixed_digest(n_bits), n_bits, nonce);
  }
  uint64_t grind(uint32_t n_bits) const {
    if (p252()) return pc.grind(n_bits);
    Hash32 pre = pow_prefixed_digest(n_bits);
    for (uint64_t nonce = 0;; nonce++) if (check_nonce(pre, n_bits, nonce)) return nonce;
  }
};

inline std::vector<size_t> draw_queries(Channel& ch, uint32_t log_domain_size, size_t n_queries) {
  std::vector<size_t> raw;
  uint32_t mask = (uint32_t)((1ull << log_domain_size) - 1);
  for (;;) {
    auto w = ch.draw_u32s();
    for (auto x : w) {
      raw.push_back(x & mask);
      if (raw.size() == n_queries) return raw;
    }
  }
}

}  // namespace orc
