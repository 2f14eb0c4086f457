// Host-side protocol pieces of the GPU prover: Blake2s hashing, the
// Fiat-Shamir channel (Blake2s, or Poseidon252 for Poseidon252MerkleChannel),
// circle points over QM31 and proof serialisation.
//
// Semantics follow the reference:
//   crates/stwo/src/core/channel/blake2s.rs:20-140   (channel: mix, draw, pow prefix)
//   crates/stwo/src/core/channel/poseidon252.rs:18-155 (the Poseidon252 channel)
//   crates/stwo/src/core/vcs/blake2_merkle.rs:53-58  (mix_root)
//   crates/stwo/src/core/queries.rs:11-28            (draw_queries)
//   crates/stwo/src/core/circle.rs:12-214            (points, random point, generators)
//   crates/stwo/src/core/constraints.rs:12-35        (coset_vanishing)
//   crates/stwo/src/core/pcs/quotients.rs:29-38, core/fri.rs:363-398 (proof layout)
#pragma once
#include <array>
#include <cstring>
#include <string>
#include <vector>
#include "../blake2s.cuh"
#include "../m31.cuh"
#include "felt252_host.h"

namespace gs {
namespace host {

using Hash = std::array<uint8_t, 32>;

// Incremental Blake2s-256 over the shared compression function.
struct Hasher {
  uint32_t h[8];
  uint8_t buf[64];
  size_t len = 0;
  uint64_t total = 0;
  Hasher() { blake2s_init(h); }
  void compress_buf(bool last) {
    uint32_t m[16];
    for (int i = 0; i < 16; i++)
      m[i] = (uint32_t)buf[4 * i] | ((uint32_t)buf[4 * i + 1] << 8) | ((uint32_t)buf[4 * i + 2] << 16) |
             ((uint32_t)buf[4 * i + 3] << 24);
    blake2s_compress(h, m, (uint32_t)total, last);
  }
  void update(const void* data, size_t n) {
    const uint8_t* p = (const uint8_t*)data;
    while (n) {
      if (len == 64) {
        total += 64;
        compress_buf(false);
        len = 0;
      }
      size_t k = 64 - len < n ? 64 - len : n;
      memcpy(buf + len, p, k);
      len += k;
      p += k;
      n -= k;
    }
  }
  void u32(uint32_t w) { uint8_t b[4] = {(uint8_t)w, (uint8_t)(w >> 8), (uint8_t)(w >> 16), (uint8_t)(w >> 24)}; update(b, 4); }
  Hash finish() {
    total += len;
    memset(buf + len, 0, 64 - len);
    compress_buf(true);
    Hash out;
    for (int i = 0; i < 8; i++)
      for (int j = 0; j < 4; j++) out[4 * i + j] = (uint8_t)(h[i] >> (8 * j));
    return out;
  }
};

inline Hash hash_bytes(const void* d, size_t n) { Hasher s; s.update(d, n); return s.finish(); }
inline Hash hash_from_words(const uint32_t w[8]) {
  Hash h;
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 4; j++) h[4 * i + j] = (uint8_t)(w[i] >> (8 * j));
  return h;
}
inline uint32_t word(const Hash& h, int i) {
  return (uint32_t)h[4 * i] | ((uint32_t)h[4 * i + 1] << 8) | ((uint32_t)h[4 * i + 2] << 16) | ((uint32_t)h[4 * i + 3] << 24);
}

// Blake2sChannel, or Poseidon252Channel when `p252` is set (then `digest`
// holds the felt252 digest as 32 big-endian bytes).
struct Channel {
  Hash digest{};
  uint32_t n_draws = 0;
  bool p252 = false;
  void set(const Hash& d) { digest = d; n_draws = 0; }
  p252::F fdigest() const { return p252::from_bytes(digest.data()); }
  void set_f(const p252::F& f) { set(p252::to_bytes(f)); }
  void mix_root(const Hash& root) {
    if (p252) return set_f(p252::hash2(fdigest(), p252::from_bytes(root.data())));
    Hasher s; s.update(digest.data(), 32); s.update(root.data(), 32); set(s.finish());
  }
  void mix_felts(const std::vector<qm31>& f) {
    if (p252) {  // two QM31 per felt252: 1, then the 8 coordinates shifted in by 31 bits
      std::vector<p252::F> res = {fdigest()};
      for (size_t i = 0; i < f.size(); i += 2) {
        uint64_t v[4] = {1, 0, 0, 0};
        for (size_t k = i; k < i + 2 && k < f.size(); k++)
          for (uint32_t c : {f[k].x.a, f[k].x.b, f[k].y.a, f[k].y.b}) {
            for (int w = 3; w > 0; w--) v[w] = (v[w] << 31) | (v[w - 1] >> 33);
            v[0] = (v[0] << 31) | c;
          }
        res.push_back(p252::from_int(v));
      }
      return set_f(p252::hash_many(res));
    }
    Hasher s;
    s.update(digest.data(), 32);
    for (auto& q : f) { s.u32(q.x.a); s.u32(q.x.b); s.u32(q.y.a); s.u32(q.y.b); }
    set(s.finish());
  }
  void mix_u64(uint64_t v) {
    if (p252) return set_f(p252::hash2(fdigest(), p252::from_u64(v)));
    Hasher s;
    s.update(digest.data(), 32);
    s.u32((uint32_t)v);
    s.u32((uint32_t)(v >> 32));
    set(s.finish());
  }
  // Words of one draw: 8 (Blake2s) or 7 (Poseidon252, 32-bit chunks of the
  // drawn felt252, low first); returns the count.
  int draw_words(uint32_t out[8]) {
    if (p252) {
      uint64_t v[4];
      p252::draw_int(fdigest(), n_draws++, v);
      for (int i = 0; i < 7; i++) out[i] = (uint32_t)p252::take_bits(v, 32);
      return 7;
    }
    uint8_t in[37];
    memcpy(in, digest.data(), 32);
    for (int i = 0; i < 4; i++) in[32 + i] = (uint8_t)(n_draws >> (8 * i));
    in[36] = 0;
    n_draws++;
    Hash h = hash_bytes(in, 37);
    for (int i = 0; i < 8; i++) out[i] = word(h, i);
    return 8;
  }
  std::array<uint32_t, 8> draw_base() {
    std::array<uint32_t, 8> u;
    if (p252) {  // 31-bit chunks, each reduced mod P
      uint64_t v[4];
      p252::draw_int(fdigest(), n_draws++, v);
      for (int i = 0; i < 8; i++) {
        uint32_t x = (uint32_t)p252::take_bits(v, 31);
        u[i] = x == P ? 0 : x;
      }
      return u;
    }
    for (;;) {
      draw_words(u.data());
      bool ok = true;
      for (auto x : u) ok = ok && x < 2 * P;
      if (ok) {
        for (auto& x : u) x = x >= P ? x - P : x;
        return u;
      }
    }
  }
  qm31 draw_felt() { auto f = draw_base(); return qm_make(f[0], f[1], f[2], f[3]); }
  std::vector<qm31> draw_felts(size_t n) {
    std::vector<qm31> r;
    while (r.size() < n) {
      auto f = draw_base();
      r.push_back(qm_make(f[0], f[1], f[2], f[3]));
      if (r.size() < n) r.push_back(qm_make(f[4], f[5], f[6], f[7]));
    }
    return r;
  }
  // H(POW_PREFIX, 0^12, digest, pow_bits) as 8 words (the Blake2s grind kernel's input).
  std::array<uint32_t, 8> pow_prefixed(uint32_t pow_bits) const {
    Hasher s;
    s.u32(0x12345678u);
    uint8_t z[12] = {0};
    s.update(z, 12);
    s.update(digest.data(), 32);
    s.u32(pow_bits);
    Hash h = s.finish();
    std::array<uint32_t, 8> w;
    for (int i = 0; i < 8; i++) w[i] = word(h, i);
    return w;
  }
};

// GrindOps::grind's acceptance test: the first little-endian word of
// Blake2s(prefixed_digest || nonce (8 B, LE)) has at least pow_bits trailing
// zeros.
inline bool pow_passes(const std::array<uint32_t, 8>& prefixed, uint64_t nonce, uint32_t pow_bits) {
  Hasher s;
  for (uint32_t w : prefixed) s.u32(w);
  s.u32((uint32_t)nonce);
  s.u32((uint32_t)(nonce >> 32));
  const Hash h = s.finish();
  const uint32_t w0 = word(h, 0);
  const uint32_t tz = w0 == 0 ? 32u : (uint32_t)__builtin_ctz(w0);
  return tz >= pow_bits;
}

inline std::vector<size_t> draw_queries(Channel& ch, uint32_t log_domain, size_t n) {
  std::vector<size_t> r;
  uint32_t mask = (uint32_t)((1ull << log_domain) - 1);
  while (r.size() < n) {
    uint32_t w[8];
    int k = ch.draw_words(w);
    for (int i = 0; i < k && r.size() < n; i++) r.push_back(w[i] & mask);
  }
  return r;
}

// --------------------------------------------------------------- circle
inline pt31 index_point(uint32_t k) {
  pt31 r = {1u, 0u}, cur = {2u, 1268011823u};
  for (int b = 0; b < 31; b++) {
    if ((k >> b) & 1u) r = pt_add(r, cur);
    cur = pt_add(cur, cur);
  }
  return r;
}
inline ptq to_ptq(pt31 p) { return {qm_from_m31(p.x), qm_from_m31(p.y)}; }
inline ptq ptq_double(ptq p) { return ptq_add(p, p); }
inline ptq ptq_rep_double(ptq p, uint32_t n) { for (uint32_t i = 0; i < n; i++) p = ptq_double(p); return p; }
inline ptq ptq_conj(ptq p) { return {p.x, qm_neg(p.y)}; }

// CanonicCoset(log): coset odds(log) = initial index 2^(30-log), step 2^(31-log).
inline uint32_t canonic_initial_index(uint32_t log) { return 1u << (31 - (log + 1)); }
inline uint32_t canonic_step_index(uint32_t log) { return (uint32_t)((1ull << (31 - log)) & 0x7fffffffu); }

// coset_vanishing(CanonicCoset(log).coset, p) for a QM31 point.
inline qm31 canonic_vanishing(uint32_t log, ptq p) {
  pt31 init = index_point(canonic_initial_index(log));
  pt31 half_step = index_point(canonic_step_index(log) >> 1);
  p = ptq_add(p, to_ptq(pt_conj(init)));
  p = ptq_add(p, to_ptq(half_step));
  qm31 x = p.x;
  for (uint32_t i = 1; i < log; i++) x = qm_double_x(x);
  return x;
}
inline uint32_t canonic_vanishing_m31(uint32_t log, pt31 p) {
  pt31 init = index_point(canonic_initial_index(log));
  pt31 half_step = index_point(canonic_step_index(log) >> 1);
  p = pt_add(pt_add(p, pt_conj(init)), half_step);
  uint32_t x = p.x;
  for (uint32_t i = 1; i < log; i++) x = double_x(x);
  return x;
}

inline ptq random_point(Channel& ch) {
  qm31 t = ch.draw_felt();
  qm31 t2 = qm_sqr(t);
  qm31 iv = qm_inv(qm_add(t2, qm_one()));
  return {qm_mul(qm_sub(qm_one(), t2), iv), qm_mul(qm_add(t, t), iv)};
}

inline size_t bitrev(size_t i, uint32_t log) {
  size_t r = 0;
  for (uint32_t b = 0; b < log; b++) r |= ((i >> b) & 1) << (log - 1 - b);
  return r;
}

// ------------------------------------------------------------- proof
// bincode-1.x style: little-endian fixed width, u64 sequence lengths,
// Option as a 1-byte tag, hash = 32 raw bytes, QM31 = 4 x u32; field order of
// CommitmentSchemeProof (config, commitments, sampled_values, decommitments,
// queried_values, proof_of_work, fri_proof).
static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "proof serialization assumes a little-endian host");
// A proof is written in passes over one layout: a counting pass (no output),
// then a pass of the bytes the host holds (`fixed`) and a pass of the bytes
// gathered on the device (`gathered`), each advancing over the other kind,
// so the first can run while the gather is still on its way.
struct Writer {
  char* out = nullptr;  // null: counting pass
  size_t len = 0;
  bool fixed = false, gathered = false;
  void put(const void* p, size_t n) {
    if (out && fixed) memcpy(out + len, p, n);
    len += n;
  }
  void put_gathered(const void* p, size_t n) {
    if (out && gathered && n) memcpy(out + len, p, n);
    len += n;
  }
  void u8(uint8_t v) { put(&v, 1); }
  void u32(uint32_t v) { put(&v, 4); }
  void u64(uint64_t v) { put(&v, 8); }
  void hash(const Hash& h) { put(h.data(), 32); }
  void qm(const qm31& q) {
    const uint32_t w[4] = {q.x.a, q.x.b, q.y.a, q.y.b};
    put(w, 16);
  }
};

}  // namespace host
}  // namespace gs
