// Blake2s-256 compression for the device (RFC 7693; the reference uses the
// `blake2 = 0.10.6` crate at crates/stwo/src/core/vcs/blake2_merkle.rs:18-39).
//
// Each thread keeps the 16 message words and the 16-word working state in
// registers; the message schedule is resolved at compile time (fully unrolled
// rounds), so a compression is pure 32-bit add/xor/rotate work: IADD3 for the
// three-input adds, LOP3 for xors, PRMT/SHF for the rotations.
#pragma once
#include <cstdint>
#include "m31.cuh"

namespace gs {


constexpr uint32_t BLAKE_IV0 = 0x6A09E667u, BLAKE_IV1 = 0xBB67AE85u, BLAKE_IV2 = 0x3C6EF372u, BLAKE_IV3 = 0xA54FF53Au,
                   BLAKE_IV4 = 0x510E527Fu, BLAKE_IV5 = 0x9B05688Cu, BLAKE_IV6 = 0x1F83D9ABu, BLAKE_IV7 = 0x5BE0CD19u;
// Initial chaining value for an unkeyed 32-byte digest: IV0 ^ 0x01010020.
constexpr uint32_t BLAKE_H0 = BLAKE_IV0 ^ 0x01010020u;

GS_HD uint32_t rotr32(uint32_t x, int n) {
#ifdef __CUDA_ARCH__
  return __funnelshift_r(x, x, n);
#else
  return (x >> n) | (x << (32 - n));
#endif
}

// Rotations by 16 and 8 are byte permutes (PRMT) on the device.
GS_HD uint32_t rotr16(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __byte_perm(x, 0, 0x1032);
#else
  return rotr32(x, 16);
#endif
}
GS_HD uint32_t rotr8(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __byte_perm(x, 0, 0x0321);
#else
  return rotr32(x, 8);
#endif
}

#define GS_G(a, b, c, d, x, y)         \
  do {                                 \
    v[a] = v[a] + v[b] + (x);          \
    v[d] = rotr16(v[d] ^ v[a]);        \
    v[c] = v[c] + v[d];                \
    v[b] = rotr32(v[b] ^ v[c], 12);    \
    v[a] = v[a] + v[b] + (y);          \
    v[d] = rotr8(v[d] ^ v[a]);         \
    v[c] = v[c] + v[d];                \
    v[b] = rotr32(v[b] ^ v[c], 7);     \
  } while (0)

#define GS_ROUND(s0, s1, s2, s3, s4, s5, s6, s7, s8, s9, s10, s11, s12, s13, s14, s15) \
  do {                                                                                 \
    GS_G(0, 4, 8, 12, m[s0], m[s1]);                                                   \
    GS_G(1, 5, 9, 13, m[s2], m[s3]);                                                   \
    GS_G(2, 6, 10, 14, m[s4], m[s5]);                                                  \
    GS_G(3, 7, 11, 15, m[s6], m[s7]);                                                  \
    GS_G(0, 5, 10, 15, m[s8], m[s9]);                                                  \
    GS_G(1, 6, 11, 12, m[s10], m[s11]);                                                \
    GS_G(2, 7, 8, 13, m[s12], m[s13]);                                                 \
    GS_G(3, 4, 9, 14, m[s14], m[s15]);                                                 \
  } while (0)

// h <- compress(h, m, t, last). t = total bytes hashed so far including this block.
GS_HD void blake2s_compress(uint32_t h[8], const uint32_t m[16], uint32_t t, bool last) {
  uint32_t v[16];
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = h[i];
  v[8] = BLAKE_IV0; v[9] = BLAKE_IV1; v[10] = BLAKE_IV2; v[11] = BLAKE_IV3;
  v[12] = BLAKE_IV4 ^ t; v[13] = BLAKE_IV5; v[14] = last ? ~BLAKE_IV6 : BLAKE_IV6; v[15] = BLAKE_IV7;
  GS_ROUND(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15);
  GS_ROUND(14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3);
  GS_ROUND(11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4);
  GS_ROUND(7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8);
  GS_ROUND(9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13);
  GS_ROUND(2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9);
  GS_ROUND(12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11);
  GS_ROUND(13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10);
  GS_ROUND(6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5);
  GS_ROUND(10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0);
#pragma unroll
  for (int i = 0; i < 8; i++) h[i] ^= v[i] ^ v[i + 8];
}

#ifdef __CUDACC__
// The same compression with every add issued as an IMAD against a runtime 1
// (`one`): the xors and rotations keep the integer ALU pipe busy, the adds
// move to the FMA pipe, which would otherwise sit idle.
__device__ __forceinline__ uint32_t b2_imad(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
}
#define GS_GF(a, b, c, d, x, y)                                    \
  do {                                                             \
    v[a] = b2_imad(b2_imad(v[a], one, v[b]), one, (x));            \
    v[d] = rotr16(v[d] ^ v[a]);                                  \
    v[c] = b2_imad(v[c], one, v[d]);                               \
    v[b] = rotr32(v[b] ^ v[c], 12);                                \
    v[a] = b2_imad(b2_imad(v[a], one, v[b]), one, (y));            \
    v[d] = rotr8(v[d] ^ v[a]);                                   \
    v[c] = b2_imad(v[c], one, v[d]);                               \
    v[b] = rotr32(v[b] ^ v[c], 7);                                 \
  } while (0)
#define GS_ROUNDF(s0, s1, s2, s3, s4, s5, s6, s7, s8, s9, s10, s11, s12, s13, s14, s15) \
  do {                                                                                  \
    GS_GF(0, 4, 8, 12, m[s0], m[s1]);                                                   \
    GS_GF(1, 5, 9, 13, m[s2], m[s3]);                                                   \
    GS_GF(2, 6, 10, 14, m[s4], m[s5]);                                                  \
    GS_GF(3, 7, 11, 15, m[s6], m[s7]);                                                  \
    GS_GF(0, 5, 10, 15, m[s8], m[s9]);                                                  \
    GS_GF(1, 6, 11, 12, m[s10], m[s11]);                                                \
    GS_GF(2, 7, 8, 13, m[s12], m[s13]);                                                 \
    GS_GF(3, 4, 9, 14, m[s14], m[s15]);                                                 \
  } while (0)
__device__ __forceinline__ void blake2s_compress_f(uint32_t h[8], const uint32_t m[16], uint32_t t, bool last,
                                                   uint32_t one) {
  uint32_t v[16];
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = h[i];
  v[8] = BLAKE_IV0; v[9] = BLAKE_IV1; v[10] = BLAKE_IV2; v[11] = BLAKE_IV3;
  v[12] = BLAKE_IV4 ^ t; v[13] = BLAKE_IV5; v[14] = last ? ~BLAKE_IV6 : BLAKE_IV6; v[15] = BLAKE_IV7;
  GS_ROUNDF(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15);
  GS_ROUNDF(14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3);
  GS_ROUNDF(11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4);
  GS_ROUNDF(7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8);
  GS_ROUNDF(9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13);
  GS_ROUNDF(2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9);
  GS_ROUNDF(12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11);
  GS_ROUNDF(13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10);
  GS_ROUNDF(6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5);
  GS_ROUNDF(10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0);
#pragma unroll
  for (int i = 0; i < 8; i++) h[i] ^= v[i] ^ v[i + 8];
}
#endif

GS_HD void blake2s_init(uint32_t h[8]) {
  h[0] = BLAKE_H0; h[1] = BLAKE_IV1; h[2] = BLAKE_IV2; h[3] = BLAKE_IV3;
  h[4] = BLAKE_IV4; h[5] = BLAKE_IV5; h[6] = BLAKE_IV6; h[7] = BLAKE_IV7;
}

}  // namespace gs
