// Poseidon252 Merkle hashing on the device: MerkleOps<Poseidon252MerkleHasher>
// ::commit_on_layer (crates/stwo/src/core/vcs/poseidon252_merkle.rs:18-72;
// reference CUDA poseidon252_commit_on_first_layer / _with_previous,
// stwo_cuda/bindings.rs:592-612).
//
// The hash is Starknet's Poseidon (the Hades permutation of the crate
// starknet-crypto 0.6.2 that the reference calls): field p = 2^251 +
// 17·2^192 + 1, state of 3 elements, x^3 S-box, 4 full + 83 partial + 4 full
// rounds, MDS [[3, 1, 1], [1, -1, 1], [1, 1, -2]], round constants from
// poseidon252_constants.py.
//
//   hash_node(children, values): poseidon_hash(l, r) when there are children
//   and no values; otherwise poseidon_hash_many([l, r,] felts of the values,
//   8 M31 values per felt shifted in 31 bits at a time, a shorter last word
//   carrying its length at bit 248).
//
// Field elements live in registers as 8 little-endian 32-bit limbs in
// Montgomery form (R = 2^256). The modulus is sparse, limbs [1, 0, 0, 0, 0, 0,
// 17, 2^27], and p = 1 mod 2^32, so the Montgomery quotient digit of each
// reduction step is -t0 and adding m·p touches limbs 0, 6, 7 and 8. Hashes in
// memory are the reference's device layout: 32 bytes, big-endian.
#include "runtime.cuh"
#include <cstring>

namespace gs {

struct Felt {
  uint32_t v[8];
};

#include "poseidon252_constants.inc"

// Carry chains in PTX (add.cc / addc, mad.lo.cc / madc.hi.cc): one
// instruction per limb, the carry in the flag.

// t -> t - p when t >= p (t < 2p); branch-free select
__device__ __forceinline__ void reduce_once(uint32_t t[8]) {
  uint32_t d[8], bw;
  asm("sub.cc.u32 %0, %9, 1;\n\t"
      "subc.cc.u32 %1, %10, 0;\n\t"
      "subc.cc.u32 %2, %11, 0;\n\t"
      "subc.cc.u32 %3, %12, 0;\n\t"
      "subc.cc.u32 %4, %13, 0;\n\t"
      "subc.cc.u32 %5, %14, 0;\n\t"
      "subc.cc.u32 %6, %15, 17;\n\t"
      "subc.cc.u32 %7, %16, 0x08000000;\n\t"
      "subc.u32 %8, 0, 0;"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]), "=r"(bw)
      : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]));
#pragma unroll
  for (int j = 0; j < 8; j++) t[j] = (t[j] & bw) | (d[j] & ~bw);  // borrow: t < p, keep it
}

// Montgomery product a·b·R^-1 mod p (CIOS), for a, b < p. Per limb b_i:
// t += a·b_i, then t += m·p with m = -t0 (p = 1 mod 2^32), which zeroes
// t0 and touches limbs 6, 7, 8 (17·2^192 and 2^251), then a one-limb shift.
// t0 + m is 0 with a carry exactly when t0 != 0; that carry is fed into
// limb 1 directly, and m·17 is formed outside the carry chain, which holds
// plain add-with-carry only (a chain that mixed multiply-add-with-carry
// with an immediate operand into the reduction produced wrong carries on
// sm_100a). After each shift t < 2p < 2^253, so limb 8 is 0 before the next
// product.
template <bool FULL>
__device__ __forceinline__ Felt fmul_t(const Felt& a, const Felt& b) {
  uint32_t t[10];
#pragma unroll
  for (int j = 0; j < 10; j++) t[j] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    asm("mad.lo.cc.u32 %0, %10, %18, %0;\n\t"
        "madc.lo.cc.u32 %1, %11, %18, %1;\n\t"
        "madc.lo.cc.u32 %2, %12, %18, %2;\n\t"
        "madc.lo.cc.u32 %3, %13, %18, %3;\n\t"
        "madc.lo.cc.u32 %4, %14, %18, %4;\n\t"
        "madc.lo.cc.u32 %5, %15, %18, %5;\n\t"
        "madc.lo.cc.u32 %6, %16, %18, %6;\n\t"
        "madc.lo.cc.u32 %7, %17, %18, %7;\n\t"
        "addc.u32 %8, %8, 0;\n\t"
        "mad.hi.cc.u32 %1, %10, %18, %1;\n\t"
        "madc.hi.cc.u32 %2, %11, %18, %2;\n\t"
        "madc.hi.cc.u32 %3, %12, %18, %3;\n\t"
        "madc.hi.cc.u32 %4, %13, %18, %4;\n\t"
        "madc.hi.cc.u32 %5, %14, %18, %5;\n\t"
        "madc.hi.cc.u32 %6, %15, %18, %6;\n\t"
        "madc.hi.cc.u32 %7, %16, %18, %7;\n\t"
        "madc.hi.cc.u32 %8, %17, %18, %8;\n\t"
        "addc.u32 %9, 0, 0;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]),
          "+r"(t[8]), "=r"(t[9])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
          "r"(a.v[7]), "r"(b.v[i]));
    // reduction with plain add-with-carry: t0 + m is 0 with a carry exactly
    // when t0 != 0; m·17 at limb 6 (two words); m·2^251 at limbs 7 and 8
    const uint32_t m = 0u - t[0];
    const uint64_t m17 = (uint64_t)m * 17u;
    asm("add.cc.u32 %0, %0, %9;\n\t"
        "addc.cc.u32 %1, %1, 0;\n\t"
        "addc.cc.u32 %2, %2, 0;\n\t"
        "addc.cc.u32 %3, %3, 0;\n\t"
        "addc.cc.u32 %4, %4, 0;\n\t"
        "addc.cc.u32 %5, %5, %10;\n\t"
        "addc.cc.u32 %6, %6, %11;\n\t"
        "addc.cc.u32 %7, %7, 0;\n\t"
        "addc.u32 %8, %8, 0;\n\t"
        "add.cc.u32 %6, %6, %12;\n\t"
        "addc.cc.u32 %7, %7, %13;\n\t"
        "addc.u32 %8, %8, 0;"
        : "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8]),
          "+r"(t[9])
        : "r"(t[0] != 0u ? 1u : 0u), "r"((uint32_t)m17), "r"((uint32_t)(m17 >> 32)), "r"(m << 27), "r"(m >> 5));
#pragma unroll
    for (int j = 0; j < 9; j++) t[j] = t[j + 1];
  }
  if (FULL) reduce_once(t);
  Felt r;
#pragma unroll
  for (int j = 0; j < 8; j++) r.v[j] = t[j];
  return r;
}

// Fully reduced product (inputs below 2p): below p.
__device__ __forceinline__ Felt fmul(const Felt& a, const Felt& b) { return fmul_t<true>(a, b); }
// Lazy product: for inputs below 5.6p the result a·b/R + (< p) stays below
// 2p; the permutation keeps every product input below 4.5p.
__device__ __forceinline__ Felt fmul_l(const Felt& a, const Felt& b) { return fmul_t<false>(a, b); }

// a + b without reduction (callers keep the sum below 2^256)
__device__ __forceinline__ Felt ladd(const Felt& a, const Felt& b) {
  Felt r;
  asm("add.cc.u32 %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32 %7, %15, %23;"
      : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]),
        "=r"(r.v[7])
      : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
        "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
  return r;
}
// a - b without reduction (callers guarantee a >= b)
__device__ __forceinline__ Felt lsub(const Felt& a, const Felt& b) {
  Felt r;
  asm("sub.cc.u32 %0, %8, %16;\n\t"
      "subc.cc.u32 %1, %9, %17;\n\t"
      "subc.cc.u32 %2, %10, %18;\n\t"
      "subc.cc.u32 %3, %11, %19;\n\t"
      "subc.cc.u32 %4, %12, %20;\n\t"
      "subc.cc.u32 %5, %13, %21;\n\t"
      "subc.cc.u32 %6, %14, %22;\n\t"
      "subc.u32 %7, %15, %23;"
      : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]),
        "=r"(r.v[7])
      : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
        "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
  return r;
}
// x < 2^255 -> below 2p: with q = x >> 251, x - max(q - 1, 0)·p lies in
// [p - q·(17·2^192 + 1), 2^251 + p) when q > 0 (and is x < 2^251 when q = 0):
// no compare, no select.
__device__ __forceinline__ Felt lreduce(const Felt& x) {
  const uint32_t q = x.v[7] >> 27;
  const uint32_t k = q > 0 ? q - 1 : 0;
  Felt r;
  asm("sub.cc.u32 %0, %8, %16;\n\t"
      "subc.cc.u32 %1, %9, 0;\n\t"
      "subc.cc.u32 %2, %10, 0;\n\t"
      "subc.cc.u32 %3, %11, 0;\n\t"
      "subc.cc.u32 %4, %12, 0;\n\t"
      "subc.cc.u32 %5, %13, 0;\n\t"
      "subc.cc.u32 %6, %14, %17;\n\t"
      "subc.u32 %7, %15, %18;"
      : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]),
        "=r"(r.v[7])
      : "r"(x.v[0]), "r"(x.v[1]), "r"(x.v[2]), "r"(x.v[3]), "r"(x.v[4]), "r"(x.v[5]), "r"(x.v[6]), "r"(x.v[7]),
        "r"(k), "r"(k * 17u), "r"(k << 27));
  return r;
}

__device__ __forceinline__ Felt fadd(const Felt& a, const Felt& b) {
  uint32_t t[8];
  asm("add.cc.u32 %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32 %7, %15, %23;"
      : "=r"(t[0]), "=r"(t[1]), "=r"(t[2]), "=r"(t[3]), "=r"(t[4]), "=r"(t[5]), "=r"(t[6]), "=r"(t[7])
      : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
        "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
  reduce_once(t);  // a + b < 2p < 2^253
  Felt r;
#pragma unroll
  for (int j = 0; j < 8; j++) r.v[j] = t[j];
  return r;
}

__device__ __forceinline__ Felt fsub(const Felt& a, const Felt& b) {
  uint32_t t[8], bw;
  asm("sub.cc.u32 %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32 %8, 0, 0;"
      : "=r"(t[0]), "=r"(t[1]), "=r"(t[2]), "=r"(t[3]), "=r"(t[4]), "=r"(t[5]), "=r"(t[6]), "=r"(t[7]), "=r"(bw)
      : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
        "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
  // a borrow (a < b): add p back
  asm("add.cc.u32 %0, %0, %8;\n\t"
      "addc.cc.u32 %1, %1, 0;\n\t"
      "addc.cc.u32 %2, %2, 0;\n\t"
      "addc.cc.u32 %3, %3, 0;\n\t"
      "addc.cc.u32 %4, %4, 0;\n\t"
      "addc.cc.u32 %5, %5, 0;\n\t"
      "addc.cc.u32 %6, %6, %9;\n\t"
      "addc.u32 %7, %7, %10;"
      : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7])
      : "r"(bw & 1u), "r"(bw & 17u), "r"(bw & 0x08000000u));
  Felt r;
#pragma unroll
  for (int j = 0; j < 8; j++) r.v[j] = t[j];
  return r;
}

__device__ __forceinline__ Felt fcube(const Felt& x) { return fmul_l(fmul_l(x, x), x); }

// 4p and 6p as plain integers (limbs 0, 6, 7 nonzero)
__device__ __forceinline__ Felt p_times(uint32_t k) {
  Felt r{};
  r.v[0] = k;
  r.v[6] = 17u * k;
  r.v[7] = k << 27;
  return r;
}

// MDS [[3, 1, 1], [1, -1, 1], [1, 1, -2]] on inputs below 2p:
// t = s0 + s1 + s2 < 6p; (t + 2 s0, t + 4p - 2 s1, t + 6p - 3 s2), each
// non-negative and below 12p, brought back below 2p.
__device__ __forceinline__ void mds(Felt s[3]) {
  const Felt t = ladd(ladd(s[0], s[1]), s[2]);
  const Felt s1x2 = ladd(s[1], s[1]);
  const Felt s2x3 = ladd(ladd(s[2], s[2]), s[2]);
  const Felt a0 = ladd(t, ladd(s[0], s[0]));
  const Felt a1 = lsub(ladd(t, p_times(4)), s1x2);
  const Felt a2 = lsub(ladd(t, p_times(6)), s2x3);
  s[0] = lreduce(a0);
  s[1] = lreduce(a1);
  s[2] = lreduce(a2);
}

// The permutation with compressed partial rounds (one constant each, added
// to s2; the folded remainder sits in the first of the last 4 full rounds'
// constants): the same permutation, two constant additions fewer per
// partial round (poseidon252_constants.py derives and checks the form).
// Bounds: each round starts below 2p (below 3.5p right after absorbing a
// block), adding a constant keeps every product input below 4.5p, products
// return below 2p, and the MDS output is brought back below 2p.
__device__ __forceinline__ void hades(Felt s[3]) {
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int j = 0; j < 3; j++) s[j] = fcube(ladd(s[j], P252_FULL_RC[3 * r + j]));
    mds(s);
  }
#pragma unroll 1
  for (int k = 0; k < 83; k++) {
    s[2] = fcube(ladd(s[2], P252_PARTIAL_RC[k]));
    mds(s);
  }
#pragma unroll 1
  for (int r = 4; r < 8; r++) {
#pragma unroll
    for (int j = 0; j < 3; j++) s[j] = fcube(ladd(s[j], P252_FULL_RC[3 * r + j]));
    mds(s);
  }
}

// 32 big-endian bytes (as 8 little-endian-stored words) <-> canonical limbs
__device__ __forceinline__ Felt from_be_words(const uint32_t w[8]) {
  Felt x;
#pragma unroll
  for (int k = 0; k < 8; k++) x.v[7 - k] = __byte_perm(w[k], 0, 0x0123);
  return x;
}
__device__ __forceinline__ void to_be_words(const Felt& x, uint32_t w[8]) {
#pragma unroll
  for (int k = 0; k < 8; k++) w[k] = __byte_perm(x.v[7 - k], 0, 0x0123);
}
__device__ __forceinline__ Felt to_mont(const Felt& x) { return fmul_l(x, P252_R2); }  // below 2p
__device__ __forceinline__ Felt from_mont(const Felt& x) {
  Felt one{};
  one.v[0] = 1;
  return fmul(x, one);
}

__device__ __forceinline__ Felt load_hash(const uint8_t* base, size_t i) {
  const uint4* p = reinterpret_cast<const uint4*>(base + 32 * i);
  const uint4 a = __ldg(p), b = __ldg(p + 1);
  const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  return to_mont(from_be_words(w));
}
__device__ __forceinline__ void store_hash(uint8_t* base, size_t i, const Felt& m) {
  uint32_t w[8];
  to_be_words(from_mont(m), w);
  uint4* p = reinterpret_cast<uint4*>(base + 32 * i);
  p[0] = make_uint4(w[0], w[1], w[2], w[3]);
  p[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

// Value k of a node's input sequence: the children (when there is a previous
// layer), then the column words of 8 values each.
__device__ __forceinline__ Felt node_value(uint32_t k, size_t i, const uint8_t* prev,
                                           const uint32_t* const* cols, uint32_t n_cols) {
  if (prev) {
    if (k < 2) return load_hash(prev, 2 * i + k);
    k -= 2;
  }
  const uint32_t c0 = 8 * k;
  const uint32_t len = n_cols - c0 < 8 ? n_cols - c0 : 8;
  Felt f{};
  for (uint32_t q = 0; q < len; q++) {
    const uint32_t v = __ldg(cols[c0 + q] + i);
    // f = f << 31 | v
#pragma unroll
    for (int j = 7; j >= 1; j--) f.v[j] = (f.v[j] << 31) | (f.v[j - 1] >> 1);
    f.v[0] = (f.v[0] << 31) | v;
  }
  if (len < 8) f.v[7] += len << 24;  // length at bit 248
  return to_mont(f);
}

// One node per thread: children from `prev` (or none) and columns [0, n_cols).
// poseidon_hash_many of m values absorbs blocks of two from the sequence
// values, 1, 0: m / 2 + 1 permutations; poseidon_hash(l, r) (children and no
// columns) is one permutation of (l, r, 2). Either way one call site of the
// permutation, inlined with the state in registers.
__global__ void __launch_bounds__(128) poseidon252_layer_kernel(uint32_t log_size, const uint8_t* __restrict__ prev,
                                                                const uint32_t* const* __restrict__ cols,
                                                                uint32_t n_cols, uint8_t* __restrict__ out) {
  const size_t n = (size_t)1 << log_size;
  const bool node_only = prev && n_cols == 0;
  const uint32_t m = (prev ? 2u : 0u) + (n_cols + 7) / 8;  // values
  const uint32_t n_blocks = node_only ? 1u : m / 2 + 1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    Felt s[3] = {};
    if (node_only) s[2] = P252_TWO;
    for (uint32_t b = 0; b < n_blocks; b++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const uint32_t k = 2 * b + h;
        if (k < m) s[h] = ladd(s[h], node_value(k, i, prev, cols, n_cols));
        else if (k == m && !node_only) s[h] = ladd(s[h], P252_ONE);
      }
      hades(s);
    }
    store_hash(out, i, s[0]);
  }
}

// A batch of permutations: states of 3 big-endian hashes each (tests).
__global__ void poseidon252_permute_kernel(const uint8_t* __restrict__ in, uint32_t n, uint8_t* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Felt s[3] = {load_hash(in, 3 * (size_t)i), load_hash(in, 3 * (size_t)i + 1), load_hash(in, 3 * (size_t)i + 2)};
    hades(s);
#pragma unroll
    for (int j = 0; j < 3; j++) store_hash(out, 3 * (size_t)i + j, s[j]);
  }
}

int poseidon252_commit_on_layer(cudaStream_t st, uint32_t log_size, const uint8_t* d_prev,
                                const uint32_t* const* d_cols, uint32_t n_cols, uint8_t* d_out) {
  GS_REQUIRE(log_size <= 30, "layer log size out of range");
  GS_REQUIRE(d_out != nullptr, "null output");
  GS_REQUIRE(n_cols == 0 || d_cols != nullptr, "null column table");
  GS_REQUIRE(((uintptr_t)d_out & 15) == 0 && ((uintptr_t)d_prev & 15) == 0, "hash buffers must be 16-byte aligned");
  const size_t n = (size_t)1 << log_size;
  size_t blocks = (n + 127) / 128;
  const size_t cap = (size_t)num_sms() * 16;
  if (blocks > cap) blocks = cap;
  poseidon252_layer_kernel<<<(unsigned)blocks, 128, 0, st>>>(log_size, d_prev, d_cols, n_cols, d_out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

int poseidon252_permute(cudaStream_t st, const uint8_t* d_in, uint32_t n, uint8_t* d_out) {
  if (n == 0) return OK;
  GS_REQUIRE(((uintptr_t)d_in & 15) == 0 && ((uintptr_t)d_out & 15) == 0, "state buffers must be 16-byte aligned");
  const uint32_t blocks = (n + 127) / 128;
  poseidon252_permute_kernel<<<blocks, 128, 0, st>>>(d_in, n, d_out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

}  // namespace gs

namespace gs {

// ------------------------------------------------ proof of work, Poseidon252
// GrindOps<Poseidon252Channel>::grind (prover/backend/simd/grind.rs:152-190;
// the reference's CUDA backend hands it to that CPU code, cuda/backend.rs:
// 52-56): prefixed = poseidon_hash_many([POW_PREFIX, digest, pow_bits]); the
// answer is the smallest nonce (hi << 32) | low, low < 2^14, hi = 0, 1, ...,
// whose poseidon_hash(prefixed, nonce) has at least pow_bits trailing zero
// bits in its low 128 bits.
constexpr uint32_t P252_POW_PREFIX = 0x12345678u;
constexpr uint32_t P252_GRIND_LOW_LOG = 14, P252_GRIND_STEP = 128;

__device__ __forceinline__ Felt small_felt(uint32_t lo, uint32_t hi) {
  Felt x{};
  x.v[0] = lo;
  x.v[1] = hi;
  return to_mont(x);
}

// One thread: poseidon_hash_many of three values (two permutations).
__global__ void poseidon252_pow_prefix_kernel(const uint8_t* __restrict__ digest, uint32_t pow_bits,
                                              uint8_t* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Felt s[3] = {};
  for (int b = 0; b < 2; b++) {
    if (b == 0) {
      s[0] = fadd(s[0], small_felt(P252_POW_PREFIX, 0));
      s[1] = fadd(s[1], load_hash(digest, 0));
    } else {
      s[0] = fadd(s[0], small_felt(pow_bits, 0));
      s[1] = fadd(s[1], P252_ONE);
    }
    hades(s);
  }
  store_hash(out, 0, s[0]);
}

// Persistent grid over 128-nonce steps of high words [hi0, hi0 + n_hi), in
// increasing nonce order; a block stops at the first step above the recorded
// minimum (a plain read, nothing waits), so the answer is still the smallest
// passing nonce (atomicMin over the 64-bit nonce).
__global__ void __launch_bounds__(P252_GRIND_STEP) poseidon252_grind_kernel(const uint8_t* __restrict__ prefixed,
                                                                           uint32_t hi0, uint32_t n_hi,
                                                                           uint32_t pow_bits,
                                                                           unsigned long long* result) {
  const volatile unsigned long long* best = result;
  const Felt pre = load_hash(prefixed, 0);
  constexpr uint32_t STEPS_PER_HI = (1u << P252_GRIND_LOW_LOG) / P252_GRIND_STEP;
  for (uint32_t step = blockIdx.x; step < n_hi * STEPS_PER_HI; step += gridDim.x) {
    const uint32_t hi = hi0 + step / STEPS_PER_HI;
    const uint32_t low0 = (step % STEPS_PER_HI) * P252_GRIND_STEP;
    if (*best < (((unsigned long long)hi << 32) | low0)) return;
    const uint32_t low = low0 + threadIdx.x;
    Felt s[3] = {pre, small_felt(low, hi), P252_TWO};
    hades(s);
    const Felt h = from_mont(s[0]);
    // trailing zeros of the low 128 bits (limbs 0..3)
    uint32_t tz = 128;
#pragma unroll
    for (int j = 3; j >= 0; j--)
      if (h.v[j]) tz = 32u * j + (uint32_t)(__ffs(h.v[j]) - 1);
    if (tz >= pow_bits) atomicMin(result, ((unsigned long long)hi << 32) | low);
  }
}

int poseidon252_grind(cudaStream_t st, const uint8_t* d_digest, uint32_t pow_bits, uint8_t* d_scratch,
                      uint32_t* h_word, uint64_t* nonce_out, bool digest_is_prefixed) {
  GS_REQUIRE(pow_bits <= 128, "pow_bits > 128 is not supported");
  GS_REQUIRE(((uintptr_t)d_digest & 15) == 0 && ((uintptr_t)d_scratch & 15) == 0, "buffers must be 16-byte aligned");
  const uint8_t* d_pre = d_digest;
  unsigned long long* d_res = reinterpret_cast<unsigned long long*>(d_scratch + 32);  // 8 bytes
  if (!digest_is_prefixed) {  // one thread, two permutations
    d_pre = d_scratch;        // 32 bytes
    poseidon252_pow_prefix_kernel<<<1, 32, 0, st>>>(d_digest, pow_bits, d_scratch);
    note_launch();
    GS_CUDA_TRY(cudaGetLastError());
  }
  // high words per launch: about twice the expected number of chunks
  // (2^(pow_bits - 14) each), 1 to 64
  const uint32_t e = pow_bits > P252_GRIND_LOW_LOG ? pow_bits - P252_GRIND_LOW_LOG + 1 : 0;
  const uint32_t n_hi = e >= 6 ? 64u : 1u << e;
  const uint32_t steps = n_hi * ((1u << P252_GRIND_LOW_LOG) / P252_GRIND_STEP);
  const uint32_t cap = 8u * (uint32_t)num_sms();
  const unsigned blocks = steps < cap ? steps : cap;
  // Bounded search: 2^20 high words cover pow_bits far beyond 40 with
  // overwhelming probability; running out is reported, never looped on.
  for (uint32_t hi = 0; hi < (1u << 20); hi += n_hi) {
    GS_CUDA_TRY(cudaMemsetAsync(d_res, 0xff, 8, st));
    poseidon252_grind_kernel<<<blocks, P252_GRIND_STEP, 0, st>>>(d_pre, hi, n_hi, pow_bits, d_res);
    note_launch();
    GS_CUDA_TRY(cudaGetLastError());
    GS_CUDA_TRY(cudaMemcpyAsync(h_word, d_res, 8, cudaMemcpyDeviceToHost, st));
    GS_TRY(stream_sync(st));
    uint64_t found;
    memcpy(&found, h_word, 8);
    if (found != ~0ull) {
      *nonce_out = found;
      return OK;
    }
  }
  set_error("poseidon252 grind: no nonce found within the search bound");
  return ERR_TIMEOUT;
}

}  // namespace gs
