// Mersenne-31 field tower for the device (and host) side of gpustark.
//
// M31:  p = 2^31 - 1, canonical values in [0, p).
// CM31: M31[i] / (i^2 + 1).
// QM31: CM31[u] / (u^2 - (2 + i)), stored in device memory as 4 coordinate
//       planes (a, b, c, d) for (a + b i) + (c + d i) u.
//
// Semantics follow the reference field code (crates/stwo/src/core/fields/
// m31.rs:58-110, cm31.rs:43-78, qm31.rs:87-135). Every operation returns the
// canonical representative, so results are bit-identical to the reference no
// matter how the product is reduced.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define GS_HD __host__ __device__ __forceinline__
#else
#define GS_HD inline
#endif

namespace gs {

constexpr uint32_t P = 0x7fffffffu;

GS_HD uint32_t umin32(uint32_t a, uint32_t b) { return a < b ? a : b; }

// a + b for a, b < p: with s = a + b - p (mod 2^32), the result is
// min(s + p, s) (s wraps above s + p exactly when a + b < p). On the device
// that is one three-input add and one add-then-min (VIADDMNMX).
GS_HD uint32_t add(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  uint32_t s = a + b - P;
  return __viaddmin_u32(s, P, s);
#else
  uint32_t r = a + b;
  return umin32(r, r - P);
#endif
}
// a - b: d = a - b (mod 2^32), result min(d, d + p).
GS_HD uint32_t sub(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  uint32_t d = a - b;
  return __viaddmin_u32(d, P, d);
#else
  uint32_t r = a + (P - b);
  return umin32(r, r - P);
#endif
}
GS_HD uint32_t neg(uint32_t a) { uint32_t r = P - a; return umin32(r, r - P); }
GS_HD uint32_t mul(uint32_t a, uint32_t b);

// a * b: 62-bit product folded once (lo 31 bits + hi 31 bits < 2p), then one
// conditional subtract.
//
// Device form: with b2 = 2b < 2^32, the 64-bit product a * b2 = 2(ab) has
// high word (ab) >> 31 and low word 2((ab) mod 2^31), so one wide multiply
// and one shift-add (LEA.HI) give r = (ab >> 31) + (ab mod 2^31) < 2p, and
// an add-then-min finishes the reduction.
__device__ __forceinline__ uint32_t mul_b2(uint32_t a, uint32_t b2) {
  uint64_t p = (uint64_t)a * b2;
  uint32_t r = (uint32_t)(p >> 32) + ((uint32_t)p >> 1);
  return __viaddmin_u32(r, 0u - P, r);
}
// FMA-pipe forms. The integer ALU pipe bounds the FFT, Blake2s and
// constraint kernels while the FMA pipe idles; an add issued as an IMAD
// against a runtime 1 (or -1), which the compiler cannot fold, runs there
// instead, leaving one add-then-min per field add/sub on the ALU pipe.
__device__ __forceinline__ uint32_t imad_u32(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
}
// a + b (one = 1 at run time)
__device__ __forceinline__ uint32_t add_f(uint32_t a, uint32_t b, uint32_t one) {
  uint32_t s = imad_u32(a, one, b);
  return __viaddmin_u32(s, 0u - P, s);
}
// a - b (neg1 = 2^32 - 1 at run time)
__device__ __forceinline__ uint32_t sub_f(uint32_t a, uint32_t b, uint32_t neg1) {
  uint32_t d = imad_u32(b, neg1, a);
  return __viaddmin_u32(d, P, d);
}
// a * b with the doubling of b on the FMA pipe
__device__ __forceinline__ uint32_t mul_f(uint32_t a, uint32_t b, uint32_t one) {
  return mul_b2(a, imad_u32(b, one, b));
}
GS_HD uint32_t mul(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return mul_b2(a, b << 1);
#else
  uint64_t p = (uint64_t)a * b;
  uint32_t r = (uint32_t)(p & P) + (uint32_t)(p >> 31);
  return umin32(r, r - P);
#endif
}
// Fold of a 64-bit lazy accumulator of products to below 2^34, congruent
// mod p but not reduced: x = hi * 2^32 + lo and 2^32 = 2 (mod p), so x = 2 hi
// + lo (mod p), one wide multiply-add on the device. Three more products of
// two values below 2^31 fit after it (3 * 2^62 + 2^34 < 2^64).
__device__ __forceinline__ uint64_t fold64h(uint64_t x) {
  uint64_t r;
  asm("mad.wide.u32 %0, %1, 2, %2;" : "=l"(r) : "r"((uint32_t)(x >> 32)), "l"(x & 0xffffffffull));
  return r;
}
// Reduce any 64-bit value (used for lazily accumulated sums of products).
GS_HD uint32_t reduce64(uint64_t v) {
  // v = h * 2^62 + m * 2^31 + l  ->  h + m + l (mod p), each part < 2^31
  uint32_t l = (uint32_t)v & P;
  uint32_t m = (uint32_t)(v >> 31) & P;
  uint32_t h = (uint32_t)(v >> 62);
  uint32_t r = l + m;                 // < 2^32
  r = umin32(r, r - P);               // < p + small
  r = r + h;
  r = umin32(r, r - P);
  return umin32(r, r - P);
}

GS_HD uint32_t sqr(uint32_t a) { return mul(a, a); }
GS_HD uint32_t sqn(uint32_t v, int n) { for (int i = 0; i < n; i++) v = sqr(v); return v; }
// a^(p-2) by a fixed addition chain (37 multiplications).
GS_HD uint32_t inv(uint32_t v) {
  uint32_t t0 = mul(sqn(v, 2), v);
  uint32_t t1 = mul(sqn(t0, 1), t0);
  uint32_t t2 = mul(sqn(t1, 3), t0);
  uint32_t t3 = mul(sqn(t2, 1), t0);
  uint32_t t4 = mul(sqn(t3, 8), t3);
  uint32_t t5 = mul(sqn(t4, 8), t3);
  return mul(sqn(t5, 7), t2);
}

struct cm31 { uint32_t a, b; };
GS_HD cm31 cm_add(cm31 x, cm31 y) { return {add(x.a, y.a), add(x.b, y.b)}; }
GS_HD cm31 cm_sub(cm31 x, cm31 y) { return {sub(x.a, y.a), sub(x.b, y.b)}; }
GS_HD cm31 cm_neg(cm31 x) { return {neg(x.a), neg(x.b)}; }
GS_HD cm31 cm_mul(cm31 x, cm31 y) {
  // (a + bi)(c + di) = (ac - bd) + ((a+b)(c+d) - ac - bd) i
  uint32_t ac = mul(x.a, y.a), bd = mul(x.b, y.b);
  uint32_t s = mul(add(x.a, x.b), add(y.a, y.b));
  return {sub(ac, bd), sub(sub(s, ac), bd)};
}
GS_HD cm31 cm_mul_m31(cm31 x, uint32_t s) { return {mul(x.a, s), mul(x.b, s)}; }
GS_HD cm31 cm_sqr(cm31 x) { return cm_mul(x, x); }
GS_HD cm31 cm_inv(cm31 x) {
  uint32_t n = inv(add(sqr(x.a), sqr(x.b)));
  return {mul(x.a, n), mul(neg(x.b), n)};
}
// Multiply by R = 2 + i.
GS_HD cm31 cm_mul_r(cm31 x) {
  // (a + bi)(2 + i) = (2a - b) + (a + 2b) i
  return {sub(add(x.a, x.a), x.b), add(x.a, add(x.b, x.b))};
}

struct qm31 { cm31 x, y; };
GS_HD qm31 qm_zero() { return {{0, 0}, {0, 0}}; }
GS_HD qm31 qm_one() { return {{1, 0}, {0, 0}}; }
GS_HD qm31 qm_from_m31(uint32_t v) { return {{v, 0}, {0, 0}}; }
GS_HD qm31 qm_make(uint32_t a, uint32_t b, uint32_t c, uint32_t d) { return {{a, b}, {c, d}}; }
GS_HD bool qm_eq(qm31 p, qm31 q) { return p.x.a == q.x.a && p.x.b == q.x.b && p.y.a == q.y.a && p.y.b == q.y.b; }
GS_HD qm31 qm_add(qm31 p, qm31 q) { return {cm_add(p.x, q.x), cm_add(p.y, q.y)}; }
GS_HD qm31 qm_sub(qm31 p, qm31 q) { return {cm_sub(p.x, q.x), cm_sub(p.y, q.y)}; }
GS_HD qm31 qm_neg(qm31 p) { return {cm_neg(p.x), cm_neg(p.y)}; }
GS_HD qm31 qm_mul(qm31 p, qm31 q) {
  // (x0 + y0 u)(x1 + y1 u) = (x0 x1 + R y0 y1) + ((x0+y0)(x1+y1) - x0 x1 - y0 y1) u
  cm31 xx = cm_mul(p.x, q.x), yy = cm_mul(p.y, q.y);
  cm31 s = cm_mul(cm_add(p.x, p.y), cm_add(q.x, q.y));
  return {cm_add(xx, cm_mul_r(yy)), cm_sub(cm_sub(s, xx), yy)};
}
GS_HD qm31 qm_mul_m31(qm31 p, uint32_t s) { return {cm_mul_m31(p.x, s), cm_mul_m31(p.y, s)}; }
GS_HD qm31 qm_mul_cm31(qm31 p, cm31 c) { return {cm_mul(p.x, c), cm_mul(p.y, c)}; }
GS_HD qm31 qm_add_m31(qm31 p, uint32_t s) { return {{add(p.x.a, s), p.x.b}, p.y}; }
GS_HD qm31 qm_sqr(qm31 p) { return qm_mul(p, p); }
GS_HD qm31 qm_inv(qm31 p) {
  cm31 b2 = cm_sqr(p.y);
  cm31 ib2 = {neg(b2.b), b2.a};
  cm31 denom = cm_sub(cm_sqr(p.x), cm_add(cm_add(b2, b2), ib2));
  cm31 di = cm_inv(denom);
  return {cm_mul(p.x, di), cm_neg(cm_mul(p.y, di))};
}
GS_HD qm31 qm_conj(qm31 p) { return {p.x, cm_neg(p.y)}; }

// Circle-group helpers over M31 and QM31.
struct pt31 { uint32_t x, y; };
GS_HD pt31 pt_add(pt31 a, pt31 b) {
  return {sub(mul(a.x, b.x), mul(a.y, b.y)), add(mul(a.x, b.y), mul(a.y, b.x))};
}
GS_HD pt31 pt_conj(pt31 a) { return {a.x, neg(a.y)}; }
struct ptq { qm31 x, y; };
GS_HD ptq ptq_add(ptq a, ptq b) {
  return {qm_sub(qm_mul(a.x, b.x), qm_mul(a.y, b.y)), qm_add(qm_mul(a.x, b.y), qm_mul(a.y, b.x))};
}
GS_HD qm31 qm_double_x(qm31 x) { qm31 s = qm_sqr(x); return qm_sub(qm_add(s, s), qm_one()); }
GS_HD uint32_t double_x(uint32_t x) { uint32_t s = sqr(x); return sub(add(s, s), 1); }

}  // namespace gs
