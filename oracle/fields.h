// ORACLE — test infrastructure only. CPU restatement of the reference's
// Mersenne-31 field tower; only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg may use anything under oracle/.
//
// Follows (reference paths within the Stwo fork):
//   crates/stwo/src/core/fields/m31.rs:14,48-60  (P, partial_reduce, reduce)
//   crates/stwo/src/core/fields/m31.rs:78-110    (add, neg, sub, mul)
//   crates/stwo/src/core/fields/m31.rs:168-188   (pow2147483645 inverse chain)
//   crates/stwo/src/core/fields/cm31.rs:43-78    (CM31 mul / inverse)
//   crates/stwo/src/core/fields/qm31.rs:14,87-135 (R = 2+i, QM31 mul / inverse)
//   crates/stwo/src/core/fields/mod.rs:44-107    (batch inverse)
//   crates/stwo/src/core/fields/mod.rs:412-415   (complex conjugate)
#pragma once
#include <cstdint>
#include <cstddef>
#include <vector>
#include <cassert>

namespace orc {

constexpr uint32_t P = 2147483647u;

// M31::reduce for val in [0, P^2): m31.rs:58-60.
inline uint32_t reduce64(uint64_t v) {
  return (uint32_t)(((((v >> 31) + v + 1) >> 31) + v) & (uint64_t)P);
}
inline uint32_t partial_reduce(uint32_t v) { return v >= P ? v - P : v; }

struct M31 {
  uint32_t v = 0;
  M31() = default;
  constexpr explicit M31(uint32_t x) : v(x) {}
  static M31 from_u64(uint64_t x) { return M31(reduce64(x)); }
  static M31 from_i64(int64_t x) {
    int64_t r = x % (int64_t)P;
    if (r < 0) r += P;
    return M31((uint32_t)r);
  }
  bool operator==(const M31& o) const { return v == o.v; }
  bool operator!=(const M31& o) const { return v != o.v; }
  bool is_zero() const { return v == 0; }
};
inline M31 operator+(M31 a, M31 b) { return M31(partial_reduce(a.v + b.v)); }
inline M31 operator-(M31 a, M31 b) { return M31(partial_reduce(a.v + P - b.v)); }
inline M31 operator-(M31 a) { return M31(partial_reduce(P - a.v)); }
inline M31 operator*(M31 a, M31 b) { return M31(reduce64((uint64_t)a.v * b.v)); }
inline M31& operator+=(M31& a, M31 b) { return a = a + b; }
inline M31& operator-=(M31& a, M31 b) { return a = a - b; }
inline M31& operator*=(M31& a, M31 b) { return a = a * b; }

template <class T> inline T sqn(T v, int n) { for (int i = 0; i < n; i++) v = v * v; return v; }
// m31.rs:168-176: v^(P-2) with 37 multiplications.
inline M31 pow2147483645(M31 v) {
  M31 t0 = sqn(v, 2) * v;
  M31 t1 = sqn(t0, 1) * t0;
  M31 t2 = sqn(t1, 3) * t0;
  M31 t3 = sqn(t2, 1) * t0;
  M31 t4 = sqn(t3, 8) * t3;
  M31 t5 = sqn(t4, 8) * t3;
  return sqn(t5, 7) * t2;
}
inline M31 inv(M31 v) { assert(!v.is_zero()); return pow2147483645(v); }

struct CM31 {
  M31 a, b;  // a + b i
  CM31() = default;
  constexpr CM31(M31 a_, M31 b_) : a(a_), b(b_) {}
  explicit CM31(M31 x) : a(x), b(0) {}
  static CM31 u(uint32_t x, uint32_t y) { return CM31(M31(x), M31(y)); }
  bool operator==(const CM31& o) const { return a == o.a && b == o.b; }
  bool operator!=(const CM31& o) const { return !(*this == o); }
  bool is_zero() const { return a.is_zero() && b.is_zero(); }
};
inline CM31 operator+(CM31 x, CM31 y) { return CM31(x.a + y.a, x.b + y.b); }
inline CM31 operator-(CM31 x, CM31 y) { return CM31(x.a - y.a, x.b - y.b); }
inline CM31 operator-(CM31 x) { return CM31(-x.a, -x.b); }
inline CM31 operator*(CM31 x, CM31 y) { return CM31(x.a * y.a - x.b * y.b, x.a * y.b + x.b * y.a); }
inline CM31 operator*(CM31 x, M31 y) { return CM31(x.a * y, x.b * y); }
inline CM31 inv(CM31 x) {
  assert(!x.is_zero());
  return CM31(x.a, -x.b) * inv(x.a * x.a + x.b * x.b);
}

struct QM31 {
  CM31 x, y;  // x + y u, u^2 = 2 + i
  QM31() = default;
  constexpr QM31(CM31 x_, CM31 y_) : x(x_), y(y_) {}
  explicit QM31(M31 v) : x(v), y() {}
  static QM31 u(uint32_t a, uint32_t b, uint32_t c, uint32_t d) { return QM31(CM31::u(a, b), CM31::u(c, d)); }
  static QM31 from_m31(M31 a, M31 b, M31 c, M31 d) { return QM31(CM31(a, b), CM31(c, d)); }
  uint32_t coord(int i) const { return i == 0 ? x.a.v : i == 1 ? x.b.v : i == 2 ? y.a.v : y.b.v; }
  bool operator==(const QM31& o) const { return x == o.x && y == o.y; }
  bool operator!=(const QM31& o) const { return !(*this == o); }
  bool is_zero() const { return x.is_zero() && y.is_zero(); }
  // Lexicographic order over (a, b, c, d), as the derived Ord of the reference type.
  bool operator<(const QM31& o) const {
    for (int i = 0; i < 4; i++) if (coord(i) != o.coord(i)) return coord(i) < o.coord(i);
    return false;
  }
};
inline const CM31 R_CM31 = CM31::u(2, 1);
inline QM31 operator+(QM31 p, QM31 q) { return QM31(p.x + q.x, p.y + q.y); }
inline QM31 operator-(QM31 p, QM31 q) { return QM31(p.x - q.x, p.y - q.y); }
inline QM31 operator-(QM31 p) { return QM31(-p.x, -p.y); }
inline QM31 operator*(QM31 p, QM31 q) { return QM31(p.x * q.x + R_CM31 * p.y * q.y, p.x * q.y + p.y * q.x); }
inline QM31 operator*(QM31 p, M31 s) { return QM31(p.x * s, p.y * s); }
inline QM31 operator*(M31 s, QM31 p) { return p * s; }
inline QM31 operator+(QM31 p, M31 s) { return QM31(CM31(p.x.a + s, p.x.b), p.y); }
inline QM31 operator-(QM31 p, M31 s) { return QM31(CM31(p.x.a - s, p.x.b), p.y); }
inline QM31 mul_cm31(QM31 p, CM31 c) { return QM31(p.x * c, p.y * c); }
inline QM31& operator+=(QM31& a, QM31 b) { return a = a + b; }
inline QM31& operator-=(QM31& a, QM31 b) { return a = a - b; }
inline QM31& operator*=(QM31& a, QM31 b) { return a = a * b; }
inline QM31 inv(QM31 p) {
  assert(!p.is_zero());
  CM31 b2 = p.y * p.y;
  CM31 ib2 = CM31(-b2.b, b2.a);
  CM31 denom = p.x * p.x - (b2 + b2 + ib2);
  CM31 di = inv(denom);
  return QM31(p.x * di, -p.y * di);
}
inline QM31 conj(QM31 p) { return QM31(p.x, -p.y); }
inline QM31 qm31_from_partial_evals(const QM31 e[4]) {
  QM31 r = e[0];
  r += e[1] * QM31::u(0, 1, 0, 0);
  r += e[2] * QM31::u(0, 0, 1, 0);
  r += e[3] * QM31::u(0, 0, 0, 1);
  return r;
}
inline M31 operator/(M31 a, M31 b) { return a * inv(b); }
inline QM31 operator/(QM31 a, QM31 b) { return a * inv(b); }
inline QM31 operator/(QM31 a, M31 b) { return a * inv(b); }

// Generic helpers used by the circle code.
inline M31 one_of(M31) { return M31(1); }
inline QM31 one_of(QM31) { return QM31(M31(1)); }
inline M31 zero_of(M31) { return M31(0); }
inline QM31 zero_of(QM31) { return QM31(); }

// batch_inverse_in_place (fields/mod.rs:71-101); any correct inverse gives the
// same canonical values, the classic Montgomery trick is used here.
template <class F>
void batch_inverse(const F* in, F* out, size_t n) {
  if (n == 0) return;
  out[0] = in[0];
  for (size_t i = 1; i < n; i++) out[i] = out[i - 1] * in[i];
  F cur = inv(out[n - 1]);
  for (size_t i = n - 1; i > 0; i--) {
    out[i] = out[i - 1] * cur;
    cur = cur * in[i];
  }
  out[0] = cur;
}

}  // namespace orc
