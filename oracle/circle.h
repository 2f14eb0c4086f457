// ORACLE — test infrastructure only (see fields.h).
// Circle group, cosets, circle domains and index helpers.
// Follows:
//   crates/stwo/src/core/circle.rs:12-131        (CirclePoint, add, double_x, mul, conjugate)
//   crates/stwo/src/core/circle.rs:163-214       (random point from channel, generators)
//   crates/stwo/src/core/circle.rs:221-412       (CirclePointIndex, Coset)
//   crates/stwo/src/core/poly/circle/canonic.rs  (CanonicCoset)
//   crates/stwo/src/core/poly/circle/domain.rs   (CircleDomain)
//   crates/stwo/src/core/utils.rs                (bit_reverse_index, offset index)
//   crates/stwo/src/core/constraints.rs:12-93    (coset_vanishing, point_vanishing)
#pragma once
#include "fields.h"
#include <algorithm>

namespace orc {

template <class F>
struct CirclePoint {
  F x, y;
  static CirclePoint zero() { return {one_of(F()), zero_of(F())}; }
  bool operator==(const CirclePoint& o) const { return x == o.x && y == o.y; }
  bool operator!=(const CirclePoint& o) const { return !(*this == o); }
};
template <class F> CirclePoint<F> operator+(const CirclePoint<F>& a, const CirclePoint<F>& b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <class F> CirclePoint<F> conjugate(const CirclePoint<F>& a) { return {a.x, -a.y}; }
template <class F> CirclePoint<F> operator-(const CirclePoint<F>& a) { return conjugate(a); }
template <class F> CirclePoint<F> operator-(const CirclePoint<F>& a, const CirclePoint<F>& b) { return a + conjugate(b); }
template <class F> CirclePoint<F> antipode(const CirclePoint<F>& a) { return {-a.x, -a.y}; }
template <class F> CirclePoint<F> dbl(const CirclePoint<F>& a) { return a + a; }
template <class F> F double_x(F x) { F sx = x * x; return sx + sx - one_of(F()); }
template <class F> CirclePoint<F> repeated_double(CirclePoint<F> a, uint32_t n) {
  for (uint32_t i = 0; i < n; i++) a = dbl(a);
  return a;
}
template <class F> CirclePoint<F> mul_scalar(const CirclePoint<F>& p, unsigned __int128 scalar) {
  CirclePoint<F> res = CirclePoint<F>::zero(), cur = p;
  while (scalar > 0) {
    if (scalar & 1) res = res + cur;
    cur = dbl(cur);
    scalar >>= 1;
  }
  return res;
}
inline CirclePoint<QM31> to_qm31(const CirclePoint<M31>& p) { return {QM31(p.x), QM31(p.y)}; }
inline CirclePoint<QM31> operator+(const CirclePoint<QM31>& a, const CirclePoint<M31>& b) { return a + to_qm31(b); }

constexpr uint32_t M31_CIRCLE_LOG_ORDER = 31;
inline const CirclePoint<M31> M31_CIRCLE_GEN = {M31(2), M31(1268011823)};
inline const CirclePoint<QM31> SECURE_FIELD_CIRCLE_GEN = {
    QM31::u(1, 0, 478637715, 513582971), QM31::u(992285211, 649143431, 740191619, 1186584352)};

// CirclePointIndex: integers mod 2^31 (circle.rs:221-282).
struct CPI {
  uint64_t v;
  static constexpr uint64_t MASK = (1ull << M31_CIRCLE_LOG_ORDER) - 1;
  CPI reduce() const { return CPI{v & MASK}; }
  static CPI subgroup_gen(uint32_t log_size) { return CPI{1ull << (M31_CIRCLE_LOG_ORDER - log_size)}; }
  CirclePoint<M31> to_point() const { return mul_scalar(M31_CIRCLE_GEN, (unsigned __int128)v); }
  CPI half() const { assert((v & 1) == 0); return CPI{v >> 1}; }
  bool operator==(const CPI& o) const { return v == o.v; }
};
inline CPI operator+(CPI a, CPI b) { return CPI{a.v + b.v}.reduce(); }
inline CPI operator-(CPI a, CPI b) { return CPI{a.v + (1ull << M31_CIRCLE_LOG_ORDER) - b.v}.reduce(); }
inline CPI operator*(CPI a, uint64_t s) { return CPI{a.v * s}.reduce(); }
inline CPI operator-(CPI a) { return CPI{(1ull << M31_CIRCLE_LOG_ORDER) - a.v}.reduce(); }

struct Coset {
  CPI initial_index;
  CirclePoint<M31> initial;
  CPI step_size;
  CirclePoint<M31> step;
  uint32_t log_size;
  static Coset make(CPI initial_index, uint32_t log_size) {
    CPI step_size = CPI::subgroup_gen(log_size);
    return Coset{initial_index, initial_index.to_point(), step_size, step_size.to_point(), log_size};
  }
  static Coset subgroup(uint32_t log_size) { return make(CPI{0}, log_size); }
  static Coset odds(uint32_t log_size) { return make(CPI::subgroup_gen(log_size + 1), log_size); }
  static Coset half_odds(uint32_t log_size) { return make(CPI::subgroup_gen(log_size + 2), log_size); }
  size_t size() const { return (size_t)1 << log_size; }
  Coset dbl() const {
    assert(log_size > 0);
    return Coset{initial_index * 2, orc::dbl(initial), step_size * 2, orc::dbl(step), log_size - 1};
  }
  Coset repeated_double(uint32_t n) const { Coset c = *this; for (uint32_t i = 0; i < n; i++) c = c.dbl(); return c; }
  CPI index_at(size_t i) const { return initial_index + step_size * i; }
  CirclePoint<M31> at(size_t i) const { return index_at(i).to_point(); }
  Coset conjugate() const {
    CPI ii = -initial_index, ss = -step_size;
    return Coset{ii, ii.to_point(), ss, ss.to_point(), log_size};
  }
  // Points in coset order, by repeated addition of the step (CosetIterator).
  std::vector<CirclePoint<M31>> points() const {
    std::vector<CirclePoint<M31>> r(size());
    CirclePoint<M31> cur = initial;
    for (size_t i = 0; i < size(); i++) { r[i] = cur; cur = cur + step; }
    return r;
  }
  bool operator==(const Coset& o) const {
    return initial_index == o.initial_index && step_size == o.step_size && log_size == o.log_size;
  }
};

struct CircleDomain {
  Coset half_coset;
  uint32_t log_size() const { return half_coset.log_size + 1; }
  size_t size() const { return (size_t)1 << log_size(); }
  CPI index_at(size_t i) const {
    if (i < half_coset.size()) return half_coset.index_at(i);
    return -half_coset.index_at(i - half_coset.size());
  }
  CirclePoint<M31> at(size_t i) const { return index_at(i).to_point(); }
  bool is_canonic() const { return half_coset.initial_index * 4 == half_coset.step_size; }
  // All points in natural (circle domain) order: half coset then its conjugate.
  std::vector<CirclePoint<M31>> points() const {
    std::vector<CirclePoint<M31>> r = half_coset.points();
    size_t h = r.size();
    r.resize(2 * h);
    for (size_t i = 0; i < h; i++) r[h + i] = conjugate(r[i]);
    return r;
  }
};

struct CanonicCoset {
  Coset coset;
  static CanonicCoset make(uint32_t log_size) { assert(log_size > 0); return CanonicCoset{Coset::odds(log_size)}; }
  Coset half_coset() const { return Coset::half_odds(coset.log_size - 1); }
  CircleDomain circle_domain() const { return CircleDomain{half_coset()}; }
  uint32_t log_size() const { return coset.log_size; }
  CirclePoint<M31> step() const { return coset.step; }
  CirclePoint<M31> at(size_t i) const { return coset.at(i); }
};

inline size_t bit_reverse_index(size_t i, uint32_t log_size) {
  if (log_size == 0) return i;
  size_t r = 0;
  for (uint32_t b = 0; b < log_size; b++) r |= ((i >> b) & 1) << (log_size - 1 - b);
  return r;
}
template <class T> void bit_reverse(std::vector<T>& v) {
  size_t n = v.size();
  uint32_t log_n = 0;
  while (((size_t)1 << log_n) < n) log_n++;
  assert(((size_t)1 << log_n) == n);
  for (size_t i = 0; i < n; i++) {
    size_t j = bit_reverse_index(i, log_n);
    if (j > i) std::swap(v[i], v[j]);
  }
}
inline uint32_t ilog2(size_t n) { uint32_t r = 0; while (((size_t)1 << (r + 1)) <= n) r++; return r; }

// utils.rs offset_bit_reversed_circle_domain_index.
inline size_t offset_bit_reversed_circle_domain_index(size_t i, uint32_t domain_log_size, uint32_t eval_log_size, int64_t offset) {
  int64_t prev = (int64_t)bit_reverse_index(i, eval_log_size);
  int64_t half = (int64_t)1 << (eval_log_size - 1);
  int64_t step = offset * ((int64_t)1 << (eval_log_size - domain_log_size - 1));
  auto rem = [](int64_t a, int64_t m) { int64_t r = a % m; return r < 0 ? r + m : r; };
  if (prev < half) prev = rem(prev + step, half);
  else prev = rem(prev - step, half) + half;
  return bit_reverse_index((size_t)prev, eval_log_size);
}

// constraints.rs:12-35.
template <class F> F coset_vanishing(const Coset& coset, CirclePoint<F> p) {
  CirclePoint<F> init{F(coset.initial.x), F(coset.initial.y)};
  CirclePoint<M31> hs = coset.step_size.half().to_point();
  CirclePoint<F> half_step{F(hs.x), F(hs.y)};
  p = p - init + half_step;
  F x = p.x;
  for (uint32_t i = 1; i < coset.log_size; i++) x = double_x(x);
  return x;
}
inline M31 coset_vanishing(const Coset& coset, CirclePoint<M31> p) {
  p = p - coset.initial + coset.step_size.half().to_point();
  M31 x = p.x;
  for (uint32_t i = 1; i < coset.log_size; i++) x = double_x(x);
  return x;
}

// circle.rs:169-181.
template <class Ch> CirclePoint<QM31> get_random_point(Ch& ch) {
  QM31 t = ch.draw_secure_felt();
  QM31 t2 = t * t;
  QM31 inv_ = inv(t2 + M31(1));
  QM31 x = (QM31(M31(1)) + (-t2)) * inv_;
  QM31 y = (t + t) * inv_;
  return {x, y};
}

}  // namespace orc
