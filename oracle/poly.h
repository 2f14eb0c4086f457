// ORACLE — test infrastructure only (see fields.h).
// Circle FFT (interpolate / evaluate), twiddle tree, line interpolation and
// point evaluation of coefficient polynomials.
// Follows:
//   crates/stwo/src/core/fft.rs:5-21                            (butterfly / ibutterfly)
//   crates/stwo/src/prover/backend/cpu/circle.rs:28-80          (interpolate)
//   crates/stwo/src/prover/backend/cpu/circle.rs:82-98          (eval_at_point)
//   crates/stwo/src/prover/backend/cpu/circle.rs:182-228        (evaluate)
//   crates/stwo/src/prover/backend/cpu/circle.rs:230-305        (twiddles, layer loop, circle twiddles)
//   crates/stwo/src/core/poly/utils.rs:8-68                     (fold, folding alphas, line twiddles)
//   crates/stwo/src/prover/line.rs:45-70                        (line interpolate / line_ifft)
#pragma once
#include "circle.h"
#include <functional>

namespace orc {

template <class F> inline void butterfly(F& v0, F& v1, M31 t) { F tmp = v1 * t; v1 = v0 - tmp; v0 = v0 + tmp; }
template <class F> inline void ibutterfly(F& v0, F& v1, M31 it) { F tmp = v0; v0 = tmp + v1; v1 = (tmp - v1) * it; }

struct TwiddleTree {
  Coset root_coset;
  std::vector<M31> twiddles, itwiddles;
};

// slow_precompute_twiddles (cpu/circle.rs:273-289).
inline std::vector<M31> slow_precompute_twiddles(Coset coset) {
  std::vector<M31> tw;
  tw.reserve(coset.size());
  uint32_t levels = coset.log_size;
  for (uint32_t l = 0; l < levels; l++) {
    size_t i0 = tw.size();
    auto pts = coset.points();
    std::vector<M31> xs(coset.size() / 2);
    for (size_t i = 0; i < xs.size(); i++) xs[i] = pts[i].x;
    bit_reverse(xs);
    tw.insert(tw.end(), xs.begin(), xs.end());
    (void)i0;
    coset = coset.dbl();
  }
  tw.push_back(M31(1));
  return tw;
}

inline TwiddleTree precompute_twiddles(Coset coset) {
  TwiddleTree t;
  t.root_coset = coset;
  t.twiddles = slow_precompute_twiddles(coset);
  t.itwiddles.resize(t.twiddles.size());
  batch_inverse(t.twiddles.data(), t.itwiddles.data(), t.twiddles.size());
  return t;
}

// domain_line_twiddles_from_tree: line layer j of a domain of log size n is the
// slice of length 2^(n-2-j) that ends 2^(n-2-j) elements before the buffer end.
inline const M31* line_twiddles(const std::vector<M31>& buf, uint32_t domain_log_size, uint32_t j) {
  uint32_t k = domain_log_size - 1;  // line domain log size
  size_t len = (size_t)1 << (k - 1 - j);
  assert(buf.size() >= ((size_t)1 << k));
  return buf.data() + buf.size() - 2 * len;
}

template <class F>
inline void fft_layer_loop(std::vector<F>& values, uint32_t i, size_t h, M31 t, bool inverse) {
  for (size_t l = 0; l < ((size_t)1 << i); l++) {
    size_t idx0 = (h << (i + 1)) + l;
    size_t idx1 = idx0 + ((size_t)1 << i);
    if (inverse) ibutterfly(values[idx0], values[idx1], t);
    else butterfly(values[idx0], values[idx1], t);
  }
}

// circle_twiddles_from_line_twiddles: pairs [x, y] -> [y, -y, -x, x].
inline std::vector<M31> circle_twiddles(const M31* first_line, size_t first_line_len) {
  std::vector<M31> c;
  c.reserve(first_line_len * 2);
  for (size_t q = 0; 2 * q + 1 < first_line_len; q++) {
    M31 x = first_line[2 * q], y = first_line[2 * q + 1];
    c.push_back(y); c.push_back(-y); c.push_back(-x); c.push_back(x);
  }
  return c;
}

// interpolate: bit-reversed evaluations on `domain` -> coefficients (in place).
inline void interpolate(std::vector<M31>& values, const CircleDomain& domain, const TwiddleTree& tw) {
  uint32_t n = domain.log_size();
  assert(values.size() == domain.size());
  assert(n <= tw.root_coset.log_size + 1);
  if (n == 1) {
    M31 y = domain.half_coset.initial.y;
    M31 two(2);
    M31 yn_inv = inv(y * two);
    M31 y_inv = yn_inv * two;
    M31 n_inv = yn_inv * y;
    M31 v0 = values[0], v1 = values[1];
    ibutterfly(v0, v1, y_inv);
    values = {v0 * n_inv, v1 * n_inv};
    return;
  }
  if (n == 2) {
    M31 x = domain.half_coset.initial.x, y = domain.half_coset.initial.y;
    M31 four(4);
    M31 xyn_inv = inv(x * y * four);
    M31 x_inv = xyn_inv * y * four;
    M31 y_inv = xyn_inv * x * four;
    M31 n_inv = xyn_inv * x * y;
    M31 v0 = values[0], v1 = values[1], v2 = values[2], v3 = values[3];
    ibutterfly(v0, v1, y_inv);
    ibutterfly(v2, v3, -y_inv);
    ibutterfly(v0, v2, x_inv);
    ibutterfly(v1, v3, x_inv);
    values = {v0 * n_inv, v1 * n_inv, v2 * n_inv, v3 * n_inv};
    return;
  }
  size_t first_len = (size_t)1 << (n - 2);
  auto ct = circle_twiddles(line_twiddles(tw.itwiddles, n, 0), first_len);
  for (size_t h = 0; h < ct.size(); h++) fft_layer_loop(values, 0, h, ct[h], true);
  for (uint32_t j = 0; j + 1 < n; j++) {
    const M31* lt = line_twiddles(tw.itwiddles, n, j);
    size_t len = (size_t)1 << (n - 2 - j);
    for (size_t h = 0; h < len; h++) fft_layer_loop(values, j + 1, h, lt[h], true);
  }
  M31 inv_n = inv(M31((uint32_t)domain.size()));
  for (auto& v : values) v = v * inv_n;
}

// evaluate: coefficients (zero-extended to the domain size) -> bit-reversed evaluations.
inline std::vector<M31> evaluate(const std::vector<M31>& coeffs, const CircleDomain& domain, const TwiddleTree& tw) {
  uint32_t n = domain.log_size();
  assert(coeffs.size() <= domain.size());
  std::vector<M31> values(coeffs);
  values.resize(domain.size(), M31(0));
  if (n == 1) {
    M31 v0 = values[0], v1 = values[1];
    butterfly(v0, v1, domain.half_coset.initial.y);
    return {v0, v1};
  }
  if (n == 2) {
    M31 v0 = values[0], v1 = values[1], v2 = values[2], v3 = values[3];
    M31 x = domain.half_coset.initial.x, y = domain.half_coset.initial.y;
    butterfly(v0, v2, x);
    butterfly(v1, v3, x);
    butterfly(v0, v1, y);
    butterfly(v2, v3, -y);
    return {v0, v1, v2, v3};
  }
  for (int j = (int)n - 2; j >= 0; j--) {
    const M31* lt = line_twiddles(tw.twiddles, n, (uint32_t)j);
    size_t len = (size_t)1 << (n - 2 - j);
    for (size_t h = 0; h < len; h++) fft_layer_loop(values, (uint32_t)j + 1, h, lt[h], false);
  }
  size_t first_len = (size_t)1 << (n - 2);
  auto ct = circle_twiddles(line_twiddles(tw.twiddles, n, 0), first_len);
  for (size_t h = 0; h < ct.size(); h++) fft_layer_loop(values, 0, h, ct[h], false);
  return values;
}

// poly/utils.rs fold: values (base or extension) folded by factors.
template <class V>
QM31 fold(const V* values, size_t n, const QM31* factors, size_t n_factors) {
  assert(n == ((size_t)1 << n_factors));
  if (n == 1) return QM31(values[0]);
  QM31 l = fold(values, n / 2, factors + 1, n_factors - 1);
  QM31 r = fold(values + n / 2, n / 2, factors + 1, n_factors - 1);
  return l + r * factors[0];
}
inline QM31 fold_qm(const QM31* values, size_t n, const QM31* factors, size_t n_factors) {
  if (n == 1) return values[0];
  QM31 l = fold_qm(values, n / 2, factors + 1, n_factors - 1);
  QM31 r = fold_qm(values + n / 2, n / 2, factors + 1, n_factors - 1);
  return l + r * factors[0];
}

// cpu/circle.rs:82-98: coefficient polynomial evaluated at a secure point.
inline QM31 eval_at_point(const std::vector<M31>& coeffs, CirclePoint<QM31> p) {
  uint32_t log_size = ilog2(coeffs.size());
  if (log_size == 0) return QM31(coeffs[0]);
  std::vector<QM31> mappings{p.y};
  QM31 x = p.x;
  for (uint32_t i = 1; i < log_size; i++) { mappings.push_back(x); x = double_x(x); }
  std::reverse(mappings.begin(), mappings.end());
  return fold(coeffs.data(), coeffs.size(), mappings.data(), mappings.size());
}

// line.rs:45-70: bit-reversed line evaluation -> LinePoly coefficients (stored
// in the reference's internal, bit-reversed coefficient order).
inline std::vector<QM31> line_interpolate(std::vector<QM31> values, Coset domain) {
  bit_reverse(values);
  Coset d = domain;
  while (d.size() > 1) {
    auto pts = d.points();
    for (size_t c = 0; c < values.size(); c += d.size()) {
      size_t half = d.size() / 2;
      for (size_t i = 0; i < half; i++) ibutterfly(values[c + i], values[c + half + i], inv(pts[i].x));
    }
    d = d.dbl();
  }
  M31 len_inv = inv(M31((uint32_t)values.size()));
  for (auto& v : values) v = v * len_inv;
  return values;
}

// LinePoly::eval_at_point (core/poly/line.rs:110-117); coeffs in internal order.
inline QM31 line_poly_eval(const std::vector<QM31>& coeffs, QM31 x) {
  uint32_t log_size = ilog2(coeffs.size());
  std::vector<QM31> d;
  for (uint32_t i = 0; i < log_size; i++) { d.push_back(x); x = double_x(x); }
  return fold_qm(coeffs.data(), coeffs.size(), d.data(), d.size());
}

}  // namespace orc
