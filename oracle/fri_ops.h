// ORACLE — test infrastructure only (see fields.h).
// FRI folding, DEEP-quotient numerators/combination and lifted accumulation.
// QM31 columns are held as std::vector<QM31> here (the device layout is 4 planes).
// Follows:
//   crates/stwo/src/prover/backend/cpu/fri.rs:64-124           (fold_line_cpu, fold_circle_into_line_cpu)
//   crates/stwo/src/core/pcs/quotients.rs:206-263               (partial numerators, line coeffs, denominators)
//   crates/stwo/src/core/constraints.rs:119-134                 (complex_conjugate_line_coeffs)
//   crates/stwo/src/prover/backend/cpu/quotients.rs:21-75       (accumulate_numerators, compute_quotients_and_combine)
//   crates/stwo/src/prover/backend/cpu/accumulation.rs:9-48     (accumulate, powers, lift_and_accumulate)
#pragma once
#include "poly.h"

namespace orc {

// Line domain fold: eval on a line domain (coset) in bit-reversed order.
inline std::vector<QM31> fold_line(const std::vector<QM31>& eval, const Coset& domain, QM31 alpha) {
  size_t n = eval.size();
  assert(n >= 2 && n == domain.size());
  auto pts = domain.points();
  std::vector<QM31> out(n / 2);
#pragma omp parallel for schedule(static)
  for (long long ii = 0; ii < (long long)(n / 2); ii++) {
    size_t i = (size_t)ii;
    M31 x = pts[bit_reverse_index(i << 1, domain.log_size)].x;
    QM31 f0 = eval[2 * i], f1 = eval[2 * i + 1];
    ibutterfly(f0, f1, inv(x));
    out[i] = f0 + alpha * f1;
  }
  return out;
}

// dst (line eval of size n/2) <- dst * alpha^2 + fold(src).
inline void fold_circle_into_line(std::vector<QM31>& dst, const std::vector<QM31>& src, const CircleDomain& domain, QM31 alpha) {
  assert(src.size() / 2 == dst.size());
  QM31 alpha_sq = alpha * alpha;
  auto pts = domain.points();
#pragma omp parallel for schedule(static)
  for (long long ii = 0; ii < (long long)dst.size(); ii++) {
    size_t i = (size_t)ii;
    CirclePoint<M31> p = pts[bit_reverse_index(i << 1, domain.log_size())];
    QM31 f0 = src[2 * i], f1 = src[2 * i + 1];
    ibutterfly(f0, f1, inv(p.y));
    QM31 f_prime = alpha * f1 + f0;
    dst[i] = dst[i] * alpha_sq + f_prime;
  }
}

struct LineCoeffs { QM31 a, b, c; };
// constraints.rs:119-134.
inline LineCoeffs complex_conjugate_line_coeffs(const CirclePoint<QM31>& point, QM31 value, QM31 alpha) {
  assert(point.y != conj(point.y));
  QM31 a = conj(value) - value;
  QM31 c = conj(point.y) - point.y;
  QM31 b = value * c - a * point.y;
  return {alpha * a, alpha * b, alpha * c};
}

// One batch = one sample point with its (column index, value, random coeff) entries.
struct NumeratorData { size_t column_index; QM31 sample_value; QM31 random_coeff; };
struct ColumnSampleBatch { CirclePoint<QM31> point; std::vector<NumeratorData> entries; };

struct AccumulatedNumerators {
  CirclePoint<QM31> sample_point;
  std::vector<QM31> partial;  // length 2^log_size of the batch's columns
  QM31 first_linear_term;
};

// cpu/quotients.rs:21-45 for one log-size group.
inline void accumulate_numerators(const std::vector<const std::vector<M31>*>& columns,
                                  const std::vector<ColumnSampleBatch>& batches,
                                  std::vector<AccumulatedNumerators>& out) {
  size_t size = columns[0]->size();
  for (auto& batch : batches) {
    std::vector<LineCoeffs> coeffs;
    for (auto& e : batch.entries) coeffs.push_back(complex_conjugate_line_coeffs(batch.point, e.sample_value, e.random_coeff));
    AccumulatedNumerators acc;
    acc.sample_point = batch.point;
    acc.partial.resize(size);
#pragma omp parallel for schedule(static)
    for (long long rr = 0; rr < (long long)size; rr++) {
      size_t row = (size_t)rr;
      QM31 num;
      for (size_t k = 0; k < batch.entries.size(); k++) {
        QM31 v = coeffs[k].c * (*columns[batch.entries[k].column_index])[row];
        num += v - coeffs[k].b;
      }
      acc.partial[row] = num;
    }
    QM31 s;
    for (auto& c : coeffs) s += c.a;
    acc.first_linear_term = s;
    out.push_back(std::move(acc));
  }
}

// quotients.rs:223-242: CM31 denominator (Re px - x) Im py - (Re py - y) Im px.
inline CM31 quotient_denominator(const CirclePoint<QM31>& sp, const CirclePoint<M31>& dp) {
  CM31 prx = sp.x.x, pry = sp.y.x, pix = sp.x.y, piy = sp.y.y;
  return (prx - CM31(dp.x)) * piy - (pry - CM31(dp.y)) * pix;
}

inline size_t lifted_index(size_t row, uint32_t log_ratio) { return ((row >> (log_ratio + 1)) << 1) + (row & 1); }

// cpu/quotients.rs:47-75.
inline std::vector<QM31> compute_quotients_and_combine(const std::vector<AccumulatedNumerators>& accs, uint32_t lifting_log_size) {
  CircleDomain domain = CanonicCoset::make(lifting_log_size).circle_domain();
  auto pts = domain.points();
  size_t n = (size_t)1 << lifting_log_size;
  std::vector<QM31> out(n);
#pragma omp parallel for schedule(static)
  for (long long rr = 0; rr < (long long)n; rr++) {
    size_t row = (size_t)rr;
    CirclePoint<M31> dp = pts[bit_reverse_index(row, lifting_log_size)];
    QM31 q;
    for (auto& acc : accs) {
      CM31 den_inv = inv(quotient_denominator(acc.sample_point, dp));
      uint32_t log_ratio = lifting_log_size - ilog2(acc.partial.size());
      QM31 full = acc.partial[lifted_index(row, log_ratio)] - acc.first_linear_term * dp.y;
      q += mul_cm31(full, den_inv);
    }
    out[row] = q;
  }
  return out;
}

// cpu/accumulation.rs:27-47: columns sorted by increasing size.
inline std::vector<QM31> lift_and_accumulate(std::vector<std::vector<QM31>> cols) {
  assert(!cols.empty());
  std::vector<QM31> curr(2);
  for (auto& col : cols) {
    uint32_t log_ratio = ilog2(col.size()) - ilog2(curr.size());
    for (size_t i = 0; i < col.size(); i++) col[i] = col[i] + curr[lifted_index(i, log_ratio)];
    curr = std::move(col);
  }
  return curr;
}

inline std::vector<QM31> secure_powers(QM31 felt, size_t n) {
  std::vector<QM31> r(n);
  QM31 acc(M31(1));
  for (size_t i = 0; i < n; i++) { r[i] = acc; acc = acc * felt; }
  return r;
}

}  // namespace orc
