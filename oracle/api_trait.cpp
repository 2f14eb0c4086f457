// ORACLE — test infrastructure only (see fields.h).
// CPU restatements of the per-trait operations the C ABI exposes besides the
// kernels in api_kernels.cpp, checked against the library by the GPU tests:
//   crates/stwo/src/prover/backend/cpu/circle.rs:101-141      (barycentric_weights, barycentric_eval_at_point)
//   crates/stwo/src/core/constraints.rs:12-55,87-93           (coset_vanishing, coset_vanishing_derivative,
//                                                              point_vanishing)
//   crates/stwo/src/prover/backend/cpu/accumulation.rs        (generate_secure_powers)
//   crates/constraint-framework/src/prover/component_prover.rs:177-245 (the CPU evaluation of constraint
//                                                              quotients over the domain: row_res times
//                                                              denom_inv[row >> trace_log])
#include "prover.h"

using namespace orc;

static QM31 qin(const uint32_t* v) { return QM31::u(v[0], v[1], v[2], v[3]); }
static void qout(QM31 q, uint32_t* o) {
  for (int i = 0; i < 4; i++) o[i] = q.coord(i);
}

// coset_vanishing_derivative (core/constraints.rs:38-55): 4^(log-1) times
// the product of the vanishing polynomials of CanonicCoset(i), i < log.
static M31 coset_vanishing_derivative(uint32_t log_size, CirclePoint<M31> p) {
  M31 exp(1);
  for (uint32_t i = 1; i < log_size; i++) exp = exp * M31(4);
  M31 v(1);
  for (uint32_t i = 1; i < log_size; i++) v = v * coset_vanishing(CanonicCoset::make(i).coset, p);
  return exp * v;
}

// point_vanishing (core/constraints.rs:87-93): h = p - vanish_point; h.y / (1 + h.x).
static QM31 point_vanishing(CirclePoint<M31> vanish, CirclePoint<QM31> p) {
  CirclePoint<QM31> h = p - to_qm31(vanish);
  return h.y / (QM31(M31(1)) + h.x);
}

extern "C" {

// PolyOps::barycentric_weights(CanonicCoset(log_size), p): 4 output planes of 2^log_size.
void oracle_barycentric_weights(uint32_t log_size, const uint32_t* point8, uint32_t* const* out) {
  CircleDomain d = CanonicCoset::make(log_size).circle_domain();
  CirclePoint<QM31> p{qin(point8), qin(point8 + 4)};
  QM31 vn_p = coset_vanishing(CanonicCoset::make(log_size).coset, p);
  size_t n = d.size();
#pragma omp parallel for schedule(static)
  for (long long ii = 0; ii < (long long)n; ii++) {
    size_t i = (size_t)ii;
    CirclePoint<M31> q = d.at(bit_reverse_index(i, log_size));
    M31 minus_two_y = q.y * (-M31(2));
    QM31 si = QM31(minus_two_y * coset_vanishing_derivative(log_size, q));
    QM31 vi = point_vanishing(q, p);
    QM31 w = vn_p / (si * vi);
    for (int c = 0; c < 4; c++) out[c][i] = w.coord(c);
  }
}

// PolyOps::barycentric_eval_at_point: sum_i evals[i] * weights[i].
void oracle_barycentric_eval(const uint32_t* evals, const uint32_t* const* w, uint32_t log_size, uint32_t* out4) {
  QM31 acc;
  for (size_t i = 0; i < ((size_t)1 << log_size); i++)
    acc += QM31::u(w[0][i], w[1][i], w[2][i], w[3][i]) * M31(evals[i]);
  qout(acc, out4);
}

// generate_secure_powers: felt^i, i < n.
void oracle_secure_powers(const uint32_t* felt4, size_t n, uint32_t* const* out) {
  auto v = secure_powers(qin(felt4), n);
  for (size_t i = 0; i < n; i++)
    for (int c = 0; c < 4; c++) out[c][i] = v[i].coord(c);
}

// Constraint quotients on the evaluation domain for one of the two example
// components: air 0 = wide fibonacci (n_cols trace columns), 1 = poseidon2
// (158 trace columns, 4 interaction columns, lookup z / alpha). Columns are
// bit-reversed evaluations on CanonicCoset(eval_log); powers: the reversed
// random-coefficient powers (n_constraints QM31 words); denom_inv: 2^(eval_log
// - trace_log) words; shift: the logup cumsum shift. Writes 4 planes.
void oracle_constraint_quotients(uint32_t air, uint32_t n_cols, uint32_t trace_log, uint32_t eval_log,
                                 const uint32_t* const* trace, const uint32_t* const* inter, const uint32_t* powers,
                                 uint32_t n_constraints, const uint32_t* denom_inv, const uint32_t* z4,
                                 const uint32_t* alpha4, const uint32_t* shift4, uint32_t* const* out) {
  size_t n = (size_t)1 << eval_log;
  AirSpec spec;
  spec.kind = air == 0 ? AirKind::WideFibonacci : AirKind::Poseidon;
  spec.log_n = trace_log;
  spec.n_cols = n_cols;
  uint32_t n_trace = air == 0 ? n_cols : (uint32_t)PN_COLUMNS;
  std::vector<std::vector<M31>> tcols(n_trace, std::vector<M31>(n)), icols(air == 0 ? 0 : 4, std::vector<M31>(n));
  for (uint32_t c = 0; c < n_trace; c++)
    for (size_t i = 0; i < n; i++) tcols[c][i] = M31(trace[c][i]);
  for (size_t c = 0; c < icols.size(); c++)
    for (size_t i = 0; i < n; i++) icols[c][i] = M31(inter[c][i]);
  std::vector<std::vector<const std::vector<M31>*>> cols(3);
  for (auto& c : tcols) cols[1].push_back(&c);
  for (auto& c : icols) cols[2].push_back(&c);
  if (air == 1) {
    spec.le.z = qin(z4);
    spec.le.alpha = qin(alpha4);
    QM31 cur(M31(1));
    for (int i = 0; i < 16; i++) {
      spec.le.alpha_powers[i] = cur;
      cur = cur * spec.le.alpha;
    }
  }
  std::vector<QM31> pw(n_constraints);
  for (uint32_t k = 0; k < n_constraints; k++) pw[k] = qin(powers + 4 * k);
  QM31 shift = shift4 ? qin(shift4) : QM31();
#pragma omp parallel for schedule(static)
  for (long long rr = 0; rr < (long long)n; rr++) {
    DomainEval e{&cols, (size_t)rr, trace_log, eval_log, &pw, QM31(), 0, 0, shift};
    eval_air(spec, e);
    QM31 v = e.row_res * M31(denom_inv[(size_t)rr >> trace_log]);
    for (int c = 0; c < 4; c++) out[c][rr] = v.coord(c);
  }
}

}  // extern "C"
