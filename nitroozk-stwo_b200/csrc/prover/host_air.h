// The two components as the prover's host side sees them: sizes, mask
// offsets, and their constraints evaluated at the out-of-domain point (for
// prove_ex's composition sanity check).
//   crates/examples/src/wide_fibonacci/mod.rs:48-58   (WideFibonacciEval)
//   crates/examples/src/poseidon/mod.rs:79-220        (Poseidon2 constraints, LOG_EXPAND = 2)
//   crates/constraint-framework/src/point.rs           (PointEvaluator: acc = acc * alpha + c / V)
//   crates/constraint-framework/src/lib.rs:218-262    (finalize_logup_in_pairs)
#pragma once
#include <vector>
#include "../air.cuh"
#include "host.h"

namespace gs {
namespace prover {

enum class AirKind { WideFibonacci, Poseidon };

struct AirHost {
  AirKind kind = AirKind::WideFibonacci;
  uint32_t log_n = 0;
  uint32_t n_cols = 100;       // wide fibonacci width
  LookupParams lookup{};       // poseidon
  qm31 claimed_sum{};          // poseidon
  uint32_t log_expand() const { return kind == AirKind::WideFibonacci ? 1 : 2; }
  uint32_t max_constraint_log() const { return log_n + log_expand(); }
  uint32_t n_trace_cols() const { return kind == AirKind::WideFibonacci ? n_cols : 158; }
  uint32_t n_constraints() const { return kind == AirKind::WideFibonacci ? n_cols - 2 : 143; }
};

// Constraint combination at a point: mask[t][c][k] = value of column c of
// tree t at its k-th mask point (tree 1 trace: offset 0; tree 2 interaction:
// offsets -1, 0). Returns sum over constraints in order of acc*alpha + c*dinv.
struct PointAcc {
  qm31 acc = qm_zero(), alpha, dinv;
  void add(qm31 c) { acc = qm_add(qm_mul(acc, alpha), qm_mul(dinv, c)); }
};

inline void p2h_m4(qm31* x) {
  qm31 t0 = qm_add(x[0], x[1]), t02 = qm_add(t0, t0), t1 = qm_add(x[2], x[3]), t12 = qm_add(t1, t1);
  qm31 t2 = qm_add(qm_add(x[1], x[1]), t1), t3 = qm_add(qm_add(x[3], x[3]), t0);
  qm31 t4 = qm_add(qm_add(t12, t12), t3), t5 = qm_add(qm_add(t02, t02), t2);
  x[0] = qm_add(t3, t5); x[1] = t5; x[2] = qm_add(t2, t4); x[3] = t4;
}
inline void p2h_external(qm31* s) {
  for (int i = 0; i < 4; i++) p2h_m4(s + 4 * i);
  for (int j = 0; j < 4; j++) {
    qm31 t = qm_add(qm_add(s[j], s[j + 4]), qm_add(s[j + 8], s[j + 12]));
    for (int i = 0; i < 4; i++) s[4 * i + j] = qm_add(s[4 * i + j], t);
  }
}
inline void p2h_internal(qm31* s) {
  qm31 sum = s[0];
  for (int i = 1; i < 16; i++) sum = qm_add(sum, s[i]);
  for (int i = 0; i < 16; i++) s[i] = qm_add(qm_mul_m31(s[i], 1u << (i + 1)), sum);
}
inline qm31 p2h_pow5(qm31 x) { qm31 x2 = qm_sqr(x); return qm_mul(qm_sqr(x2), x); }

inline qm31 from_partial_evals(const qm31 e[4]) {
  qm31 r = e[0];
  r = qm_add(r, qm_mul(e[1], qm_make(0, 1, 0, 0)));
  r = qm_add(r, qm_mul(e[2], qm_make(0, 0, 1, 0)));
  r = qm_add(r, qm_mul(e[3], qm_make(0, 0, 0, 1)));
  return r;
}

inline qm31 eval_at_point(const AirHost& air, const std::vector<std::vector<std::vector<qm31>>>& mask, qm31 alpha,
                          qm31 denom_inv) {
  PointAcc pa;
  pa.alpha = alpha;
  pa.dinv = denom_inv;
  const auto& tr = mask[1];
  if (air.kind == AirKind::WideFibonacci) {
    qm31 a = tr[0][0], b = tr[1][0];
    for (uint32_t k = 2; k < air.n_cols; k++) {
      qm31 c = tr[k][0];
      pa.add(qm_sub(c, qm_add(qm_sqr(a), qm_sqr(b))));
      a = b;
      b = c;
    }
    return pa.acc;
  }
  const qm31 rc = qm_from_m31(1234);
  qm31 s[16], init[16];
  size_t col = 0;
  for (int i = 0; i < 16; i++) init[i] = s[i] = tr[col++][0];
  auto full = [&]() {
    for (int i = 0; i < 16; i++) s[i] = qm_add(s[i], rc);
    p2h_external(s);
    for (int i = 0; i < 16; i++) {
      qm31 m = tr[col++][0];
      pa.add(qm_sub(p2h_pow5(s[i]), m));
      s[i] = m;
    }
  };
  for (int r = 0; r < 4; r++) full();
  for (int r = 0; r < 14; r++) {
    s[0] = qm_add(s[0], rc);
    p2h_internal(s);
    qm31 m = tr[col++][0];
    pa.add(qm_sub(p2h_pow5(s[0]), m));
    s[0] = m;
  }
  for (int r = 0; r < 4; r++) full();
  auto combine = [&](const qm31* v) {
    qm31 acc = qm_zero();
    for (int i = 0; i < 16; i++) {
      const uint32_t* ap = air.lookup.alpha_pow + 4 * i;
      acc = qm_add(acc, qm_mul(qm_make(ap[0], ap[1], ap[2], ap[3]), v[i]));
    }
    return qm_sub(acc, qm_make(air.lookup.z[0], air.lookup.z[1], air.lookup.z[2], air.lookup.z[3]));
  };
  qm31 d0 = combine(init), d1 = combine(s);
  qm31 prev[4], cur[4];
  for (int k = 0; k < 4; k++) { prev[k] = mask[2][k][0]; cur[k] = mask[2][k][1]; }
  qm31 shift = qm_mul_m31(air.claimed_sum, inv((uint32_t)((1ull << air.log_n) % P)));
  qm31 diff = qm_add(qm_sub(from_partial_evals(cur), from_partial_evals(prev)), shift);
  pa.add(qm_sub(qm_mul(diff, qm_mul(d0, d1)), qm_sub(d1, d0)));
  return pa.acc;
}

}  // namespace prover
}  // namespace gs
