// ORACLE — test infrastructure only (see fields.h).
// The two benchmark AIRs written once over an abstract row evaluator, used on
// the evaluation domain (F = M31) and at the out-of-domain point (F = QM31).
// Follows:
//   crates/examples/src/wide_fibonacci/mod.rs:34-58     (WideFibonacciEval)
//   crates/examples/src/poseidon/mod.rs:38-220          (Poseidon2 rounds, constraints, lookups)
//   crates/constraint-framework/src/lib.rs:131-300      (EvalAtRow, logup proxy, finalize_logup_in_pairs)
//   crates/constraint-framework/src/logup.rs:17-110     (LogupAtRow cumsum_shift, LookupElements)
//   crates/stwo/src/core/fraction.rs:22-60              (projective fraction add / sum)
#pragma once
#include "fields.h"
#include <array>

namespace orc {

struct LookupElements16 {
  QM31 z, alpha;
  std::array<QM31, 16> alpha_powers;
};

template <class F> inline QM31 to_ef(const F& v) { return QM31(v); }
template <> inline QM31 to_ef<QM31>(const QM31& v) { return v; }

// ---------------------------------------------------------------- WideFib
template <class E>
void eval_wide_fibonacci(E& eval, uint32_t n_cols) {
  using F = typename E::F;
  F a = eval.next_trace_mask();
  F b = eval.next_trace_mask();
  for (uint32_t i = 2; i < n_cols; i++) {
    F c = eval.next_trace_mask();
    eval.add_constraint(to_ef(c - (a * a + b * b)));
    a = b;
    b = c;
  }
}

// ---------------------------------------------------------------- Poseidon2
constexpr int PN_STATE = 16, PN_PARTIAL = 14, PN_HALF_FULL = 4;
constexpr uint32_t P_ROUND_CONST = 1234;  // the reference's placeholder constants (poseidon/mod.rs:48-51)
constexpr int PN_COLUMNS = PN_STATE * (1 + 2 * PN_HALF_FULL) + PN_PARTIAL;  // 158

template <class F> inline void apply_m4(F x[4]) {
  F t0 = x[0] + x[1];
  F t02 = t0 + t0;
  F t1 = x[2] + x[3];
  F t12 = t1 + t1;
  F t2 = x[1] + x[1] + t1;
  F t3 = x[3] + x[3] + t0;
  F t4 = t12 + t12 + t3;
  F t5 = t02 + t02 + t2;
  F t6 = t3 + t5;
  F t7 = t2 + t4;
  x[0] = t6; x[1] = t5; x[2] = t7; x[3] = t4;
}
template <class F> inline void apply_external_round_matrix(F s[16]) {
  for (int i = 0; i < 4; i++) apply_m4(s + 4 * i);
  for (int j = 0; j < 4; j++) {
    F t = s[j] + s[j + 4] + s[j + 8] + s[j + 12];
    for (int i = 0; i < 4; i++) s[4 * i + j] = s[4 * i + j] + t;
  }
}
template <class F> inline void apply_internal_round_matrix(F s[16]) {
  F sum = s[0];
  for (int i = 1; i < 16; i++) sum = sum + s[i];
  for (int i = 0; i < 16; i++) s[i] = s[i] * M31(1u << (i + 1)) + sum;
}
template <class F> inline F pow5(F x) { F x2 = x * x; F x4 = x2 * x2; return x4 * x; }

// Projective fraction over QM31.
struct Frac { QM31 num, den; };
inline Frac frac_add(const Frac& a, const Frac& b) { return {b.den * a.num + a.den * b.num, a.den * b.den}; }

template <class F> inline QM31 combine16(const LookupElements16& le, const F v[16]) {
  QM31 acc;
  for (int i = 0; i < 16; i++) acc = acc + le.alpha_powers[i] * to_ef(v[i]);
  return acc - le.z;
}

template <class E>
void eval_poseidon(E& eval, const LookupElements16& le) {
  using F = typename E::F;
  F state[16];
  for (int i = 0; i < 16; i++) state[i] = eval.next_trace_mask();
  F initial[16];
  for (int i = 0; i < 16; i++) initial[i] = state[i];
  const M31 rc(P_ROUND_CONST);
  for (int round = 0; round < PN_HALF_FULL; round++) {
    for (int i = 0; i < 16; i++) state[i] = state[i] + F(rc);
    apply_external_round_matrix(state);
    for (int i = 0; i < 16; i++) state[i] = pow5(state[i]);
    for (int i = 0; i < 16; i++) {
      F m = eval.next_trace_mask();
      eval.add_constraint(to_ef(state[i] - m));
      state[i] = m;
    }
  }
  for (int round = 0; round < PN_PARTIAL; round++) {
    state[0] = state[0] + F(rc);
    apply_internal_round_matrix(state);
    state[0] = pow5(state[0]);
    F m = eval.next_trace_mask();
    eval.add_constraint(to_ef(state[0] - m));
    state[0] = m;
  }
  for (int round = 0; round < PN_HALF_FULL; round++) {
    for (int i = 0; i < 16; i++) state[i] = state[i] + F(rc);
    apply_external_round_matrix(state);
    for (int i = 0; i < 16; i++) state[i] = pow5(state[i]);
    for (int i = 0; i < 16; i++) {
      F m = eval.next_trace_mask();
      eval.add_constraint(to_ef(state[i] - m));
      state[i] = m;
    }
  }
  // add_to_relation(+1, initial), add_to_relation(-1, final), finalize_logup_in_pairs:
  // a single batch, so the whole sum goes into the last (cumsum) column.
  Frac f0{QM31(M31(1)), combine16(le, initial)};
  Frac f1{-QM31(M31(1)), combine16(le, state)};
  Frac frac = frac_add(f0, f1);
  QM31 prev, cur;
  eval.next_cumsum_mask(prev, cur);
  QM31 diff = cur - prev;  // minus the (zero) previous-column cumsum
  QM31 shifted = diff + eval.cumsum_shift();
  eval.add_constraint(shifted * frac.den - frac.num);
}

// Reference trace-generation input rule (poseidon/mod.rs:242): row r, lane i
// of state: r + state_i (one instance per row). Returns the 158 columns and
// the initial/final states for the lookup.
inline void poseidon_trace_row(const M31 init_state[16], M31 cols_out[PN_COLUMNS], M31 final_state[16]) {
  M31 s[16];
  for (int i = 0; i < 16; i++) s[i] = init_state[i];
  int c = 0;
  for (int i = 0; i < 16; i++) cols_out[c++] = s[i];
  const M31 rc(P_ROUND_CONST);
  for (int round = 0; round < PN_HALF_FULL; round++) {
    for (int i = 0; i < 16; i++) s[i] = s[i] + rc;
    apply_external_round_matrix(s);
    for (int i = 0; i < 16; i++) s[i] = pow5(s[i]);
    for (int i = 0; i < 16; i++) cols_out[c++] = s[i];
  }
  for (int round = 0; round < PN_PARTIAL; round++) {
    s[0] = s[0] + rc;
    apply_internal_round_matrix(s);
    s[0] = pow5(s[0]);
    cols_out[c++] = s[0];
  }
  for (int round = 0; round < PN_HALF_FULL; round++) {
    for (int i = 0; i < 16; i++) s[i] = s[i] + rc;
    apply_external_round_matrix(s);
    for (int i = 0; i < 16; i++) s[i] = pow5(s[i]);
    for (int i = 0; i < 16; i++) cols_out[c++] = s[i];
  }
  for (int i = 0; i < 16; i++) final_state[i] = s[i];
}

}  // namespace orc
