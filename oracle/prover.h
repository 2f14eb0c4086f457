// ORACLE — test infrastructure only (see fields.h).
// prove() for one component over the CPU restatement.
// Follows:
//   crates/stwo/src/prover/mod.rs:37-150                    (prove_ex)
//   crates/stwo/src/prover/air/accumulation.rs:21-125        (DomainEvaluationAccumulator)
//   crates/constraint-framework/src/prover/component_prover.rs:177-280 (domain evaluation, denominators)
//   crates/constraint-framework/src/prover/cpu_domain.rs     (row evaluator, offsets)
//   crates/constraint-framework/src/component.rs:255-300     (mask points, point evaluation)
//   crates/constraint-framework/src/point.rs                 (PointEvaluator)
//   crates/stwo/src/core/air/accumulation.rs                 (PointEvaluationAccumulator)
//   crates/stwo/src/core/proof.rs:26-56                      (extract_composition_oods_eval)
#pragma once
#include "pcs.h"
#include "air.h"
#include <functional>

namespace orc {

enum class AirKind { WideFibonacci, Poseidon };

struct AirSpec {
  AirKind kind;
  uint32_t log_n;          // trace rows (log)
  uint32_t n_cols = 100;   // wide fibonacci width
  LookupElements16 le;     // poseidon
  QM31 claimed_sum;        // poseidon
  uint32_t max_constraint_log() const { return log_n + (kind == AirKind::WideFibonacci ? 1 : 2); }
  uint32_t n_constraints() const { return kind == AirKind::WideFibonacci ? n_cols - 2 : 143; }
  // mask offsets per tree: tree 1 trace columns, tree 2 interaction columns
  std::vector<std::vector<std::vector<int>>> mask_offsets() const {
    std::vector<std::vector<std::vector<int>>> m(kind == AirKind::WideFibonacci ? 2 : 3);
    uint32_t tc = kind == AirKind::WideFibonacci ? n_cols : PN_COLUMNS;
    m[1].assign(tc, std::vector<int>{0});
    if (kind == AirKind::Poseidon) m[2].assign(4, std::vector<int>{-1, 0});
    return m;
  }
};

// Row evaluator on the evaluation domain (F = M31).
struct DomainEval {
  using F = M31;
  const std::vector<std::vector<const std::vector<M31>*>>* cols;  // per tree
  size_t row;
  uint32_t trace_log, eval_log;
  const std::vector<QM31>* powers;  // reversed random coefficient powers
  QM31 row_res;
  size_t ci = 0, tcol = 0;
  QM31 shift;
  M31 next_trace_mask() { return (*(*cols)[1][tcol++])[row]; }
  void next_cumsum_mask(QM31& prev, QM31& cur) {
    size_t pr = offset_bit_reversed_circle_domain_index(row, trace_log, eval_log, -1);
    M31 p[4], c[4];
    for (int k = 0; k < 4; k++) { p[k] = (*(*cols)[2][k])[pr]; c[k] = (*(*cols)[2][k])[row]; }
    prev = QM31::from_m31(p[0], p[1], p[2], p[3]);
    cur = QM31::from_m31(c[0], c[1], c[2], c[3]);
  }
  QM31 cumsum_shift() const { return shift; }
  void add_constraint(QM31 c) { row_res += (*powers)[ci++] * c; }
};

// Evaluator at the out-of-domain point (F = QM31).
struct PointEval {
  using F = QM31;
  const std::vector<std::vector<std::vector<QM31>>>* mask;  // per tree, per column, per offset
  QM31 acc, random_coeff, denom_inv, shift;
  size_t tcol = 0;
  QM31 next_trace_mask() { return (*mask)[1][tcol++][0]; }
  void next_cumsum_mask(QM31& prev, QM31& cur) {
    QM31 p[4], c[4];
    for (int k = 0; k < 4; k++) { p[k] = (*mask)[2][k][0]; c[k] = (*mask)[2][k][1]; }
    prev = qm31_from_partial_evals(p);
    cur = qm31_from_partial_evals(c);
  }
  QM31 cumsum_shift() const { return shift; }
  void add_constraint(QM31 c) { acc = acc * random_coeff + denom_inv * c; }
};

template <class E> void eval_air(const AirSpec& a, E& e) {
  if (a.kind == AirKind::WideFibonacci) eval_wide_fibonacci(e, a.n_cols);
  else eval_poseidon(e, a.le);
}

inline const TwiddleTree& twiddles_for(std::map<uint32_t, TwiddleTree>& cache, uint32_t root_log) {
  auto it = cache.find(root_log);
  if (it == cache.end()) it = cache.emplace(root_log, precompute_twiddles(Coset::half_odds(root_log))).first;
  return it->second;
}

// compute_composition_polynomial: returns the 4 coordinate coefficient polys.
inline std::array<std::vector<M31>, 4> composition_poly(const CommitmentScheme& cs, const AirSpec& air, QM31 random_coeff) {
  uint32_t eval_log = air.max_constraint_log(), trace_log = air.log_n;
  CircleDomain ed = CanonicCoset::make(eval_log).circle_domain();
  TwiddleTree tw = precompute_twiddles(Coset::half_odds(eval_log - 1));
  // component trace on the evaluation domain (extend from coefficients if needed)
  std::vector<std::vector<std::vector<M31>>> ext(cs.trees.size());
  std::vector<std::vector<const std::vector<M31>*>> cols(cs.trees.size());
  for (size_t t = 1; t < cs.trees.size(); t++) {
    auto& tree = cs.trees[t];
    ext[t].resize(tree.polys.size());
#pragma omp parallel for schedule(dynamic)
    for (long long c = 0; c < (long long)tree.polys.size(); c++) {
      if (tree.polys[c].eval_log() != eval_log) ext[t][c] = evaluate(tree.polys[c].coeffs, ed, tw);
    }
    for (size_t c = 0; c < tree.polys.size(); c++)
      cols[t].push_back(tree.polys[c].eval_log() != eval_log ? &ext[t][c] : &tree.polys[c].evals);
  }
  // denominators: 1 / coset_vanishing(trace coset, eval_domain.at(i)), bit-reversed
  uint32_t log_expand = eval_log - trace_log;
  std::vector<M31> denom_inv((size_t)1 << log_expand);
  Coset tc = CanonicCoset::make(trace_log).coset;
  for (size_t i = 0; i < denom_inv.size(); i++) denom_inv[i] = inv(coset_vanishing(tc, ed.at(i)));
  bit_reverse(denom_inv);
  std::vector<QM31> powers = secure_powers(random_coeff, air.n_constraints());
  std::reverse(powers.begin(), powers.end());
  QM31 shift = air.kind == AirKind::Poseidon ? air.claimed_sum / M31(1u << air.log_n) : QM31();
  size_t n = (size_t)1 << eval_log;
  std::array<std::vector<M31>, 4> acc;
  for (auto& a : acc) a.resize(n);
#pragma omp parallel for schedule(static)
  for (long long rr = 0; rr < (long long)n; rr++) {
    DomainEval e{&cols, (size_t)rr, trace_log, eval_log, &powers, QM31(), 0, 0, shift};
    eval_air(air, e);
    QM31 v = e.row_res * denom_inv[(size_t)rr >> trace_log];
    for (int c = 0; c < 4; c++) acc[c][rr] = M31(v.coord(c));
  }
  // finalize: single size (lift is the identity), interpolate coordinates
  for (int c = 0; c < 4; c++) interpolate(acc[c], ed, tw);
  return acc;
}

struct ProveResult {
  StarkProof proof;
  bool constraints_ok = false;
  QM31 composition_at_oods, constraints_at_oods;
};

// prove_ex for a single component; `cs` holds the committed preprocessed,
// trace (and interaction) trees, `ch` the channel after those commitments.
// split_log: the composition polynomial is split into 2^split_log parts by the
// top coefficient-index bits (the reference fixes split_log = 1,
// core/verifier.rs:17 COMPOSITION_LOG_SPLIT); parts are committed in part
// order, each as its 4 coordinate polynomials.
inline ProveResult prove(CommitmentScheme& cs, Channel& ch, const AirSpec& air, uint32_t split_log = 1) {
  ProveResult R;
  const PcsConfig& cfg = cs.config;
  QM31 random_coeff = ch.draw_secure_felt();
  auto comp = composition_poly(cs, air, random_coeff);
  // split_at_mid (generalised): part t holds coefficients [t*len, (t+1)*len)
  std::vector<std::vector<M31>> split;
  size_t parts = (size_t)1 << split_log, plen = comp[0].size() / parts;
  for (size_t t = 0; t < parts; t++)
    for (int c = 0; c < 4; c++) split.emplace_back(comp[c].begin() + t * plen, comp[c].begin() + (t + 1) * plen);
  cs.commit_polys(std::move(split), ch);
  CirclePoint<QM31> oods = get_random_point(ch);
  uint32_t lifting = cs.trees.back().max_log();
  uint32_t lifting_cfg = cfg.has_lifting ? cfg.lifting : lifting;
  uint32_t max_log_degree_bound = lifting_cfg - cfg.log_blowup;
  // sample points
  SampleSet s;
  s.points.resize(cs.trees.size());
  s.values.resize(cs.trees.size());
  auto offs = air.mask_offsets();
  CirclePoint<M31> step = CanonicCoset::make(max_log_degree_bound).step();
  for (size_t t = 0; t < cs.trees.size(); t++) {
    size_t ncols = cs.trees[t].polys.size();
    s.points[t].resize(ncols);
    for (size_t c = 0; c < ncols; c++) {
      if (t + 1 == cs.trees.size()) { s.points[t][c] = {oods}; continue; }
      if (t >= offs.size() || c >= offs[t].size()) continue;
      for (int off : offs[t][c]) {
        CirclePoint<M31> d = off > 0 ? mul_scalar(step, (unsigned __int128)off) : mul_scalar(conjugate(step), (unsigned __int128)(-off));
        s.points[t][c].push_back(oods + to_qm31(d));
      }
    }
  }
  // sampled values at the lifted (doubled) points
  for (size_t t = 0; t < cs.trees.size(); t++) {
    s.values[t].resize(s.points[t].size());
#pragma omp parallel for schedule(dynamic)
    for (long long c = 0; c < (long long)s.points[t].size(); c++) {
      auto& poly = cs.trees[t].polys[c];
      for (auto& p : s.points[t][c])
        s.values[t][c].push_back(eval_at_point(poly.coeffs, repeated_double(p, lifting - poly.eval_log())));
    }
  }
  std::vector<QM31> flat;
  for (auto& t : s.values) for (auto& c : t) for (auto& v : c) flat.push_back(v);
  ch.mix_felts(flat);
  QM31 qrc = ch.draw_secure_felt();
  auto quot = compute_fri_quotients(cs, s, qrc, lifting);
  auto fri = fri_commit(ch, cfg, quot, lifting);
  uint64_t pow = ch.grind(cfg.pow_bits);
  ch.mix_u64(pow);
  // FRI decommit
  auto raw = draw_queries(ch, lifting, cfg.n_queries);
  std::set<size_t> qs(raw.begin(), raw.end());
  std::vector<size_t> queries(qs.begin(), qs.end());
  StarkProof& P = R.proof;
  P.config = cfg;
  P.fri.first = decommit_fri_layer(fri.first, queries);
  std::vector<size_t> lq = queries;
  for (auto& L : fri.inner) {
    std::vector<size_t> f;
    for (size_t q : lq) if (f.empty() || f.back() != (q >> 1)) f.push_back(q >> 1);
    lq = f;
    P.fri.inner.push_back(decommit_fri_layer(L, lq));
  }
  P.fri.last_layer_coeffs = fri.last_coeffs;
  P.fri.last_layer_log = ilog2(fri.last_coeffs.size());
  P.proof_of_work = pow;
  // trees
  for (auto& tree : cs.trees) {
    P.commitments.push_back(tree.merkle.root());
    auto tq = prepare_query_positions(queries, lifting, tree.max_log());
    std::map<uint32_t, std::vector<size_t>> qpl;
    std::set<uint32_t> logs;
    for (auto& p : tree.polys) logs.insert(p.eval_log());
    for (uint32_t ls : logs) {
      uint32_t shift = tree.max_log() - ls;
      std::set<size_t> pos;
      for (size_t q : tq) pos.insert(((q >> (shift + 1)) << 1) + (q & 1));
      qpl[ls] = std::vector<size_t>(pos.begin(), pos.end());
    }
    std::vector<const std::vector<M31>*> cols;
    for (auto& p : tree.polys) cols.push_back(&p.evals);
    auto [vals, dec] = tree.merkle.decommit(qpl, cols);
    P.queried_values.push_back(vals);
    P.decommitments.push_back(dec);
  }
  P.sampled_values = s.values;
  // sanity check: composition at the OODS point vs constraints from the mask
  // extract_composition_oods_eval: sum_t part_t(oods) * prod_{bits b of t} F_{n-s+b},
  // F_k = pi^{k-1}(x) the fold factor of coefficient-index bit k (n = composition log).
  auto& cv = s.values.back();
  uint32_t comp_log = air.max_constraint_log();
  QM31 total;
  for (size_t t = 0; t < parts; t++) {
    QM31 e4[4] = {cv[4 * t][0], cv[4 * t + 1][0], cv[4 * t + 2][0], cv[4 * t + 3][0]};
    QM31 v = qm31_from_partial_evals(e4);
    for (uint32_t b = 0; b < split_log; b++)
      if ((t >> b) & 1) v = v * repeated_double(oods, comp_log - split_log + b - 1).x;
    total += v;
  }
  R.composition_at_oods = total;
  PointEval pe;
  pe.mask = &s.values;
  pe.random_coeff = random_coeff;
  pe.denom_inv = inv(coset_vanishing(CanonicCoset::make(max_log_degree_bound).coset, oods));
  pe.shift = air.kind == AirKind::Poseidon ? air.claimed_sum / M31(1u << air.log_n) : QM31();
  eval_air(air, pe);
  R.constraints_at_oods = pe.acc;
  R.constraints_ok = R.composition_at_oods == R.constraints_at_oods;
  return R;
}

}  // namespace orc
