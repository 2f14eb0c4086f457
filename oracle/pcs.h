// ORACLE — test infrastructure only (see fields.h).
// Commitment scheme and FRI prover.
// Follows:
//   crates/stwo/src/prover/pcs/mod.rs:57-66,367-457   (tree builder, commit: interpolate, LDE, Merkle, mix_root)
//   crates/stwo/src/prover/pcs/mod.rs:151-357         (prove_values)
//   crates/stwo/src/prover/pcs/mod.rs:459-494         (CommitmentTreeProver::decommit, lifted positions)
//   crates/stwo/src/prover/pcs/quotient_ops.rs:45-145 (compute_fri_quotients)
//   crates/stwo/src/core/pcs/quotients.rs:80-103,306-347 (ColumnSampleBatch, samples with periodicity)
//   crates/stwo/src/core/pcs/utils.rs:200-218         (prepare_preprocessed_query_positions)
//   crates/stwo/src/prover/fri.rs:85-330              (FriProver commit / decommit)
//   crates/stwo/src/core/queries.rs                   (Queries::new, fold)
// Deviation shared with the GPU prover: every tree is decommitted at its own
// (tree-local, lifted) query positions, the rule the reference verifier's
// reshape_flat_to_per_column (core/pcs/quotients.rs:350-420) expects; the
// reference prover passes lifting-domain positions to trees smaller than the
// lifting domain, which indexes past their end.
#pragma once
#include "fri_ops.h"
#include "channel.h"
#include "proof.h"
#include <map>
#include <set>

namespace orc {

struct Poly {
  std::vector<M31> coeffs;  // 2^log coefficients
  std::vector<M31> evals;   // bit-reversed evaluations on CanonicCoset(log + blowup)
  uint32_t eval_log() const { return ilog2(evals.size()); }
};

struct TreeProver {
  std::vector<Poly> polys;
  MerkleProver merkle;
  uint32_t max_log() const { return (uint32_t)merkle.layers.size() - 1; }
};

struct SampleSet {  // per tree, per column, per point
  std::vector<std::vector<std::vector<CirclePoint<QM31>>>> points;
  std::vector<std::vector<std::vector<QM31>>> values;
};

inline std::vector<size_t> prepare_query_positions(const std::vector<size_t>& q, uint32_t max_log, uint32_t tree_log) {
  std::vector<size_t> r;
  if (tree_log == 0) return r;
  for (size_t pos : q) {
    if (max_log < tree_log) r.push_back(((pos >> 1) << (tree_log - max_log + 1)) + (pos & 1));
    else r.push_back(((pos >> (max_log - tree_log + 1)) << 1) + (pos & 1));
  }
  return r;
}

struct CommitmentScheme {
  PcsConfig config;
  std::vector<TreeProver> trees;

  // TreeBuilder::extend_evals + commit: evaluations (bit-reversed, on
  // CanonicCoset(log)) are interpolated, extended by the blowup and committed.
  void commit_evals(const std::vector<std::vector<M31>>& evals, Channel& ch) {
    std::vector<std::vector<M31>> coeffs(evals.size());
#pragma omp parallel for schedule(dynamic)
    for (long long c = 0; c < (long long)evals.size(); c++) {
      uint32_t log = ilog2(evals[c].size());
      coeffs[c] = evals[c];
      interpolate(coeffs[c], CanonicCoset::make(log).circle_domain(),
                  precompute_twiddles(Coset::half_odds(log > 1 ? log - 1 : 1)));
    }
    commit_polys(std::move(coeffs), ch);
  }
  void commit_polys(std::vector<std::vector<M31>> coeffs, Channel& ch) {
    TreeProver t;
    t.polys.resize(coeffs.size());
#pragma omp parallel for schedule(dynamic)
    for (long long c = 0; c < (long long)coeffs.size(); c++) {
      uint32_t log = ilog2(coeffs[c].size());
      uint32_t el = log + config.log_blowup;
      t.polys[c].evals = evaluate(coeffs[c], CanonicCoset::make(el).circle_domain(),
                                  precompute_twiddles(Coset::half_odds(el - 1)));
      t.polys[c].coeffs = std::move(coeffs[c]);
    }
    std::vector<const std::vector<M31>*> cols;
    for (auto& p : t.polys) cols.push_back(&p.evals);
    t.merkle = MerkleProver::commit(cols, ch.kind);
    ch.mix_root(t.merkle.root());
    trees.push_back(std::move(t));
  }
};

// ---------------------------------------------------------------- quotients
inline std::vector<QM31> compute_fri_quotients(const CommitmentScheme& cs, const SampleSet& s, QM31 random_coeff,
                                               uint32_t lifting) {
  // build_samples_with_randomness_and_periodicity
  struct ColSamples { const std::vector<M31>* col; uint32_t log; std::vector<std::pair<CirclePoint<QM31>, QM31>> pv; std::vector<QM31> rnd; };
  std::vector<ColSamples> all;
  QM31 pw(M31(1));
  CirclePoint<M31> lift_gen = CanonicCoset::make(lifting).step();
  for (size_t t = 0; t < cs.trees.size(); t++) {
    for (size_t c = 0; c < cs.trees[t].polys.size(); c++) {
      ColSamples cs_;
      cs_.col = &cs.trees[t].polys[c].evals;
      cs_.log = cs.trees[t].polys[c].eval_log();
      const auto& pts = s.points[t][c];
      const auto& vals = s.values[t][c];
      if (pts.empty()) { all.push_back(cs_); continue; }
      if (pts.size() == 2) {
        CirclePoint<M31> period = repeated_double(lift_gen, cs_.log);
        cs_.pv.push_back({pts[1] + to_qm31(period), vals[1]});
        cs_.rnd.push_back(pw); pw = pw * random_coeff;
      }
      for (size_t k = 0; k < pts.size(); k++) {
        cs_.pv.push_back({pts[k], vals[k]});
        cs_.rnd.push_back(pw); pw = pw * random_coeff;
      }
      all.push_back(cs_);
    }
  }
  // group by column log size (ascending, stable), then batches by point (first appearance)
  std::map<uint32_t, std::vector<size_t>> by_log;
  for (size_t i = 0; i < all.size(); i++) by_log[all[i].log].push_back(i);
  std::vector<AccumulatedNumerators> accs;
  for (auto& [log, idxs] : by_log) {
    std::vector<const std::vector<M31>*> cols;
    std::vector<ColumnSampleBatch> batches;
    for (size_t ci = 0; ci < idxs.size(); ci++) {
      auto& cs_ = all[idxs[ci]];
      cols.push_back(cs_.col);
      for (size_t k = 0; k < cs_.pv.size(); k++) {
        auto it = std::find_if(batches.begin(), batches.end(), [&](const ColumnSampleBatch& b) { return b.point == cs_.pv[k].first; });
        if (it == batches.end()) { batches.push_back({cs_.pv[k].first, {}}); it = batches.end() - 1; }
        it->entries.push_back({ci, cs_.pv[k].second, cs_.rnd[k]});
      }
    }
    if (!batches.empty()) accumulate_numerators(cols, batches, accs);
  }
  // per distinct point: sum first linear terms, lift-and-accumulate partials (ascending size)
  std::vector<AccumulatedNumerators> per_point;
  std::vector<bool> used(accs.size(), false);
  for (size_t i = 0; i < accs.size(); i++) {
    if (used[i]) continue;
    std::vector<std::vector<QM31>> parts;
    QM31 flt;
    for (size_t j = i; j < accs.size(); j++) {
      if (used[j] || accs[j].sample_point != accs[i].sample_point) continue;
      used[j] = true;
      flt += accs[j].first_linear_term;
      parts.push_back(accs[j].partial);
    }
    std::stable_sort(parts.begin(), parts.end(), [](auto& a, auto& b) { return a.size() < b.size(); });
    AccumulatedNumerators a;
    a.sample_point = accs[i].sample_point;
    a.first_linear_term = flt;
    a.partial = lift_and_accumulate(parts);
    per_point.push_back(std::move(a));
  }
  return compute_quotients_and_combine(per_point, lifting);
}

// ---------------------------------------------------------------- FRI
struct FriLayer {
  std::vector<QM31> values;  // bit-reversed line (or circle, first layer) evaluation
  MerkleProver merkle;
  std::vector<std::vector<M31>> coords;  // 4 coordinate columns committed
};

inline void split_coords(const std::vector<QM31>& v, std::vector<std::vector<M31>>& coords) {
  coords.assign(4, std::vector<M31>(v.size()));
  for (size_t i = 0; i < v.size(); i++)
    for (int c = 0; c < 4; c++) coords[c][i] = M31(v[i].coord(c));
}
inline void commit_fri_layer(FriLayer& L, MerkleHash kind) {
  split_coords(L.values, L.coords);
  std::vector<const std::vector<M31>*> cols;
  for (auto& c : L.coords) cols.push_back(&c);
  L.merkle = MerkleProver::commit(cols, kind);
}

// compute_decommitment_positions_and_witness_evals (prover/fri.rs:301-330), fold step 1.
inline FriLayerProof decommit_fri_layer(const FriLayer& L, const std::vector<size_t>& queries) {
  FriLayerProof pr;
  std::vector<size_t> positions;
  size_t qi = 0;
  while (qi < queries.size()) {
    size_t start = (queries[qi] >> 1) << 1;
    size_t qj = qi;
    while (qj < queries.size() && (queries[qj] >> 1) == (queries[qi] >> 1)) qj++;
    size_t k = qi;
    for (size_t pos = start; pos < start + 2; pos++) {
      positions.push_back(pos);
      if (k < qj && queries[k] == pos) k++;
      else pr.fri_witness.push_back(L.values[pos]);
    }
    qi = qj;
  }
  std::map<uint32_t, std::vector<size_t>> qpl{{ilog2(L.values.size()), positions}};
  std::vector<const std::vector<M31>*> cols;
  for (auto& c : L.coords) cols.push_back(&c);
  pr.decommitment = L.merkle.decommit(qpl, cols).second;
  pr.commitment = L.merkle.root();
  return pr;
}

struct FriProverState {
  FriLayer first;
  std::vector<FriLayer> inner;
  std::vector<QM31> last_coeffs;
};

inline FriProverState fri_commit(Channel& ch, const PcsConfig& cfg, const std::vector<QM31>& column, uint32_t lifting) {
  FriProverState st;
  st.first.values = column;
  commit_fri_layer(st.first, ch.kind);
  ch.mix_root(st.first.merkle.root());
  uint32_t log = lifting - 1;
  std::vector<QM31> layer(1u << log);
  QM31 alpha = ch.draw_secure_felt();
  fold_circle_into_line(layer, column, CanonicCoset::make(lifting).circle_domain(), alpha);
  uint32_t last_log = cfg.log_last_layer + cfg.log_blowup;
  Coset domain = Coset::half_odds(log);
  if (log != last_log) {
    while (ilog2(layer.size()) > last_log + cfg.fold_step) {
      FriLayer L;
      L.values = layer;
      commit_fri_layer(L, ch.kind);
      ch.mix_root(L.merkle.root());
      alpha = ch.draw_secure_felt();
      layer = fold_line(L.values, domain, alpha);
      domain = domain.dbl();
      st.inner.push_back(std::move(L));
    }
    // last fold (step 1 in every configuration used here)
    FriLayer L;
    L.values = layer;
    commit_fri_layer(L, ch.kind);
    ch.mix_root(L.merkle.root());
    alpha = ch.draw_secure_felt();
    layer = fold_line(L.values, domain, alpha);
    domain = domain.dbl();
    st.inner.push_back(std::move(L));
  }
  // last layer polynomial
  auto coeffs = line_interpolate(layer, domain);   // internal order
  bit_reverse(coeffs);                              // into_ordered_coefficients
  size_t bound = (size_t)1 << cfg.log_last_layer;
  for (size_t i = bound; i < coeffs.size(); i++) assert(coeffs[i].is_zero() && "invalid degree");
  coeffs.resize(bound);
  bit_reverse(coeffs);                              // from_ordered_coefficients
  st.last_coeffs = coeffs;
  ch.mix_felts(coeffs);
  return st;
}

}  // namespace orc
