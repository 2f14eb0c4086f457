// ORACLE — test infrastructure only (see fields.h).
// STARK verifier: a restatement of the reference's verification rule, used by
// the tests to accept the proofs that both provers produce and to reject
// tampered ones. It shares with the oracle prover only the primitives pinned
// on the reference's known answers (fields, circle geometry, the Fiat-Shamir
// channel, the Merkle node hash) and the AIR definitions (the statement); it
// uses none of the prover's protocol code, and it reads the proof from its
// serialised bytes.
//
// Follows:
//   crates/stwo/src/core/verifier.rs:19-122          (verify / verify_ex)
//   crates/stwo/src/core/pcs/verifier.rs:45-182      (commit, verify_values, build_queries_per_log_size)
//   crates/stwo/src/core/pcs/quotients.rs:80-420     (ColumnSampleBatch::new_vec, fri_answers,
//                                                     accumulate_row_quotients, denominator_inverses,
//                                                     build_samples_with_randomness_and_periodicity,
//                                                     reshape_flat_to_per_column)
//   crates/stwo/src/core/pcs/utils.rs:200-225        (prepare_preprocessed_query_positions, get_lifting_log_size)
//   crates/stwo/src/core/constraints.rs:119-134      (complex_conjugate_line_coeffs)
//   crates/stwo/src/core/fri.rs:83-700,750-777       (FriVerifier::commit / decommit, first and inner layer
//                                                     verifiers, SparseEvaluation, fold_coset,
//                                                     fold_circle_into_line)
//   crates/stwo/src/core/vcs/verifier.rs:85-200      (MerkleVerifier::verify)
//   crates/stwo/src/core/vcs/utils.rs:5-16           (next_decommitment_node)
//   crates/stwo/src/core/queries.rs:11-60            (draw_queries, Queries::new / fold)
//   crates/stwo/src/core/poly/line.rs:138-145        (LinePoly::eval_at_point), core/poly/utils.rs:27-38 (fold)
//   crates/stwo/src/core/proof.rs:26-56              (extract_composition_oods_eval)
//   crates/stwo/src/core/air/components.rs:28-80     (mask points, eval_composition_polynomial_at_point)
//   crates/stwo/src/core/air/accumulation.rs:10-40   (PointEvaluationAccumulator)
//   crates/constraint-framework/src/component.rs:264-320 (mask_points, evaluate_constraint_quotients_at_point)
//   crates/constraint-framework/src/point.rs:12-64   (PointEvaluator)
//   crates/constraint-framework/src/logup.rs:31-40   (cumsum_shift = claimed_sum / 2^log_size)
//   crates/examples/src/poseidon/mod.rs:905-922      (the verifier side of the Poseidon2 test: tree
//                                                     commits, lookup elements drawn after the trace)
//
// One generalisation, in the composition split only: the reference fixes
// COMPOSITION_LOG_SPLIT = 1 (core/verifier.rs:17); here it is a parameter s.
// The composition polynomial of 2^(m) coefficients is committed as 2^s parts,
// part t holding coefficients [t 2^(m-s), (t+1) 2^(m-s)), each as 4
// coordinate columns; its value at the OODS point p is
//   sum_t part_t(p) * prod_{bits j of t} pi^(m-s-1+j)(p.x)
// which for s = 1 is the reference's left + pi^(m-2)(p.x) * right.
#pragma once
#include "air.h"
#include "channel.h"
#include "circle.h"
#include "merkle.h"
#include "proof.h"
#include <map>
#include <string>

namespace orc {
namespace ver {

enum Code {
  OK = 0,
  INVALID_STRUCTURE = 1,
  MERKLE = 2,
  OODS_NOT_MATCHING = 3,
  FRI = 4,
  PROOF_OF_WORK = 5,
};

struct Result {
  int code = OK;
  std::string msg;
};
inline Result fail(int code, const std::string& msg) { return Result{code, msg}; }

// ------------------------------------------------------------ deserialisation
// The byte layout written by the provers (bincode-1.x style: little-endian
// fixed-width integers, u64 sequence lengths, Option as a one-byte tag, a
// hash as 32 raw bytes, M31 as u32, QM31 as 4 x u32), field order of the
// reference's serde structs (core/pcs/quotients.rs:29-38, core/fri.rs:363-398,
// core/vcs/verifier.rs:13-22, core/poly/line.rs:96-101). Every length is
// checked against the bytes left before anything is allocated, and a field
// value >= P is rejected.
struct Reader {
  const uint8_t* p;
  size_t n, off = 0;
  bool ok = true;
  bool need(size_t k) {
    if (!ok || n - off < k) ok = false;
    return ok;
  }
  uint8_t u8() { return need(1) ? p[off++] : 0; }
  uint32_t u32() {
    if (!need(4)) return 0;
    uint32_t v = 0;
    for (int i = 0; i < 4; i++) v |= (uint32_t)p[off + i] << (8 * i);
    off += 4;
    return v;
  }
  uint64_t u64() {
    if (!need(8)) return 0;
    uint64_t v = 0;
    for (int i = 0; i < 8; i++) v |= (uint64_t)p[off + i] << (8 * i);
    off += 8;
    return v;
  }
  // a sequence length whose elements take at least elem_bytes each
  size_t len(size_t elem_bytes) {
    uint64_t v = u64();
    if (ok && elem_bytes && v > (n - off) / elem_bytes) ok = false;
    return ok ? (size_t)v : 0;
  }
  Hash32 hash() {
    Hash32 h{};
    if (need(32)) {
      memcpy(h.data(), p + off, 32);
      off += 32;
    }
    return h;
  }
  M31 m31() {
    uint32_t v = u32();
    if (v >= P) ok = false;
    return M31(ok ? v : 0);
  }
  QM31 qm() {
    M31 a = m31(), b = m31(), c = m31(), d = m31();
    return QM31::from_m31(a, b, c, d);
  }
  MerkleDecommitment decommitment() {
    MerkleDecommitment d;
    size_t nh = len(32);
    for (size_t i = 0; ok && i < nh; i++) d.hash_witness.push_back(hash());
    size_t nc = len(4);
    for (size_t i = 0; ok && i < nc; i++) d.column_witness.push_back(m31());
    return d;
  }
  FriLayerProof fri_layer() {
    FriLayerProof l;
    size_t nw = len(16);
    for (size_t i = 0; ok && i < nw; i++) l.fri_witness.push_back(qm());
    l.decommitment = decommitment();
    l.commitment = hash();
    return l;
  }
};

inline bool deserialize(const uint8_t* bytes, size_t n, StarkProof& out) {
  Reader r{bytes, n};
  StarkProof& p = out;
  p.config.pow_bits = r.u32();
  p.config.log_blowup = r.u32();
  p.config.log_last_layer = r.u32();
  uint64_t nq = r.u64();
  p.config.n_queries = nq > 0xffffffffull ? (r.ok = false, 0u) : (uint32_t)nq;
  p.config.fold_step = r.u32();
  uint8_t tag = r.u8();
  if (tag > 1) r.ok = false;
  p.config.has_lifting = tag == 1;
  if (p.config.has_lifting) p.config.lifting = r.u32();
  size_t nc = r.len(32);
  for (size_t i = 0; r.ok && i < nc; i++) p.commitments.push_back(r.hash());
  size_t nt = r.len(8);
  for (size_t t = 0; r.ok && t < nt; t++) {
    std::vector<std::vector<QM31>> tree;
    size_t ncol = r.len(8);
    for (size_t c = 0; r.ok && c < ncol; c++) {
      std::vector<QM31> col;
      size_t nv = r.len(16);
      for (size_t v = 0; r.ok && v < nv; v++) col.push_back(r.qm());
      tree.push_back(std::move(col));
    }
    p.sampled_values.push_back(std::move(tree));
  }
  size_t nd = r.len(16);
  for (size_t i = 0; r.ok && i < nd; i++) p.decommitments.push_back(r.decommitment());
  size_t nqv = r.len(8);
  for (size_t t = 0; r.ok && t < nqv; t++) {
    std::vector<M31> vals;
    size_t nv = r.len(4);
    for (size_t v = 0; r.ok && v < nv; v++) vals.push_back(r.m31());
    p.queried_values.push_back(std::move(vals));
  }
  p.proof_of_work = r.u64();
  p.fri.first = r.fri_layer();
  size_t ni = r.len(56);
  for (size_t i = 0; r.ok && i < ni; i++) p.fri.inner.push_back(r.fri_layer());
  size_t nl = r.len(16);
  for (size_t i = 0; r.ok && i < nl; i++) p.fri.last_layer_coeffs.push_back(r.qm());
  p.fri.last_layer_log = r.u32();
  // LinePoly's invariant: 2^log_size coefficients
  if (r.ok && (p.fri.last_layer_log > 20 || p.fri.last_layer_coeffs.size() != ((size_t)1 << p.fri.last_layer_log)))
    r.ok = false;
  return r.ok && r.off == n;
}

// ------------------------------------------------------------- statement
// The verifier's knowledge of the component: the AIR, its size, the
// composition split and, for Poseidon2, the logup claimed sum the prover
// reports beside the proof (the reference hands it over inside the
// component, poseidon/mod.rs:398-407).
enum class Air { WideFibonacci, Poseidon };
struct Statement {
  Air kind = Air::WideFibonacci;
  uint32_t log_n = 0;
  uint32_t n_cols = 100;
  uint32_t split_log = 1;
  QM31 claimed_sum;
  MerkleHash hash = MerkleHash::Blake2s;
  uint32_t n_trace_cols() const { return kind == Air::WideFibonacci ? n_cols : (uint32_t)PN_COLUMNS; }
  uint32_t max_constraint_log_degree_bound() const { return log_n + (kind == Air::WideFibonacci ? 1 : 2); }
};

// --------------------------------------------------------------- Merkle
// MerkleVerifier::verify (core/vcs/verifier.rs:85-200): rebuild the nodes on
// the queried paths layer by layer from the largest column size down, taking
// sibling hashes and unqueried column values from the witness in order.
// Returns an empty string on success, else the reference's error name.
inline std::string merkle_verify(const Hash32& root, const std::vector<uint32_t>& column_log_sizes,
                                 const std::map<uint32_t, std::vector<size_t>>& queries_per_log_size,
                                 const std::vector<M31>& queried_values, const MerkleDecommitment& decommitment,
                                 MerkleHash kind) {
  if (column_log_sizes.empty()) return "";
  uint32_t max_log = *std::max_element(column_log_sizes.begin(), column_log_sizes.end());
  std::map<uint32_t, size_t> n_columns_per_log_size;
  for (uint32_t l : column_log_sizes) n_columns_per_log_size[l]++;
  size_t qv = 0, hw = 0, cw = 0;
  const auto& hash_witness = decommitment.hash_witness;
  const auto& column_witness = decommitment.column_witness;
  bool has_last = false;
  std::vector<std::pair<size_t, Hash32>> last;
  for (int64_t layer = max_log; layer >= 0; layer--) {
    auto it_n = n_columns_per_log_size.find((uint32_t)layer);
    size_t n_in_layer = it_n == n_columns_per_log_size.end() ? 0 : it_n->second;
    auto it_q = queries_per_log_size.find((uint32_t)layer);
    const std::vector<size_t>* col_queries = it_q == queries_per_log_size.end() ? nullptr : &it_q->second;
    size_t pq = 0, ph = 0, cq = 0;  // cursors: previous-layer queries, previous-layer hashes, column queries
    std::vector<std::pair<size_t, Hash32>> cur;
    for (;;) {
      // next_decommitment_node: the smaller of the next parent and the next column query
      bool have = false;
      size_t node = 0;
      if (has_last && pq < last.size()) { node = last[pq].first / 2; have = true; }
      if (col_queries && cq < col_queries->size()) {
        size_t c = (*col_queries)[cq];
        if (!have || c < node) node = c;
        have = true;
      }
      if (!have) break;
      while (has_last && pq < last.size() && last[pq].first / 2 == node) pq++;
      Hash32 left{}, right{};
      if (has_last) {
        if (ph < last.size() && last[ph].first == 2 * node) left = last[ph++].second;
        else if (hw < hash_witness.size()) left = hash_witness[hw++];
        else return "WitnessTooShort";
        if (ph < last.size() && last[ph].first == 2 * node + 1) right = last[ph++].second;
        else if (hw < hash_witness.size()) right = hash_witness[hw++];
        else return "WitnessTooShort";
      }
      std::vector<M31> values;
      if (col_queries && cq < col_queries->size() && (*col_queries)[cq] == node) {
        cq++;
        if (queried_values.size() - qv < n_in_layer) return "TooFewQueriedValues";
        values.assign(queried_values.begin() + qv, queried_values.begin() + qv + n_in_layer);
        qv += n_in_layer;
      } else {
        if (column_witness.size() - cw < n_in_layer) return "WitnessTooShort";
        values.assign(column_witness.begin() + cw, column_witness.begin() + cw + n_in_layer);
        cw += n_in_layer;
      }
      cur.push_back({node, hash_node(has_last ? &left : nullptr, has_last ? &right : nullptr, values.data(),
                                     values.size(), kind)});
    }
    last = std::move(cur);
    has_last = true;
  }
  if (hw != hash_witness.size()) return "WitnessTooLong";
  if (qv != queried_values.size()) return "TooManyQueriedValues";
  if (cw != column_witness.size()) return "WitnessTooLong";
  if (last.size() != 1 || last[0].first != 0) return "RootMismatch";
  if (last[0].second != root) return "RootMismatch";
  return "";
}

// ------------------------------------------------------------------ helpers
// prepare_preprocessed_query_positions (core/pcs/utils.rs:200-218).
inline std::vector<size_t> prepare_query_positions(const std::vector<size_t>& positions, uint32_t max_log_size,
                                                   uint32_t pp_max_log_size) {
  std::vector<size_t> r;
  if (pp_max_log_size == 0) return r;
  for (size_t pos : positions) {
    if (max_log_size < pp_max_log_size)
      r.push_back(((pos >> 1) << (pp_max_log_size - max_log_size + 1)) + (pos & 1));
    else
      r.push_back(((pos >> (max_log_size - pp_max_log_size + 1)) << 1) + (pos & 1));
  }
  return r;
}

inline std::vector<size_t> sorted_unique(std::vector<size_t> v) {
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  return v;
}

inline size_t lifted_position(size_t pos, uint32_t shift) { return ((pos >> (shift + 1)) << 1) + (pos & 1); }

// build_queries_per_log_size (core/pcs/verifier.rs:160-182).
inline std::map<uint32_t, std::vector<size_t>> queries_per_log_size(const std::vector<uint32_t>& log_sizes,
                                                                    const std::vector<size_t>& positions) {
  std::map<uint32_t, std::vector<size_t>> r;
  uint32_t max_log = log_sizes.empty() ? 0 : *std::max_element(log_sizes.begin(), log_sizes.end());
  for (uint32_t l : log_sizes) {
    if (r.count(l)) continue;
    std::vector<size_t> v;
    for (size_t p : positions) v.push_back(lifted_position(p, max_log - l));
    r[l] = sorted_unique(v);
  }
  return r;
}

// LinePoly::eval_at_point: fold(coeffs, [x, pi(x), pi^2(x), ...]).
inline QM31 fold_values(const QM31* v, size_t n, const QM31* factors) {
  if (n == 1) return v[0];
  QM31 l = fold_values(v, n / 2, factors + 1), r = fold_values(v + n / 2, n / 2, factors + 1);
  return l + r * factors[0];
}
inline QM31 line_poly_eval(const std::vector<QM31>& coeffs, uint32_t log_size, QM31 x) {
  std::vector<QM31> doublings;
  for (uint32_t i = 0; i < log_size; i++) {
    doublings.push_back(x);
    x = double_x(x);
  }
  return fold_values(coeffs.data(), coeffs.size(), doublings.data());
}

inline void ibfly(QM31& v0, QM31& v1, M31 itw) {
  QM31 t = v0;
  v0 = t + v1;
  v1 = (t - v1) * itw;
}

// fold_coset (core/fri.rs:680-700): folds 2^n values on a line coset by n.
inline QM31 fold_coset(std::vector<QM31> eval, Coset domain, QM31 alpha) {
  uint32_t n = domain.log_size;
  for (uint32_t i = 0; i < n; i++) {
    for (size_t j = 0; j < ((size_t)1 << (n - i)); j += 2) {
      M31 x = domain.at(bit_reverse_index(j, domain.log_size)).x;
      QM31 f0 = eval[j], f1 = eval[j + 1];
      ibfly(f0, f1, inv(x));
      eval[j >> 1] = f0 + alpha * f1;
    }
    alpha = alpha * alpha;
    domain = domain.dbl();
  }
  return eval[0];
}

// compute_decommitment_positions_and_rebuild_evals (core/fri.rs:593-632).
struct Sparse {
  std::vector<std::vector<QM31>> subset_evals;
  std::vector<size_t> subset_initial_indexes;
};
inline bool rebuild_evals(const std::vector<size_t>& queries, uint32_t log_domain_size,
                          const std::vector<QM31>& query_evals, const std::vector<QM31>& witness, size_t& wi,
                          uint32_t fold_step, std::vector<size_t>& decommitment_positions, Sparse& sparse) {
  size_t qi = 0, ei = 0;
  while (qi < queries.size()) {
    size_t subset = queries[qi] >> fold_step;
    size_t start = subset << fold_step;
    std::vector<QM31> ev;
    for (size_t pos = start; pos < start + ((size_t)1 << fold_step); pos++) {
      decommitment_positions.push_back(pos);
      if (qi < queries.size() && queries[qi] == pos) {
        if (ei >= query_evals.size()) return false;
        ev.push_back(query_evals[ei++]);
        qi++;
      } else {
        if (wi >= witness.size()) return false;
        ev.push_back(witness[wi++]);
      }
    }
    sparse.subset_evals.push_back(std::move(ev));
    sparse.subset_initial_indexes.push_back(bit_reverse_index(start, log_domain_size));
  }
  return true;
}

inline std::vector<M31> flat_coordinates(const Sparse& s) {
  std::vector<M31> r;
  for (auto& e : s.subset_evals)
    for (auto& q : e)
      for (int k = 0; k < 4; k++) r.push_back(M31(q.coord(k)));
  return r;
}

inline std::vector<size_t> fold_queries(const std::vector<size_t>& q, uint32_t n_folds) {
  std::vector<size_t> r;
  for (size_t x : q) {
    size_t f = x >> n_folds;
    if (r.empty() || r.back() != f) r.push_back(f);
  }
  return r;
}

// Evaluator of the AIR at the out-of-domain point (PointEvaluator,
// constraint-framework/src/point.rs): mask values from the proof, each
// constraint times the vanishing polynomial's inverse accumulated with the
// random coefficient (PointEvaluationAccumulator::accumulate).
struct PointEvaluator {
  using F = QM31;
  const std::vector<std::vector<std::vector<QM31>>>* mask;  // per tree, column, mask offset
  QM31 random_coeff, denom_inverse, shift, acc;
  size_t trace_col = 0;
  QM31 next_trace_mask() { return (*mask)[1][trace_col++][0]; }
  void next_cumsum_mask(QM31& prev, QM31& cur) {
    QM31 p[4], c[4];
    for (int k = 0; k < 4; k++) {
      p[k] = (*mask)[2][k][0];
      c[k] = (*mask)[2][k][1];
    }
    prev = qm31_from_partial_evals(p);
    cur = qm31_from_partial_evals(c);
  }
  QM31 cumsum_shift() const { return shift; }
  void add_constraint(QM31 c) { acc = acc * random_coeff + denom_inverse * c; }
};

// ------------------------------------------------------------------- verify
// cfg: the verifier's PcsConfig (CommitmentSchemeVerifier::new(config)); as
// in the reference, the copy serialised inside the proof is not consulted.
inline Result verify(const Statement& st, const StarkProof& proof, const PcsConfig& cfg) {
  // FriConfig::new's ranges (core/fri.rs:43-70)
  if (cfg.log_blowup < 1 || cfg.log_blowup > 16 || cfg.log_last_layer > 10 || cfg.fold_step < 1)
    return fail(INVALID_STRUCTURE, "PcsConfig out of range");
  const bool poseidon = st.kind == Air::Poseidon;
  const size_t n_trees = poseidon ? 3 : 2;  // preprocessed, trace (, interaction)
  if (proof.commitments.size() != n_trees + 1) return fail(INVALID_STRUCTURE, "number of commitments");
  Channel ch(st.hash);
  std::vector<Hash32> roots;
  std::vector<std::vector<uint32_t>> tree_log_sizes;  // extended by the blowup
  auto commit = [&](const Hash32& root, uint32_t n_columns, uint32_t log_size) {
    ch.mix_root(root);
    roots.push_back(root);
    tree_log_sizes.push_back(std::vector<uint32_t>(n_columns, log_size + cfg.log_blowup));
  };
  // the caller's side of the protocol (poseidon/mod.rs:905-922)
  commit(proof.commitments[0], 0, st.log_n);
  commit(proof.commitments[1], st.n_trace_cols(), st.log_n);
  LookupElements16 le{};
  if (poseidon) {
    auto zs = ch.draw_secure_felts(2);
    le.z = zs[0];
    le.alpha = zs[1];
    QM31 cur(M31(1));
    for (int i = 0; i < 16; i++) {
      le.alpha_powers[i] = cur;
      cur = cur * le.alpha;
    }
    commit(proof.commitments[2], 4, st.log_n);
  }

  // verify_ex (core/verifier.rs:35-122)
  uint32_t comp_bound = st.max_constraint_log_degree_bound();
  if (st.split_log < 1 || st.split_log >= comp_bound) return fail(INVALID_STRUCTURE, "composition split");
  uint32_t split_bound = comp_bound - st.split_log;
  uint32_t lifting = cfg.has_lifting ? cfg.lifting : split_bound + cfg.log_blowup;
  if (split_bound + cfg.log_blowup > lifting || lifting > 30) return fail(INVALID_STRUCTURE, "lifting log size");
  uint32_t max_ldb = lifting - cfg.log_blowup;
  QM31 random_coeff = ch.draw_secure_felt();
  const uint32_t n_comp_cols = 4u << st.split_log;
  commit(proof.commitments.back(), n_comp_cols, max_ldb);
  CirclePoint<QM31> oods = get_random_point(ch);

  // mask points per tree and column
  CirclePoint<M31> step = CanonicCoset::make(max_ldb).step();
  CirclePoint<M31> identity{M31(1), M31(0)};
  std::vector<std::vector<std::vector<CirclePoint<QM31>>>> points(tree_log_sizes.size());
  points[1].assign(st.n_trace_cols(), {oods + identity});
  if (poseidon) points[2].assign(4, {oods + conjugate(step), oods + identity});
  points.back().assign(n_comp_cols, {oods});

  const auto& sv = proof.sampled_values;
  if (sv.size() != points.size()) return fail(INVALID_STRUCTURE, "sampled_values trees");
  for (size_t t = 0; t < points.size(); t++) {
    if (sv[t].size() != points[t].size()) return fail(INVALID_STRUCTURE, "sampled_values columns");
    for (size_t c = 0; c < points[t].size(); c++)
      if (sv[t][c].size() != points[t][c].size()) return fail(INVALID_STRUCTURE, "sampled_values per column");
  }

  // extract_composition_oods_eval, for 2^split parts
  QM31 composition_oods;
  {
    const auto& comp = sv.back();
    for (uint32_t part = 0; part < (1u << st.split_log); part++) {
      QM31 e[4];
      for (int k = 0; k < 4; k++) e[k] = comp[4 * part + k][0];
      QM31 v = qm31_from_partial_evals(e);
      for (uint32_t j = 0; j < st.split_log; j++)
        if ((part >> j) & 1) v = v * repeated_double(oods, max_ldb - 1 + j).x;
      composition_oods += v;
    }
  }
  // eval_composition_polynomial_at_point
  PointEvaluator pe;
  pe.mask = &sv;
  pe.random_coeff = random_coeff;
  pe.denom_inverse = inv(coset_vanishing(CanonicCoset::make(max_ldb).coset, oods));
  pe.shift = st.claimed_sum * inv(M31((uint32_t)(((uint64_t)1 << st.log_n) % P)));
  if (poseidon) eval_poseidon(pe, le);
  else eval_wide_fibonacci(pe, st.n_cols);
  if (pe.acc != composition_oods) return fail(OODS_NOT_MATCHING, "composition OODS value does not match");

  // verify_values (core/pcs/verifier.rs:60-157)
  {
    std::vector<QM31> flat;
    for (auto& tree : sv)
      for (auto& col : tree) flat.insert(flat.end(), col.begin(), col.end());
    ch.mix_felts(flat);
  }
  QM31 fri_coeff = ch.draw_secure_felt();
  uint32_t lift2 = 0;
  for (size_t t = 0; t < points.size(); t++)
    for (size_t c = 0; c < points[t].size(); c++)
      if (!points[t][c].empty()) lift2 = std::max(lift2, tree_log_sizes[t][c]);
  uint32_t bound = lift2 - cfg.log_blowup;

  // FriVerifier::commit (core/fri.rs:109-183)
  const FriProof& fri = proof.fri;
  ch.mix_root(fri.first.commitment);
  const CircleDomain first_domain = CanonicCoset::make(bound + cfg.log_blowup).circle_domain();
  QM31 first_alpha = ch.draw_secure_felt();
  struct Inner {
    Coset domain;  // the line domain's coset
    QM31 alpha;
    uint32_t fold_step;
  };
  std::vector<Inner> inner;
  if (bound < 1) return fail(FRI, "InvalidNumFriLayers");
  uint32_t layer_bound = bound - 1;
  Coset layer_domain = Coset::half_odds(layer_bound + cfg.log_blowup);
  for (size_t i = 0; i < fri.inner.size(); i++) {
    ch.mix_root(fri.inner[i].commitment);
    uint32_t fold_step = cfg.fold_step;
    if (i + 1 == fri.inner.size()) {
      if (layer_bound < cfg.log_last_layer) return fail(FRI, "InvalidNumFriLayers");
      fold_step = layer_bound - cfg.log_last_layer;
      if (fold_step < 1 || fold_step > cfg.fold_step) return fail(FRI, "InvalidNumFriLayers");
    }
    QM31 alpha = ch.draw_secure_felt();
    inner.push_back({layer_domain, alpha, fold_step});
    if (layer_bound < fold_step || layer_domain.log_size < fold_step) return fail(FRI, "InvalidNumFriLayers");
    layer_bound -= fold_step;
    layer_domain = layer_domain.repeated_double(fold_step);
  }
  if (layer_bound != cfg.log_last_layer) return fail(FRI, "InvalidNumFriLayers");
  const Coset last_domain = layer_domain;
  if (fri.last_layer_coeffs.size() > ((size_t)1 << cfg.log_last_layer)) return fail(FRI, "LastLayerDegreeInvalid");
  ch.mix_felts(fri.last_layer_coeffs);

  // proof of work, query positions
  if (!ch.verify_pow_nonce(cfg.pow_bits, proof.proof_of_work)) return fail(PROOF_OF_WORK, "proof of work");
  ch.mix_u64(proof.proof_of_work);
  const uint32_t query_log = first_domain.log_size();
  std::vector<size_t> positions = sorted_unique(draw_queries(ch, query_log, cfg.n_queries));

  // Merkle decommitments of the committed trees
  if (proof.decommitments.size() != tree_log_sizes.size() || proof.queried_values.size() != tree_log_sizes.size())
    return fail(INVALID_STRUCTURE, "decommitments / queried_values trees");
  for (size_t t = 0; t < tree_log_sizes.size(); t++) {
    const auto& ls = tree_log_sizes[t];
    uint32_t tmax = ls.empty() ? 0 : *std::max_element(ls.begin(), ls.end());
    std::vector<size_t> tree_positions = t == 0 ? prepare_query_positions(positions, lift2, tmax) : positions;
    std::string e = merkle_verify(roots[t], ls, queries_per_log_size(ls, tree_positions), proof.queried_values[t],
                                  proof.decommitments[t], st.hash);
    if (!e.empty()) return fail(MERKLE, "tree " + std::to_string(t) + ": " + e);
  }

  // fri_answers (core/pcs/quotients.rs:120-165)
  std::vector<std::vector<M31>> column_values;  // per column over every tree, one value per query position
  for (size_t t = 0; t < tree_log_sizes.size(); t++) {
    const auto& ls = tree_log_sizes[t];
    const auto& flat = proof.queried_values[t];
    uint32_t tmax = ls.empty() ? 0 : *std::max_element(ls.begin(), ls.end());
    std::vector<size_t> tq = prepare_query_positions(positions, lift2, tmax);
    std::map<uint32_t, std::vector<size_t>> cols_by_log;
    for (size_t c = 0; c < ls.size(); c++) cols_by_log[ls[c]].push_back(c);
    std::map<uint32_t, std::vector<size_t>> qpl;
    for (auto& kv : cols_by_log) {
      std::vector<size_t> v;
      for (size_t p : tq) v.push_back(lifted_position(p, tmax - kv.first));
      qpl[kv.first] = sorted_unique(v);
    }
    std::vector<std::vector<M31>> natural(ls.size());
    size_t fi = 0;
    for (auto it = cols_by_log.rbegin(); it != cols_by_log.rend(); ++it)
      for (size_t k = 0; k < qpl[it->first].size(); k++)
        for (size_t c : it->second) {
          if (fi >= flat.size()) return fail(INVALID_STRUCTURE, "too few queried values");
          natural[c].push_back(flat[fi++]);
        }
    if (fi != flat.size()) return fail(INVALID_STRUCTURE, "too many queried values");
    for (size_t c = 0; c < ls.size(); c++) {
      const auto& pos = qpl[ls[c]];
      std::vector<M31> vals;
      for (size_t p : tq) {
        size_t lp = lifted_position(p, tmax - ls[c]);
        size_t idx = std::lower_bound(pos.begin(), pos.end(), lp) - pos.begin();
        vals.push_back(natural[c][idx]);
      }
      if (vals.size() != positions.size()) return fail(INVALID_STRUCTURE, "queried values per column");
      column_values.push_back(std::move(vals));
    }
  }
  // samples with random coefficients (powers of fri_coeff in column order) and periodicity samples
  struct Sample {
    CirclePoint<QM31> point;
    QM31 value;
    QM31 coeff;
  };
  std::vector<std::vector<Sample>> col_samples;
  {
    QM31 pow(M31(1));
    CirclePoint<M31> lift_gen = CanonicCoset::make(lift2).step();
    for (size_t t = 0; t < points.size(); t++)
      for (size_t c = 0; c < points[t].size(); c++) {
        std::vector<Sample> s;
        const auto& pts = points[t][c];
        const auto& vals = sv[t][c];
        if (pts.size() == 2) {
          CirclePoint<M31> period = repeated_double(lift_gen, tree_log_sizes[t][c]);
          s.push_back({pts[1] + period, vals[1], pow});
          pow = pow * fri_coeff;
        }
        for (size_t k = 0; k < pts.size(); k++) {
          s.push_back({pts[k], vals[k], pow});
          pow = pow * fri_coeff;
        }
        col_samples.push_back(std::move(s));
      }
  }
  if (col_samples.size() != column_values.size()) return fail(INVALID_STRUCTURE, "column count");
  // ColumnSampleBatch::new_vec: group by point in first-seen order; line coefficients per entry
  struct Entry {
    size_t column;
    QM31 a, b, c;
  };
  struct Batch {
    CirclePoint<QM31> point;
    std::vector<Entry> entries;
  };
  std::vector<Batch> batches;
  for (size_t col = 0; col < col_samples.size(); col++)
    for (const Sample& s : col_samples[col]) {
      size_t b = 0;
      while (b < batches.size() && !(batches[b].point.x == s.point.x && batches[b].point.y == s.point.y)) b++;
      if (b == batches.size()) batches.push_back({s.point, {}});
      // complex_conjugate_line_coeffs (core/constraints.rs:119-134)
      if (s.point.y == conj(s.point.y)) return fail(INVALID_STRUCTURE, "sample point on the base circle");
      QM31 a = conj(s.value) - s.value;
      QM31 c = conj(s.point.y) - s.point.y;
      QM31 bb = s.value * c - a * s.point.y;
      batches[b].entries.push_back({col, s.coeff * a, s.coeff * bb, s.coeff * c});
    }
  std::vector<QM31> answers;
  const CircleDomain lift_domain = CanonicCoset::make(lift2).circle_domain();
  for (size_t qi = 0; qi < positions.size(); qi++) {
    CirclePoint<M31> dp = lift_domain.at(bit_reverse_index(positions[qi], lift2));
    std::vector<CM31> den(batches.size()), den_inv(batches.size());
    for (size_t b = 0; b < batches.size(); b++) {
      const auto& sp = batches[b].point;
      // (Re px - x) * Im py - (Re py - y) * Im px
      den[b] = (sp.x.x - CM31(dp.x, M31(0))) * sp.y.y - (sp.y.x - CM31(dp.y, M31(0))) * sp.x.y;
    }
    batch_inverse(den.data(), den_inv.data(), den.size());
    QM31 row;
    for (size_t b = 0; b < batches.size(); b++) {
      QM31 num;
      for (const Entry& e : batches[b].entries) num += e.c * column_values[e.column][qi] - (e.a * dp.y + e.b);
      row += mul_cm31(num, den_inv[b]);
    }
    answers.push_back(row);
  }

  // FriVerifier::decommit (core/fri.rs:195-290, 431-590)
  size_t wi = 0;
  std::vector<size_t> decommit_positions;
  Sparse first;
  if (!rebuild_evals(positions, query_log, answers, fri.first.fri_witness, wi, 1, decommit_positions, first) ||
      wi != fri.first.fri_witness.size())
    return fail(FRI, "FirstLayerEvaluationsInvalid");
  {
    std::string e = merkle_verify(fri.first.commitment, std::vector<uint32_t>(4, query_log),
                                  {{query_log, decommit_positions}}, flat_coordinates(first),
                                  fri.first.decommitment, st.hash);
    if (!e.empty()) return fail(FRI, "FirstLayerCommitmentInvalid: " + e);
  }
  // fold_circle: each pair (p, conj p) into one line value
  std::vector<QM31> evals;
  for (size_t s = 0; s < first.subset_evals.size(); s++) {
    CirclePoint<M31> p = first_domain.index_at(first.subset_initial_indexes[s]).to_point();
    QM31 f0 = first.subset_evals[s][0], f1 = first.subset_evals[s][1];
    ibfly(f0, f1, inv(p.y));
    evals.push_back(first_alpha * f1 + f0);
  }
  std::vector<size_t> queries = fold_queries(positions, 1);
  uint32_t qlog = query_log - 1;
  for (size_t i = 0; i < inner.size(); i++) {
    const Inner& L = inner[i];
    const FriLayerProof& lp = fri.inner[i];
    if (qlog != L.domain.log_size) return fail(FRI, "InnerLayerEvaluationsInvalid");
    size_t w = 0;
    std::vector<size_t> dpos;
    Sparse sp;
    if (!rebuild_evals(queries, qlog, evals, lp.fri_witness, w, L.fold_step, dpos, sp) || w != lp.fri_witness.size())
      return fail(FRI, "InnerLayerEvaluationsInvalid " + std::to_string(i));
    std::string e = merkle_verify(lp.commitment, std::vector<uint32_t>(4, qlog), {{qlog, dpos}},
                                  flat_coordinates(sp), lp.decommitment, st.hash);
    if (!e.empty()) return fail(FRI, "InnerLayerCommitmentInvalid " + std::to_string(i) + ": " + e);
    std::vector<QM31> folded;
    for (size_t s = 0; s < sp.subset_evals.size(); s++) {
      CPI init = L.domain.index_at(sp.subset_initial_indexes[s]);
      folded.push_back(fold_coset(sp.subset_evals[s], Coset::make(init, L.fold_step), L.alpha));
    }
    evals = std::move(folded);
    queries = fold_queries(queries, L.fold_step);
    qlog -= L.fold_step;
  }
  for (size_t k = 0; k < queries.size(); k++) {
    QM31 x(last_domain.at(bit_reverse_index(queries[k], last_domain.log_size)).x);
    if (evals[k] != line_poly_eval(fri.last_layer_coeffs, fri.last_layer_log, x))
      return fail(FRI, "LastLayerEvaluationsInvalid");
  }
  return Result{};
}

}  // namespace ver
}  // namespace orc
