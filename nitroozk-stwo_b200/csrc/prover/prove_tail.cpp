// prove_ex after the trace commitments: composition commit, OODS samples,
// DEEP quotients, FRI, proof of work, decommitment and the composition sanity
// check (crates/stwo/src/prover/mod.rs:50-150, prover/pcs/mod.rs:151-357).
#include "prover_impl.h"
#include "prove_api.h"
#include <functional>

namespace gs {
namespace prover {

int fri_commit(Prover& pv, uint32_t* quot[4], uint32_t lifting, FriLayerDev& first, std::vector<FriLayerDev>& inner,
               std::vector<qm31>& last_coeffs, const std::function<void()>& while_busy, uint64_t* nonce,
               bool* have_nonce, std::function<int()>* replay);
size_t fri_witness_positions(const std::vector<size_t>& q, std::vector<size_t>& wit, std::vector<size_t>* pos);

int prove_tail(Prover& pv, AirHost& air, uint32_t split, std::string* proof_bytes, ProveStats* stats,
               uint8_t* out_buf, size_t out_cap) {
  cudaStream_t st = pv.st;
  const PcsConfig& cfg = pv.cfg;
  const uint32_t E = air.max_constraint_log();
  // composition polynomial and its commitment (split into 2^split parts)
  qm31 random_coeff = pv.ch.draw_felt();
  uint32_t* comp[4];
  GS_TRY(pv.composition(air, random_coeff, comp));
  pv.mark("composition");
  // The sample requests and the DEEP quotients' plan depend on the trees'
  // shapes and on the sample points' offsets from the OODS point, not on the
  // point itself (p + a = p + b exactly when a = b): both are built, and the
  // plan uploaded, while the composition's root is on its way to the host.
  // The points of tree t are oods + off for the requests [req0[t], req0[t] +
  // n_pts[t]); every column of a tree is sampled at all of them, the values
  // staying in the read-back array.
  struct SampleReq {
    size_t t;
    pt31 off;
    size_t slot;
    ptq p;  // once the OODS point is drawn
  };
  std::vector<SampleReq> reqs;
  std::vector<size_t> req0, n_pts;
  size_t n_trees = 0, n_vals = 0, scratch_bytes = 0;
  uint32_t lifting = 0, max_ldb = 0;
  // DEEP quotients (compute_fri_quotients, prover/pcs/quotient_ops.rs): the
  // terms (column, sample point) are grouped in batches of one column size
  // and one point; each batch accumulates its numerators, each point lifts
  // and combines its batches. One kernel computes the line coefficients and
  // their sums once the random coefficient is drawn.
  struct Batch {
    pt31 off;
    uint32_t log, point_id;
    std::vector<NumEntry> entries;
    std::vector<LineTerm> terms;
    uint32_t* planes = nullptr;
  };
  std::vector<Batch> batches;
  std::vector<pt31> qoffs;  // the distinct sample points' offsets
  struct PointAcc {
    std::vector<std::pair<uint32_t, uint32_t*>> parts;  // (log, planes base of 4 x 2^log)
    const void* d_lift = nullptr;                       // LiftCol array when more than one part
    uint32_t* res = nullptr;
    uint32_t top = 0;
  };
  std::vector<PointAcc> per_point;
  uint32_t* d_vals = nullptr;
  void* eval_scratch = nullptr;
  void* eval_scratch_big = nullptr;
  NumEntry* d_entries = nullptr;
  const LineTerm* d_terms = nullptr;
  const uint32_t* d_bfirst = nullptr;
  const uint32_t* d_bpoint = nullptr;
  uint32_t* d_bsums = nullptr;
  uint32_t* d_lscratch = nullptr;
  std::vector<uint32_t> bfirst;
  uint32_t n_terms = 0;
  auto plan_samples = [&](Tree& comp_tree) -> int {
    n_trees = pv.trees.size() + 1;
    auto tree = [&](size_t t) -> Tree& { return t + 1 == n_trees ? comp_tree : pv.trees[t]; };
    lifting = comp_tree.max_log();
    max_ldb = lifting - cfg.log_blowup;
    const pt31 step = host::index_point(host::canonic_step_index(max_ldb));
    const pt31 zero = {1u, 0u};
    req0.assign(n_trees, 0);
    n_pts.assign(n_trees, 0);
    for (size_t t = 0; t < n_trees; t++) {
      Tree& tr = tree(t);
      req0[t] = reqs.size();
      if (tr.n_cols == 0) continue;
      std::vector<pt31> offs;  // mask points of every column of this tree
      if (t + 1 == n_trees || t == 1) offs = {zero};
      else offs = {pt_conj(step), zero};  // interaction: offsets -1, 0
      for (auto& o : offs) {
        reqs.push_back({t, o, n_vals, {}});
        n_vals += tr.n_cols;
        scratch_bytes = std::max(scratch_bytes, eval_at_point_scratch_bytes(tr.n_cols, tr.coeff_log));
      }
      n_pts[t] = offs.size();
    }
    GS_TRY(pv.A.alloc_n(4 * n_vals + 4, &d_vals));
    GS_TRY(pv.A.alloc(scratch_bytes + 16, &eval_scratch));
    GS_TRY(pv.A.alloc(scratch_bytes + 16, &eval_scratch_big));
    // the quotients' batches, in the order the terms are met
    uint32_t kterm = 0;  // the random coefficient's power of the next term
    const pt31 lift_step = host::index_point(host::canonic_step_index(lifting));
    for (size_t t = 0; t < n_trees; t++) {
      Tree& tr = tree(t);
      if (tr.n_cols == 0 || n_pts[t] == 0) continue;
      // the terms of each column: with two points, the second point shifted
      // by the tree's period first (its value repeated), then every point;
      // all columns of a tree share the points, hence the batches
      pt31 offs[3];
      size_t src[3], n_t = 0;
      if (n_pts[t] == 2) {
        pt31 period = lift_step;
        for (uint32_t k = 0; k < tr.eval_log; k++) period = pt_add(period, period);
        offs[n_t] = pt_add(reqs[req0[t] + 1].off, period);
        src[n_t++] = 1;
      }
      for (size_t k = 0; k < n_pts[t]; k++) {
        offs[n_t] = reqs[req0[t] + k].off;
        src[n_t++] = k;
      }
      auto same = [](const pt31& a, const pt31& b) { return a.x == b.x && a.y == b.y; };
      size_t bidx[3];
      for (size_t j = 0; j < n_t; j++) {
        bidx[j] = batches.size();
        for (size_t x = 0; x < batches.size(); x++)
          if (batches[x].log == tr.eval_log && same(batches[x].off, offs[j])) bidx[j] = x;
        if (bidx[j] == batches.size()) {
          uint32_t pid = (uint32_t)qoffs.size();
          for (size_t q = 0; q < qoffs.size(); q++)
            if (same(qoffs[q], offs[j])) pid = (uint32_t)q;
          if (pid == qoffs.size()) qoffs.push_back(offs[j]);
          batches.push_back(Batch{offs[j], tr.eval_log, pid, {}, {}, nullptr});
        }
        batches[bidx[j]].entries.reserve(batches[bidx[j]].entries.size() + tr.n_cols);
        batches[bidx[j]].terms.reserve(batches[bidx[j]].terms.size() + tr.n_cols);
      }
      for (uint32_t c = 0; c < tr.n_cols; c++)
        for (size_t j = 0; j < n_t; j++) {
          Batch& bt = batches[bidx[j]];
          NumEntry e{};
          e.col = tr.eval_col(c);
          bt.entries.push_back(e);
          bt.terms.push_back(LineTerm{(uint32_t)(4 * (reqs[req0[t] + src[j]].slot + c)), bt.point_id, kterm++, 0});
        }
    }
    GS_REQUIRE(batches.size() <= QUOT_MAX_BATCHES && qoffs.size() <= QUOT_MAX_POINTS,
               "too many quotient batches or sample points");
    // numerator planes per batch; per point the lifted sum of its batches
    per_point.resize(qoffs.size());
    for (auto& bt : batches) {
      GS_TRY(pv.A.alloc_n((size_t)4 << bt.log, &bt.planes));
      per_point[bt.point_id].parts.push_back({bt.log, bt.planes});
    }
    std::vector<std::vector<LiftCol>> lifts(qoffs.size());
    for (size_t q = 0; q < qoffs.size(); q++) {
      PointAcc& pa = per_point[q];
      std::sort(pa.parts.begin(), pa.parts.end(), [](auto& x, auto& y) { return x.first < y.first; });
      pa.top = pa.parts.back().first;
      pa.res = pa.parts.back().second;
      if (pa.parts.size() > 1) {
        for (auto& [lg, base] : pa.parts) {
          size_t nn = (size_t)1 << lg;
          lifts[q].push_back(LiftCol{{base, base + nn, base + 2 * nn, base + 3 * nn}, lg, 0});
        }
        GS_TRY(pv.A.alloc_n((size_t)4 << pa.top, &pa.res));
      }
    }
    // one upload: entries | terms | batch_first | batch_point | lift columns
    std::vector<uint8_t> up;
    auto put = [&up](const void* p, size_t n) {
      const size_t o = up.size();
      up.resize(o + ((n + 15) & ~(size_t)15));
      if (n) memcpy(up.data() + o, p, n);
      return o;
    };
    std::vector<uint32_t> bpoint;
    bfirst.assign(1, 0);
    for (auto& bt : batches) {
      bfirst.push_back(bfirst.back() + (uint32_t)bt.entries.size());
      bpoint.push_back(bt.point_id);
    }
    n_terms = bfirst.back();
    std::vector<NumEntry> entries;
    std::vector<LineTerm> terms;
    entries.reserve(n_terms);
    terms.reserve(n_terms);
    for (auto& bt : batches) {
      entries.insert(entries.end(), bt.entries.begin(), bt.entries.end());
      terms.insert(terms.end(), bt.terms.begin(), bt.terms.end());
    }
    const size_t o_entries = put(entries.data(), entries.size() * sizeof(NumEntry));
    const size_t o_terms = put(terms.data(), terms.size() * sizeof(LineTerm));
    const size_t o_bfirst = put(bfirst.data(), bfirst.size() * 4);
    const size_t o_bpoint = put(bpoint.data(), bpoint.size() * 4);
    std::vector<size_t> o_lift(qoffs.size(), 0);
    for (size_t q = 0; q < qoffs.size(); q++)
      if (!lifts[q].empty()) o_lift[q] = put(lifts[q].data(), lifts[q].size() * sizeof(LiftCol));
    const void* d = nullptr;
    GS_TRY(pv.ctx.stage_bytes(up.data(), up.size(), &d));
    const uint8_t* db = (const uint8_t*)d;
    d_entries = (NumEntry*)(db + o_entries);  // the coefficient kernel writes c in place
    d_terms = (const LineTerm*)(db + o_terms);
    d_bfirst = (const uint32_t*)(db + o_bfirst);
    d_bpoint = (const uint32_t*)(db + o_bpoint);
    for (size_t q = 0; q < qoffs.size(); q++)
      if (!lifts[q].empty()) per_point[q].d_lift = db + o_lift[q];
    GS_TRY(pv.A.alloc_n(4 * batches.size() + 4, &d_bsums));
    GS_TRY(pv.A.alloc_n(8 * (size_t)n_terms + 8, &d_lscratch));
    return OK;
  };
  {
    std::vector<const uint32_t*> parts;
    const uint32_t plog = E - split;
    for (uint32_t t = 0; t < (1u << split); t++)
      for (int c = 0; c < 4; c++) parts.push_back(comp[c] + ((size_t)t << plog));
    GS_TRY(pv.commit_coeffs(parts, plog, plan_samples));
  }
  pv.mark("composition_commit");
  GS_REQUIRE(pv.trees.size() == n_trees, "sample plan out of step with the trees");
  ptq oods = host::random_point(pv.ch);
  for (auto& r : reqs) r.p = ptq_add(oods, host::to_ptq(r.off));
  std::vector<uint32_t> h(4 * n_vals);
  auto sample_value = [&](size_t t, uint32_t c, size_t k) {
    const uint32_t* v = h.data() + 4 * (reqs[req0[t] + k].slot + c);
    return qm_make(v[0], v[1], v[2], v[3]);
  };
  QuotAcc* d_qaccs = nullptr;
  const ptq* d_qpoints = nullptr;
  {
    // every (tree, mask point) evaluation is enqueued, then read back once;
    // the largest evaluation (the trace's) runs on the side stream with a
    // scratch of its own, next to the small ones on the work stream
    size_t big = 0;
    auto cost = [&](const SampleReq& r) { return (size_t)pv.trees[r.t].n_cols << pv.trees[r.t].coeff_log; };
    for (size_t i = 1; i < reqs.size(); i++)
      if (cost(reqs[i]) > cost(reqs[big])) big = i;
    const bool split_streams = reqs.size() > 1 && pv.ctx.side != nullptr;
    if (split_streams) GS_TRY(pv.ctx.fork_side());
    for (size_t i = 0; i < reqs.size(); i++) {
      const SampleReq& r = reqs[i];
      Tree& tr = pv.trees[r.t];
      bool vec = true;
      for (auto* c : tr.coeff_ptrs) vec = vec && ((uintptr_t)c & 15) == 0;
      const bool side = split_streams && i == big;
      GS_TRY(batch_eval_at_point(side ? pv.ctx.side : st, tr.coeff_tab, tr.n_cols, tr.coeff_log,
                                 host::ptq_rep_double(r.p, lifting - tr.eval_log), d_vals + 4 * r.slot,
                                 (uint32_t*)(side ? eval_scratch_big : eval_scratch), 12, vec));
    }
    // the sample points and the quotient accumulators (one upload)
    std::vector<ptq> qpoints;
    std::vector<QuotAcc> qaccs;
    for (size_t q = 0; q < qoffs.size(); q++) {
      const ptq pt = ptq_add(oods, host::to_ptq(qoffs[q]));
      qpoints.push_back(pt);
      const PointAcc& pa = per_point[q];
      const size_t nn = (size_t)1 << pa.top;
      QuotAcc qa{};
      qa.p[0] = pa.res; qa.p[1] = pa.res + nn; qa.p[2] = pa.res + 2 * nn; qa.p[3] = pa.res + 3 * nn;
      qa.log_size = pa.top;
      qa.first_linear = qm_zero();  // written by the coefficient kernel
      qa.prx = pt.x.x; qa.pix = pt.x.y; qa.pry = pt.y.x; qa.piy = pt.y.y;
      qaccs.push_back(qa);
    }
    const size_t o_acc = ((qpoints.size() * sizeof(ptq)) + 15) & ~(size_t)15;
    std::vector<uint8_t> up(o_acc + qaccs.size() * sizeof(QuotAcc));
    memcpy(up.data(), qpoints.data(), qpoints.size() * sizeof(ptq));
    memcpy(up.data() + o_acc, qaccs.data(), qaccs.size() * sizeof(QuotAcc));
    const void* d = nullptr;
    GS_TRY(pv.ctx.stage_bytes(up.data(), up.size(), &d));
    d_qpoints = (const ptq*)d;
    d_qaccs = (QuotAcc*)((uint8_t*)d + o_acc);
    GS_TRY(pv.ctx.join_side());
    GS_TRY(pv.ctx.read_back_published(d_vals, h.size() * 4, h.data()));
  }
  // mixed tree by tree, column by column, point by point
  std::vector<qm31> flat;
  flat.reserve(n_vals);
  for (size_t t = 0; t < n_trees; t++)
    for (uint32_t c = 0; c < pv.trees[t].n_cols; c++)
      for (size_t k = 0; k < n_pts[t]; k++) flat.push_back(sample_value(t, c, k));
  pv.ch.mix_felts(flat);
  pv.mark("oods_mix");
  pv.mark("oods_sample");
  // Sanity check (composition at the OODS point vs the constraints evaluated
  // from the mask values), run on this thread while the device works on the
  // FRI layers (fri_commit calls it before its read-back).
  bool sane = false;
  auto sanity = [&, split, oods, E, max_ldb, random_coeff]() {
    std::vector<std::vector<std::vector<qm31>>> sv(n_trees);
    for (size_t t = 0; t < n_trees; t++) {
      sv[t].resize(pv.trees[t].n_cols);
      for (uint32_t c = 0; c < pv.trees[t].n_cols; c++)
        for (size_t k = 0; k < n_pts[t]; k++) sv[t][c].push_back(sample_value(t, c, k));
    }
    auto& cv = sv.back();
    qm31 total = qm_zero();
    for (uint32_t t = 0; t < (1u << split); t++) {
      qm31 e4[4] = {cv[4 * t][0], cv[4 * t + 1][0], cv[4 * t + 2][0], cv[4 * t + 3][0]};
      qm31 v = from_partial_evals(e4);
      for (uint32_t b = 0; b < split; b++)
        if ((t >> b) & 1) v = qm_mul(v, host::ptq_rep_double(oods, E - split + b - 1).x);
      total = qm_add(total, v);
    }
    qm31 dinv = qm_inv(host::canonic_vanishing(max_ldb, oods));
    qm31 cons = eval_at_point(air, sv, random_coeff, dinv);
    sane = qm_eq(total, cons);
  };
  qm31 qrc = pv.ch.draw_felt();
  GS_TRY(quot_line_coeffs(st, d_terms, n_terms, d_vals, d_qpoints, qrc, d_entries, d_bfirst, d_bpoint,
                          (uint32_t)batches.size(), d_bsums, d_qaccs, (uint32_t)qoffs.size(), d_lscratch));
  pv.mark("quot_plan");
  for (size_t b = 0; b < batches.size(); b++) {
    const Batch& bt = batches[b];
    const size_t nn = (size_t)1 << bt.log;
    bool vec = bt.log >= 2;  // tree columns and these planes sit at multiples of 2^log words
    for (auto& e : bt.entries) vec = vec && ((uintptr_t)e.col & 15) == 0;
    GS_TRY(accumulate_numerators(st, d_entries + bfirst[b], bfirst[b + 1] - bfirst[b], qm_zero(), bt.log,
                                 Planes{{bt.planes, bt.planes + nn, bt.planes + 2 * nn, bt.planes + 3 * nn}}, vec,
                                 d_bsums + 4 * b));
  }
  for (auto& pa : per_point)
    if (pa.d_lift) {
      size_t nn = (size_t)1 << pa.top;
      GS_TRY(lift_and_accumulate(st, pa.d_lift, (uint32_t)pa.parts.size(), pa.top,
                                 Planes{{pa.res, pa.res + nn, pa.res + 2 * nn, pa.res + 3 * nn}}));
    }
  uint32_t* quot[4];
  for (int c = 0; c < 4; c++) GS_TRY(pv.A.alloc_n((size_t)1 << lifting, &quot[c]));
  {
    DomainTables dt;
    GS_TRY(pv.ctx.domain_tables(lifting, &dt));
    GS_TRY(compute_quotients_and_combine(st, d_qaccs, (uint32_t)qoffs.size(), dt,
                                         Planes{{quot[0], quot[1], quot[2], quot[3]}}));
  }
  pv.mark("quotients");
  // FRI commit, proof of work
  FriLayerDev first;
  std::vector<FriLayerDev> inner;
  std::vector<qm31> last;
  uint64_t nonce = 0;
  bool have_nonce = false;
  std::function<int()> replay;  // the FRI channel's host replay, when deferred
  GS_TRY(fri_commit(pv, quot, lifting, first, inner, last, sanity, &nonce, &have_nonce, &replay));
  pv.mark("fri_commit");
  if (have_nonce) {
    // found by the device right after the FRI layers (Blake2s channel)
  } else if (pv.ch.p252) {  // GrindOps<Poseidon252Channel>; the prefix hash on the host
    namespace f = host::p252;
    const auto pre = f::to_bytes(f::hash_many({f::from_u64(0x12345678u), pv.ch.fdigest(), f::from_u64(cfg.pow_bits)}));
    const void* d_pre = nullptr;
    GS_TRY(pv.ctx.stage_bytes(pre.data(), 32, &d_pre));
    GS_TRY(poseidon252_grind(st, (const uint8_t*)d_pre, cfg.pow_bits, pv.ctx.d_small, (uint32_t*)pv.ctx.h_small,
                             &nonce, true));
  } else {
    auto pre = pv.ch.pow_prefixed(cfg.pow_bits);
    GS_TRY(grind_blake2s(st, pre.data(), cfg.pow_bits, (uint32_t*)pv.ctx.d_small, &nonce,
                         (uint32_t*)pv.ctx.h_small));
  }
  pv.ch.mix_u64(nonce);
  pv.mark("grind");
  // queries
  auto raw = host::draw_queries(pv.ch, lifting, cfg.n_queries);
  std::vector<size_t> queries(raw);
  std::sort(queries.begin(), queries.end());
  queries.erase(std::unique(queries.begin(), queries.end()), queries.end());
  pv.mark("queries");
  // plan all gathers of the decommitment
  // The plan keeps its capacity across proofs; proofs on fibers of one
  // thread interleave at every wait, so nothing of it is read after launch
  // (the results are this proof's GatherOut).
  static thread_local GatherPlan g;
  g.clear();
  struct FriPlan {
    size_t n_wit = 0;  // witness values (only theirs are gathered)
    size_t val_base = 0;
    MerkleDecommitPlan merkle;
  };
  // the witness lists of every level of the query set, shared by the FRI
  // layers and the lifting-size trees
  static thread_local SharedWitness sw;
  sw.build(g, queries, lifting);
  // FRI layer i (the first layer is i = 0) is queried at S_i, its leaves
  // decommitted as the pairs of S_i. The position lists are scratch of this
  // thread, reused from layer to layer: planning never waits, and a plan
  // keeps only counts and offsets.
  static thread_local std::vector<size_t> s_pos, s_wpos, s_lq, s_f;
  static const std::vector<const uint32_t*> no_cols;
  auto plan_fri = [&](FriLayerDev& L, const std::vector<size_t>& q, size_t i, FriPlan& fp) -> int {
    const bool shared = L.layers.size() == (size_t)lifting - i + 1;
    const size_t n_pos = fri_witness_positions(q, s_wpos, shared ? nullptr : &s_pos);
    fp.n_wit = s_wpos.size();
    const uint32_t* cols[4] = {L.planes[0], L.planes[1], L.planes[2], L.planes[3]};
    GS_TRY(g.add_cols(cols, 4, s_wpos, &fp.val_base));
    if (shared) return fp.merkle.plan_shared_hashes(g, L.layers, n_pos, sw, (int)L.layers.size() - 3, i + 1);
    return fp.merkle.plan(g, L.layers, no_cols, s_pos, false);
  };
  FriPlan first_plan;
  GS_TRY(plan_fri(first, queries, 0, first_plan));
  std::vector<FriPlan> inner_plans(inner.size());
  s_lq.assign(queries.begin(), queries.end());
  for (size_t i = 0; i < inner.size(); i++) {
    s_f.clear();
    for (size_t q : s_lq)
      if (s_f.empty() || s_f.back() != (q >> 1)) s_f.push_back(q >> 1);
    s_lq.swap(s_f);
    GS_TRY(plan_fri(inner[i], s_lq, i + 1, inner_plans[i]));
  }
  pv.mark("fri_plans");
  std::vector<MerkleDecommitPlan> tree_plans(n_trees);
  for (size_t t = 0; t < n_trees; t++) {
    Tree& tr = pv.trees[t];
    if (tr.n_cols == 0) continue;
    std::vector<size_t> pos = prepare_positions(queries, lifting, tr.max_log());
    std::vector<const uint32_t*> cols;
    for (uint32_t c = 0; c < tr.n_cols; c++) cols.push_back(tr.eval_col(c));
    if (tr.layers.size() == (size_t)lifting + 1 && pos == sw.s0)
      GS_TRY(tree_plans[t].plan_shared(g, tr.layers, cols, pos, sw, (int)lifting - 1, 0));
    else
      GS_TRY(tree_plans[t].plan(g, tr.layers, cols, pos));
  }
  pv.mark("decommit_plan");
  GatherOut go;
  GS_TRY(g.launch(pv.ctx, pv.A, &go));
  if (replay) GS_TRY(replay());
  // The proof, written straight from the plans: every size is known now, so
  // the bytes the host holds are written while the gather runs, the gathered
  // ones after it lands.
  uint32_t last_layer_log = 0;
  while ((1u << last_layer_log) < last.size()) last_layer_log++;
  auto fri_layer = [&](host::Writer& w, const FriPlan& fp, const FriLayerDev& L) {
    // the witness values (4 coordinates each), consecutive in the gather
    w.u64(fp.n_wit);
    w.put_gathered(w.gathered ? go.word_out + fp.val_base : nullptr, 16 * fp.n_wit);
    fp.merkle.write_decommitment(w, go);
    w.hash(L.root);
  };
  auto write = [&](host::Writer& w) {
    w.u32(cfg.pow_bits);
    w.u32(cfg.log_blowup);
    w.u32(cfg.log_last_layer);
    w.u64(cfg.n_queries);
    w.u32(cfg.fold_step);
    w.u8(0);  // lifting_log_size: None
    w.u64(n_trees);
    for (auto& tr : pv.trees) w.hash(tr.root);
    w.u64(n_trees);
    for (size_t t = 0; t < n_trees; t++) {
      w.u64(pv.trees[t].n_cols);
      for (uint32_t c = 0; c < pv.trees[t].n_cols; c++) {
        w.u64(n_pts[t]);
        for (size_t k = 0; k < n_pts[t]; k++) w.qm(sample_value(t, c, k));
      }
    }
    w.u64(n_trees);
    for (size_t t = 0; t < n_trees; t++) {
      if (pv.trees[t].n_cols) {
        tree_plans[t].write_decommitment(w, go);
      } else {
        w.u64(0);
        w.u64(0);
      }
    }
    w.u64(n_trees);
    for (size_t t = 0; t < n_trees; t++) {
      if (pv.trees[t].n_cols) tree_plans[t].write_queried(w, go);
      else w.u64(0);
    }
    w.u64(nonce);
    fri_layer(w, first_plan, first);
    w.u64(inner.size());
    for (size_t i = 0; i < inner.size(); i++) fri_layer(w, inner_plans[i], inner[i]);
    w.u64(last.size());
    for (auto& q : last) w.qm(q);
    w.u32(last_layer_log);
  };
  host::Writer count;
  write(count);
  const size_t len = count.len;
  const bool direct = out_buf && len <= out_cap;
  char* dst = (char*)out_buf;
  if (!direct) {
    proof_bytes->resize(len);
    dst = len ? &(*proof_bytes)[0] : nullptr;
  }
  host::Writer fixed;
  fixed.out = dst;
  fixed.fixed = true;
  write(fixed);
  if (stats) {
    stats->constraint_check = sane ? 1.0 : 0.0;
    stats->proof_len = len;
    stats->in_out_buf = direct;
  }
  pv.mark("assemble");
  GS_TRY(go.wait(pv.ctx));
  pv.mark("decommit_gather");
  host::Writer gathered;
  gathered.out = dst;
  gathered.gathered = true;
  write(gathered);
  pv.mark("serialize");
  if (!sane) {
    set_error("constraints not satisfied: composition OODS value differs from the constraints at the mask");
    return ERR_PROOF;
  }
  return OK;
}

}  // namespace prover
}  // namespace gs
