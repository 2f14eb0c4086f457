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
void fri_positions(const std::vector<size_t>& q, std::vector<size_t>& pos, std::vector<uint8_t>& is_witness);

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
  {
    std::vector<const uint32_t*> parts;
    const uint32_t plog = E - split;
    for (uint32_t t = 0; t < (1u << split); t++)
      for (int c = 0; c < 4; c++) parts.push_back(comp[c] + ((size_t)t << plog));
    GS_TRY(pv.commit_coeffs(parts, plog));
  }
  pv.mark("composition_commit");
  ptq oods = host::random_point(pv.ch);
  const uint32_t lifting = pv.trees.back().max_log();
  const uint32_t max_ldb = lifting - cfg.log_blowup;
  // sample points and values per tree / column: the points of tree t are
  // those of requests [req0[t], req0[t] + n_pts[t]); every column of a tree is
  // sampled at all of them, the values staying in the read-back array
  const size_t n_trees = pv.trees.size();
  std::vector<size_t> req0(n_trees, 0), n_pts(n_trees, 0);
  pt31 step = host::index_point(host::canonic_step_index(max_ldb));
  // every (tree, mask point) evaluation is enqueued, then read back once
  struct SampleReq {
    size_t t;
    ptq p;
    size_t slot;
  };
  std::vector<SampleReq> reqs;
  size_t n_vals = 0, scratch_bytes = 0;
  for (size_t t = 0; t < n_trees; t++) {
    Tree& tr = pv.trees[t];
    req0[t] = reqs.size();
    if (tr.n_cols == 0) continue;
    std::vector<ptq> pts;  // mask points of every column of this tree
    if (t + 1 == n_trees || t == 1) pts = {oods};
    else pts = {ptq_add(oods, host::to_ptq(pt_conj(step))), oods};  // interaction: offsets -1, 0
    for (auto& p : pts) {
      reqs.push_back({t, p, n_vals});
      n_vals += tr.n_cols;
      scratch_bytes = std::max(scratch_bytes, eval_at_point_scratch_bytes(tr.n_cols, tr.coeff_log));
    }
    n_pts[t] = pts.size();
  }
  std::vector<uint32_t> h(4 * n_vals);
  auto sample_point = [&](size_t t, size_t k) -> const ptq& { return reqs[req0[t] + k].p; };
  auto sample_value = [&](size_t t, uint32_t c, size_t k) {
    const uint32_t* v = h.data() + 4 * (reqs[req0[t] + k].slot + c);
    return qm_make(v[0], v[1], v[2], v[3]);
  };
  {
    uint32_t* d_vals = nullptr;
    void* scratch = nullptr;
    GS_TRY(pv.A.alloc_n(4 * n_vals + 4, &d_vals));
    GS_TRY(pv.A.alloc(scratch_bytes + 16, &scratch));
    // the largest evaluation (the trace's) runs on the side stream with a
    // scratch of its own, next to the small ones on the work stream
    size_t big = 0;
    auto cost = [&](const SampleReq& r) { return (size_t)pv.trees[r.t].n_cols << pv.trees[r.t].coeff_log; };
    for (size_t i = 1; i < reqs.size(); i++)
      if (cost(reqs[i]) > cost(reqs[big])) big = i;
    const bool split_streams = reqs.size() > 1 && pv.ctx.side != nullptr;
    void* scratch_big = scratch;
    if (split_streams) {
      GS_TRY(pv.A.alloc(scratch_bytes + 16, &scratch_big));
      GS_TRY(pv.ctx.fork_side());
    }
    for (size_t i = 0; i < reqs.size(); i++) {
      const SampleReq& r = reqs[i];
      Tree& tr = pv.trees[r.t];
      bool vec = true;
      for (auto* c : tr.coeff_ptrs) vec = vec && ((uintptr_t)c & 15) == 0;
      const bool side = split_streams && i == big;
      GS_TRY(batch_eval_at_point(side ? pv.ctx.side : st, tr.coeff_tab, tr.n_cols, tr.coeff_log,
                                 host::ptq_rep_double(r.p, lifting - tr.eval_log), d_vals + 4 * r.slot,
                                 (uint32_t*)(side ? scratch_big : scratch), 12, vec));
    }
    GS_TRY(pv.ctx.join_side());
    GS_TRY(pv.ctx.read_back(d_vals, h.size() * 4, h.data()));
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
  // DEEP quotients: per (column size, point) batches of line-coefficient
  // terms, lifted per point, combined over the lifting domain.
  qm31 qrc = pv.ch.draw_felt();
  struct Batch {
    ptq point;
    uint32_t log;
    std::vector<NumEntry> entries;
    qm31 b_sum = qm_zero(), a_sum = qm_zero();
  };
  std::vector<Batch> batches;
  qm31 pw = qm_one();
  pt31 lift_step = host::index_point(host::canonic_step_index(lifting));
  for (size_t t = 0; t < n_trees; t++) {
    Tree& tr = pv.trees[t];
    if (tr.n_cols == 0 || n_pts[t] == 0) continue;
    // the terms of each column: with two points, the second point shifted by
    // the tree's period first (its value repeated), then every point; all
    // columns of a tree share the points, hence the batches
    ptq pts[3];
    size_t src[3], n_terms = 0;
    if (n_pts[t] == 2) {
      pt31 period = lift_step;
      for (uint32_t k = 0; k < tr.eval_log; k++) period = pt_add(period, period);
      pts[n_terms] = ptq_add(sample_point(t, 1), host::to_ptq(period));
      src[n_terms++] = 1;
    }
    for (size_t k = 0; k < n_pts[t]; k++) {
      pts[n_terms] = sample_point(t, k);
      src[n_terms++] = k;
    }
    size_t bidx[3];
    for (size_t j = 0; j < n_terms; j++) {
      bidx[j] = batches.size();
      for (size_t x = 0; x < batches.size(); x++)
        if (batches[x].log == tr.eval_log && pt_eq(batches[x].point, pts[j])) bidx[j] = x;
      if (bidx[j] == batches.size()) batches.push_back(Batch{pts[j], tr.eval_log, {}, qm_zero(), qm_zero()});
      batches[bidx[j]].entries.reserve(batches[bidx[j]].entries.size() + tr.n_cols);
    }
    for (uint32_t c = 0; c < tr.n_cols; c++)
      for (size_t j = 0; j < n_terms; j++) {
        qm31 a, b, cc;
        line_coeffs(pts[j], sample_value(t, c, src[j]), pw, a, b, cc);
        pw = qm_mul(pw, qrc);
        Batch& bt = batches[bidx[j]];
        NumEntry e;
        e.col = tr.eval_col(c);
        e.c[0] = cc.x.a; e.c[1] = cc.x.b; e.c[2] = cc.y.a; e.c[3] = cc.y.b;
        bt.entries.push_back(e);
        bt.b_sum = qm_add(bt.b_sum, b);
        bt.a_sum = qm_add(bt.a_sum, a);
      }
  }
  pv.mark("quot_plan");
  struct PointAcc2 {
    ptq point;
    std::vector<std::pair<uint32_t, uint32_t*>> parts;  // (log, planes base of 4 x 2^log)
    qm31 flt = qm_zero();
  };
  std::vector<PointAcc2> per_point;
  for (auto& bt : batches) {
    uint32_t* planes = nullptr;
    GS_TRY(pv.A.alloc_n((size_t)4 << bt.log, &planes));
    const void* d_entries = nullptr;
    GS_TRY(pv.ctx.stage_bytes(bt.entries.data(), bt.entries.size() * sizeof(NumEntry), &d_entries));
    size_t nn = (size_t)1 << bt.log;
    bool vec = bt.log >= 2;  // tree columns and these planes sit at multiples of 2^log words
    for (auto& e : bt.entries) vec = vec && ((uintptr_t)e.col & 15) == 0;
    GS_TRY(accumulate_numerators(st, d_entries, (uint32_t)bt.entries.size(), bt.b_sum, bt.log,
                                 Planes{{planes, planes + nn, planes + 2 * nn, planes + 3 * nn}}, vec));
    PointAcc2* pa = nullptr;
    for (auto& x : per_point)
      if (pt_eq(x.point, bt.point)) pa = &x;
    if (!pa) {
      per_point.push_back(PointAcc2{bt.point, {}, qm_zero()});
      pa = &per_point.back();
    }
    pa->parts.push_back({bt.log, planes});
    pa->flt = qm_add(pa->flt, bt.a_sum);
  }
  std::vector<QuotAcc> qaccs;
  for (auto& pa : per_point) {
    std::sort(pa.parts.begin(), pa.parts.end(), [](auto& x, auto& y) { return x.first < y.first; });
    uint32_t top = pa.parts.back().first;
    uint32_t* res = pa.parts.back().second;
    if (pa.parts.size() > 1) {
      std::vector<LiftCol> lc;
      for (auto& [lg, base] : pa.parts) {
        size_t nn = (size_t)1 << lg;
        lc.push_back(LiftCol{{base, base + nn, base + 2 * nn, base + 3 * nn}, lg, 0});
      }
      GS_TRY(pv.A.alloc_n((size_t)4 << top, &res));
      const void* d = nullptr;
      GS_TRY(pv.ctx.stage_bytes(lc.data(), lc.size() * sizeof(LiftCol), &d));
      size_t nn = (size_t)1 << top;
      GS_TRY(lift_and_accumulate(st, d, (uint32_t)lc.size(), top, Planes{{res, res + nn, res + 2 * nn, res + 3 * nn}}));
    }
    size_t nn = (size_t)1 << top;
    QuotAcc q;
    q.p[0] = res; q.p[1] = res + nn; q.p[2] = res + 2 * nn; q.p[3] = res + 3 * nn;
    q.log_size = top;
    q.pad = 0;
    q.first_linear = pa.flt;
    q.prx = pa.point.x.x; q.pix = pa.point.x.y; q.pry = pa.point.y.x; q.piy = pa.point.y.y;
    qaccs.push_back(q);
  }
  uint32_t* quot[4];
  for (int c = 0; c < 4; c++) GS_TRY(pv.A.alloc_n((size_t)1 << lifting, &quot[c]));
  {
    DomainTables dt;
    GS_TRY(pv.ctx.domain_tables(lifting, &dt));
    const void* d = nullptr;
    GS_TRY(pv.ctx.stage_bytes(qaccs.data(), qaccs.size() * sizeof(QuotAcc), &d));
    GS_TRY(compute_quotients_and_combine(st, d, (uint32_t)qaccs.size(), dt, Planes{{quot[0], quot[1], quot[2], quot[3]}}));
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
    std::vector<size_t> pos;
    std::vector<uint8_t> wit;  // 1: the position is a witness value
    std::vector<size_t> wpos;  // the witness positions: only their values are gathered
    size_t val_base = 0;
    MerkleDecommitPlan merkle;
  };
  // the witness lists of every level of the query set, shared by the FRI
  // layers and the lifting-size trees
  static thread_local SharedWitness sw;
  sw.build(g, queries, lifting);
  // FRI layer i (the first layer is i = 0) is queried at S_i, its leaves
  // decommitted as the pairs of S_i
  auto plan_fri = [&](FriLayerDev& L, const std::vector<size_t>& q, size_t i, FriPlan& fp) -> int {
    fri_positions(q, fp.pos, fp.wit);
    fp.wpos.clear();
    fp.wpos.reserve(fp.pos.size());
    for (size_t k = 0; k < fp.pos.size(); k++)
      if (fp.wit[k]) fp.wpos.push_back(fp.pos[k]);
    std::vector<const uint32_t*> cols = {L.planes[0], L.planes[1], L.planes[2], L.planes[3]};
    GS_TRY(g.add_cols(cols, fp.wpos, &fp.val_base));
    if (L.layers.size() == (size_t)lifting - i + 1)
      return fp.merkle.plan_shared(g, L.layers, cols, fp.pos, sw, (int)L.layers.size() - 3, i + 1, false);
    return fp.merkle.plan(g, L.layers, cols, fp.pos, false);
  };
  FriPlan first_plan;
  GS_TRY(plan_fri(first, queries, 0, first_plan));
  std::vector<FriPlan> inner_plans(inner.size());
  std::vector<size_t> lq = queries;
  std::vector<size_t> f;
  for (size_t i = 0; i < inner.size(); i++) {
    f.clear();
    f.reserve(lq.size());
    for (size_t q : lq)
      if (f.empty() || f.back() != (q >> 1)) f.push_back(q >> 1);
    lq.swap(f);
    GS_TRY(plan_fri(inner[i], lq, i + 1, inner_plans[i]));
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
    w.u64(fp.wpos.size());
    w.put_gathered(w.gathered ? go.word_out + fp.val_base : nullptr, 16 * fp.wpos.size());
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
