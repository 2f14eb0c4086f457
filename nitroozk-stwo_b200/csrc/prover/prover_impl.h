#pragma once
#include <functional>
// GPU prover (see prover.h): commitment trees, composition polynomial,
// out-of-domain sampling, DEEP quotients, FRI, proof of work, decommitment.
#include "prover.h"
#include "host_air.h"
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>

namespace gs {
int fold_line_fused(cudaStream_t st, CPlanes src, uint32_t log_n, qm31 alpha, Planes dst, const uint32_t* d_itw,
                    uint32_t tw_log, uint32_t* leaf_out);
int fold_circle_into_line_fused(cudaStream_t st, CPlanes src, uint32_t log_n, qm31 alpha, Planes dst,
                                const uint32_t* d_itw, uint32_t tw_log, uint32_t* leaf_out);
int fold_line_dev_alpha(cudaStream_t st, CPlanes src, uint32_t log_n, const uint32_t* d_alpha, Planes dst,
                        const uint32_t* d_itw, uint32_t tw_log, uint32_t* leaf_out);
int fold_circle_into_line_dev_alpha(cudaStream_t st, CPlanes src, uint32_t log_n, const uint32_t* d_alpha, Planes dst,
                                    const uint32_t* d_itw, uint32_t tw_log, uint32_t* leaf_out);
int interpolate_columns_to(cudaStream_t st, const uint32_t* const* d_src, uint32_t* const* d_dst, uint32_t n_cols,
                           uint32_t log_n, const uint32_t* d_itwiddles, uint32_t tw_log);

namespace prover {

using host::Hash;

// Phase timeline of one proof, enabled by the environment variable
// GS_PHASE_LOG=1: at each mark, a CUDA event on the prover's stream and the
// host clock. At the end one JSON line goes to stderr with, per phase, the
// device time between events and the host time spent enqueuing it; a phase
// whose host time exceeds its device time leaves the GPU idle.
struct PhaseLog {
  bool on = false;
  cudaStream_t st = nullptr;
  std::vector<const char*> names;
  std::vector<cudaEvent_t> ev;
  std::vector<std::chrono::steady_clock::time_point> host;
  void init(cudaStream_t s) {
    static const bool enabled = [] {  // read once per process
      const char* e = getenv("GS_PHASE_LOG");
      return e && e[0] == '1';
    }();
    on = enabled;
    st = s;
  }
  void mark(const char* name) {
    if (!on) return;
    cudaEvent_t x;
    cudaEventCreate(&x);
    cudaEventRecord(x, st);
    names.push_back(name);
    ev.push_back(x);
    host.push_back(std::chrono::steady_clock::now());
  }
  void report(size_t pool_allocs = 0, size_t requests = 0) {
    if (!on || ev.size() < 2) return;
    cudaEventSynchronize(ev.back());
    std::string js = "{\"phases\": [";
    for (size_t i = 1; i < ev.size(); i++) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[i - 1], ev[i]);
      double hms = std::chrono::duration<double, std::milli>(host[i] - host[i - 1]).count();
      char buf[160];
      snprintf(buf, sizeof buf, "%s[\"%s\", %.3f, %.3f]", i > 1 ? ", " : "", names[i], ms, hms);
      js += buf;
    }
    float tot = 0;
    cudaEventElapsedTime(&tot, ev.front(), ev.back());
    double htot = std::chrono::duration<double, std::milli>(host.back() - host.front()).count();
    char buf[160];
    snprintf(buf, sizeof buf, "], \"device_ms\": %.3f, \"host_ms\": %.3f, \"pool_allocs\": %zu, \"requests\": %zu}\n",
             tot, htot, pool_allocs, requests);
    js += buf;
    fputs(js.c_str(), stderr);
    for (auto x : ev) cudaEventDestroy(x);
    ev.clear();
  }
  ~PhaseLog() {
    for (auto x : ev) cudaEventDestroy(x);
  }
};

struct Prover {
  Context& ctx;
  cudaStream_t st;
  PcsConfig cfg;
  host::Channel ch;
  Arena A;
  std::vector<Tree> trees;
  const uint32_t* tw = nullptr;
  const uint32_t* itw = nullptr;
  uint32_t tw_log = 0;
  PhaseLog phases;

  Prover(Context& c, const PcsConfig& p) : ctx(c), st(c.stream), cfg(p) {
    A.st = st;
    A.pool = c.pool;
    if (c.keep_buffers) A.spare = &c.spare;
    phases.init(st);
  }
  void mark(const char* name) { phases.mark(name); }

  int twiddles_for(uint32_t root_log) {
    GS_TRY(ctx.twiddles(root_log, &tw, &itw));
    tw_log = root_log;
    return OK;
  }

  int table(const std::vector<const uint32_t*>& ptrs, const uint32_t* const** out) {
    const void* const* d = nullptr;
    GS_TRY(ctx.stage_ptrs((const void* const*)ptrs.data(), ptrs.size(), &d));
    *out = (const uint32_t* const*)d;
    return OK;
  }

  int merkle(Tree& t) {
    t.layers.assign(t.eval_log + 1, nullptr);
    for (uint32_t L = 0; L <= t.eval_log; L++) GS_TRY(A.alloc_n((size_t)8 << L, &t.layers[L]));
    std::vector<const uint32_t*> cols;
    for (uint32_t c = 0; c < t.n_cols; c++) cols.push_back(t.eval_col(c));
    const uint32_t* const* tab = nullptr;
    GS_TRY(table(cols, &tab));
    if (ch.p252) {  // Poseidon252MerkleHasher: one launch per layer
      GS_TRY(poseidon252_commit_on_layer(st, t.eval_log, nullptr, tab, t.n_cols, (uint8_t*)t.layers[t.eval_log]));
      for (int L = (int)t.eval_log - 1; L >= 0; L--)
        GS_TRY(poseidon252_commit_on_layer(st, (uint32_t)L, (const uint8_t*)t.layers[L + 1], nullptr, 0,
                                           (uint8_t*)t.layers[L]));
    } else {
      GS_TRY(commit_on_layer(st, t.eval_log, nullptr, tab, t.n_cols, t.layers[t.eval_log]));
      if (ctx.d_mail) {  // the tree kernel writes the root into mailbox slot 0 itself
        GS_TRY(commit_node_layers_to(st, t.eval_log, t.layers.data(), ctx.tree_counters, (uint32_t*)ctx.d_mail));
        return ctx.mail_record(0);
      }
      GS_TRY(commit_node_layers(st, t.eval_log, t.layers.data(), ctx.tree_counters));
    }
    // the root comes back through mailbox slot 0; commit_coeffs waits for it
    return ctx.mail_start(0, t.layers[0], 32);
  }

  // Extends columns [t.ext_done, c_end) of a committed tree to the constraint
  // domain 2^E (the composition needs every column there; the work depends
  // on nothing the channel draws, so it can fill a wait for the host). With
  // on_side it runs on the context's low-priority side stream, joined
  // before the composition reads it.
  int extend(Tree& t, uint32_t E, uint32_t c_end, bool on_side = false) {
    if (t.eval_log == E || c_end <= t.ext_done) return OK;
    if (!t.ext) {
      GS_TRY(A.alloc_n((size_t)t.n_cols << E, &t.ext));
      t.ext_log = E;
    }
    std::vector<const uint32_t*> src(t.coeff_ptrs.begin() + t.ext_done, t.coeff_ptrs.begin() + c_end);
    std::vector<const uint32_t*> dst;
    for (uint32_t c = t.ext_done; c < c_end; c++) dst.push_back(t.ext + ((size_t)c << E));
    const uint32_t* const* stab = nullptr;
    const uint32_t* const* dtab = nullptr;
    GS_TRY(table(src, &stab));
    GS_TRY(table(dst, &dtab));
    cudaStream_t s = st;
    if (on_side && ctx.side) {
      GS_TRY(ctx.fork_side());
      s = ctx.side;
    }
    GS_TRY(evaluate_columns(s, stab, t.coeff_log, (uint32_t* const*)dtab, c_end - t.ext_done, E, tw, tw_log));
    t.ext_done = c_end;
    return OK;
  }

  // TreeBuilder::commit on coefficient columns (given by pointer). `overlap`
  // enqueues device work that needs neither this root nor anything drawn
  // after it; it runs while the root is on its way to the host.
  // `early` runs as soon as the coefficients are known, before the tree's
  // own evaluation and hashing are enqueued (for side-stream work that can
  // then fill the gaps of all of them).
  int commit_coeffs(const std::vector<const uint32_t*>& coeffs, uint32_t coeff_log,
                    const std::function<int(Tree&)>& overlap = nullptr,
                    const std::function<int(Tree&)>& early = nullptr) {
    Tree t;
    t.n_cols = (uint32_t)coeffs.size();
    t.coeff_log = coeff_log;
    t.eval_log = coeff_log + cfg.log_blowup;
    t.coeff_ptrs = coeffs;
    if (early) GS_TRY(early(t));
    GS_TRY(table(coeffs, &t.coeff_tab));
    GS_TRY(A.alloc_n((size_t)t.n_cols << t.eval_log, &t.evals));
    std::vector<const uint32_t*> dst;
    for (uint32_t c = 0; c < t.n_cols; c++) dst.push_back(t.eval_col(c));
    const uint32_t* const* dtab = nullptr;
    GS_TRY(table(dst, &dtab));
    GS_TRY(evaluate_columns(st, t.coeff_tab, coeff_log, (uint32_t* const*)dtab, t.n_cols, t.eval_log, tw, tw_log));
    GS_TRY(merkle(t));
    if (overlap) GS_TRY(overlap(t));
    const void* h = nullptr;
    GS_TRY(ctx.mail_wait(0, &h));
    t.root = host::hash_from_words((const uint32_t*)h);
    ch.mix_root(t.root);
    trees.push_back(std::move(t));
    return OK;
  }

  // TreeBuilder::extend_evals + commit: contiguous evaluations on
  // CanonicCoset(log) (bit-reversed) are interpolated into new buffers.
  int commit_evals(const uint32_t* evals, uint32_t n_cols, uint32_t log,
                   const std::function<int(Tree&)>& overlap = nullptr,
                   const std::function<int(Tree&)>& early = nullptr) {
    uint32_t* coeffs = nullptr;
    GS_TRY(A.alloc_n((size_t)n_cols << log, &coeffs));
    std::vector<const uint32_t*> src, dst;
    for (uint32_t c = 0; c < n_cols; c++) {
      src.push_back(evals + ((size_t)c << log));
      dst.push_back(coeffs + ((size_t)c << log));
    }
    const uint32_t* const* stab = nullptr;
    const uint32_t* const* dtab = nullptr;
    GS_TRY(table(src, &stab));
    GS_TRY(table(dst, &dtab));
    GS_TRY(interpolate_columns_to(st, stab, (uint32_t* const*)dtab, n_cols, log, itw, tw_log));
    return commit_coeffs(dst, log, overlap, early);
  }

  int commit_empty() {
    Tree t;
    // MerkleProver::commit of no columns: hash_node(None, []) of one node
    t.root = ch.p252 ? host::p252::to_bytes(host::p252::hash_many({})) : host::hash_bytes(nullptr, 0);
    ch.mix_root(t.root);
    trees.push_back(std::move(t));
    return OK;
  }

  // What the composition needs before its random coefficient is drawn: the
  // constraint denominators, the output planes and their pointer table.
  // Called while the last trace root is read back; composition() calls it
  // itself when nothing did.
  struct CompositionPrep {
    bool ready = false;
    ConstraintParams prm;
    uint32_t* comp[4] = {nullptr, nullptr, nullptr, nullptr};
    const uint32_t* const* ctab = nullptr;
  } cprep;
  int prepare_composition(const AirHost& air) {
    if (cprep.ready) return OK;
    const uint32_t E = air.max_constraint_log(), T = air.log_n;
    ConstraintParams& prm = cprep.prm;
    memset(&prm, 0, sizeof(prm));
    // denominators 1 / vanishing(CanonicCoset(T), eval_domain.at(i)), bit-reversed
    const uint32_t log_expand = E - T;
    GS_REQUIRE(log_expand <= 3, "constraint blowup above 8");
    std::vector<uint32_t> dn(1u << log_expand);
    for (uint32_t i = 0; i < dn.size(); i++) {
      // eval_domain = CanonicCoset(E).circle_domain(): half coset half_odds(E-1),
      // point i (i < half) = index 2^(31-(E+1)) + i * 2^(31-(E-1)).
      uint32_t idx = (uint32_t)(((1ull << (31 - (E + 1))) + (uint64_t)i * (1ull << (31 - (E - 1)))) & 0x7fffffffu);
      dn[i] = inv(host::canonic_vanishing_m31(T, host::index_point(idx)));
    }
    for (uint32_t i = 0; i < dn.size(); i++) prm.denom_inv[host::bitrev(i, log_expand)] = dn[i];
    for (int c = 0; c < 4; c++) GS_TRY(A.alloc_n((size_t)1 << E, &cprep.comp[c]));
    std::vector<const uint32_t*> cp = {cprep.comp[0], cprep.comp[1], cprep.comp[2], cprep.comp[3]};
    GS_TRY(table(cp, &cprep.ctab));
    cprep.ready = true;
    return OK;
  }

  // Composition polynomial coefficients (4 planes of 2^eval_log) for the component.
  int composition(const AirHost& air, qm31 random_coeff, uint32_t* comp[4]) {
    const uint32_t E = air.max_constraint_log(), T = air.log_n;
    GS_TRY(prepare_composition(air));
    // trace columns on the evaluation domain
    std::vector<const uint32_t*> on_domain(trees.size(), nullptr);
    for (size_t t = 1; t < trees.size(); t++) {
      Tree& tr = trees[t];
      if (tr.eval_log == E) { on_domain[t] = tr.evals; continue; }
      GS_TRY(extend(tr, E, tr.n_cols));  // the columns not extended earlier
      on_domain[t] = tr.ext;
    }
    GS_TRY(ctx.join_side());
    ConstraintParams& prm = cprep.prm;
    const uint32_t nc = air.n_constraints();
    GS_REQUIRE(nc <= (uint32_t)MAX_CONSTRAINTS, "too many constraints");
    qm31 pw = qm_one();
    for (uint32_t k = 0; k < nc; k++) {  // constraint k gets alpha^(nc-1-k)
      uint32_t* p = prm.powers + 4 * (nc - 1 - k);
      p[0] = pw.x.a; p[1] = pw.x.b; p[2] = pw.y.a; p[3] = pw.y.b;
      pw = qm_mul(pw, random_coeff);
    }
    for (int c = 0; c < 4; c++) comp[c] = cprep.comp[c];
    Planes out{{comp[0], comp[1], comp[2], comp[3]}};
    if (air.kind == AirKind::WideFibonacci) {
      GS_TRY(wf_constraints(st, on_domain[1], air.n_cols, E, T, prm, out));
    } else {
      qm31 shift = qm_mul_m31(air.claimed_sum, inv((uint32_t)((1ull << T) % P)));
      GS_TRY(poseidon_constraints(st, on_domain[1], on_domain[2], E, T, prm, air.lookup, shift, out));
    }
    // finalize: interpolate the 4 coordinates on CanonicCoset(E)
    const uint32_t* const* ctab = cprep.ctab;
    GS_TRY(interpolate_columns(st, (uint32_t* const*)ctab, 4, E, itw, tw_log));
    return OK;
  }
};

static bool pt_eq(const ptq& a, const ptq& b) { return qm_eq(a.x, b.x) && qm_eq(a.y, b.y); }

// Line interpolation of the last FRI layer (prover/line.rs:45-70) on
// half_odds(log) from bit-reversed values; returns LinePoly coefficients in
// the reference's internal order.
static std::vector<qm31> line_interpolate_host(std::vector<qm31> v, uint32_t log) {
  size_t n = v.size();
  std::vector<qm31> t(n);
  for (size_t i = 0; i < n; i++) t[host::bitrev(i, log)] = v[i];
  v = t;
  for (uint32_t l = log; l >= 1; l--) {  // domain half_odds(l) = index 2^(29-l) + i * 2^(31-l)
    size_t size = (size_t)1 << l;
    for (size_t c = 0; c < n; c += size)
      for (size_t i = 0; i < size / 2; i++) {
        uint32_t idx = (uint32_t)(((1ull << (31 - (l + 2))) + (uint64_t)i * (1ull << (31 - l))) & 0x7fffffffu);
        uint32_t xinv = inv(host::index_point(idx).x);
        qm31 a = v[c + i], b = v[c + size / 2 + i];
        v[c + i] = qm_add(a, b);
        v[c + size / 2 + i] = qm_mul_m31(qm_sub(a, b), xinv);
      }
  }
  uint32_t ninv = inv((uint32_t)n);
  for (auto& x : v) x = qm_mul_m31(x, ninv);
  return v;
}

// FRI layer data kept for decommitment.
struct FriLayerDev {
  uint32_t log = 0;
  uint32_t* planes[4] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<uint32_t*> layers;
  Hash root{};
};

static std::vector<size_t> prepare_positions(const std::vector<size_t>& q, uint32_t lifting, uint32_t tree_log) {
  std::vector<size_t> r;
  if (tree_log == 0) return r;
  for (size_t pos : q) {
    if (lifting < tree_log) r.push_back(((pos >> 1) << (tree_log - lifting + 1)) + (pos & 1));
    else r.push_back(((pos >> (lifting - tree_log + 1)) << 1) + (pos & 1));
  }
  std::sort(r.begin(), r.end());
  r.erase(std::unique(r.begin(), r.end()), r.end());
  return r;
}

}  // namespace prover
}  // namespace gs
