// prove() driver for the two benchmark components on the GPU prover.
#include "prover_impl.h"
#include "prove_api.h"

namespace gs {
void fft_set_columns_aligned(bool aligned);
namespace prover {

// FRI commit (prover/fri.rs:99-199) on the combined quotient planes (2^lifting).
int fri_commit(Prover& pv, uint32_t* quot[4], uint32_t lifting, FriLayerDev& first,
                      std::vector<FriLayerDev>& inner, std::vector<qm31>& last_coeffs) {
  cudaStream_t st = pv.st;
  Arena& A = pv.A;
  auto alloc_layer = [&](FriLayerDev& L, uint32_t log) -> int {
    L.log = log;
    for (int c = 0; c < 4; c++) GS_TRY(A.alloc_n((size_t)1 << log, &L.planes[c]));
    L.layers.assign(log + 1, nullptr);
    for (uint32_t k = 0; k <= log; k++) GS_TRY(A.alloc_n((size_t)8 << k, &L.layers[k]));
    return OK;
  };
  auto root_of = [&](FriLayerDev& L) -> int {
    GS_TRY(commit_node_layers(st, L.log, L.layers.data()));
    uint32_t w[8];
    GS_CUDA_TRY(cudaMemcpyAsync(w, L.layers[0], 32, cudaMemcpyDeviceToHost, st));
    GS_CUDA_TRY(cudaStreamSynchronize(st));
    L.root = host::hash_from_words(w);
    return OK;
  };
  // first layer: the quotient columns themselves
  first.log = lifting;
  for (int c = 0; c < 4; c++) first.planes[c] = quot[c];
  first.layers.assign(lifting + 1, nullptr);
  for (uint32_t k = 0; k <= lifting; k++) GS_TRY(A.alloc_n((size_t)8 << k, &first.layers[k]));
  {
    std::vector<const uint32_t*> cols = {quot[0], quot[1], quot[2], quot[3]};
    const uint32_t* const* tab = nullptr;
    GS_TRY(pv.table(cols, &tab));
    GS_TRY(commit_on_layer(st, lifting, nullptr, tab, 4, first.layers[lifting]));
  }
  GS_TRY(root_of(first));
  pv.ch.mix_root(first.root);
  const uint32_t last_log = pv.cfg.log_last_layer + pv.cfg.log_blowup;
  // fold the circle evaluation into the first line layer (zero-initialised)
  FriLayerDev cur;
  GS_TRY(alloc_layer(cur, lifting - 1));
  for (int c = 0; c < 4; c++) GS_CUDA_TRY(cudaMemsetAsync(cur.planes[c], 0, (size_t)4 << cur.log, st));
  qm31 alpha = pv.ch.draw_felt();
  GS_TRY(fold_circle_into_line_fused(st, CPlanes{{quot[0], quot[1], quot[2], quot[3]}}, lifting, alpha,
                                     Planes{{cur.planes[0], cur.planes[1], cur.planes[2], cur.planes[3]}}, pv.itw,
                                     pv.tw_log, cur.layers[cur.log]));
  if (cur.log != last_log) {
    for (;;) {
      GS_TRY(root_of(cur));
      pv.ch.mix_root(cur.root);
      alpha = pv.ch.draw_felt();
      FriLayerDev next;
      GS_TRY(alloc_layer(next, cur.log - 1));
      GS_TRY(fold_line_fused(st, CPlanes{{cur.planes[0], cur.planes[1], cur.planes[2], cur.planes[3]}}, cur.log, alpha,
                             Planes{{next.planes[0], next.planes[1], next.planes[2], next.planes[3]}}, pv.itw,
                             pv.tw_log, next.layers[next.log]));
      inner.push_back(std::move(cur));
      cur = std::move(next);
      if (cur.log <= last_log) break;
    }
  }
  // last layer: 2^last_log values -> line polynomial, degree check, mix
  size_t n = (size_t)1 << cur.log;
  std::vector<uint32_t> h(4 * n);
  for (int c = 0; c < 4; c++)
    GS_CUDA_TRY(cudaMemcpyAsync(h.data() + c * n, cur.planes[c], 4 * n, cudaMemcpyDeviceToHost, st));
  GS_CUDA_TRY(cudaStreamSynchronize(st));
  std::vector<qm31> vals(n);
  for (size_t i = 0; i < n; i++) vals[i] = qm_make(h[i], h[n + i], h[2 * n + i], h[3 * n + i]);
  std::vector<qm31> coeffs = line_interpolate_host(vals, cur.log);
  // into ordered coefficients (bit reverse), keep the degree bound, back
  std::vector<qm31> ordered(n);
  for (size_t i = 0; i < n; i++) ordered[host::bitrev(i, cur.log)] = coeffs[i];
  size_t bound = (size_t)1 << pv.cfg.log_last_layer;
  for (size_t i = bound; i < n; i++)
    if (!qm_eq(ordered[i], qm_zero())) {
      set_error("FRI last layer: invalid degree");
      return ERR_PROOF;
    }
  ordered.resize(bound);
  uint32_t blog = pv.cfg.log_last_layer;
  last_coeffs.assign(bound, qm_zero());
  for (size_t i = 0; i < bound; i++) last_coeffs[host::bitrev(i, blog)] = ordered[i];
  pv.ch.mix_felts(last_coeffs);
  return OK;
}

// compute_decommitment_positions_and_witness_evals (prover/fri.rs:301-330),
// fold step 1: positions are both members of each queried pair; the witness
// values are the pair members that were not queried.
void fri_positions(const std::vector<size_t>& q, std::vector<size_t>& pos, std::vector<bool>& is_witness) {
  size_t i = 0;
  while (i < q.size()) {
    size_t start = (q[i] >> 1) << 1;
    size_t j = i;
    while (j < q.size() && (q[j] >> 1) == (q[i] >> 1)) j++;
    size_t k = i;
    for (size_t p = start; p < start + 2; p++) {
      pos.push_back(p);
      if (k < j && q[k] == p) { k++; is_witness.push_back(false); }
      else is_witness.push_back(true);
    }
    i = j;
  }
}

int prove_component(Context& ctx, const ProveRequest& req, std::string* proof_bytes, ProveStats* stats) {
  PcsConfig cfg = req.cfg;
  Prover pv(ctx, cfg);
  cudaStream_t st = ctx.stream;
  AirHost air;
  air.kind = req.air == 0 ? AirKind::WideFibonacci : AirKind::Poseidon;
  air.log_n = req.log_n;
  air.n_cols = req.n_cols;
  const uint32_t split = req.split_log;
  const uint32_t E = air.max_constraint_log();
  GS_REQUIRE(air.log_n >= 2 && air.log_n <= 26, "trace log size out of range");
  GS_REQUIRE(split >= 1 && split <= air.log_expand(), "composition split must be in [1, constraint blowup]");
  GS_REQUIRE(cfg.fold_step == 1, "only line_fold_step 1 is supported (as the reference's CUDA FRI)");
  GS_REQUIRE(cfg.log_blowup >= 1 && cfg.log_blowup <= 4, "log_blowup out of range");
  // twiddles for the largest domain used: LDEs, the constraint domain, FRI
  uint32_t comp_tree = E - split + cfg.log_blowup;
  GS_REQUIRE(comp_tree >= cfg.log_last_layer + cfg.log_blowup + 1, "trace too small for the FRI last layer");
  uint32_t root = std::max({air.log_n + cfg.log_blowup, E, comp_tree}) - 1;
  GS_TRY(pv.twiddles_for(root));
  // every column buffer of the prover starts at a multiple of 4 words
  fft_set_columns_aligned(true);
  // preprocessed tree (empty)
  GS_TRY(pv.commit_empty());
  // trace
  const uint32_t T = air.log_n;
  const size_t n = (size_t)1 << T;
  uint32_t* trace = nullptr;
  GS_TRY(pv.A.alloc_n((size_t)air.n_trace_cols() << T, &trace));
  if (air.kind == AirKind::WideFibonacci) {
    if (req.input_mode == 2) {
      GS_CUDA_TRY(cudaMemcpyAsync(trace, req.host_inputs, 4 * n, cudaMemcpyHostToDevice, st));
      GS_CUDA_TRY(cudaMemcpyAsync(trace + n, req.host_inputs + n, 4 * n, cudaMemcpyHostToDevice, st));
    }
    GS_TRY(wf_trace(st, trace, T, air.n_cols, req.seed, req.input_mode));
  } else {
    if (req.input_mode == 2)
      GS_CUDA_TRY(cudaMemcpyAsync(trace, req.host_inputs, 16 * 4 * n, cudaMemcpyHostToDevice, st));
    GS_TRY(poseidon_trace(st, trace, T, req.seed, req.input_mode));
  }
  GS_TRY(pv.commit_evals(trace, air.n_trace_cols(), T));
  if (air.kind == AirKind::Poseidon) {
    auto z = pv.ch.draw_felts(2);
    qm31 alpha = z[1], cur = qm_one();
    for (int i = 0; i < 16; i++) {
      air.lookup.alpha_pow[4 * i] = cur.x.a; air.lookup.alpha_pow[4 * i + 1] = cur.x.b;
      air.lookup.alpha_pow[4 * i + 2] = cur.y.a; air.lookup.alpha_pow[4 * i + 3] = cur.y.b;
      cur = qm_mul(cur, alpha);
    }
    air.lookup.z[0] = z[0].x.a; air.lookup.z[1] = z[0].x.b; air.lookup.z[2] = z[0].y.a; air.lookup.z[3] = z[0].y.b;
    void* scratch = nullptr;
    GS_TRY(pv.A.alloc(logup_scratch_bytes(T), &scratch));
    uint32_t* inter = nullptr;
    GS_TRY(pv.A.alloc_n((size_t)4 << T, &inter));
    GS_TRY(poseidon_interaction(st, trace, T, air.lookup, inter, scratch, &air.claimed_sum));
    GS_TRY(pv.commit_evals(inter, 4, T));
  }
  return prove_tail(pv, air, split, proof_bytes, stats);
}

}  // namespace prover
}  // namespace gs
