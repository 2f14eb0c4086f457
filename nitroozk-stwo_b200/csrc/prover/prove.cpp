// prove() driver for the two benchmark components on the GPU prover.
#include "prover_impl.h"
#include <functional>
#include "prove_api.h"

namespace gs {
void fft_set_columns_aligned(bool aligned);
namespace prover {

static int last_layer_coeffs(Prover& pv, const uint32_t* h, uint32_t log, std::vector<qm31>& last_coeffs);
static int finish_last_layer(Prover& pv, const uint32_t* h, uint32_t log, std::vector<qm31>& last_coeffs);

// FRI commit with Poseidon252MerkleChannel (prover/fri.rs:99-199 over
// MerkleProver<Poseidon252MerkleHasher>): per layer, the leaves (the 4
// coordinates packed into one felt252 each) and node layers of its tree, then
// its root back to the host channel (mix_root, draw_secure_felt) for the fold
// into the next layer.
static int fri_commit_p252(Prover& pv, uint32_t* quot[4], uint32_t lifting, FriLayerDev& first,
                           std::vector<FriLayerDev>& inner, std::vector<qm31>& last_coeffs,
                           const std::function<void()>& while_busy) {
  cudaStream_t st = pv.st;
  const uint32_t last_log = pv.cfg.log_last_layer + pv.cfg.log_blowup;
  GS_REQUIRE(lifting >= last_log + 1, "FRI: lifting domain below the last layer");
  auto planes_of = [&](FriLayerDev& L, uint32_t log) -> int {
    L.log = log;
    for (int c = 0; c < 4; c++) GS_TRY(pv.A.alloc_n((size_t)1 << log, &L.planes[c]));
    return OK;
  };
  bool busy_done = false;
  auto commit_layer = [&](FriLayerDev& L) -> int {
    L.layers.assign(L.log + 1, nullptr);
    for (uint32_t k = 0; k <= L.log; k++) GS_TRY(pv.A.alloc_n((size_t)8 << k, &L.layers[k]));
    std::vector<const uint32_t*> cols = {L.planes[0], L.planes[1], L.planes[2], L.planes[3]};
    const uint32_t* const* tab = nullptr;
    GS_TRY(pv.table(cols, &tab));
    GS_TRY(poseidon252_commit_on_layer(st, L.log, nullptr, tab, 4, (uint8_t*)L.layers[L.log]));
    for (int k = (int)L.log - 1; k >= 0; k--)
      GS_TRY(poseidon252_commit_on_layer(st, (uint32_t)k, (const uint8_t*)L.layers[k + 1], nullptr, 0,
                                         (uint8_t*)L.layers[k]));
    if (!busy_done && while_busy) while_busy();  // overlaps the first tree
    busy_done = true;
    GS_TRY(pv.ctx.read_back(L.layers[0], 32, L.root.data()));
    pv.ch.mix_root(L.root);
    return OK;
  };
  first.log = lifting;
  for (int c = 0; c < 4; c++) first.planes[c] = quot[c];
  GS_TRY(commit_layer(first));
  qm31 alpha = pv.ch.draw_felt();
  FriLayerDev cur;
  GS_TRY(planes_of(cur, lifting - 1));
  for (int c = 0; c < 4; c++) GS_CUDA_TRY(cudaMemsetAsync(cur.planes[c], 0, (size_t)4 << cur.log, st));
  GS_TRY(fold_circle_into_line_fused(st, CPlanes{{quot[0], quot[1], quot[2], quot[3]}}, lifting, alpha,
                                     Planes{{cur.planes[0], cur.planes[1], cur.planes[2], cur.planes[3]}}, pv.itw,
                                     pv.tw_log, nullptr));
  while (cur.log > last_log) {
    GS_TRY(commit_layer(cur));
    alpha = pv.ch.draw_felt();
    FriLayerDev next;
    GS_TRY(planes_of(next, cur.log - 1));
    GS_TRY(fold_line_fused(st, CPlanes{{cur.planes[0], cur.planes[1], cur.planes[2], cur.planes[3]}}, cur.log, alpha,
                           Planes{{next.planes[0], next.planes[1], next.planes[2], next.planes[3]}}, pv.itw,
                           pv.tw_log, nullptr));
    inner.push_back(std::move(cur));
    cur = std::move(next);
  }
  const size_t n = (size_t)1 << cur.log;
  uint32_t* d_last = nullptr;
  GS_TRY(pv.A.alloc_n(4 * n, &d_last));
  for (int c = 0; c < 4; c++)
    GS_CUDA_TRY(cudaMemcpyAsync(d_last + c * n, cur.planes[c], 4 * n, cudaMemcpyDeviceToDevice, st));
  std::vector<uint32_t> h(4 * n);
  GS_TRY(pv.ctx.read_back(d_last, 16 * n, h.data()));
  return finish_last_layer(pv, h.data(), cur.log, last_coeffs);
}

// FRI commit (prover/fri.rs:99-199) on the combined quotient planes (2^lifting).
//
// The whole phase is enqueued without a host round trip: each layer's Merkle
// root goes through the device channel (mix_root + draw_secure_felt), whose
// challenge the next fold reads from device memory. Roots, challenges and the
// last layer come back in one read at the end; the host replays the channel
// on the roots and checks every challenge.
// `while_busy` runs on the host after every FRI launch is enqueued and before
// the one blocking read-back, overlapping host work with the device's.
// With the Blake2s channel and a last layer of at most 2^FRI_POW_MAX_LOG
// values, the proof of work follows on the device too (the last layer's
// coefficients mixed into the device channel, the prefixed digest, the
// grind's first chunk of nonces) and comes back in the same read: *nonce
// is then set and *have_nonce true. The host channel then takes the device's
// digest at once (the queries need it), and the replay of the layers' roots
// and challenges, the last layer's mix and the comparison with the device's
// digest go to *replay, which the caller runs before the proof is returned
// (while the decommitment's gather is on the device).
int fri_commit(Prover& pv, uint32_t* quot[4], uint32_t lifting, FriLayerDev& first,
                      std::vector<FriLayerDev>& inner, std::vector<qm31>& last_coeffs,
                      const std::function<void()>& while_busy, uint64_t* nonce, bool* have_nonce,
                      std::function<int()>* replay) {
  *have_nonce = false;
  *replay = nullptr;
  if (pv.ch.p252) return fri_commit_p252(pv, quot, lifting, first, inner, last_coeffs, while_busy);
  cudaStream_t st = pv.st;
  const uint32_t last_log = pv.cfg.log_last_layer + pv.cfg.log_blowup;
  GS_REQUIRE(lifting >= last_log + 1, "FRI: lifting domain below the last layer");
  const uint32_t n_roots = lifting - last_log;  // the first layer and the committed line layers
  const bool dev_pow = last_log <= FRI_POW_MAX_LOG && pv.cfg.log_last_layer <= 3 && pv.cfg.pow_bits <= 32;
  // one allocation for every FRI buffer, carved at 256-byte boundaries
  auto up = [](size_t w) { return (w + 63) & ~(size_t)63; };
  auto tree_words = [&](uint32_t log) {
    size_t w = 0;
    for (uint32_t k = 0; k <= log; k++) w += up((size_t)8 << k);
    return w;
  };
  // channel state, roots, challenges, a copy of the last layer, then the
  // proof of work's words
  const size_t pow_off = 16 + 16 * (size_t)n_roots + 4 * ((size_t)1 << last_log);
  const size_t ctl_used = pow_off + (dev_pow ? fri_last_layer_pow_words(pv.cfg.log_last_layer) : 0);
  const size_t ctl_words = up(ctl_used);
  size_t words = ctl_words + tree_words(lifting);
  for (uint32_t lg = lifting - 1;; lg--) {
    words += 4 * up((size_t)1 << lg);
    if (lg > last_log) words += tree_words(lg);
    if (lg == last_log) break;
  }
  uint32_t* block = nullptr;
  GS_TRY(pv.A.alloc_n(words, &block));
  uint32_t* carve = block;
  auto take = [&](size_t w) {
    uint32_t* p = carve;
    carve += up(w);
    return p;
  };
  uint32_t* ctl = take(ctl_words);  // [0,16): channel state; then roots, then challenges
  uint32_t* d_roots = ctl + 16;
  uint32_t* d_felts = d_roots + 8 * (size_t)n_roots;
  auto take_tree = [&](FriLayerDev& L) {
    L.layers.assign(L.log + 1, nullptr);
    for (uint32_t k = 0; k <= L.log; k++) L.layers[k] = take((size_t)8 << k);
  };
  auto take_layer = [&](FriLayerDev& L, uint32_t log) {
    L.log = log;
    for (int c = 0; c < 4; c++) L.planes[c] = take((size_t)1 << log);
    if (log > last_log) take_tree(L);
  };
  {
    uint32_t h[16] = {0};
    for (int j = 0; j < 8; j++) h[j] = host::word(pv.ch.digest, j);
    h[8] = pv.ch.n_draws;
    const void* d = nullptr;
    GS_TRY(pv.ctx.stage_bytes(h, sizeof h, &d));
    GS_CUDA_TRY(cudaMemcpyAsync(ctl, d, sizeof h, cudaMemcpyDeviceToDevice, st));
  }
  // first layer: the quotient columns themselves
  first.log = lifting;
  for (int c = 0; c < 4; c++) first.planes[c] = quot[c];
  take_tree(first);
  {
    std::vector<const uint32_t*> cols = {quot[0], quot[1], quot[2], quot[3]};
    const uint32_t* const* tab = nullptr;
    GS_TRY(pv.table(cols, &tab));
    GS_TRY(commit_on_layer(st, lifting, nullptr, tab, 4, first.layers[lifting]));
  }
  GS_TRY(commit_node_layers_ch(st, first.log, first.layers.data(), pv.ctx.tree_counters, ctl, d_roots, d_felts));
  // fold the circle evaluation into the first line layer (zero-initialised)
  FriLayerDev cur;
  take_layer(cur, lifting - 1);
  for (int c = 0; c < 4; c++) GS_CUDA_TRY(cudaMemsetAsync(cur.planes[c], 0, (size_t)4 << cur.log, st));
  GS_TRY(fold_circle_into_line_dev_alpha(st, CPlanes{{quot[0], quot[1], quot[2], quot[3]}}, lifting, d_felts,
                                         Planes{{cur.planes[0], cur.planes[1], cur.planes[2], cur.planes[3]}},
                                         pv.itw, pv.tw_log, cur.log > last_log ? cur.layers[cur.log] : nullptr));
  uint32_t k = 1;
  while (cur.log > last_log) {
    if (cur.log <= FRI_TAIL_LOG) {
      // every remaining layer in one fused launch
      FriTail ft;
      ft.log0 = cur.log;
      ft.n = cur.log - last_log;
      ft.roots = d_roots + 8 * k;
      ft.felts = d_felts + 8 * k;
      std::vector<FriLayerDev> rest(ft.n + 1);
      rest[0] = std::move(cur);
      for (uint32_t j = 1; j <= ft.n; j++) take_layer(rest[j], rest[0].log - j);
      for (uint32_t j = 0; j <= ft.n; j++) {
        for (int c = 0; c < 4; c++) ft.planes[j][c] = rest[j].planes[c];
        if (j < ft.n)
          for (uint32_t L = 0; L <= rest[j].log; L++) ft.tree[j][L] = rest[j].layers[L];
      }
      GS_TRY(fri_tail(st, ft, ctl, pv.itw, pv.tw_log));
      for (uint32_t j = 0; j < ft.n; j++) inner.push_back(std::move(rest[j]));
      cur = std::move(rest[ft.n]);
      k += ft.n;
      break;
    }
    GS_TRY(commit_node_layers_ch(st, cur.log, cur.layers.data(), pv.ctx.tree_counters, ctl, d_roots + 8 * k,
                                 d_felts + 8 * k));
    FriLayerDev next;
    take_layer(next, cur.log - 1);
    GS_TRY(fold_line_dev_alpha(st, CPlanes{{cur.planes[0], cur.planes[1], cur.planes[2], cur.planes[3]}}, cur.log,
                               d_felts + 8 * k, Planes{{next.planes[0], next.planes[1], next.planes[2], next.planes[3]}},
                               pv.itw, pv.tw_log, next.log > last_log ? next.layers[next.log] : nullptr));
    inner.push_back(std::move(cur));
    cur = std::move(next);
    k++;
  }
  // one read-back through pinned memory: channel state, roots, challenges
  // and the last layer (copied next to them on the device)
  size_t n = (size_t)1 << cur.log;
  uint32_t* d_last = ctl + 16 + 16 * (size_t)n_roots;
  for (int c = 0; c < 4; c++)
    GS_CUDA_TRY(cudaMemcpyAsync(d_last + c * n, cur.planes[c], 4 * n, cudaMemcpyDeviceToDevice, st));
  if (dev_pow) GS_TRY(fri_last_layer_pow(st, d_last, cur.log, pv.cfg.log_last_layer, pv.cfg.pow_bits, ctl, ctl + pow_off));
  std::vector<uint32_t> hc(ctl_used);
  if (while_busy) while_busy();
  GS_TRY(pv.ctx.read_back_published(ctl, hc.size() * 4, hc.data()));
  std::vector<uint32_t> h(hc.begin() + 16 + 16 * (size_t)n_roots, hc.begin() + pow_off);
  GS_REQUIRE(hc[9] == 0, "device channel: no challenge within the draw bound");
  if (dev_pow) {
    for (uint32_t r = 0; r < n_roots; r++) {
      host::Hash root = host::hash_from_words(hc.data() + 16 + 8 * r);
      if (r == 0) first.root = root;
      else inner[r - 1].root = root;
    }
    GS_TRY(last_layer_coeffs(pv, h.data(), cur.log, last_coeffs));
    const size_t nc = (size_t)4 << pv.cfg.log_last_layer;
    const uint32_t* pw = hc.data() + pow_off;
    host::Channel before = pv.ch;
    pv.ch.set(host::hash_from_words(pw + nc));  // the digest after the last layer's mix
    const auto pre = pv.ch.pow_prefixed(pv.cfg.pow_bits);
    for (int j = 0; j < 8; j++)
      if (pw[nc + 8 + j] != pre[j]) {
        set_error("device channel diverged from the host channel (proof-of-work prefix)");
        return ERR_CUDA;
      }
    const uint32_t best = pw[nc + 16];
    if (best == 0xffffffffu) {  // no nonce below 2^20: the search goes on from the next chunk
      GS_TRY(grind_blake2s(st, pre.data(), pv.cfg.pow_bits, (uint32_t*)pv.ctx.d_small, nonce,
                           (uint32_t*)pv.ctx.h_small, 1));
    } else {
      if (!host::pow_passes(pre, best, pv.cfg.pow_bits)) {
        set_error("device grind returned a nonce that does not pass");
        return ERR_CUDA;
      }
      *nonce = best;
    }
    *have_nonce = true;
    *replay = [&pv, &first, &inner, &last_coeffs, before, hc = std::move(hc), n_roots,
               digest = pv.ch.digest]() mutable -> int {
      for (uint32_t r = 0; r < n_roots; r++) {
        before.mix_root(r == 0 ? first.root : inner[r - 1].root);
        const qm31 a = before.draw_felt();
        const uint32_t* f = hc.data() + 16 + 8 * (size_t)n_roots + 8 * r;
        if (!qm_eq(a, qm_make(f[0], f[1], f[2], f[3]))) {
          set_error("device channel diverged from the host channel");
          return ERR_CUDA;
        }
      }
      before.mix_felts(last_coeffs);
      if (before.digest != digest) {
        set_error("device channel diverged from the host channel (last FRI layer)");
        return ERR_CUDA;
      }
      return OK;
    };
    return OK;
  }
  for (uint32_t r = 0; r < n_roots; r++) {
    host::Hash root = host::hash_from_words(hc.data() + 16 + 8 * r);
    pv.ch.mix_root(root);
    qm31 a = pv.ch.draw_felt();
    const uint32_t* f = hc.data() + 16 + 8 * (size_t)n_roots + 8 * r;
    if (!qm_eq(a, qm_make(f[0], f[1], f[2], f[3]))) {
      set_error("device channel diverged from the host channel");
      return ERR_CUDA;
    }
    if (r == 0) first.root = root;
    else inner[r - 1].root = root;
  }
  return finish_last_layer(pv, h.data(), cur.log, last_coeffs);
}

// The last FRI layer (4 planes of 2^log values, host memory) into the line
// polynomial's coefficients: interpolation, degree check, mix into the channel.
static int finish_last_layer(Prover& pv, const uint32_t* h, uint32_t log, std::vector<qm31>& last_coeffs) {
  GS_TRY(last_layer_coeffs(pv, h, log, last_coeffs));
  pv.ch.mix_felts(last_coeffs);
  return OK;
}

// The interpolation and degree check of finish_last_layer, without the mix.
static int last_layer_coeffs(Prover& pv, const uint32_t* h, uint32_t log, std::vector<qm31>& last_coeffs) {
  const size_t n = (size_t)1 << log;
  std::vector<qm31> vals(n);
  for (size_t i = 0; i < n; i++) vals[i] = qm_make(h[i], h[n + i], h[2 * n + i], h[3 * n + i]);
  std::vector<qm31> coeffs = line_interpolate_host(vals, log);
  // into ordered coefficients (bit reverse), keep the degree bound, back
  std::vector<qm31> ordered(n);
  for (size_t i = 0; i < n; i++) ordered[host::bitrev(i, log)] = coeffs[i];
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
  return OK;
}

// compute_decommitment_positions_and_witness_evals (prover/fri.rs:301-330),
// fold step 1: the decommitted positions are both members of each queried
// pair; the witness values are the pair members that were not queried. Fills
// `wit` with the witness positions (and `pos`, when given, with every
// decommitted position) and returns the number of decommitted positions.
size_t fri_witness_positions(const std::vector<size_t>& q, std::vector<size_t>& wit, std::vector<size_t>* pos) {
  // q is sorted and unique. A query starts a pair unless its left neighbour
  // is in the same pair; the witness of a pair is the member that was not
  // queried: q ^ 1 after a starting query, unless q is even and q + 1 follows
  // (both members queried). The flags are computed as integers: for random
  // queries a branch on them mispredicts half the time.
  const size_t n = q.size();
  wit.resize(n);
  size_t n_pos = 0, nw = 0;
  for (size_t i = 0; i < n; i++) {
    const size_t v = q[i];
    const size_t left = i > 0 ? q[i - 1] : ~(size_t)0;
    const size_t right = i + 1 < n ? q[i + 1] : ~(size_t)0;
    const size_t starts = (size_t)(((left ^ v) >> 1) != 0);
    const size_t both = ((v & 1) ^ 1) & (size_t)(right == v + 1);
    wit[nw] = v ^ 1;
    nw += starts & (both ^ 1);
    n_pos += starts << 1;
  }
  wit.resize(nw);
  if (pos) {
    pos->clear();
    for (size_t i = 0; i < n; i++)
      if (i == 0 || ((q[i - 1] ^ q[i]) >> 1) != 0) {
        pos->push_back(q[i] & ~(size_t)1);
        pos->push_back(q[i] | 1);
      }
  }
  return n_pos;
}

int validate_request(const ProveRequest& r) {
  GS_REQUIRE(r.air <= 1, "unknown component");
  GS_REQUIRE(r.merkle_channel <= 1, "merkle channel must be 0 (Blake2s) or 1 (Poseidon252)");
  GS_REQUIRE(r.input_mode <= 2, "unknown input mode");
  GS_REQUIRE(r.input_mode != 2 || r.host_inputs != nullptr, "host inputs required");
  GS_REQUIRE(r.cfg.pow_bits <= 32 && r.cfg.n_queries >= 1 && r.cfg.log_last_layer <= 10, "bad PCS config");
  GS_REQUIRE(r.air != 0 || (r.n_cols >= 3 && r.n_cols <= 160), "wide fibonacci needs 3..160 columns");
  return OK;
}

// The context's proof streams for one proof: entered after the caller's
// stream, left (side work joined, the caller's stream ordered after) when
// the proof returns on any path. Declared before the Prover, so the Prover's
// buffers are released on the work stream first.
struct ProofStreams {
  Context& c;
  bool on = false;
  explicit ProofStreams(Context& x) : c(x) {}
  int begin() {
    GS_TRY(c.begin_proof());
    on = true;
    return OK;
  }
  ~ProofStreams() {
    if (on) c.end_proof();
  }
};

int prove_component(Context& ctx, const ProveRequest& req, std::string* proof_bytes, ProveStats* stats) {
  PcsConfig cfg = req.cfg;
  ProofStreams streams(ctx);
  GS_TRY(streams.begin());
  Prover pv(ctx, cfg);
  GS_REQUIRE(req.merkle_channel <= 1, "merkle channel must be 0 (Blake2s) or 1 (Poseidon252)");
  pv.ch.p252 = req.merkle_channel == 1;
  pv.mark("start");
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
  pv.mark("twiddles");
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
  pv.mark("trace");
  // The trace's extension to the constraint domain (Poseidon2: 2^(T+2), the
  // largest FFT of the proof) depends on no channel draw: it is enqueued on
  // the low-priority side stream as soon as the trace's coefficients exist,
  // and its blocks fill the SMs that the work up to the composition leaves
  // idle (the tails of the trace's own evaluation and hashing, the tree
  // kernel's upper levels, the interaction phase, the host's draws); the
  // composition joins it.
  const uint32_t n_trace = air.n_trace_cols();
  // Wide-Fibonacci: the composition's preparation fills the trace root's wait
  const std::function<int(Tree&)> prep = [&](Tree&) { return pv.prepare_composition(air); };
  GS_TRY(pv.commit_evals(trace, n_trace, T, air.kind == AirKind::WideFibonacci ? prep : nullptr,
                         [&](Tree& t) { return pv.extend(t, E, n_trace, true); }));
  pv.mark("trace_commit");
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
    // the claimed sum stays on the device (the finalize kernel reads it) and
    // comes back through mailbox slot 1 while the interaction is committed
    GS_TRY(poseidon_interaction(st, trace, T, air.lookup, inter, scratch, nullptr));
    GS_TRY(pv.ctx.mail_start(1, logup_claimed_sum_ptr(scratch, T), 16));
    pv.mark("interaction");
    GS_TRY(pv.commit_evals(inter, 4, T, prep, [&](Tree& t) { return pv.extend(t, E, t.n_cols, true); }));
    const void* h = nullptr;
    GS_TRY(pv.ctx.mail_wait(1, &h));
    const uint32_t* cs = (const uint32_t*)h;
    air.claimed_sum = qm_make(cs[0], cs[1], cs[2], cs[3]);
    pv.mark("interaction_commit");
  }
  int rc = prove_tail(pv, air, split, proof_bytes, stats, req.out_buf, req.out_cap);
  pv.mark("end");
  pv.phases.report(pv.A.ptrs.size(), pv.A.n_requests);
  return rc;
}

}  // namespace prover
}  // namespace gs
