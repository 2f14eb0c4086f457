// Batched commitment of columns of mixed sizes: TreeBuilder::extend_evals +
// commit (crates/stwo/src/prover/pcs/mod.rs:388-430) followed by
// MerkleProver::commit (crates/stwo/src/prover/vcs/prover.rs:39-62).
//
// A plan fixes the shape (the columns' log sizes and the blowup) and owns every
// buffer: coefficients, extended evaluations and Merkle layers. One run
//   1. interpolates each size group's columns (one launch per pass per group),
//   2. evaluates them on the blown-up domain (one launch per pass per group),
//   3. commits every column in one Merkle tree: columns sorted by size
//      (stable), each size group hashed into the layer of its size together
//      with the two children from the layer above, node-only layers between,
//   4. reads the root back.
// With `use_graph`, steps 1-3 are captured once into a CUDA graph on the
// plan's own stream and replayed on later runs; the input pointers live in a
// device table that each run rewrites before the replay, so one graph serves
// any inputs of the same shape.
#include <algorithm>
#include <map>
#include <memory>
#include "../../../include/gpustark.h"
#include "prover_impl.h"

namespace gs {
void fft_set_columns_aligned(bool aligned);
namespace prover {

struct CommitPlan {
  Context* ctx = nullptr;
  cudaStream_t st = nullptr;  // the plan's own stream (graph capture needs one)
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  uint32_t n_cols = 0, blowup = 0, max_eval = 0;
  std::vector<uint32_t> log_sizes;
  // size groups in decreasing log size; members keep their input order
  struct Group {
    uint32_t log = 0;
    std::vector<uint32_t> cols;         // input indices
    uint32_t* coeffs = nullptr;         // contiguous, column stride `stride_c`
    uint32_t* evals = nullptr;          // contiguous, column stride `stride_e`
    size_t stride_c = 0, stride_e = 0;
    const uint32_t* const* d_src = nullptr;  // into d_src_table
    uint32_t* const* d_coeffs = nullptr;
    uint32_t* const* d_evals = nullptr;
  };
  std::vector<Group> groups;
  std::vector<uint32_t*> layers;        // layers[L]: 2^L hashes
  uint32_t* counters = nullptr;         // Merkle tree kernel tickets (in `block`)
  void* block = nullptr;                // one device allocation for everything
  const void** d_src_table = nullptr;   // input pointers in group order (rewritten per run)
  const uint32_t* tw = nullptr;
  const uint32_t* itw = nullptr;
  uint32_t tw_log = 0;
  bool use_graph = false;
  cudaGraphExec_t graph = nullptr;
  bool graph_aligned = true;            // input alignment the graph was captured with

  int enqueue(bool inputs_aligned);
  int run(const uint32_t* const* inputs, uint32_t root[8]);
  void destroy();
};

static size_t up64(size_t w) { return (w + 63) & ~(size_t)63; }

int CommitPlan::enqueue(bool inputs_aligned) {
  // 1-2. interpolate each group out of place, then extend it
  for (auto& g : groups) {
    fft_set_columns_aligned(inputs_aligned);
    GS_TRY(interpolate_columns_to(st, g.d_src, g.d_coeffs, (uint32_t)g.cols.size(), g.log, itw, tw_log));
    fft_set_columns_aligned(true);
    GS_TRY(evaluate_columns(st, (const uint32_t* const*)g.d_coeffs, g.log, g.d_evals, (uint32_t)g.cols.size(),
                            g.log + blowup, tw, tw_log));
  }
  // 3. Merkle tree, from the largest layer down
  uint32_t L = max_eval;
  size_t gi = 0;
  for (;;) {
    const Group* inj = (gi < groups.size() && groups[gi].log + blowup == L) ? &groups[gi] : nullptr;
    if (inj) gi++;
    const uint32_t* prev = L == max_eval ? nullptr : layers[L + 1];
    if (inj || L == max_eval) {
      GS_TRY(commit_on_layer(st, L, prev, inj ? (const uint32_t* const*)inj->d_evals : nullptr,
                             inj ? (uint32_t)inj->cols.size() : 0, layers[L]));
      if (L == 0) break;
      L--;
      continue;
    }
    // node-only layers down to the next injected size (or the root)
    uint32_t stop = gi < groups.size() ? groups[gi].log + blowup : 0;  // next injected layer
    if (stop == 0) {
      GS_TRY(commit_node_layers(st, L + 1, layers.data(), counters));
      break;
    }
    while (L > stop) {
      GS_TRY(commit_on_layer(st, L, layers[L + 1], nullptr, 0, layers[L]));
      L--;
    }
  }
  fft_set_columns_aligned(true);
  return OK;
}

int CommitPlan::run(const uint32_t* const* inputs, uint32_t root[8]) {
  bool aligned = true;
  for (uint32_t i = 0; i < n_cols; i++) {
    GS_REQUIRE(inputs[i] != nullptr, "null input column");
    aligned = aligned && ((uintptr_t)inputs[i] & 15) == 0;
  }
  // the input pointers in group order, then the work, ordered after the
  // caller's stream
  std::vector<const void*> ordered;
  ordered.reserve(n_cols);
  for (auto& g : groups)
    for (uint32_t i : g.cols) ordered.push_back(inputs[i]);
  const void* staged = nullptr;
  GS_TRY(ctx->stage_bytes(ordered.data(), n_cols * sizeof(void*), &staged));
  GS_CUDA_TRY(
      cudaMemcpyAsync(d_src_table, staged, n_cols * sizeof(void*), cudaMemcpyDeviceToDevice, ctx->stream));
  GS_CUDA_TRY(cudaEventRecord(ev_in, ctx->stream));
  GS_CUDA_TRY(cudaStreamWaitEvent(st, ev_in, 0));
  if (use_graph && graph && graph_aligned == aligned) {
    GS_CUDA_TRY(cudaGraphLaunch(graph, st));
    note_launch();
  } else if (use_graph && !graph) {
    cudaGraph_t g = nullptr;
    GS_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue(aligned);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    GS_CUDA_TRY(e);
    e = cudaGraphInstantiate(&graph, g, 0);
    cudaGraphDestroy(g);
    GS_CUDA_TRY(e);
    graph_aligned = aligned;
    GS_CUDA_TRY(cudaGraphLaunch(graph, st));
    note_launch();
  } else {
    GS_TRY(enqueue(aligned));
  }
  GS_CUDA_TRY(cudaEventRecord(ev_out, st));
  GS_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ev_out, 0));
  return ctx->read_back(layers[0], 32, root);
}

void CommitPlan::destroy() {
  if (st) cudaStreamSynchronize(st);
  if (graph) cudaGraphExecDestroy(graph);
  if (block) cudaFree(block);
  if (ev_in) cudaEventDestroy(ev_in);
  if (ev_out) cudaEventDestroy(ev_out);
  if (st) cudaStreamDestroy(st);
  graph = nullptr;
  block = nullptr;
  ev_in = ev_out = nullptr;
  st = nullptr;
}

int plan_create(Context& ctx, const uint32_t* log_sizes, uint32_t n, uint32_t blowup, bool use_graph,
                CommitPlan** out) {
  GS_REQUIRE(n >= 1 && n <= (1u << 20), "column count out of range");
  GS_REQUIRE(blowup <= 4, "log blowup out of range");
  auto p = std::make_unique<CommitPlan>();
  p->ctx = &ctx;
  p->n_cols = n;
  p->blowup = blowup;
  p->use_graph = use_graph;
  p->log_sizes.assign(log_sizes, log_sizes + n);
  std::map<uint32_t, std::vector<uint32_t>, std::greater<uint32_t>> by_log;
  for (uint32_t i = 0; i < n; i++) {
    GS_REQUIRE(log_sizes[i] >= 1 && log_sizes[i] + blowup <= 28, "column log size out of range");
    by_log[log_sizes[i]].push_back(i);
  }
  p->max_eval = by_log.begin()->first + blowup;
  GS_REQUIRE(p->max_eval >= 2, "the largest extended column needs at least 4 rows");
  for (auto& [lg, cols] : by_log) {
    GS_REQUIRE(cols.size() <= 65535, "too many columns of one size");
    CommitPlan::Group g;
    g.log = lg;
    g.cols = cols;
    g.stride_c = up64((size_t)1 << lg);
    g.stride_e = up64((size_t)1 << (lg + blowup));
    p->groups.push_back(g);
  }
  // one device block: pointer tables, coefficients, evaluations, layers
  size_t words = 3 * up64(2 * (size_t)n);  // src / coeff / eval tables (8 bytes per pointer)
  for (auto& g : p->groups) words += g.cols.size() * (g.stride_c + g.stride_e);
  for (uint32_t L = 0; L <= p->max_eval; L++) words += up64((size_t)8 << L);
  words += up64(TREE_COUNTERS);  // the tree kernel's tickets, owned by the plan's stream
  GS_CUDA_TRY(cudaMalloc(&p->block, words * 4));
  uint32_t* carve = (uint32_t*)p->block;
  auto take = [&](size_t w) { uint32_t* q = carve; carve += up64(w); return q; };
  uint32_t* t_src = take(2 * (size_t)n);
  uint32_t* t_coef = take(2 * (size_t)n);
  uint32_t* t_eval = take(2 * (size_t)n);
  p->d_src_table = (const void**)t_src;
  std::vector<const void*> h_src, h_coef, h_eval;  // host images of the tables
  for (auto& g : p->groups) {
    g.coeffs = take(g.cols.size() * g.stride_c);
    g.evals = take(g.cols.size() * g.stride_e);
    // the group's slice of the source table, written at each run
    g.d_src = (const uint32_t* const*)((const void**)t_src + h_src.size());
    g.d_coeffs = (uint32_t* const*)((const void**)t_coef + h_coef.size());
    g.d_evals = (uint32_t* const*)((const void**)t_eval + h_eval.size());
    for (size_t k = 0; k < g.cols.size(); k++) {
      h_src.push_back(nullptr);
      h_coef.push_back(g.coeffs + k * g.stride_c);
      h_eval.push_back(g.evals + k * g.stride_e);
    }
  }
  p->layers.resize(p->max_eval + 1);
  for (uint32_t L = 0; L <= p->max_eval; L++) p->layers[L] = take((size_t)8 << L);
  p->counters = take(TREE_COUNTERS);
  GS_CUDA_TRY(cudaMemcpy(t_coef, h_coef.data(), h_coef.size() * sizeof(void*), cudaMemcpyHostToDevice));
  GS_CUDA_TRY(cudaMemcpy(t_eval, h_eval.data(), h_eval.size() * sizeof(void*), cudaMemcpyHostToDevice));
  p->tw_log = p->max_eval - 1;
  GS_TRY(ctx.twiddles(p->tw_log, &p->tw, &p->itw));
  GS_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
  GS_CUDA_TRY(cudaStreamCreateWithFlags(&p->st, cudaStreamNonBlocking));
  GS_CUDA_TRY(cudaMemsetAsync(p->counters, 0, 4 * TREE_COUNTERS, p->st));  // ordered before every run
  GS_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_in, cudaEventDisableTiming));
  GS_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_out, cudaEventDisableTiming));
  *out = p.release();
  return OK;
}

int plan_run(CommitPlan* p, const uint32_t* const* inputs, uint32_t root[8]) { return p->run(inputs, root); }

int plan_extended(CommitPlan* p, uint32_t column, const uint32_t** out) {
  GS_REQUIRE(column < p->n_cols, "column index out of range");
  for (auto& g : p->groups)
    for (size_t k = 0; k < g.cols.size(); k++)
      if (g.cols[k] == column) {
        *out = g.evals + k * g.stride_e;
        return OK;
      }
  set_error("column not found");
  return ERR_INVALID;
}

int plan_layer(CommitPlan* p, uint32_t log_size, const uint32_t** out) {
  GS_REQUIRE(log_size <= p->max_eval, "layer log size out of range");
  *out = p->layers[log_size];
  return OK;
}

void plan_destroy(CommitPlan* p) {
  if (!p) return;
  p->destroy();
  delete p;
}

}  // namespace prover
}  // namespace gs
