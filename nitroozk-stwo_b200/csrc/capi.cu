// C ABI (include/gpustark.h) over the internal launch interface.
#include "../../include/gpustark.h"
#include "runtime.cuh"
#include "air.cuh"
#include "prover/prove_api.h"
#include <cstring>
#include <algorithm>
#include <vector>

struct gs_ctx {
  gs::Context c;
};

using namespace gs;

namespace gs {
void fft_set_columns_aligned(bool aligned);
int fold_line_fused(cudaStream_t st, CPlanes src, uint32_t log_n, qm31 alpha, Planes dst, const uint32_t* d_itw,
                    uint32_t tw_log, uint32_t* leaf_out);
int fold_circle_into_line_fused(cudaStream_t st, CPlanes src, uint32_t log_n, qm31 alpha, Planes dst,
                                const uint32_t* d_itw, uint32_t tw_log, uint32_t* leaf_out);
}

#define CTX_REQUIRED(ctx) GS_REQUIRE((ctx) != nullptr, "null context")

static qm31 to_qm(gs_qm31 v) { return qm_make(v.a, v.b, v.c, v.d); }

extern "C" {

const char* gs_last_error(void) { return last_error(); }

int gs_ctx_create(void* cuda_stream, gs_ctx** out) {
  GS_REQUIRE(out != nullptr, "null output");
  gs_ctx* c = new gs_ctx();
  int s = c->c.init(cuda_stream);
  if (s != OK) {
    c->c.destroy();
    delete c;
    return s;
  }
  *out = c;
  return OK;
}

int gs_ctx_destroy(gs_ctx* ctx) {
  if (!ctx) return OK;
  ctx->c.destroy();
  delete ctx;
  return OK;
}

int gs_ctx_synchronize(gs_ctx* ctx) {
  CTX_REQUIRED(ctx);
  return ctx->c.sync();
}

void* gs_ctx_stream(gs_ctx* ctx) { return ctx ? (void*)ctx->c.stream : nullptr; }

unsigned long long gs_launch_count(void) { return launch_count(); }

int gs_malloc(gs_ctx* ctx, size_t bytes, void** out) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(out != nullptr, "null output");
  cudaError_t e = cudaMallocAsync(out, bytes ? bytes : 16, ctx->c.stream);
  if (e != cudaSuccess) {
    set_error(std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? ERR_OOM : ERR_CUDA;
  }
  return OK;
}

int gs_free(gs_ctx* ctx, void* ptr) {
  CTX_REQUIRED(ctx);
  if (!ptr) return OK;
  GS_CUDA_TRY(cudaFreeAsync(ptr, ctx->c.stream));
  return OK;
}

int gs_memset_zero(gs_ctx* ctx, void* dst, size_t bytes) {
  CTX_REQUIRED(ctx);
  GS_CUDA_TRY(cudaMemsetAsync(dst, 0, bytes, ctx->c.stream));
  return OK;
}

int gs_memcpy_h2d(gs_ctx* ctx, void* dst, const void* src, size_t bytes) {
  CTX_REQUIRED(ctx);
  GS_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->c.stream));
  return OK;
}

int gs_memcpy_d2h(gs_ctx* ctx, void* dst, const void* src, size_t bytes) {
  CTX_REQUIRED(ctx);
  GS_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->c.stream));
  GS_CUDA_TRY(cudaStreamSynchronize(ctx->c.stream));
  return OK;
}

int gs_memcpy_d2d(gs_ctx* ctx, void* dst, const void* src, size_t bytes) {
  CTX_REQUIRED(ctx);
  GS_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx->c.stream));
  return OK;
}

int gs_bit_reverse_base_field(gs_ctx* ctx, uint32_t* col, uint32_t log_size) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(col != nullptr, "null column");
  return bit_reverse(ctx->c.stream, col, log_size);
}

int gs_bit_reverse_secure_field(gs_ctx* ctx, uint32_t* const planes[4], uint32_t log_size) {
  CTX_REQUIRED(ctx);
  for (int i = 0; i < 4; i++) {
    GS_REQUIRE(planes[i] != nullptr, "null plane");
    GS_TRY(bit_reverse(ctx->c.stream, planes[i], log_size));
  }
  return OK;
}

int gs_batch_inverse_base_field(gs_ctx* ctx, const uint32_t* src, uint32_t* dst, size_t n) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(n == 0 || (src && dst), "null buffer");
  return batch_inverse(ctx->c.stream, src, dst, n);
}

int gs_precompute_twiddles(gs_ctx* ctx, uint32_t initial_index, uint32_t step_index, uint32_t log_size,
                           uint32_t* twiddles, uint32_t* itwiddles) {
  CTX_REQUIRED(ctx);
  return precompute_twiddles(ctx->c.stream, initial_index, step_index, log_size, twiddles, itwiddles);
}

int gs_interpolate_columns(gs_ctx* ctx, uint32_t* const* cols, uint32_t n_cols, uint32_t log_size,
                           const uint32_t* itwiddles, uint32_t twiddles_log_size) {
  CTX_REQUIRED(ctx);
  if (n_cols == 0) return OK;
  GS_REQUIRE(cols != nullptr, "null column list");
  for (uint32_t i = 0; i < n_cols; i++) GS_REQUIRE(cols[i] != nullptr, "null column");
  GS_REQUIRE(log_size <= 2 || itwiddles != nullptr, "null itwiddles");
  bool aligned = true;
  for (uint32_t i = 0; i < n_cols; i++) aligned = aligned && (((uintptr_t)cols[i] & 15) == 0);
  fft_set_columns_aligned(aligned);
  const void* const* d = nullptr;
  GS_TRY(ctx->c.stage_ptrs((const void* const*)cols, n_cols, &d));
  return interpolate_columns(ctx->c.stream, (uint32_t* const*)d, n_cols, log_size, itwiddles, twiddles_log_size);
}

int gs_fft_worklist(gs_ctx* ctx, const gs_fft_item* items, uint32_t n_items, const uint32_t* twiddles,
                    const uint32_t* itwiddles, uint32_t twiddles_log_size) {
  CTX_REQUIRED(ctx);
  if (n_items == 0) return OK;
  GS_REQUIRE(items != nullptr, "null item list");
  static_assert(sizeof(gs_fft_item) == sizeof(FftItem) && offsetof(gs_fft_item, log_size) == offsetof(FftItem, log) &&
                    offsetof(gs_fft_item, inverse) == offsetof(FftItem, inverse),
                "gs_fft_item and FftItem differ");
  bool aligned = true;  // the per-size path's vector access, for the items that take it
  for (uint32_t k = 0; k < n_items; k++) {
    const gs_fft_item& x = items[k];
    GS_REQUIRE(x.inverse <= 1, "inverse must be 0 or 1");
    GS_REQUIRE(x.inverse || x.src != x.dst, "an evaluation needs distinct source and destination");
    aligned = aligned && (((uintptr_t)x.src & 15) == 0) && (((uintptr_t)x.dst & 15) == 0);
  }
  fft_set_columns_aligned(aligned);
  // the same fields in the same order (checked above)
  return fft_worklist(ctx->c, reinterpret_cast<const FftItem*>(items), n_items, twiddles, itwiddles, twiddles_log_size);
}

int gs_evaluate_columns(gs_ctx* ctx, const uint32_t* const* coeffs, uint32_t coeffs_log_size, uint32_t* const* evals,
                        uint32_t n_cols, uint32_t log_size, const uint32_t* twiddles, uint32_t twiddles_log_size) {
  CTX_REQUIRED(ctx);
  if (n_cols == 0) return OK;
  GS_REQUIRE(coeffs != nullptr && evals != nullptr, "null column list");
  for (uint32_t i = 0; i < n_cols; i++) GS_REQUIRE(coeffs[i] && evals[i] && coeffs[i] != evals[i], "bad column pair");
  GS_REQUIRE(log_size <= 2 || twiddles != nullptr, "null twiddles");
  bool aligned = true;
  for (uint32_t i = 0; i < n_cols; i++)
    aligned = aligned && (((uintptr_t)coeffs[i] & 15) == 0) && (((uintptr_t)evals[i] & 15) == 0);
  fft_set_columns_aligned(aligned);
  const void* const* ds = nullptr;
  const void* const* dd = nullptr;
  GS_TRY(ctx->c.stage_ptrs((const void* const*)coeffs, n_cols, &ds));
  GS_TRY(ctx->c.stage_ptrs((const void* const*)evals, n_cols, &dd));
  return evaluate_columns(ctx->c.stream, (const uint32_t* const*)ds, coeffs_log_size, (uint32_t* const*)dd, n_cols,
                          log_size, twiddles, twiddles_log_size);
}

int gs_fft_autotune(gs_ctx* ctx, uint32_t min_log, uint32_t max_log, uint32_t max_extension, uint32_t* tile_logs,
                    uint32_t* coalesce_bits) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(min_log >= 3 && min_log <= max_log && max_log <= 27, "autotune range must satisfy 3 <= min <= max <= 27");
  GS_REQUIRE(max_extension <= 3, "extension must be at most 3");
  const uint32_t root = std::min<uint32_t>(max_log + max_extension, 28) - 1;
  const uint32_t* tw = nullptr;
  const uint32_t* itw = nullptr;
  GS_TRY(ctx->c.twiddles(root, &tw, &itw));
  GS_TRY(fft_autotune(ctx->c.stream, min_log, max_log, max_extension, tw, itw, root, tile_logs, coalesce_bits));
  return ctx->c.sync();
}

int gs_fft_set_tuning(uint32_t log_size, uint32_t extension, uint32_t tile_log, uint32_t coalesce_bits) {
  return set_fft_tuning(log_size, extension, tile_log, coalesce_bits);
}

int gs_fft_get_tuning(uint32_t log_size, uint32_t extension, uint32_t* tile_log, uint32_t* coalesce_bits) {
  GS_REQUIRE(log_size < 32 && tile_log && coalesce_bits, "bad arguments");
  get_fft_tuning(log_size, extension, tile_log, coalesce_bits);
  return OK;
}

int gs_commit_on_layer(gs_ctx* ctx, uint32_t log_size, const uint32_t* prev_layer, uint32_t n_cols,
                       const uint32_t* const* cols, uint32_t* out) {
  CTX_REQUIRED(ctx);
  const void* const* d = nullptr;
  if (n_cols) {
    GS_REQUIRE(cols != nullptr, "null column list");
    for (uint32_t i = 0; i < n_cols; i++) GS_REQUIRE(cols[i] != nullptr, "null column");
    GS_TRY(ctx->c.stage_ptrs((const void* const*)cols, n_cols, &d));
  }
  return commit_on_layer(ctx->c.stream, log_size, prev_layer, (const uint32_t* const*)d, n_cols, out);
}

int gs_merkle_worklist(gs_ctx* ctx, const gs_merkle_item* items, uint32_t n_items) {
  CTX_REQUIRED(ctx);
  if (n_items == 0) return OK;
  GS_REQUIRE(items != nullptr, "null tree list");
  static_assert(sizeof(gs_merkle_item) == sizeof(MerkleItem) && offsetof(gs_merkle_item, n_cols) == offsetof(MerkleItem, n_cols) &&
                    offsetof(gs_merkle_item, layers) == offsetof(MerkleItem, layers),
                "gs_merkle_item and MerkleItem differ");
  return merkle_worklist(ctx->c, reinterpret_cast<const MerkleItem*>(items), n_items);
}

int gs_commit_node_layers(gs_ctx* ctx, uint32_t top_log, uint32_t* const* layers) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(layers != nullptr, "null layer list");
  for (uint32_t k = 0; k <= top_log; k++) GS_REQUIRE(layers[k] != nullptr, "null layer buffer");
  return commit_node_layers(ctx->c.stream, top_log, layers, ctx->c.tree_counters);
}

int gs_poseidon252_commit_on_layer(gs_ctx* ctx, uint32_t log_size, const uint8_t* prev_layer, uint32_t n_cols,
                                   const uint32_t* const* cols, uint8_t* out) {
  CTX_REQUIRED(ctx);
  const void* const* d = nullptr;
  if (n_cols) {
    GS_REQUIRE(cols != nullptr, "null column list");
    for (uint32_t i = 0; i < n_cols; i++) GS_REQUIRE(cols[i] != nullptr, "null column");
    GS_TRY(ctx->c.stage_ptrs((const void* const*)cols, n_cols, &d));
  }
  return poseidon252_commit_on_layer(ctx->c.stream, log_size, prev_layer, (const uint32_t* const*)d, n_cols, out);
}

int gs_poseidon252_grind(gs_ctx* ctx, const uint8_t digest[32], uint32_t pow_bits, uint64_t* nonce) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(digest != nullptr && nonce != nullptr, "null digest/nonce");
  const void* d_digest = nullptr;
  GS_TRY(ctx->c.stage_bytes(digest, 32, &d_digest));
  return poseidon252_grind(ctx->c.stream, (const uint8_t*)d_digest, pow_bits, ctx->c.d_small,
                           (uint32_t*)ctx->c.h_small, nonce);
}

int gs_poseidon252_permute(gs_ctx* ctx, const uint8_t* states, uint32_t n, uint8_t* out) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(n == 0 || (states && out), "null state buffer");
  return poseidon252_permute(ctx->c.stream, states, n, out);
}

int gs_fold_line(gs_ctx* ctx, const uint32_t* const src[4], uint32_t log_size, gs_qm31 alpha, uint32_t* const dst[4],
                 const uint32_t* itwiddles, uint32_t twiddles_log_size, uint32_t* leaf_hashes) {
  CTX_REQUIRED(ctx);
  CPlanes s;
  Planes d;
  for (int i = 0; i < 4; i++) {
    GS_REQUIRE(src[i] && dst[i], "null plane");
    GS_REQUIRE(((uintptr_t)src[i] & 7) == 0, "source planes must be 8-byte aligned");
    s.p[i] = src[i];
    d.p[i] = dst[i];
  }
  GS_REQUIRE(itwiddles != nullptr, "null itwiddles");
  return fold_line_fused(ctx->c.stream, s, log_size, to_qm(alpha), d, itwiddles, twiddles_log_size, leaf_hashes);
}

int gs_fold_circle_into_line(gs_ctx* ctx, const uint32_t* const src[4], uint32_t log_size, gs_qm31 alpha,
                             uint32_t* const dst[4], const uint32_t* itwiddles, uint32_t twiddles_log_size,
                             uint32_t* leaf_hashes) {
  CTX_REQUIRED(ctx);
  CPlanes s;
  Planes d;
  for (int i = 0; i < 4; i++) {
    GS_REQUIRE(src[i] && dst[i], "null plane");
    GS_REQUIRE(((uintptr_t)src[i] & 7) == 0, "source planes must be 8-byte aligned");
    s.p[i] = src[i];
    d.p[i] = dst[i];
  }
  GS_REQUIRE(itwiddles != nullptr || log_size < 3, "null itwiddles");
  return fold_circle_into_line_fused(ctx->c.stream, s, log_size, to_qm(alpha), d, itwiddles, twiddles_log_size,
                                     leaf_hashes);
}

int gs_accumulate_numerators(gs_ctx* ctx, uint32_t log_size, const uint32_t* const* cols, uint32_t n_cols,
                             const uint32_t* column_indices, const gs_qm31* line_coeffs_b,
                             const gs_qm31* line_coeffs_c, uint32_t n_coeffs, uint32_t* const out[4]) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(n_coeffs == 0 || (cols && column_indices && line_coeffs_b && line_coeffs_c), "null argument");
  Planes o;
  for (int i = 0; i < 4; i++) {
    GS_REQUIRE(out[i] != nullptr, "null output plane");
    o.p[i] = out[i];
  }
  std::vector<NumEntry> entries(n_coeffs);
  qm31 bsum = qm_zero();
  for (uint32_t k = 0; k < n_coeffs; k++) {
    GS_REQUIRE(column_indices[k] < n_cols && cols[column_indices[k]] != nullptr, "column index out of range");
    entries[k].col = cols[column_indices[k]];
    entries[k].c[0] = line_coeffs_c[k].a; entries[k].c[1] = line_coeffs_c[k].b;
    entries[k].c[2] = line_coeffs_c[k].c; entries[k].c[3] = line_coeffs_c[k].d;
    bsum = qm_add(bsum, to_qm(line_coeffs_b[k]));
  }
  bool vec = true;
  for (auto& e : entries) vec = vec && ((uintptr_t)e.col & 15) == 0;
  for (int i = 0; i < 4; i++) vec = vec && ((uintptr_t)o.p[i] & 15) == 0;
  const void* d = nullptr;
  if (n_coeffs) GS_TRY(ctx->c.stage_bytes(entries.data(), entries.size() * sizeof(NumEntry), &d));
  return accumulate_numerators(ctx->c.stream, d, n_coeffs, bsum, log_size, o, vec);
}

int gs_compute_quotients_and_combine(gs_ctx* ctx, const gs_quotient_acc* accs, uint32_t n_accs,
                                     uint32_t lifting_log_size, uint32_t* const out[4]) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(n_accs == 0 || accs != nullptr, "null accumulations");
  Planes o;
  for (int i = 0; i < 4; i++) {
    GS_REQUIRE(out[i] != nullptr, "null output plane");
    o.p[i] = out[i];
  }
  std::vector<QuotAcc> qa(n_accs);
  for (uint32_t a = 0; a < n_accs; a++) {
    GS_REQUIRE(accs[a].log_size <= lifting_log_size && accs[a].log_size >= 1, "accumulation larger than lifting domain");
    for (int i = 0; i < 4; i++) {
      GS_REQUIRE(accs[a].partial[i] != nullptr, "null partial plane");
      qa[a].p[i] = accs[a].partial[i];
    }
    qa[a].log_size = accs[a].log_size;
    qa[a].pad = 0;
    qa[a].first_linear = to_qm(accs[a].first_linear_term);
    qm31 px = to_qm(accs[a].sample_point.x), py = to_qm(accs[a].sample_point.y);
    qa[a].prx = px.x; qa[a].pix = px.y; qa[a].pry = py.x; qa[a].piy = py.y;
  }
  DomainTables dt;
  GS_TRY(ctx->c.domain_tables(lifting_log_size, &dt));
  const void* d = nullptr;
  if (n_accs) GS_TRY(ctx->c.stage_bytes(qa.data(), qa.size() * sizeof(QuotAcc), &d));
  return compute_quotients_and_combine(ctx->c.stream, d, n_accs, dt, o);
}

int gs_lift_and_accumulate(gs_ctx* ctx, const uint32_t* const* planes, const uint32_t* log_sizes, uint32_t n_cols,
                           uint32_t* const out[4], uint32_t out_log_size) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(n_cols > 0 && planes && log_sizes, "empty accumulation");
  Planes o;
  for (int i = 0; i < 4; i++) {
    GS_REQUIRE(out[i] != nullptr, "null output plane");
    o.p[i] = out[i];
  }
  std::vector<LiftCol> lc(n_cols);
  for (uint32_t c = 0; c < n_cols; c++) {
    GS_REQUIRE(log_sizes[c] >= 1 && log_sizes[c] <= out_log_size, "column larger than the output");
    for (int i = 0; i < 4; i++) {
      GS_REQUIRE(planes[4 * c + i] != nullptr, "null plane");
      lc[c].p[i] = planes[4 * c + i];
    }
    lc[c].log_size = log_sizes[c];
    lc[c].pad = 0;
  }
  const void* d = nullptr;
  GS_TRY(ctx->c.stage_bytes(lc.data(), lc.size() * sizeof(LiftCol), &d));
  return lift_and_accumulate(ctx->c.stream, d, n_cols, out_log_size, o);
}

int gs_accumulate(gs_ctx* ctx, uint32_t* const a[4], const uint32_t* const b[4], size_t n) {
  CTX_REQUIRED(ctx);
  Planes pa;
  CPlanes pb;
  for (int i = 0; i < 4; i++) {
    GS_REQUIRE(a[i] && b[i], "null plane");
    pa.p[i] = a[i];
    pb.p[i] = b[i];
  }
  return accumulate(ctx->c.stream, pa, pb, n);
}

int gs_batch_eval_at_point(gs_ctx* ctx, const uint32_t* const* polys, uint32_t n_polys, uint32_t log_size,
                           gs_point_qm31 point, gs_qm31* out) {
  CTX_REQUIRED(ctx);
  if (n_polys == 0) return OK;
  GS_REQUIRE(polys && out, "null argument");
  for (uint32_t i = 0; i < n_polys; i++) GS_REQUIRE(polys[i] != nullptr, "null polynomial");
  size_t need = eval_at_point_scratch_bytes(n_polys, log_size) + 16 * (size_t)n_polys;
  void* scratch = nullptr;
  GS_TRY(ctx->c.get_scratch(need, &scratch));
  const void* const* d = nullptr;
  GS_TRY(ctx->c.stage_ptrs((const void* const*)polys, n_polys, &d));
  uint32_t* d_out = (uint32_t*)((uint8_t*)scratch + eval_at_point_scratch_bytes(n_polys, log_size));
  ptq p = {to_qm(point.x), to_qm(point.y)};
  bool vec = true;
  for (uint32_t i = 0; i < n_polys; i++) vec = vec && ((uintptr_t)polys[i] & 15) == 0;
  GS_TRY(batch_eval_at_point(ctx->c.stream, (const uint32_t* const*)d, n_polys, log_size, p, d_out, (uint32_t*)scratch,
                             12, vec));
  GS_CUDA_TRY(cudaMemcpyAsync(out, d_out, 16 * (size_t)n_polys, cudaMemcpyDeviceToHost, ctx->c.stream));
  GS_CUDA_TRY(cudaStreamSynchronize(ctx->c.stream));
  return OK;
}

// ------------------------------------------------------ per-trait operations
int gs_batch_gather_multi_uint32(gs_ctx* ctx, const uint32_t* const* cols, uint32_t n_cols, size_t col_len,
                                 const uint32_t* indices, uint32_t n_indices, uint32_t* out) {
  CTX_REQUIRED(ctx);
  if (n_cols == 0 || n_indices == 0) return OK;
  GS_REQUIRE(cols && indices && out, "null argument");
  for (uint32_t c = 0; c < n_cols; c++) GS_REQUIRE(cols[c] != nullptr, "null column");
  for (uint32_t i = 0; i < n_indices; i++) GS_REQUIRE(indices[i] < col_len, "gather index out of range");
  GS_REQUIRE((size_t)n_cols * n_indices <= ((size_t)1 << 30), "gather too large");
  const void* const* d_cols = nullptr;
  const void* d_idx = nullptr;
  GS_TRY(ctx->c.stage_ptrs((const void* const*)cols, n_cols, &d_cols));
  GS_TRY(ctx->c.stage_bytes(indices, 4 * (size_t)n_indices, &d_idx));
  size_t bytes = 4 * (size_t)n_cols * n_indices;
  void* d_out = nullptr;
  GS_TRY(ctx->c.get_scratch(bytes, &d_out));
  GS_TRY(gather_multi(ctx->c.stream, (const uint32_t* const*)d_cols, n_cols, (const uint32_t*)d_idx, n_indices,
                      (uint32_t*)d_out));
  return ctx->c.read_back(d_out, bytes, out);
}

int gs_batch_get_blake2s_hash(gs_ctx* ctx, const uint32_t* layer, size_t n_hashes, const uint32_t* indices,
                              uint32_t n_indices, uint32_t* out) {
  CTX_REQUIRED(ctx);
  if (n_indices == 0) return OK;
  GS_REQUIRE(layer && indices && out, "null argument");
  GS_REQUIRE(((uintptr_t)layer & 15) == 0, "hash layer must be 16-byte aligned");
  for (uint32_t i = 0; i < n_indices; i++) GS_REQUIRE(indices[i] < n_hashes, "hash index out of range");
  const void* d_idx = nullptr;
  GS_TRY(ctx->c.stage_bytes(indices, 4 * (size_t)n_indices, &d_idx));
  size_t bytes = 32 * (size_t)n_indices;
  void* d_out = nullptr;
  GS_TRY(ctx->c.get_scratch(bytes, &d_out));
  GS_TRY(gather_hashes(ctx->c.stream, layer, (const uint32_t*)d_idx, n_indices, (uint32_t*)d_out));
  return ctx->c.read_back(d_out, bytes, out);
}

int gs_barycentric_weights(gs_ctx* ctx, uint32_t log_size, gs_point_qm31 point, uint32_t* const weights[4]) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(log_size >= 2 && log_size <= 30, "log size out of range");
  for (int q = 0; q < 4; q++) GS_REQUIRE(weights[q] != nullptr, "null weight plane");
  DomainTables dt;
  GS_TRY(ctx->c.domain_tables(log_size, &dt));
  ptq p = {to_qm(point.x), to_qm(point.y)};
  return barycentric_weights(ctx->c.stream, dt, p, Planes{{weights[0], weights[1], weights[2], weights[3]}});
}

int gs_barycentric_eval_at_point(gs_ctx* ctx, const uint32_t* evals, const uint32_t* const weights[4],
                                 uint32_t log_size, gs_qm31* out) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(evals && out, "null argument");
  GS_REQUIRE(log_size <= 30, "log size out of range");
  for (int q = 0; q < 4; q++) GS_REQUIRE(weights[q] != nullptr, "null weight plane");
  const size_t n = (size_t)1 << log_size;
  size_t words = barycentric_scratch_words(n) + 4;
  void* scratch = nullptr;
  GS_TRY(ctx->c.get_scratch(4 * words, &scratch));
  uint32_t* d_out = (uint32_t*)scratch + barycentric_scratch_words(n);
  GS_TRY(barycentric_eval(ctx->c.stream, evals, CPlanes{{weights[0], weights[1], weights[2], weights[3]}}, n,
                          (uint32_t*)scratch, d_out));
  uint32_t v[4];
  GS_TRY(ctx->c.read_back(d_out, 16, v));
  *out = gs_qm31{v[0], v[1], v[2], v[3]};
  return OK;
}

int gs_generate_secure_powers(gs_ctx* ctx, gs_qm31 felt, size_t n, uint32_t* const out[4]) {
  CTX_REQUIRED(ctx);
  if (n == 0) return OK;
  for (int q = 0; q < 4; q++) GS_REQUIRE(out[q] != nullptr, "null output plane");
  return secure_powers(ctx->c.stream, to_qm(felt), n, Planes{{out[0], out[1], out[2], out[3]}});
}

int gs_generate_wide_fibonacci_trace(gs_ctx* ctx, const uint32_t* input_a, const uint32_t* input_b,
                                     uint32_t log_size, uint32_t* const* traces, uint32_t n_columns) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(input_a && input_b && traces, "null argument");
  GS_REQUIRE(n_columns >= 2 && n_columns <= 1024 && log_size <= 28, "bad wide fibonacci shape");
  for (uint32_t c = 0; c < n_columns; c++) GS_REQUIRE(traces[c] != nullptr, "null trace column");
  const void* const* d = nullptr;
  GS_TRY(ctx->c.stage_ptrs((const void* const*)traces, n_columns, &d));
  return wf_trace_table(ctx->c.stream, input_a, input_b, log_size, (uint32_t* const*)d, n_columns);
}

int gs_generate_poseidon_traces(gs_ctx* ctx, uint32_t* const* traces, uint32_t* const* lookup_init,
                                uint32_t* const* lookup_final, uint32_t log_size) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(traces && lookup_init && lookup_final, "null argument");
  GS_REQUIRE(log_size <= 28, "log size out of range");
  for (int c = 0; c < 158; c++) GS_REQUIRE(traces[c] != nullptr, "null trace column");
  for (int c = 0; c < 16; c++) GS_REQUIRE(lookup_init[c] && lookup_final[c], "null lookup column");
  const void* const* dt = nullptr;
  const void* const* di = nullptr;
  const void* const* df = nullptr;
  GS_TRY(ctx->c.stage_ptrs((const void* const*)traces, 158, &dt));
  GS_TRY(ctx->c.stage_ptrs((const void* const*)lookup_init, 16, &di));
  GS_TRY(ctx->c.stage_ptrs((const void* const*)lookup_final, 16, &df));
  return poseidon_trace_table(ctx->c.stream, (uint32_t* const*)dt, (uint32_t* const*)di, (uint32_t* const*)df,
                              log_size);
}

int gs_generate_poseidon_interaction_traces(gs_ctx* ctx, const void* lookup_elements,
                                            const uint32_t* const* lookup_init, const uint32_t* const* lookup_final,
                                            uint32_t log_size, uint32_t* const interaction_traces[4],
                                            uint32_t claimed_sum[4]) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(lookup_elements && lookup_init && lookup_final && claimed_sum, "null argument");
  GS_REQUIRE(log_size >= 1 && log_size <= 28, "log size out of range");
  for (int c = 0; c < 16; c++) GS_REQUIRE(lookup_init[c] && lookup_final[c], "null lookup column");
  for (int c = 0; c < 4; c++) GS_REQUIRE(interaction_traces[c] != nullptr, "null interaction column");
  // LookupElements<16> { z, alpha, alpha_powers[16] }, QM31 as 4 words
  LookupParams lp;
  memcpy(lp.z, lookup_elements, 16);
  memcpy(lp.alpha_pow, (const uint8_t*)lookup_elements + 32, 16 * 16);
  const void* const* di = nullptr;
  const void* const* df = nullptr;
  GS_TRY(ctx->c.stage_ptrs((const void* const*)lookup_init, 16, &di));
  GS_TRY(ctx->c.stage_ptrs((const void* const*)lookup_final, 16, &df));
  void* scratch = nullptr;
  GS_TRY(ctx->c.get_scratch(logup_scratch_bytes(log_size), &scratch));
  qm31 cs;
  GS_TRY(poseidon_interaction_table(
      ctx->c.stream, (const uint32_t* const*)di, (const uint32_t* const*)df, log_size, lp,
      Planes{{interaction_traces[0], interaction_traces[1], interaction_traces[2], interaction_traces[3]}},
      scratch, &cs));
  claimed_sum[0] = cs.x.a;
  claimed_sum[1] = cs.x.b;
  claimed_sum[2] = cs.y.a;
  claimed_sum[3] = cs.y.b;
  return OK;
}

// FrameworkEval::cuda_eval_name ids (constraint-framework/src/lib.rs:353-363).
static constexpr uint32_t fnv1a(const char* s) {
  uint32_t h = 0x811C9DC5u;
  while (*s) {
    h ^= (uint8_t)*s++;
    h *= 0x01000193u;
  }
  return h;
}
static constexpr uint32_t EVAL_ID_WIDE_FIBONACCI = fnv1a("fibonacci_example");
static constexpr uint32_t EVAL_ID_POSEIDON = fnv1a("poseidon_example");

int gs_evaluate_constraint_quotients_on_domain(gs_ctx* ctx, uint32_t* const quotients[4],
                                               const uint32_t* const* trace0, uint32_t trace0_len,
                                               const uint32_t* const* trace1, uint32_t trace1_len,
                                               const uint32_t* const* trace2, uint32_t trace2_len,
                                               const gs_qm31* random_coeff_powers,
                                               const uint32_t* denominator_inverses, uint32_t domain_log_size,
                                               uint32_t eval_domain_log_size, uint32_t n_constraints,
                                               uint32_t logup_counts, const void* eval, size_t eval_len,
                                               gs_qm31 cumsum_shift, int should_accumulate) {
  (void)trace0;
  (void)logup_counts;
  CTX_REQUIRED(ctx);
  GS_REQUIRE(eval != nullptr && eval_len >= 12, "eval: eval_id followed by the component's Eval struct");
  for (int q = 0; q < 4; q++) GS_REQUIRE(quotients[q] != nullptr, "null quotient plane");
  GS_REQUIRE(random_coeff_powers && denominator_inverses, "null argument");
  GS_REQUIRE(eval_domain_log_size > domain_log_size && eval_domain_log_size - domain_log_size <= 3 &&
                 eval_domain_log_size <= 30,
             "evaluation domain must be 2 to 8 times the trace domain");
  GS_REQUIRE(trace0_len == 0, "the example components have no preprocessed columns");
  GS_REQUIRE(n_constraints >= 1 && n_constraints <= (uint32_t)MAX_CONSTRAINTS, "constraint count out of range");
  uint32_t w[3];
  memcpy(w, eval, 12);  // eval_id, then the Eval struct: its own eval_id, log_n_rows
  const uint32_t eval_id = w[0], log_n_rows = w[2];
  GS_REQUIRE(log_n_rows == domain_log_size, "Eval.log_n_rows differs from the trace domain");
  ConstraintParams prm;
  memset(&prm, 0, sizeof(prm));
  for (uint32_t k = 0; k < n_constraints; k++) {
    const gs_qm31& p = random_coeff_powers[k];
    prm.powers[4 * k] = p.a;
    prm.powers[4 * k + 1] = p.b;
    prm.powers[4 * k + 2] = p.c;
    prm.powers[4 * k + 3] = p.d;
  }
  for (uint32_t i = 0; i < (1u << (eval_domain_log_size - domain_log_size)); i++)
    prm.denom_inv[i] = denominator_inverses[i];
  Planes out{{quotients[0], quotients[1], quotients[2], quotients[3]}};
  const void* const* d_t1 = nullptr;
  if (eval_id == EVAL_ID_WIDE_FIBONACCI) {
    // WideFibonacciEval { eval_id, log_n_rows } (examples/src/wide_fibonacci/mod.rs:34-37);
    // constraints c_k - (c_{k-2}^2 + c_{k-1}^2), k >= 2
    GS_REQUIRE(eval_domain_log_size == domain_log_size + 1, "wide fibonacci evaluates on the doubled domain");
    GS_REQUIRE(trace1_len == n_constraints + 2 && trace2_len == 0, "wide fibonacci: n_constraints + 2 columns");
    for (uint32_t c = 0; c < trace1_len; c++) GS_REQUIRE(trace1[c] != nullptr, "null trace column");
    GS_TRY(ctx->c.stage_ptrs((const void* const*)trace1, trace1_len, &d_t1));
    return wf_constraints_table(ctx->c.stream, (const uint32_t* const*)d_t1, trace1_len, eval_domain_log_size,
                                domain_log_size, prm, out, should_accumulate != 0);
  }
  if (eval_id == EVAL_ID_POSEIDON) {
    // PoseidonEval { eval_id, log_n_rows, lookup_elements: LookupElements<16> { z, alpha,
    // alpha_powers[16] }, claimed_sum } (examples/src/poseidon/mod.rs:57-64,
    // constraint-framework/src/logup.rs:60-66), all #[repr(C)], QM31 as 4 words
    constexpr size_t QW = 16;
    GS_REQUIRE(eval_len >= 12 + QW * 19, "poseidon: Eval struct too short");
    GS_REQUIRE(eval_domain_log_size == domain_log_size + 2, "poseidon evaluates on the 4x domain");
    GS_REQUIRE(trace1_len == 158 && trace2_len == 4 && n_constraints == 143,
               "poseidon: 158 trace columns, 4 interaction columns, 143 constraints");
    for (uint32_t c = 0; c < trace1_len; c++) GS_REQUIRE(trace1[c] != nullptr, "null trace column");
    for (uint32_t c = 0; c < trace2_len; c++) GS_REQUIRE(trace2[c] != nullptr, "null interaction column");
    const uint8_t* e = (const uint8_t*)eval + 12;
    LookupParams lp;
    memcpy(lp.z, e, QW);
    memcpy(lp.alpha_pow, e + 2 * QW, 16 * QW);
    const void* const* d_t2 = nullptr;
    GS_TRY(ctx->c.stage_ptrs((const void* const*)trace1, trace1_len, &d_t1));
    GS_TRY(ctx->c.stage_ptrs((const void* const*)trace2, trace2_len, &d_t2));
    return poseidon_constraints_table(ctx->c.stream, (const uint32_t* const*)d_t1, (const uint32_t* const*)d_t2,
                                      eval_domain_log_size, domain_log_size, prm, lp, to_qm(cumsum_shift), out,
                                      should_accumulate != 0);
  }
  char msg[96];
  snprintf(msg, sizeof msg, "no device kernel for eval id 0x%08x", eval_id);
  set_error(msg);
  return ERR_UNSUPPORTED;
}

int gs_grind_blake2s(gs_ctx* ctx, const uint32_t prefixed_digest[8], uint32_t pow_bits, uint64_t* nonce) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(prefixed_digest != nullptr, "null digest");
  return grind_blake2s(ctx->c.stream, prefixed_digest, pow_bits, (uint32_t*)ctx->c.d_small, nonce,
                       (uint32_t*)ctx->c.h_small);
}

static int run_prove(gs_ctx* ctx, prover::ProveRequest& req, const gs_pcs_config* config, uint8_t* proof,
                     size_t capacity, size_t* proof_len) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(proof_len != nullptr, "null proof length");
  if (config) {
    req.cfg.pow_bits = config->pow_bits;
    req.cfg.log_blowup = config->log_blowup_factor;
    req.cfg.log_last_layer = config->log_last_layer_degree_bound;
    req.cfg.n_queries = config->n_queries;
    req.cfg.fold_step = config->line_fold_step;
  }
  GS_TRY(prover::validate_request(req));
  // serialised straight into the caller's buffer when it fits; the string
  // (reused per thread) only holds a proof that does not, for its length
  static thread_local std::string bytes;
  req.out_buf = proof;
  req.out_cap = proof ? capacity : 0;
  prover::ProveStats stats;
  int st = prover::prove_component(ctx->c, req, &bytes, &stats);
  *proof_len = stats.proof_len;
  if (st != OK) {
    cudaStreamSynchronize(ctx->c.stream);
    return st;
  }
  if (!stats.in_out_buf) {
    set_error("proof buffer too small");
    return ERR_INVALID;
  }
  return OK;
}

static int prove_wf(gs_ctx* ctx, uint32_t log_n_rows, uint32_t n_columns, uint64_t seed, uint32_t input_mode,
                    const uint32_t* host_inputs, const gs_pcs_config* config, uint8_t* proof, size_t capacity,
                    size_t* proof_len, uint32_t merkle_channel) {
  prover::ProveRequest req;
  req.air = 0;
  req.merkle_channel = merkle_channel;
  req.log_n = log_n_rows;
  req.n_cols = n_columns;
  req.seed = seed;
  req.input_mode = input_mode;
  req.host_inputs = host_inputs;
  req.split_log = 1;
  return run_prove(ctx, req, config, proof, capacity, proof_len);
}

static int prove_p2(gs_ctx* ctx, uint32_t log_n_instances, uint64_t seed, uint32_t input_mode,
                    const uint32_t* host_inputs, uint32_t composition_log_split, const gs_pcs_config* config,
                    uint8_t* proof, size_t capacity, size_t* proof_len, uint32_t merkle_channel) {
  prover::ProveRequest req;
  req.air = 1;
  req.merkle_channel = merkle_channel;
  req.log_n = log_n_instances;
  req.seed = seed;
  req.input_mode = input_mode;
  req.host_inputs = host_inputs;
  req.split_log = composition_log_split;
  return run_prove(ctx, req, config, proof, capacity, proof_len);
}

int gs_prove_wide_fibonacci(gs_ctx* ctx, uint32_t log_n_rows, uint32_t n_columns, uint64_t seed, uint32_t input_mode,
                            const uint32_t* host_inputs, const gs_pcs_config* config, uint8_t* proof,
                            size_t capacity, size_t* proof_len) {
  return prove_wf(ctx, log_n_rows, n_columns, seed, input_mode, host_inputs, config, proof, capacity, proof_len, 0);
}
int gs_prove_wide_fibonacci_poseidon252(gs_ctx* ctx, uint32_t log_n_rows, uint32_t n_columns, uint64_t seed,
                                        uint32_t input_mode, const uint32_t* host_inputs,
                                        const gs_pcs_config* config, uint8_t* proof, size_t capacity,
                                        size_t* proof_len) {
  return prove_wf(ctx, log_n_rows, n_columns, seed, input_mode, host_inputs, config, proof, capacity, proof_len, 1);
}
int gs_prove_poseidon(gs_ctx* ctx, uint32_t log_n_instances, uint64_t seed, uint32_t input_mode,
                      const uint32_t* host_inputs, uint32_t composition_log_split, const gs_pcs_config* config,
                      uint8_t* proof, size_t capacity, size_t* proof_len) {
  return prove_p2(ctx, log_n_instances, seed, input_mode, host_inputs, composition_log_split, config, proof,
                  capacity, proof_len, 0);
}
int gs_prove_poseidon_poseidon252(gs_ctx* ctx, uint32_t log_n_instances, uint64_t seed, uint32_t input_mode,
                                  const uint32_t* host_inputs, uint32_t composition_log_split,
                                  const gs_pcs_config* config, uint8_t* proof, size_t capacity, size_t* proof_len) {
  return prove_p2(ctx, log_n_instances, seed, input_mode, host_inputs, composition_log_split, config, proof,
                  capacity, proof_len, 1);
}

// Poseidon252Channel on the host (no device work): one operation from the
// state (digest, n_draws).
int gs_poseidon252_channel_op(const uint8_t digest[32], uint32_t n_draws, uint32_t op, const uint8_t* bytes,
                              uint64_t value, const uint32_t* words, size_t n, uint32_t* out, uint8_t digest_out[32],
                              uint32_t* n_draws_out) {
  GS_REQUIRE(digest && digest_out && n_draws_out, "null digest");
  GS_REQUIRE(op <= 5 && op != 2, "channel operation must be 0, 1, 3, 4 or 5");
  GS_REQUIRE(op != 0 || bytes, "null root");
  GS_REQUIRE(op != 3 || n == 0 || words, "null words");
  GS_REQUIRE((op != 4 && op != 5) || n == 0 || out, "null output");
  host::Channel ch;
  ch.p252 = true;
  memcpy(ch.digest.data(), digest, 32);
  ch.n_draws = n_draws;
  if (op == 0) {
    host::Hash r;
    memcpy(r.data(), bytes, 32);
    ch.mix_root(r);
  } else if (op == 1) {
    ch.mix_u64(value);
  } else if (op == 3) {
    std::vector<qm31> f(n);
    for (size_t i = 0; i < n; i++) f[i] = qm_make(words[4 * i], words[4 * i + 1], words[4 * i + 2], words[4 * i + 3]);
    ch.mix_felts(f);
  } else if (op == 4) {
    auto f = ch.draw_felts(n);
    for (size_t i = 0; i < n; i++) {
      out[4 * i] = f[i].x.a; out[4 * i + 1] = f[i].x.b; out[4 * i + 2] = f[i].y.a; out[4 * i + 3] = f[i].y.b;
    }
  } else {
    for (size_t i = 0; i < n; i++) ch.draw_words(out + 7 * i);
  }
  memcpy(digest_out, ch.digest.data(), 32);
  *n_draws_out = ch.n_draws;
  return OK;
}

// ------------------------------------------------------------ lifted Merkle
int gs_lifted_build_leaves(gs_ctx* ctx, const uint32_t* const* cols, const uint32_t* log_sizes, uint32_t n_cols,
                           uint32_t lifting_log_size, uint32_t* out) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(out != nullptr && ((uintptr_t)out & 15) == 0, "output must be a 16-byte aligned device buffer");
  GS_REQUIRE(lifting_log_size <= 30, "lifting log size out of range");
  if (n_cols == 0) {  // the hash of nothing
    host::Hash h = host::hash_bytes(nullptr, 0);
    const void* d = nullptr;
    GS_TRY(ctx->c.stage_bytes(h.data(), 32, &d));
    GS_CUDA_TRY(cudaMemcpyAsync(out, d, 32, cudaMemcpyDeviceToDevice, ctx->c.stream));
    return OK;
  }
  GS_REQUIRE(cols && log_sizes, "null argument");
  std::vector<uint32_t> order(n_cols);
  for (uint32_t i = 0; i < n_cols; i++) {
    GS_REQUIRE(cols[i] != nullptr, "null column");
    GS_REQUIRE(log_sizes[i] >= 1 && log_sizes[i] <= lifting_log_size, "column log size must be in [1, lifting]");
    order[i] = i;
  }
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return log_sizes[a] < log_sizes[b]; });
  std::vector<const void*> ptrs(n_cols);
  std::vector<uint8_t> shifts(n_cols);
  for (uint32_t k = 0; k < n_cols; k++) {
    ptrs[k] = cols[order[k]];
    shifts[k] = (uint8_t)(lifting_log_size - log_sizes[order[k]]);
  }
  const void* const* d_cols = nullptr;
  const void* d_shifts = nullptr;
  GS_TRY(ctx->c.stage_ptrs(ptrs.data(), n_cols, &d_cols));
  GS_TRY(ctx->c.stage_bytes(shifts.data(), n_cols, &d_shifts));
  return lifted_leaves(ctx->c.stream, lifting_log_size, (const uint32_t* const*)d_cols, (const uint8_t*)d_shifts,
                       n_cols, out);
}

// ------------------------------------------------------------ commit plans
struct gs_commit_plan {
  prover::CommitPlan* p;
  gs_ctx* ctx;
};

int gs_commit_plan_create(gs_ctx* ctx, const uint32_t* log_sizes, uint32_t n_columns, uint32_t log_blowup,
                          uint32_t use_graph, gs_commit_plan** out) {
  CTX_REQUIRED(ctx);
  GS_REQUIRE(log_sizes && out, "null argument");
  prover::CommitPlan* p = nullptr;
  GS_TRY(prover::plan_create(ctx->c, log_sizes, n_columns, log_blowup, use_graph != 0, &p));
  *out = new gs_commit_plan{p, ctx};
  return OK;
}

int gs_commit_plan_run(gs_commit_plan* plan, const uint32_t* const* columns, uint32_t root[8]) {
  GS_REQUIRE(plan && columns && root, "null argument");
  return prover::plan_run(plan->p, columns, root);
}

int gs_commit_plan_extended(gs_commit_plan* plan, uint32_t column, const uint32_t** evals) {
  GS_REQUIRE(plan && evals, "null argument");
  return prover::plan_extended(plan->p, column, evals);
}

int gs_commit_plan_layer(gs_commit_plan* plan, uint32_t log_size, const uint32_t** layer) {
  GS_REQUIRE(plan && layer, "null argument");
  return prover::plan_layer(plan->p, log_size, layer);
}

int gs_commit_plan_destroy(gs_commit_plan* plan) {
  if (!plan) return OK;
  prover::plan_destroy(plan->p);
  delete plan;
  return OK;
}

}  // extern "C"
