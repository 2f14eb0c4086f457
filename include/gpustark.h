/*
 * gpustark — C ABI of the B200 Circle-STARK proving backend.
 *
 * Every entry point mirrors one operation of the reference's CUDA FFI
 * (crates/stwo/src/stwo_cuda/bindings.rs) or one backend-trait method of the
 * reference prover; the citation next to each declaration names the
 * reference interface it replaces. Differences from the reference ABI, all
 * deliberate:
 *   - every call takes an execution context (one CUDA stream) and returns a
 *     status code instead of calling exit(); gs_last_error() explains a
 *     non-zero status (thread-local);
 *   - column lists are HOST arrays of DEVICE pointers (the library stages
 *     them), QM31 columns are 4 device coordinate planes;
 *   - work is stream-ordered on the context's stream; only the calls that
 *     return host values (roots, nonces, proofs) synchronise. A whole proof
 *     (gs_prove_*) runs on two streams of the context's own, a high-priority
 *     one and a low-priority one for work the protocol needs only later,
 *     entered after the context's stream and left with the context's stream
 *     ordered after them, so callers see the same ordering.
 * Field values are canonical M31 words (< 2^31 - 1). Hashes are 32 bytes
 * (8 little-endian uint32 words) and hash buffers must be 16-byte aligned.
 */
#ifndef GPUSTARK_H
#define GPUSTARK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GS_OK 0
#define GS_ERR_INVALID 1
#define GS_ERR_CUDA 2
#define GS_ERR_OOM 3
#define GS_ERR_UNSUPPORTED 4
#define GS_ERR_PROOF 5
#define GS_ERR_TIMEOUT 6

typedef struct gs_ctx gs_ctx;

/* CudaSecureField (bindings.rs:9-15): QM31 (a + b i) + (c + d i) u. */
typedef struct { uint32_t a, b, c, d; } gs_qm31;
/* CirclePointSecureField (bindings.rs:68-80). */
typedef struct { gs_qm31 x, y; } gs_point_qm31;

/* ---------------------------------------------------------------- context */
const char* gs_last_error(void);
/* cuda_stream: the cudaStream_t all work of this context is ordered on;
 * NULL is CUDA's default (legacy) stream. */
int gs_ctx_create(void* cuda_stream, gs_ctx** out);
int gs_ctx_destroy(gs_ctx* ctx);
int gs_ctx_synchronize(gs_ctx* ctx);
void* gs_ctx_stream(gs_ctx* ctx);
/* Number of kernels this library has launched in this process (no reference
 * counterpart; used to account device launches in benchmarks). */
unsigned long long gs_launch_count(void);

/* ----------------------------------------------------------------- memory
 * cuda_malloc_uint32_t / cuda_alloc_zeroes_uint32_t / cuda_free_memory /
 * copy_uint32_t_vec_from_host_to_device / ..._device_to_host
 * (bindings.rs:84-131). Allocation is stream ordered (memory pool). */
int gs_malloc(gs_ctx* ctx, size_t bytes, void** out);
int gs_free(gs_ctx* ctx, void* ptr);
int gs_memset_zero(gs_ctx* ctx, void* dst, size_t bytes);
int gs_memcpy_h2d(gs_ctx* ctx, void* dst, const void* src, size_t bytes);
int gs_memcpy_d2h(gs_ctx* ctx, void* dst, const void* src, size_t bytes); /* synchronises */
int gs_memcpy_d2d(gs_ctx* ctx, void* dst, const void* src, size_t bytes);

/* -------------------------------------------------------------- ColumnOps */
/* bit_reverse_base_field (bindings.rs:133); ColumnOps::bit_reverse_column. */
int gs_bit_reverse_base_field(gs_ctx* ctx, uint32_t* col, uint32_t log_size);
/* bit_reverse_secure_field (bindings.rs:135). */
int gs_bit_reverse_secure_field(gs_ctx* ctx, uint32_t* const planes[4], uint32_t log_size);
/* batch_inverse_base_field (bindings.rs:137). */
int gs_batch_inverse_base_field(gs_ctx* ctx, const uint32_t* src, uint32_t* dst, size_t n);

/* ---------------------------------------------------------------- PolyOps */
/* precompute_twiddles (bindings.rs:165) + batch_inverse: twiddle tree of the
 * coset (initial_index, step_index, log_size) given as circle indices; writes
 * 2^log_size twiddles and, if itwiddles != NULL, their inverses.
 * PolyOps::precompute_twiddles (prover/poly/circle/ops.rs:123). */
int gs_precompute_twiddles(gs_ctx* ctx, uint32_t initial_index, uint32_t step_index, uint32_t log_size,
                           uint32_t* twiddles, uint32_t* itwiddles);
/* ntt_b2n_column (bindings.rs:503-510); PolyOps::interpolate_columns
 * (ops.rs:28-39): in place, bit-reversed evaluations on CanonicCoset(log_size)
 * -> coefficients. The twiddle tree is that of half_odds(twiddles_log_size). */
int gs_interpolate_columns(gs_ctx* ctx, uint32_t* const* cols, uint32_t n_cols, uint32_t log_size,
                           const uint32_t* itwiddles, uint32_t twiddles_log_size);
/* ntt_n2b_columns (bindings.rs:512-519); PolyOps::evaluate_polynomials /
 * extend + evaluate (ops.rs:88-120): 2^coeffs_log_size coefficients per
 * column -> bit-reversed evaluations on CanonicCoset(log_size), written to
 * evals (distinct buffers of 2^log_size words). */
int gs_evaluate_columns(gs_ctx* ctx, const uint32_t* const* coeffs, uint32_t coeffs_log_size, uint32_t* const* evals,
                        uint32_t n_cols, uint32_t log_size, const uint32_t* twiddles, uint32_t twiddles_log_size);
/* Batched FFTs of uneven sizes (the reference launches ntt_b2n_column /
 * ntt_n2b_columns once per size group, cuda/poly.rs:179-294, 409-552; this
 * entry has no single reference counterpart): item k interpolates
 * (inverse = 1) the 2^log_size bit-reversed evaluations at src into
 * coefficients at dst (src == dst: in place), or evaluates (inverse = 0) the
 * 2^coeffs_log_size coefficients at src on CanonicCoset(log_size) into dst
 * (distinct buffers). Every item of log size 3..13 runs in ONE launch of a
 * persistent grid that walks the list, largest first, each FFT whole in
 * shared memory; other sizes take the per-size path of gs_interpolate_columns
 * / gs_evaluate_columns. Results equal those entries' bit for bit. Items must
 * not overlap one another. itwiddles / twiddles: the trees of
 * half_odds(twiddles_log_size), twiddles_log_size + 1 >= every log_size;
 * itwiddles may be NULL when no item interpolates, twiddles when no item
 * evaluates. */
typedef struct {
  const uint32_t* src;
  uint32_t* dst;
  uint32_t log_size, coeffs_log_size, inverse, reserved;
} gs_fft_item;
int gs_fft_worklist(gs_ctx* ctx, const gs_fft_item* items, uint32_t n_items, const uint32_t* twiddles,
                    const uint32_t* itwiddles, uint32_t twiddles_log_size);

/* FFT pass-split tuning. No counterpart in the reference, whose CUDA FFT
 * (ntt.cu) has one fixed geometry. An FFT that computes n layers runs in
 * passes over shared-memory tiles of 2^tile_log words, 2^coalesce_bits of
 * them contiguous in memory; the split changes speed only, never the values.
 * A split is kept per (n, extension): extension 0 for an FFT of 2^n points, e
 * for an LDE of 2^n coefficients onto 2^(n+e) points (e >= 3 share one).
 * gs_fft_autotune times every split candidate for each n in [min_log,
 * max_log] (3 <= min_log <= max_log <= 27) and extension in [0,
 * max_extension] (<= 3) on scratch columns (2^max(24, max_log) output words;
 * larger LDEs keep their split) and installs the fastest for all contexts of
 * the process; tile_logs / coalesce_bits, when non-NULL, receive the choices,
 * (max_log - min_log + 1) x (max_extension + 1) entries by log size. Both
 * set-up calls: no other FFT may be in flight. gs_fft_set_tuning installs one
 * split (log_size 0: every size; extension > 3: every extension; tile_log in
 * [6, 13], coalesce_bits <= min(5, tile_log - 5)); gs_fft_get_tuning reads
 * it. Default: 13 / 4. */
int gs_fft_autotune(gs_ctx* ctx, uint32_t min_log, uint32_t max_log, uint32_t max_extension, uint32_t* tile_logs,
                    uint32_t* coalesce_bits);
int gs_fft_set_tuning(uint32_t log_size, uint32_t extension, uint32_t tile_log, uint32_t coalesce_bits);
int gs_fft_get_tuning(uint32_t log_size, uint32_t extension, uint32_t* tile_log, uint32_t* coalesce_bits);

/* -------------------------------------------------------------- MerkleOps */
/* commit_on_first_layer / commit_on_layer_with_previous (bindings.rs:262-275);
 * MerkleOps<Blake2sMerkleHasher>::commit_on_layer (prover/vcs/ops.rs:24-28).
 * prev_layer: 2^(log_size+1) hashes or NULL; out: 2^log_size hashes. */
int gs_commit_on_layer(gs_ctx* ctx, uint32_t log_size, const uint32_t* prev_layer, uint32_t n_cols,
                       const uint32_t* const* cols, uint32_t* out);

/* poseidon252_commit_on_first_layer / poseidon252_commit_on_layer_with_previous
 * (bindings.rs:592-612); MerkleOps<Poseidon252MerkleHasher>::commit_on_layer
 * (prover/backend/cuda/poseidon252.rs:21-42; hash_node at core/vcs/
 * poseidon252_merkle.rs:18-72). Hashes are felt252 values in the reference's
 * device layout, 32 bytes big-endian each (stwo_cuda/poseidon252.rs);
 * prev_layer: 2^(log_size+1) hashes or NULL; out: 2^log_size hashes; both
 * 16-byte aligned. The hash is Starknet's Poseidon (starknet-crypto 0.6.2). */
int gs_poseidon252_commit_on_layer(gs_ctx* ctx, uint32_t log_size, const uint8_t* prev_layer, uint32_t n_cols,
                                   const uint32_t* const* cols, uint8_t* out);
/* poseidon_permute_comp (starknet-crypto 0.6.2, called by core/channel/
 * poseidon252.rs:37-45) on n states of 3 felt252 values, 96 bytes each in
 * the same big-endian layout; in and out may not overlap. No counterpart in
 * the reference's C ABI (it exposes no raw permutation). */
int gs_poseidon252_permute(gs_ctx* ctx, const uint8_t* states, uint32_t n, uint8_t* out);
/* GrindOps<Poseidon252Channel>::grind (prover/backend/simd/grind.rs:152-190;
 * the reference's CUDA backend delegates it to that CPU code, prover/backend/
 * cuda/backend.rs:52-56): the smallest nonce (hi << 32) | low, low < 2^14,
 * hi = 0, 1, ..., such that poseidon_hash(poseidon_hash_many([0x12345678,
 * digest, pow_bits]), nonce) has pow_bits trailing zero bits in its low 128
 * bits. digest: the channel's felt252 digest, 32 bytes big-endian (host
 * memory). Synchronises. */
int gs_poseidon252_grind(gs_ctx* ctx, const uint8_t digest[32], uint32_t pow_bits, uint64_t* nonce);

/* The node-only part of MerkleProver::commit's layer loop (prover/vcs/
 * prover.rs:39-48) when no columns are injected below top_log: layers is a
 * host array of top_log + 1 device buffers, layers[L] holding 2^L hashes;
 * layers[top_log] is the input, all smaller layers are written. */
int gs_commit_node_layers(gs_ctx* ctx, uint32_t top_log, uint32_t* const* layers);
/* Whole Merkle trees of uneven sizes, many at once (the reference commits one
 * tree at a time through commit_on_first_layer / commit_on_layer_with_previous,
 * bindings.rs:262-275, driven by MerkleProver::commit, prover/vcs/prover.rs:
 * 39-48; this entry has no single reference counterpart). Tree k hashes its
 * n_cols >= 1 columns of 2^log_size words into the leaf layer and every node
 * layer above it: cols and layers are host arrays of device pointers,
 * layers[L] holding 2^L hashes (16-byte aligned) for L = 0..log_size. Every
 * tree of log size <= 10 is built in ONE launch of a persistent grid that
 * walks the list, largest first, each tree in one block through shared
 * memory; larger trees take gs_commit_on_layer + gs_commit_node_layers.
 * Results equal those entries' byte for byte. Trees must not share layers. */
typedef struct {
  const uint32_t* const* cols;
  uint32_t n_cols, log_size;
  uint32_t* const* layers;
} gs_merkle_item;
int gs_merkle_worklist(gs_ctx* ctx, const gs_merkle_item* items, uint32_t n_items);

/* MerkleOpsLifted::build_leaves (prover/vcs_lifted/ops.rs:8-18; CPU
 * prover/backend/cpu/merkle_lifted.rs:12-77; reference CUDA blake2s.cu:
 * 210-452): the leaves of a lifted Merkle commitment. Columns (any order;
 * sorted here by increasing size, stably) are bit-reversed evaluations of
 * log size in [1, lifting_log_size]; leaf i hashes each column's value at
 * ((i >> (lifting_log_size - log + 1)) << 1) + (i & 1). out: 2^lifting_log_size
 * hashes, or one hash (of nothing) when n_cols == 0. build_next_layer is
 * gs_commit_node_layers. */
int gs_lifted_build_leaves(gs_ctx* ctx, const uint32_t* const* cols, const uint32_t* log_sizes, uint32_t n_cols,
                           uint32_t lifting_log_size, uint32_t* out);

/* ---------------------------------------------------------------- FriOps */
/* fold_line (bindings.rs:196-203); FriOps::fold_line (prover/fri.rs:39-44),
 * fold_step 1: line evaluation on half_odds(log_size) -> 2^(log_size-1).
 * leaf_hashes: optional (NULL) output of the next layer's Merkle leaves. */
int gs_fold_line(gs_ctx* ctx, const uint32_t* const src[4], uint32_t log_size, gs_qm31 alpha, uint32_t* const dst[4],
                 const uint32_t* itwiddles, uint32_t twiddles_log_size, uint32_t* leaf_hashes);
/* fold_circle_into_line (bindings.rs:205-212); FriOps::fold_circle_into_line
 * (prover/fri.rs:61-66): dst = dst * alpha^2 + fold(src), src on
 * CanonicCoset(log_size), dst of size 2^(log_size-1). */
int gs_fold_circle_into_line(gs_ctx* ctx, const uint32_t* const src[4], uint32_t log_size, gs_qm31 alpha,
                             uint32_t* const dst[4], const uint32_t* itwiddles, uint32_t twiddles_log_size,
                             uint32_t* leaf_hashes);

/* ------------------------------------------------------------ QuotientOps */
/* accumulate_numerators_batch (bindings.rs:354-365); QuotientOps::
 * accumulate_numerators (prover/pcs/quotient_ops.rs:27-31) for one sample
 * batch: out[row] = sum_k c_k * cols[column_indices[k]][row] - sum_k b_k over
 * columns of 2^log_size rows; b/c are the batch's line coefficients (host). */
int gs_accumulate_numerators(gs_ctx* ctx, uint32_t log_size, const uint32_t* const* cols, uint32_t n_cols,
                             const uint32_t* column_indices, const gs_qm31* line_coeffs_b,
                             const gs_qm31* line_coeffs_c, uint32_t n_coeffs, uint32_t* const out[4]);

/* One accumulated numerator per sample point (AccumulatedNumerators,
 * prover/pcs/quotient_ops.rs:33-37). */
typedef struct {
  const uint32_t* partial[4]; /* 2^log_size QM31 planes (device) */
  uint32_t log_size;
  gs_qm31 first_linear_term;
  gs_point_qm31 sample_point;
} gs_quotient_acc;
/* compute_quotients_and_combine (bindings.rs:367-381); QuotientOps::
 * compute_quotients_and_combine (quotient_ops.rs:39-42): writes the combined
 * quotient on the bit-reversed CanonicCoset(lifting_log_size). */
int gs_compute_quotients_and_combine(gs_ctx* ctx, const gs_quotient_acc* accs, uint32_t n_accs,
                                     uint32_t lifting_log_size, uint32_t* const out[4]);

/* -------------------------------------------------------- AccumulationOps */
/* lift_and_accumulate (bindings.rs:216-221); AccumulationOps::
 * lift_and_accumulate (prover/air/accumulation.rs:127-145): columns in
 * increasing size; planes[4c + k] is coordinate k of column c. out has
 * 2^out_log_size rows, out_log_size = the largest column's log size. */
int gs_lift_and_accumulate(gs_ctx* ctx, const uint32_t* const* planes, const uint32_t* log_sizes, uint32_t n_cols,
                           uint32_t* const out[4], uint32_t out_log_size);
/* accumulate (bindings.rs:214); AccumulationOps::accumulate: a += b. */
int gs_accumulate(gs_ctx* ctx, uint32_t* const a[4], const uint32_t* const b[4], size_t n);

/* ----------------------------------------------------- out-of-domain eval */
/* batch_eval_at_points (bindings.rs:187-194); PolyOps::batch_eval_at_point
 * (ops.rs:51-59): values of n_polys coefficient polynomials of 2^log_size
 * coefficients at `point`, written to host memory. Synchronises. */
int gs_batch_eval_at_point(gs_ctx* ctx, const uint32_t* const* polys, uint32_t n_polys, uint32_t log_size,
                           gs_point_qm31 point, gs_qm31* out);
/* No counterpart in the reference. The same evaluation as
 * gs_batch_eval_at_point, results identical, but allocating nothing: no
 * context, no cudaMalloc/cudaFree, no pinned staging. Its device scratch is
 * one file-scope __device__ array of 4 MiB + 22 KiB per device, whose address
 * is looked up with cudaGetSymbolAddress on the first call under each CUDA
 * context (with the device's primary context, the usual case, once per
 * device; make that first call before any stream capture) and cached per
 * context. Limits, checked before
 * any launch (ERR_INVALID otherwise): n_polys <= 256 and
 * n_polys * 2^max(log_size - 10, 0) <= 2^18. Runs on `stream` (a
 * cudaStream_t; NULL = the default stream) and synchronises it. Calls that
 * overlap in time on one device race on the shared array: serialise them. */
int gs_batch_eval_at_point_noalloc(void* stream, const uint32_t* const* polys, uint32_t n_polys, uint32_t log_size,
                                   gs_point_qm31 point, gs_qm31* out);

/* ------------------------------------------------- column gathers (decommit) */
/* cuda_batch_gather_multi_uint32 (bindings.rs:314-320); Column::
 * batch_at_multi (prover/backend/mod.rs:73-89; CUDA prover/backend/cuda/
 * column.rs:198): the values of n_cols device columns (each at least col_len
 * words) at n_indices positions, written to host memory row-major:
 * out[i * n_cols + c] = cols[c][indices[i]]. Indices >= col_len are rejected
 * (ERR_INVALID) before any device work. Synchronises. */
int gs_batch_gather_multi_uint32(gs_ctx* ctx, const uint32_t* const* cols, uint32_t n_cols, size_t col_len,
                                 const uint32_t* indices, uint32_t n_indices, uint32_t* out);
/* cuda_batch_get_blake_2s_hash (bindings.rs:300-305); Column<Blake2sHash>::
 * batch_at for MerkleProver::decommit (prover/vcs/prover.rs:84-217): hashes of
 * one device layer of n_hashes (16-byte aligned) at the indices, 8 words
 * each, written to host memory. Synchronises. */
int gs_batch_get_blake2s_hash(gs_ctx* ctx, const uint32_t* layer, size_t n_hashes, const uint32_t* indices,
                              uint32_t n_indices, uint32_t* out);

/* ---------------------------------------------------- barycentric OODS */
/* barycentric_weights_cuda (bindings.rs:141-151); PolyOps::
 * barycentric_weights (prover/poly/circle/ops.rs:64-68; CPU prover/backend/
 * cpu/circle.rs:101-132): the weights of CanonicCoset(log_size) at `point`,
 * 2^log_size QM31 values in bit-reversed domain order, written to 4 device
 * planes. The point must not lie on the domain. */
int gs_barycentric_weights(gs_ctx* ctx, uint32_t log_size, gs_point_qm31 point, uint32_t* const weights[4]);
/* barycentric_eval_at_point_cuda (bindings.rs:153-158); PolyOps::
 * barycentric_eval_at_point (ops.rs:73-77; cpu/circle.rs:134-141): the sum of
 * evals[i] * weights[i] over 2^log_size bit-reversed evaluations (device), to
 * host memory. Synchronises. */
int gs_barycentric_eval_at_point(gs_ctx* ctx, const uint32_t* evals, const uint32_t* const weights[4],
                                 uint32_t log_size, gs_qm31* out);

/* ---------------------------------------------- example trace generation */
/* generate_wide_fibonacci_trace (bindings.rs:426-433; CUDA
 * evaluate_wide_fibonacci.cu:127-179): trace[0] = input_a, trace[1] =
 * input_b, trace[k] = trace[k-2]^2 + trace[k-1]^2 over 2^log_size rows;
 * inputs and the n_columns trace columns are device buffers. */
int gs_generate_wide_fibonacci_trace(gs_ctx* ctx, const uint32_t* input_a, const uint32_t* input_b,
                                     uint32_t log_size, uint32_t* const* traces, uint32_t n_columns);
/* generate_poseidon_traces (bindings.rs:435-440; CUDA
 * evaluate_poseidon_constraint.cu:270-363): the 158 Poseidon2 trace columns
 * of 2^log_size rows with the reference's inputs (row r, lane i: r + i), and
 * the 16 initial- and final-state columns the lookup uses (device). */
int gs_generate_poseidon_traces(gs_ctx* ctx, uint32_t* const* traces, uint32_t* const* lookup_init,
                                uint32_t* const* lookup_final, uint32_t log_size);
/* generate_poseidon_interaction_traces (bindings.rs:442-449; CUDA
 * evaluate_poseidon_constraint.cu:365-600; semantics crates/examples/src/
 * poseidon/mod.rs:305-335): the logup interaction column (4 device planes,
 * the shifted prefix sum in coset order) of the fractions 1/combine(init) -
 * 1/combine(final), and the claimed sum (4 words, host memory; the
 * reference writes it to device memory). lookup_elements: the #[repr(C)]
 * LookupElements<16> { z, alpha, alpha_powers[16] }, QM31 as 4 words.
 * Synchronises. */
int gs_generate_poseidon_interaction_traces(gs_ctx* ctx, const void* lookup_elements,
                                            const uint32_t* const* lookup_init, const uint32_t* const* lookup_final,
                                            uint32_t log_size, uint32_t* const interaction_traces[4],
                                            uint32_t claimed_sum[4]);

/* ------------------------------------------------- constraint accumulation */
/* AccumulationOps::generate_secure_powers (prover/air/accumulation.rs:127-145;
 * the reference's CUDA backend computes it on the host, prover/backend/cuda/
 * accumulation.rs:20-22): out[i] = felt^i for i < n, 4 device planes. */
int gs_generate_secure_powers(gs_ctx* ctx, gs_qm31 felt, size_t n, uint32_t* const out[4]);
/* evaluate_constraint_quotients_on_domain (bindings.rs:469-490), called by
 * ComponentProver<CudaBackend>::evaluate_constraint_quotients_on_domain
 * (constraint-framework/src/prover/component_prover.rs:249-498): per row of
 * the evaluation domain, sum_k random_coeff_powers[k] * C_k(row) times
 * denominator_inverses[row >> domain_log_size], written to (or, with
 * should_accumulate, added to) the 4 quotient planes. trace0/1/2: host arrays
 * of device columns on the evaluation domain (preprocessed, trace,
 * interaction); random_coeff_powers: n_constraints QM31 values in the order
 * the constraints are added (the reversed accumulator powers) and
 * denominator_inverses: 2^(eval_domain_log_size - domain_log_size) words,
 * both HOST arrays (the reference uploads them first). eval: the buffer the
 * reference's ComponentProver builds, eval_id (FNV-1a of
 * FrameworkEval::cuda_eval_name) followed by the component's #[repr(C)] Eval
 * struct, eval_len bytes. Supported ids: "fibonacci_example" (WideFibonacciEval,
 * trace1 = n_constraints + 2 columns) and "poseidon_example" (PoseidonEval,
 * 158 trace and 4 interaction columns, 143 constraints); any other id
 * returns GS_ERR_UNSUPPORTED (the reference returns false and falls back to
 * the CPU; this library has no CPU path). cumsum_shift = claimed_sum /
 * 2^domain_log_size; logup_counts is accepted and unused. */
int gs_evaluate_constraint_quotients_on_domain(gs_ctx* ctx, uint32_t* const quotients[4],
                                               const uint32_t* const* trace0, uint32_t trace0_len,
                                               const uint32_t* const* trace1, uint32_t trace1_len,
                                               const uint32_t* const* trace2, uint32_t trace2_len,
                                               const gs_qm31* random_coeff_powers,
                                               const uint32_t* denominator_inverses, uint32_t domain_log_size,
                                               uint32_t eval_domain_log_size, uint32_t n_constraints,
                                               uint32_t logup_counts, const void* eval, size_t eval_len,
                                               gs_qm31 cumsum_shift, int should_accumulate);

/* --------------------------------------------------------------- GrindOps */
/* grind_blake2s (bindings.rs:615); GrindOps<Blake2sChannel>::grind
 * (core/proof_of_work.rs): prefixed_digest = H(POW_PREFIX, 0^12, digest,
 * pow_bits) as 8 LE words; returns the smallest valid nonce. Synchronises. */
int gs_grind_blake2s(gs_ctx* ctx, const uint32_t prefixed_digest[8], uint32_t pow_bits, uint64_t* nonce);

/* ------------------------------------------------------------------ prove */
/* PcsConfig (core/pcs/mod.rs:31-36) with FriConfig (core/fri.rs:32-37);
 * lifting_log_size is None. line_fold_step must be 1 (as the reference's CUDA
 * FRI, prover/backend/cuda/fri.rs:23). */
typedef struct {
  uint32_t pow_bits;
  uint32_t log_blowup_factor;
  uint32_t log_last_layer_degree_bound;
  uint32_t n_queries;
  uint32_t line_fold_step;
} gs_pcs_config;

/* Input rule of a proof's trace: the reference examples' inputs, seeded
 * uniform M31, or columns supplied by the caller from host memory. */
#define GS_INPUT_REFERENCE 0
#define GS_INPUT_SEEDED 1
#define GS_INPUT_HOST 2

/* cuda_prove_wide_fibonacci (crates/examples/src/wide_fibonacci/mod.rs:140-184)
 * driving prove() (crates/stwo/src/prover/mod.rs:28-150): 2^log_n_rows rows
 * of n_columns. GS_INPUT_HOST: host_inputs holds columns 0 and 1 (2 x 2^log
 * words). Writes the serialised StarkProof to proof (capacity bytes); returns
 * GS_ERR_PROOF when the composition sanity check fails, GS_ERR_INVALID with
 * *proof_len set when the buffer is too small. Synchronises. */
int gs_prove_wide_fibonacci(gs_ctx* ctx, uint32_t log_n_rows, uint32_t n_columns, uint64_t seed, uint32_t input_mode,
                            const uint32_t* host_inputs, const gs_pcs_config* config, uint8_t* proof,
                            size_t capacity, size_t* proof_len);
/* cuda_prove_poseidon (crates/examples/src/poseidon/mod.rs:617-700): one
 * Poseidon2 instance per row, 2^log_n_instances rows. GS_INPUT_HOST:
 * host_inputs holds the 16 initial-state columns (16 x 2^log words).
 * composition_log_split = 1 is the reference's fixed split of the composition
 * polynomial (core/verifier.rs:17), with which the reference's own prove()
 * returns ConstraintsNotSatisfied for this component (LOG_EXPAND = 2);
 * composition_log_split = 2 splits it into 4 parts so every committed tree has
 * the trace's size, which yields a consistent proof. */
int gs_prove_poseidon(gs_ctx* ctx, uint32_t log_n_instances, uint64_t seed, uint32_t input_mode,
                      const uint32_t* host_inputs, uint32_t composition_log_split, const gs_pcs_config* config,
                      uint8_t* proof, size_t capacity, size_t* proof_len);

/* The same two proofs over Poseidon252MerkleChannel: every Merkle tree hashed
 * with Poseidon252MerkleHasher, the Fiat-Shamir transcript a
 * Poseidon252Channel, the proof of work GrindOps<Poseidon252Channel>.
 * cuda_prove_wide_fibonacci_poseidon (crates/examples/src/wide_fibonacci/
 * mod.rs:335-379) and cuda_prove_poseidon_poseidon (crates/examples/src/
 * poseidon/mod.rs:702-785). Arguments as above; hashes in the proof are the
 * felt252 values as 32 big-endian bytes. */
int gs_prove_wide_fibonacci_poseidon252(gs_ctx* ctx, uint32_t log_n_rows, uint32_t n_columns, uint64_t seed,
                                        uint32_t input_mode, const uint32_t* host_inputs,
                                        const gs_pcs_config* config, uint8_t* proof, size_t capacity,
                                        size_t* proof_len);
int gs_prove_poseidon_poseidon252(gs_ctx* ctx, uint32_t log_n_instances, uint64_t seed, uint32_t input_mode,
                                  const uint32_t* host_inputs, uint32_t composition_log_split,
                                  const gs_pcs_config* config, uint8_t* proof, size_t capacity, size_t* proof_len);

/* Poseidon252Channel (core/channel/poseidon252.rs:18-155) on the host, the
 * channel the Poseidon252 proofs use; no context and no device work. From
 * the state (digest as 32 big-endian bytes, n_draws), op 0: mix_root(bytes,
 * 32 bytes; Poseidon252MerkleChannel::mix_root), 1: mix_u64(value), 3:
 * mix_felts(n QM31 values, 4n words), 4: draw_secure_felts(n) into out (4n
 * words), 5: draw_u32s n times into out (7n words). Writes the new state. */
int gs_poseidon252_channel_op(const uint8_t digest[32], uint32_t n_draws, uint32_t op, const uint8_t* bytes,
                              uint64_t value, const uint32_t* words, size_t n, uint32_t* out, uint8_t digest_out[32],
                              uint32_t* n_draws_out);

/* ------------------------------------------------------------- serving */
/* A proof server (no reference counterpart: the reference proves one proof at
 * a time on the default stream). n_workers threads, each with its own CUDA
 * stream, prove queued jobs concurrently; a job is admitted when the
 * estimated device footprint of the jobs in flight plus its own fits
 * hbm_budget_bytes. Jobs use seeded inputs (GS_INPUT_SEEDED); air 0 = wide
 * fibonacci (n_columns), 1 = poseidon2 (composition_log_split as in
 * gs_prove_poseidon). gs_server_wait blocks until the job is done, copies its
 * proof and reports the submit-to-done latency. */
typedef struct gs_server gs_server;
int gs_server_create(uint32_t n_workers, size_t hbm_budget_bytes, gs_server** out);
/* The same server with n_threads host threads, each driving
 * fibers_per_thread proofs at once as cooperative fibers (one CUDA stream
 * and context per fiber): a proof's wait on its stream yields to the other
 * proofs of its thread instead of blocking it, so a few threads keep many
 * proofs' launches queued. Results and admission are as above;
 * gs_server_create(n, b) is gs_server_create_fibers(n, 1, b). */
int gs_server_create_fibers(uint32_t n_threads, uint32_t fibers_per_thread, size_t hbm_budget_bytes,
                            gs_server** out);
int gs_server_submit(gs_server* server, uint32_t air, uint32_t log_n, uint32_t n_columns, uint64_t seed,
                     uint32_t composition_log_split, const gs_pcs_config* config, uint64_t* job_id);
/* The same job proved over Poseidon252MerkleChannel (as
 * gs_prove_wide_fibonacci_poseidon252 / gs_prove_poseidon_poseidon252). */
int gs_server_submit_poseidon252(gs_server* server, uint32_t air, uint32_t log_n, uint32_t n_columns, uint64_t seed,
                                 uint32_t composition_log_split, const gs_pcs_config* config, uint64_t* job_id);
int gs_server_wait(gs_server* server, uint64_t job_id, uint8_t* proof, size_t capacity, size_t* proof_len,
                   double* latency_ms);
int gs_server_destroy(gs_server* server);

/* ------------------------------------------------ batched commitment plans */
/* TreeBuilder::extend_evals + commit (prover/pcs/mod.rs:388-430) followed by
 * MerkleProver::commit (prover/vcs/prover.rs:39-62) for columns of mixed
 * sizes, batched: a plan fixes the shape (log sizes, blowup) and owns every
 * buffer. gs_commit_plan_run interpolates each size group (one launch per FFT
 * pass per group), evaluates it on CanonicCoset(log + log_blowup), and commits
 * all columns in one Merkle tree (columns sorted by size, stable; each size
 * injected at its layer), then writes the 8-word root to host memory.
 * Inputs: device pointers to bit-reversed evaluations on CanonicCoset(log).
 * use_graph != 0: the first run captures the work into a CUDA graph on the
 * plan's own stream and later runs replay it (the input pointers may change
 * between runs; a change of their 16-byte alignment runs the work eagerly).
 * The extended columns and every Merkle layer stay readable until the next
 * run (gs_commit_plan_extended, gs_commit_plan_layer). Synchronises. */
typedef struct gs_commit_plan gs_commit_plan;
int gs_commit_plan_create(gs_ctx* ctx, const uint32_t* log_sizes, uint32_t n_columns, uint32_t log_blowup,
                          uint32_t use_graph, gs_commit_plan** out);
int gs_commit_plan_run(gs_commit_plan* plan, const uint32_t* const* columns, uint32_t root[8]);
int gs_commit_plan_extended(gs_commit_plan* plan, uint32_t column, const uint32_t** evals);
int gs_commit_plan_layer(gs_commit_plan* plan, uint32_t log_size, const uint32_t** layer);
int gs_commit_plan_destroy(gs_commit_plan* plan);

#ifdef __cplusplus
}
#endif
#endif /* GPUSTARK_H */
