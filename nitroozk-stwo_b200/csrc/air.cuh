// Parameters and launch interface of the AIR kernels (air.cu).
#pragma once
#include "runtime.cuh"

namespace gs {

constexpr int MAX_CONSTRAINTS = 160;

// Random-coefficient powers in the order the constraints are added
// (powers[4k..4k+3] = alpha^(n-1-k), the reversed powers of
// DomainEvaluationAccumulator::columns) and the bit-reversed denominator
// inverses 1 / vanishing(trace coset, eval_domain.at(i)), i < 2^(eval-trace).
struct ConstraintParams {
  uint32_t powers[4 * MAX_CONSTRAINTS];
  uint32_t denom_inv[8];
};

// LookupElements<16>: alpha^i (i < 16) and z, as QM31 words.
struct LookupParams {
  uint32_t alpha_pow[64];
  uint32_t z[4];
};

int wf_trace(cudaStream_t st, uint32_t* cols, uint32_t log_n, uint32_t n_cols, uint64_t seed, uint32_t mode);
int wf_constraints(cudaStream_t st, const uint32_t* cols, uint32_t n_cols, uint32_t eval_log, uint32_t trace_log,
                   const ConstraintParams& prm, Planes out);
// The same kernels over columns given by a device table of pointers (the C
// ABI's evaluate_constraint_quotients_on_domain); accumulate: add to the
// output planes instead of writing them.
int wf_constraints_table(cudaStream_t st, const uint32_t* const* d_cols, uint32_t n_cols, uint32_t eval_log,
                         uint32_t trace_log, const ConstraintParams& prm, Planes out, bool accumulate);
int poseidon_constraints_table(cudaStream_t st, const uint32_t* const* d_trace, const uint32_t* const* d_inter,
                               uint32_t eval_log, uint32_t trace_log, const ConstraintParams& prm,
                               const LookupParams& lp, qm31 cumsum_shift, Planes out, bool accumulate);
// The trace kernels of the C ABI (the reference's generate_* bindings):
// columns, initial and final lookup states as device pointer tables.
int wf_trace_table(cudaStream_t st, const uint32_t* in_a, const uint32_t* in_b, uint32_t log_n,
                   uint32_t* const* d_cols, uint32_t n_cols);
int poseidon_trace_table(cudaStream_t st, uint32_t* const* d_cols, uint32_t* const* d_init, uint32_t* const* d_final,
                         uint32_t log_n);
int poseidon_interaction_table(cudaStream_t st, const uint32_t* const* d_init, const uint32_t* const* d_final,
                               uint32_t log_n, const LookupParams& lp, Planes out, void* scratch,
                               qm31* claimed_sum);
int poseidon_trace(cudaStream_t st, uint32_t* cols, uint32_t log_n, uint64_t seed, uint32_t mode);
size_t logup_scratch_bytes(uint32_t log_n);
// Device address of the claimed sum (one QM31 as 4 words) inside the scratch
// of an interaction computed with claimed_sum = null.
const void* logup_claimed_sum_ptr(const void* scratch, uint32_t log_n);
int poseidon_interaction(cudaStream_t st, const uint32_t* trace, uint32_t log_n, const LookupParams& lp,
                         uint32_t* out, void* scratch, qm31* claimed_sum, void* h_pinned = nullptr);
int poseidon_constraints(cudaStream_t st, const uint32_t* trace, const uint32_t* inter, uint32_t eval_log,
                         uint32_t trace_log, const ConstraintParams& prm, const LookupParams& lp, qm31 cumsum_shift,
                         Planes out);

// gather.cu: hash witnesses as runs read from one Merkle layer each; item k
// of a run is hash idx[first + k] of its layer, written to output hash
// out + k (runs may share index ranges).
struct HashRun {
  const uint32_t* src;
  uint32_t first, count;
  uint32_t out, pad;
};
int gather_hash_runs(cudaStream_t st, const HashRun* d_runs, uint32_t n_runs, const uint32_t* d_idx,
                     uint32_t* d_out);
// Values of n_cols columns at a list of positions, written position-major
// (for each position, every column): columns given explicitly (n_cols <= 4)
// or as base + c * stride.
struct ColGather {
  const uint32_t* cols[4];
  const uint32_t* base;
  uint64_t stride;
  uint32_t n_cols, n_pos;
  uint64_t pos_off;  // first position in the shared position list
  uint64_t out_off;  // first output word
};
int gather_cols(cudaStream_t st, const ColGather* d_blocks, uint32_t n_blocks, uint32_t max_items,
                const uint32_t* d_positions, uint32_t* d_out);
// Both gathers in one launch: the column values to d_words, the hashes to
// d_hashes (16-byte aligned). The outputs may be mapped host memory.
int gather_all(cudaStream_t st, const ColGather* d_blocks, uint32_t n_blocks, uint32_t max_items,
               const uint32_t* d_positions, uint32_t* d_words, const HashRun* d_runs, uint32_t n_runs,
               const uint32_t* d_idx, uint32_t* d_hashes);

}  // namespace gs
