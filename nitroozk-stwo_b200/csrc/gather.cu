// Decommitment gathers (Column::batch_at / batch_at_multi, crates/stwo/src/
// prover/backend/mod.rs:70-86; reference CUDA cuda_batch_gather_multi_uint32,
// cuda_batch_get_blake_2s_hash): one launch fetches every value and hash a
// decommitment needs, listed as (buffer, index) items.
#include "air.cuh"

namespace gs {

// One block per run: the run's witnesses are spread over its threads, each
// copying one 32-byte hash as two 16-byte vectors.
__global__ void gather_hash_runs_kernel(const HashRun* __restrict__ runs, const uint32_t* __restrict__ idx,
                                        uint32_t* __restrict__ out) {
  const HashRun r = runs[blockIdx.x];
  for (uint32_t k = threadIdx.x; k < r.count; k += blockDim.x) {
    const uint4* s = reinterpret_cast<const uint4*>(r.src + 8 * (size_t)__ldg(idx + (size_t)r.first + k));
    uint4* o = reinterpret_cast<uint4*>(out + 8 * ((size_t)r.out + k));
    o[0] = __ldg(s);
    o[1] = __ldg(s + 1);
  }
}

// grid.y = descriptor, grid.x covers its n_pos * n_cols outputs.
__global__ void gather_cols_kernel(const ColGather* __restrict__ blocks, const uint32_t* __restrict__ positions,
                                   uint32_t* __restrict__ out) {
  const ColGather b = blocks[blockIdx.y];
  const uint32_t n = b.n_pos * b.n_cols;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const uint32_t p = t / b.n_cols, c = t - p * b.n_cols;
    const uint32_t* src = b.n_cols <= 4 ? b.cols[c] : b.base + c * b.stride;
    out[b.out_off + t] = __ldg(src + positions[b.pos_off + p]);
  }
}

int gather_cols(cudaStream_t st, const ColGather* d_blocks, uint32_t n_blocks, uint32_t max_items,
                const uint32_t* d_positions, uint32_t* d_out) {
  if (n_blocks == 0 || max_items == 0) return OK;
  GS_REQUIRE(n_blocks <= 65535, "too many gather descriptors");
  dim3 grid((max_items + 255) / 256 < 64 ? (max_items + 255) / 256 : 64, n_blocks);
  gather_cols_kernel<<<grid, 256, 0, st>>>(d_blocks, d_positions, d_out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

int gather_hash_runs(cudaStream_t st, const HashRun* d_runs, uint32_t n_runs, const uint32_t* d_idx,
                     uint32_t* d_out) {
  if (n_runs == 0) return OK;
  GS_REQUIRE(((uintptr_t)d_out & 15) == 0, "hash gather output must be 16-byte aligned");
  gather_hash_runs_kernel<<<n_runs, 128, 0, st>>>(d_runs, d_idx, d_out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

// The two gathers above in one grid: blocks [0, n_blocks * X) take the
// column descriptors (X blocks each), the rest one hash run each.
__global__ void __launch_bounds__(256) gather_all_kernel(const ColGather* __restrict__ blocks, uint32_t n_blocks,
                                                         uint32_t X, const uint32_t* __restrict__ positions,
                                                         uint32_t* words, const HashRun* __restrict__ runs,
                                                         const uint32_t* __restrict__ idx, uint32_t* hashes) {
  const uint32_t bid = blockIdx.x;
  if (bid < n_blocks * X) {
    const ColGather b = blocks[bid / X];
    const uint32_t n = b.n_pos * b.n_cols;
    for (uint32_t t = (bid % X) * blockDim.x + threadIdx.x; t < n; t += X * blockDim.x) {
      const uint32_t p = t / b.n_cols, c = t - p * b.n_cols;
      const uint32_t* src = b.n_cols <= 4 ? b.cols[c] : b.base + c * b.stride;
      words[b.out_off + t] = __ldg(src + positions[b.pos_off + p]);
    }
    return;
  }
  const HashRun r = runs[bid - n_blocks * X];
  for (uint32_t k = threadIdx.x; k < r.count; k += blockDim.x) {
    const uint4* s = reinterpret_cast<const uint4*>(r.src + 8 * (size_t)__ldg(idx + (size_t)r.first + k));
    uint4* o = reinterpret_cast<uint4*>(hashes + 8 * ((size_t)r.out + k));
    o[0] = __ldg(s);
    o[1] = __ldg(s + 1);
  }
}

int gather_all(cudaStream_t st, const ColGather* d_blocks, uint32_t n_blocks, uint32_t max_items,
               const uint32_t* d_positions, uint32_t* d_words, const HashRun* d_runs, uint32_t n_runs,
               const uint32_t* d_idx, uint32_t* d_hashes) {
  if (max_items == 0) n_blocks = 0;
  const uint32_t X = n_blocks ? ((max_items + 255) / 256 < 64 ? (max_items + 255) / 256 : 64) : 0;
  const uint64_t grid = (uint64_t)n_blocks * X + n_runs;
  if (grid == 0) return OK;
  GS_REQUIRE(grid <= 0x7fffffffu, "too many gather blocks");
  GS_REQUIRE(n_runs == 0 || ((uintptr_t)d_hashes & 15) == 0, "hash gather output must be 16-byte aligned");
  gather_all_kernel<<<(unsigned)grid, 256, 0, st>>>(d_blocks, n_blocks, X, d_positions, d_words, d_runs, d_idx,
                                                    d_hashes);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

// Column::batch_at_multi (crates/stwo/src/prover/backend/mod.rs:73-89):
// out[i * n_cols + c] = cols[c][idx[i]], row-major over the indices.
__global__ void gather_multi_kernel(const uint32_t* const* __restrict__ cols, uint32_t n_cols,
                                    const uint32_t* __restrict__ idx, uint32_t n_idx, uint32_t* __restrict__ out) {
  const size_t total = (size_t)n_cols * n_idx;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    uint32_t i = (uint32_t)(t / n_cols), c = (uint32_t)(t - (size_t)i * n_cols);
    out[t] = __ldg(cols[c] + __ldg(idx + i));
  }
}

// Hashes of one Merkle layer at a list of indices, 32 bytes each.
__global__ void gather_hashes_kernel(const uint4* __restrict__ layer, const uint32_t* __restrict__ idx, uint32_t n_idx,
                                     uint4* __restrict__ out) {
  const size_t total = 2 * (size_t)n_idx;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x)
    out[t] = __ldg(layer + 2 * (size_t)__ldg(idx + (t >> 1)) + (t & 1));
}

static unsigned gather_blocks(size_t items) {
  size_t b = (items + 255) / 256;
  size_t cap = (size_t)num_sms() * 8;
  return (unsigned)(b < cap ? (b ? b : 1) : cap);
}

int gather_multi(cudaStream_t st, const uint32_t* const* d_cols, uint32_t n_cols, const uint32_t* d_idx,
                 uint32_t n_idx, uint32_t* d_out) {
  if (n_cols == 0 || n_idx == 0) return OK;
  gather_multi_kernel<<<gather_blocks((size_t)n_cols * n_idx), 256, 0, st>>>(d_cols, n_cols, d_idx, n_idx, d_out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

int gather_hashes(cudaStream_t st, const uint32_t* d_layer, const uint32_t* d_idx, uint32_t n_idx, uint32_t* d_out) {
  if (n_idx == 0) return OK;
  gather_hashes_kernel<<<gather_blocks(2 * (size_t)n_idx), 256, 0, st>>>((const uint4*)d_layer, d_idx, n_idx,
                                                                          (uint4*)d_out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

}  // namespace gs
