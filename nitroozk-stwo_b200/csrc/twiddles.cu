// Twiddle tree on the device.
//
// Layout (the reference's slow_precompute_twiddles,
// crates/stwo/src/prover/backend/cpu/circle.rs:273-289): for a coset C of log
// size m, level l (l = 0..m-1) holds the x coordinates of the first half of
// C doubled l times, in bit-reversed order, at offset 2^m - 2^(m-l); the last
// slot is 1. Itwiddles are the element-wise inverses.
//
// Every entry is computed independently: the point at circle index k is the
// sum of the precomputed powers gen * 2^b over the set bits b of k, so the
// whole tree is one launch with no sequential dependency.
#include "runtime.cuh"

namespace gs {

struct GenPowers { pt31 g[31]; };

static GenPowers host_gen_powers() {
  GenPowers gp;
  pt31 cur = {2u, 1268011823u};  // M31 circle generator (core/circle.rs:202-205)
  for (int b = 0; b < 31; b++) {
    gp.g[b] = cur;
    cur = pt_add(cur, cur);
  }
  return gp;
}

__device__ __forceinline__ pt31 index_to_point(uint32_t k, const GenPowers& gp) {
  pt31 r = {1u, 0u};
#pragma unroll 1
  for (int b = 0; b < 31; b++)
    if ((k >> b) & 1u) r = pt_add(r, gp.g[b]);
  return r;
}

__global__ void twiddle_tree_kernel(GenPowers gp, uint32_t initial, uint32_t step, uint32_t m, uint32_t* tw,
                                    uint32_t* itw) {
  uint32_t total = 1u << m;
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    uint32_t x = 1;
    if (idx != total - 1) {
      // level l: offset 2^m - 2^(m-l), length 2^(m-l-1)
      uint32_t rem = total - idx;                 // in (2^(m-l-1), 2^(m-l)]
      uint32_t level = m - (32 - __clz(rem - 1)); // rem-1 in [2^(m-l-1), 2^(m-l)) -> bit length m-l
      uint32_t off = total - (1u << (m - level));
      uint32_t i = idx - off;
      uint32_t bits = m - level - 1;
      uint32_t j = bits ? (__brev(i) >> (32 - bits)) : 0u;
      uint32_t init_l = (initial << level) & 0x7fffffffu;
      uint32_t step_l = (step << level) & 0x7fffffffu;
      uint32_t k = (init_l + (uint32_t)(((uint64_t)j * step_l) & 0x7fffffffu)) & 0x7fffffffu;
      x = index_to_point(k, gp).x;
    }
    tw[idx] = x;
    if (itw) itw[idx] = inv(x);
  }
}

int precompute_twiddles(cudaStream_t st, uint32_t initial_index, uint32_t step_index, uint32_t log_size,
                        uint32_t* d_twiddles, uint32_t* d_itwiddles) {
  GS_REQUIRE(log_size >= 1 && log_size <= 30, "twiddle coset log size must be in [1, 30]");
  GS_REQUIRE(d_twiddles != nullptr, "null twiddle buffer");
  GenPowers gp = host_gen_powers();
  uint32_t total = 1u << log_size;
  int threads = 256;
  int blocks = (int)((total + threads - 1) / threads);
  int cap = num_sms() * 8;
  if (blocks > cap) blocks = cap;
  twiddle_tree_kernel<<<blocks, threads, 0, st>>>(gp, initial_index & 0x7fffffffu, step_index & 0x7fffffffu, log_size,
                                                   d_twiddles, d_itwiddles);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

__global__ void batch_inverse_kernel(const uint32_t* in, uint32_t* out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = inv(in[i]);
}

int batch_inverse(cudaStream_t st, const uint32_t* d_in, uint32_t* d_out, size_t n) {
  if (n == 0) return OK;
  int blocks = (int)((n + 255) / 256);
  int cap = num_sms() * 16;
  if (blocks > cap) blocks = cap;
  batch_inverse_kernel<<<blocks, 256, 0, st>>>(d_in, d_out, n);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

}  // namespace gs
