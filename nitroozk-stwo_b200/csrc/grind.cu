// Proof-of-work search: GrindOps<Blake2sChannel>::grind.
//
// Finds the smallest nonce = (hi << 32) | low, low < 2^20, scanning hi = 0, 1,
// ..., such that the first little-endian word of
//   Blake2s( prefixed_digest (32 B) || nonce (8 B, LE) )
// has at least pow_bits trailing zeros, where prefixed_digest =
// Blake2s(POW_PREFIX || 0^12 || digest || pow_bits) is computed by the caller.
// Same answer as the reference's SIMD grind (GRIND_LOW_BITS = 20,
// crates/stwo/src/prover/backend/simd/grind.rs) and CPU grind (cpu/grind.rs).
//
// One thread per candidate low word, one compression each; the smallest hit
// of a chunk is kept with atomicMin in a caller-provided device word.
#include "runtime.cuh"
#include "blake2s.cuh"

namespace gs {

struct Digest8 { uint32_t w[8]; };

__global__ void grind_kernel(Digest8 d, uint32_t hi, uint32_t pow_bits, uint32_t* result) {
  uint32_t low = blockIdx.x * blockDim.x + threadIdx.x;
  if (low >= (1u << 20)) return;
  uint32_t h[8], m[16];
  blake2s_init(h);
#pragma unroll
  for (int j = 0; j < 8; j++) m[j] = d.w[j];
  m[8] = low;
  m[9] = hi;
#pragma unroll
  for (int j = 10; j < 16; j++) m[j] = 0;
  blake2s_compress(h, m, 40, true);
  uint32_t tz = h[0] == 0 ? 32u : (uint32_t)__ffs(h[0]) - 1u;
  if (tz >= pow_bits) atomicMin(result, low);
}

// h_word (optional): a pinned host word for the per-chunk read-back.
int grind_blake2s(cudaStream_t st, const uint32_t prefixed_digest[8], uint32_t pow_bits, uint32_t* d_scratch,
                  uint64_t* nonce_out, uint32_t* h_word) {
  GS_REQUIRE(pow_bits <= 32, "pow_bits > 32 is not supported");
  GS_REQUIRE(d_scratch != nullptr && nonce_out != nullptr, "null scratch/result");
  Digest8 d;
  for (int j = 0; j < 8; j++) d.w[j] = prefixed_digest[j];
  // Bounded search: 2^12 chunks of 2^20 nonces covers pow_bits far beyond 32
  // with overwhelming probability; running out is reported, never looped on.
  for (uint32_t hi = 0; hi < (1u << 12); hi++) {
    GS_CUDA_TRY(cudaMemsetAsync(d_scratch, 0xff, 4, st));
    grind_kernel<<<(1u << 20) / 256, 256, 0, st>>>(d, hi, pow_bits, d_scratch);
    note_launch();
    GS_CUDA_TRY(cudaGetLastError());
    uint32_t local = 0;
    uint32_t* hw = h_word ? h_word : &local;
    GS_CUDA_TRY(cudaMemcpyAsync(hw, d_scratch, 4, cudaMemcpyDeviceToHost, st));
    GS_TRY(stream_sync(st));
    uint32_t found = *hw;
    if (found != 0xffffffffu) {
      *nonce_out = ((uint64_t)hi << 32) | found;
      return OK;
    }
  }
  set_error("grind: no nonce found within the search bound");
  return ERR_TIMEOUT;
}

}  // namespace gs
