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
// of a chunk is kept with atomicMin in a caller-provided device word. The
// grid is persistent and walks the chunk in 256-nonce steps in increasing
// order; a block stops as soon as the recorded minimum lies below its next
// step (a plain read, nothing waits), so a search that hits early costs a
// few thousand compressions instead of 2^20, and the answer is still the
// smallest hit: steps are skipped only when a smaller hit exists.
#include <cstdlib>
#include "runtime.cuh"
#include "blake2s.cuh"

namespace gs {

// High words searched before giving up: 2^12, or GS_GRIND_MAX_HI (1..4096,
// read once per process), which tests set low to reach the error path.
static uint32_t grind_max_hi() {
  static const uint32_t v = [] {
    const char* e = getenv("GS_GRIND_MAX_HI");
    long x = e ? strtol(e, nullptr, 10) : 0;
    return (uint32_t)(x >= 1 && x <= 4096 ? x : 4096);
  }();
  return v;
}

struct Digest8 { uint32_t w[8]; };

constexpr uint32_t GRIND_LOW_LOG = 20, GRIND_STEP = 256;

__global__ void __launch_bounds__(GRIND_STEP) grind_kernel(Digest8 d, uint32_t hi, uint32_t pow_bits,
                                                           uint32_t* result) {
  const volatile uint32_t* best = result;
  for (uint32_t step = blockIdx.x; step < ((1u << GRIND_LOW_LOG) / GRIND_STEP); step += gridDim.x) {
    if (*best < step * GRIND_STEP) return;  // a smaller nonce already passed
    const uint32_t low = step * GRIND_STEP + threadIdx.x;
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
  // Blocks: enough for about 16 expected hits in the first sweep of the grid
  // (2^pow_bits tries per hit), at least one per SM, at most 8 per SM.
  const uint64_t want = ((uint64_t)1 << (pow_bits < 24 ? pow_bits : 24)) * 16 / GRIND_STEP;
  const uint64_t lo_b = (uint64_t)num_sms(), hi_b = 8 * (uint64_t)num_sms();
  const unsigned blocks = (unsigned)(want < lo_b ? lo_b : want > hi_b ? hi_b : want);
  const uint32_t max_hi = grind_max_hi();
  for (uint32_t hi = 0; hi < max_hi; hi++) {
    GS_CUDA_TRY(cudaMemsetAsync(d_scratch, 0xff, 4, st));
    grind_kernel<<<blocks, GRIND_STEP, 0, st>>>(d, hi, pow_bits, d_scratch);
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
