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

// d_prefix (optional): the prefixed digest in device memory, written by an
// earlier kernel of the stream; `d` is used when it is null.
__global__ void __launch_bounds__(GRIND_STEP) grind_kernel(Digest8 d, const uint32_t* d_prefix, uint32_t hi,
                                                           uint32_t pow_bits, uint32_t* result) {
  const volatile uint32_t* best = result;
  if (d_prefix)
#pragma unroll
    for (int j = 0; j < 8; j++) d.w[j] = d_prefix[j];
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

// Blocks: enough for about 16 expected hits in the first sweep of the grid
// (2^pow_bits tries per hit), at least one per SM, at most 8 per SM.
static unsigned grind_blocks(uint32_t pow_bits) {
  const uint64_t want = ((uint64_t)1 << (pow_bits < 24 ? pow_bits : 24)) * 16 / GRIND_STEP;
  const uint64_t lo_b = (uint64_t)num_sms(), hi_b = 8 * (uint64_t)num_sms();
  return (unsigned)(want < lo_b ? lo_b : want > hi_b ? hi_b : want);
}

// h_word (optional): a pinned host word for the per-chunk read-back.
int grind_blake2s(cudaStream_t st, const uint32_t prefixed_digest[8], uint32_t pow_bits, uint32_t* d_scratch,
                  uint64_t* nonce_out, uint32_t* h_word, uint32_t hi0) {
  GS_REQUIRE(pow_bits <= 32, "pow_bits > 32 is not supported");
  GS_REQUIRE(d_scratch != nullptr && nonce_out != nullptr, "null scratch/result");
  Digest8 d;
  for (int j = 0; j < 8; j++) d.w[j] = prefixed_digest[j];
  // Bounded search: 2^12 chunks of 2^20 nonces covers pow_bits far beyond 32
  // with overwhelming probability; running out is reported, never looped on.
  const unsigned blocks = grind_blocks(pow_bits);
  const uint32_t max_hi = grind_max_hi();
  for (uint32_t hi = hi0; hi < max_hi; hi++) {
    GS_CUDA_TRY(cudaMemsetAsync(d_scratch, 0xff, 4, st));
    grind_kernel<<<blocks, GRIND_STEP, 0, st>>>(d, nullptr, hi, pow_bits, d_scratch);
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

// ------------------------------------------------ last FRI layer + prefix
// Blake2s of n_words (>= 1) little-endian words, blocks of 16 words, the last
// (possibly full) block final, as the host Hasher does.
__device__ void blake2s_words(const uint32_t* w, uint32_t n_words, uint32_t out[8]) {
  blake2s_init(out);
  const uint32_t n_blocks = (n_words + 15) / 16;
  for (uint32_t b = 0; b < n_blocks; b++) {
    uint32_t m[16];
#pragma unroll
    for (int j = 0; j < 16; j++) m[j] = 16 * b + j < n_words ? w[16 * b + j] : 0u;
    const bool last = b + 1 == n_blocks;
    blake2s_compress(out, m, last ? 4 * n_words : 64 * (b + 1), last);
  }
}

struct LastLayerArgs {
  uint32_t log, bound_log, pow_bits, ninv;
  // inverse x-coordinates of half_odds(l) for l = log, ..., 1: 2^(l-1) values
  // per level, the largest level first
  uint32_t xinv[(1u << FRI_POW_MAX_LOG) - 1];
};

__host__ __device__ inline uint32_t bitrev_u32(uint32_t i, uint32_t log) {
  uint32_t r = 0;
  for (uint32_t b = 0; b < log; b++) r |= ((i >> b) & 1u) << (log - 1 - b);
  return r;
}

size_t fri_last_layer_pow_words(uint32_t bound_log) { return ((size_t)4 << bound_log) + 8 + 8 + 1; }

// One thread: LineEvaluation::interpolate of the last layer (prover/line.rs:
// 45-70) with the degree bound's coefficients kept, mix_felts of them
// (Blake2sChannel, core/channel/blake2s.rs), then the grind's prefixed digest
// Blake2s(POW_PREFIX || 0^12 || digest || pow_bits) (GrindOps, prover/
// backend/simd/grind.rs). The host restates every step and compares.
__global__ void fri_last_layer_prefix_kernel(const uint32_t* last, LastLayerArgs a, const uint32_t* state,
                                             uint32_t* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const uint32_t n = 1u << a.log;
  qm31 v[1u << FRI_POW_MAX_LOG];
  for (uint32_t i = 0; i < n; i++)
    v[bitrev_u32(i, a.log)] = qm_make(last[i], last[n + i], last[2 * n + i], last[3 * n + i]);
  uint32_t off = 0;
  for (uint32_t l = a.log; l >= 1; l--) {
    const uint32_t size = 1u << l;
    for (uint32_t c = 0; c < n; c += size)
      for (uint32_t i = 0; i < size / 2; i++) {
        const qm31 x = v[c + i], y = v[c + size / 2 + i];
        v[c + i] = qm_add(x, y);
        v[c + size / 2 + i] = qm_mul_m31(qm_sub(x, y), a.xinv[off + i]);
      }
    off += size / 2;
  }
  // coefficients in the channel's order: ordered[bitrev(i, log)] = v[i],
  // then coeffs[bitrev(i, bound_log)] = ordered[i] for i < 2^bound_log
  uint32_t msg[8 + (4u << 3)];
#pragma unroll
  for (int j = 0; j < 8; j++) msg[j] = state[j];
  const uint32_t bound = 1u << a.bound_log;
  for (uint32_t i = 0; i < n; i++) {
    const uint32_t o = bitrev_u32(i, a.log);
    if (o >= bound) continue;
    const qm31 c = qm_mul_m31(v[i], a.ninv);
    const uint32_t k = bitrev_u32(o, a.bound_log);
    msg[8 + 4 * k] = c.x.a; msg[9 + 4 * k] = c.x.b; msg[10 + 4 * k] = c.y.a; msg[11 + 4 * k] = c.y.b;
  }
  for (uint32_t j = 0; j < 4 * bound; j++) out[j] = msg[8 + j];
  uint32_t dg[8];
  blake2s_words(msg, 8 + 4 * bound, dg);
  uint32_t pre[13] = {0x12345678u, 0, 0, 0};
#pragma unroll
  for (int j = 0; j < 8; j++) {
    out[4 * bound + j] = dg[j];
    pre[4 + j] = dg[j];
  }
  pre[12] = a.pow_bits;
  uint32_t pd[8];
  blake2s_words(pre, 13, pd);
#pragma unroll
  for (int j = 0; j < 8; j++) out[4 * bound + 8 + j] = pd[j];
  out[4 * bound + 16] = 0xffffffffu;  // the grind's running minimum
}

// The point of index k of the circle group M31 (generator (2, 1268011823),
// order 2^31).
static pt31 circle_index_point(uint32_t k) {
  pt31 r = {1u, 0u}, cur = {2u, 1268011823u};
  for (int b = 0; b < 31; b++) {
    if ((k >> b) & 1u) r = pt_add(r, cur);
    cur = pt_add(cur, cur);
  }
  return r;
}

int fri_last_layer_pow(cudaStream_t st, const uint32_t* d_last, uint32_t log, uint32_t bound_log, uint32_t pow_bits,
                       const uint32_t* d_state, uint32_t* d_out) {
  GS_REQUIRE(log >= 1 && log <= FRI_POW_MAX_LOG && bound_log <= 3 && bound_log <= log && pow_bits <= 32,
             "last layer out of the device form's range");
  GS_REQUIRE(d_last && d_state && d_out, "null buffer");
  LastLayerArgs a{};
  a.log = log;
  a.bound_log = bound_log;
  a.pow_bits = pow_bits;
  a.ninv = inv(1u << log);
  uint32_t off = 0;
  for (uint32_t l = log; l >= 1; l--) {  // half_odds(l): index 2^(29-l) + i * 2^(31-l)
    for (uint32_t i = 0; i < (1u << (l - 1)); i++) {
      const uint32_t idx = (uint32_t)(((1ull << (31 - (l + 2))) + (uint64_t)i * (1ull << (31 - l))) & 0x7fffffffu);
      a.xinv[off + i] = inv(circle_index_point(idx).x);
    }
    off += 1u << (l - 1);
  }
  fri_last_layer_prefix_kernel<<<1, 32, 0, st>>>(d_last, a, d_state, d_out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  const uint32_t* d_prefix = d_out + ((size_t)4 << bound_log) + 8;
  uint32_t* d_best = d_out + ((size_t)4 << bound_log) + 16;
  grind_kernel<<<grind_blocks(pow_bits), GRIND_STEP, 0, st>>>(Digest8{}, d_prefix, 0, pow_bits, d_best);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

}  // namespace gs
