// Out-of-domain evaluation of coefficient polynomials at a QM31 point
// (PolyOps::eval_at_point / batch_eval_at_point, crates/stwo/src/prover/
// backend/cpu/circle.rs:82-98, reference CUDA batch_eval_at_points).
//
// The reference folds the coefficients with the factors
// [pi^{n-2}(x), ..., pi(x), x, y] (pi(x) = 2x^2 - 1): unrolled, the value is
//   sum_i c_i * prod_{b in bits(i)} F_b,   F_0 = y, F_1 = x, F_b = pi^{b-1}(x).
// Split i = k * 2^s + j: the low-bit weights W[j] (2^s QM31 values) are built
// once per call, a block sums c_i * W[j] over its chunk with M31 x QM31
// products accumulated lazily in 64-bit, multiplies the chunk sum by the
// high-bit weight of k and writes one partial; a second kernel adds the
// partials of each polynomial. Scratch: weights + partials (caller-provided).
#include "runtime.cuh"

namespace gs {

constexpr uint32_t EAP_S = 10;                 // low bits per chunk: 1024 coefficients

struct Factors { qm31 f[31]; };

// W[j] = prod over set bits b < s of j of F_b, for j < 2^s (one block).
__global__ void eap_weights_kernel(Factors fs, uint32_t s, uint32_t* w /* 4 planes of 2^s, interleaved as [j][4] */) {
  extern __shared__ uint32_t sw[];  // 4 * 2^s
  uint32_t n = 1u << s;
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    qm31 acc = qm_one();
    for (uint32_t b = 0; b < s; b++)
      if ((j >> b) & 1u) acc = qm_mul(acc, fs.f[b]);
    w[4 * j + 0] = acc.x.a; w[4 * j + 1] = acc.x.b; w[4 * j + 2] = acc.y.a; w[4 * j + 3] = acc.y.b;
  }
  (void)sw;
}

__device__ __forceinline__ uint64_t fold64e(uint64_t x) { return (x & P) + (x >> 31); }

// grid: (chunks per poly, n_polys). Each block handles one chunk of one poly.
__global__ void __launch_bounds__(256) eap_chunk_kernel(const uint32_t* const* __restrict__ polys, uint32_t log_n,
                                                        const uint32_t* __restrict__ w, Factors fs, uint32_t* partials) {
  __shared__ uint32_t red[4][256 / 32];
  const uint32_t poly = blockIdx.y;
  const uint32_t chunk = blockIdx.x;
  const uint32_t s = log_n < EAP_S ? log_n : EAP_S;
  const uint32_t clen = 1u << s;
  const uint32_t* c = polys[poly] + ((size_t)chunk << s);
  uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  int cnt = 0;
  for (uint32_t j = threadIdx.x; j < clen; j += blockDim.x) {
    uint32_t v = __ldg(c + j);
    uint4 wj = __ldg(reinterpret_cast<const uint4*>(w) + j);
    a0 += (uint64_t)wj.x * v; a1 += (uint64_t)wj.y * v; a2 += (uint64_t)wj.z * v; a3 += (uint64_t)wj.w * v;
    if (++cnt == 2) { a0 = fold64e(a0); a1 = fold64e(a1); a2 = fold64e(a2); a3 = fold64e(a3); cnt = 0; }
  }
  uint32_t r0 = reduce64(a0), r1 = reduce64(a1), r2 = reduce64(a2), r3 = reduce64(a3);
  // warp reduction (field adds)
  for (int off = 16; off > 0; off >>= 1) {
    r0 = add(r0, __shfl_down_sync(0xffffffffu, r0, off));
    r1 = add(r1, __shfl_down_sync(0xffffffffu, r1, off));
    r2 = add(r2, __shfl_down_sync(0xffffffffu, r2, off));
    r3 = add(r3, __shfl_down_sync(0xffffffffu, r3, off));
  }
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { red[0][warp] = r0; red[1][warp] = r1; red[2][warp] = r2; red[3][warp] = r3; }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0;
    for (uint32_t k = 0; k < blockDim.x / 32; k++) {
      t0 = add(t0, red[0][k]); t1 = add(t1, red[1][k]); t2 = add(t2, red[2][k]); t3 = add(t3, red[3][k]);
    }
    qm31 sum = qm_make(t0, t1, t2, t3);
    // high-bit weight of the chunk index
    for (uint32_t b = 0; s + b < log_n; b++)
      if ((chunk >> b) & 1u) sum = qm_mul(sum, fs.f[s + b]);
    uint32_t* o = partials + 4 * ((size_t)poly * gridDim.x + chunk);
    o[0] = sum.x.a; o[1] = sum.x.b; o[2] = sum.y.a; o[3] = sum.y.b;
  }
}

__global__ void eap_finalize_kernel(const uint32_t* partials, uint32_t n_chunks, uint32_t n_polys, uint32_t* out) {
  uint32_t poly = blockIdx.x * blockDim.x + threadIdx.x;
  if (poly >= n_polys) return;
  uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0;
  const uint32_t* p = partials + 4 * (size_t)poly * n_chunks;
  for (uint32_t k = 0; k < n_chunks; k++) {
    t0 = add(t0, p[4 * k]); t1 = add(t1, p[4 * k + 1]); t2 = add(t2, p[4 * k + 2]); t3 = add(t3, p[4 * k + 3]);
  }
  out[4 * poly] = t0; out[4 * poly + 1] = t1; out[4 * poly + 2] = t2; out[4 * poly + 3] = t3;
}

// Factors F_b for a point (host).
static Factors eap_factors(const ptq& p, uint32_t log_n) {
  Factors fs;
  fs.f[0] = p.y;
  qm31 x = p.x;
  for (uint32_t b = 1; b < log_n && b < 31; b++) {
    fs.f[b] = x;
    x = qm_double_x(x);
  }
  return fs;
}

size_t eval_at_point_scratch_bytes(uint32_t n_polys, uint32_t log_n) {
  uint32_t s = log_n < EAP_S ? log_n : EAP_S;
  size_t chunks = (size_t)1 << (log_n - s);
  return 16 * ((size_t)1 << s) + 16 * chunks * n_polys;
}

// out: 4 words per polynomial (device). scratch: eval_at_point_scratch_bytes().
int batch_eval_at_point(cudaStream_t st, const uint32_t* const* d_polys, uint32_t n_polys, uint32_t log_n, ptq point,
                        uint32_t* d_out, uint32_t* d_scratch) {
  GS_REQUIRE(log_n <= 30, "log size out of range");
  if (n_polys == 0) return OK;
  Factors fs = eap_factors(point, log_n);
  uint32_t s = log_n < EAP_S ? log_n : EAP_S;
  uint32_t chunks = 1u << (log_n - s);
  GS_REQUIRE(chunks <= 65535 * 32768u, "too many chunks");
  uint32_t* w = d_scratch;
  uint32_t* partials = d_scratch + 4 * (1u << s);
  eap_weights_kernel<<<1, 256, 0, st>>>(fs, s, w);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  dim3 grid(chunks, n_polys);
  eap_chunk_kernel<<<grid, 256, 0, st>>>(d_polys, log_n, w, fs, partials);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  eap_finalize_kernel<<<(n_polys + 127) / 128, 128, 0, st>>>(partials, chunks, n_polys, d_out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

}  // namespace gs
