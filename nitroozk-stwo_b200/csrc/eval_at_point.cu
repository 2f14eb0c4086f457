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

struct Factors { qm31 f[31]; };

// W[j] = prod over set bits b < s of j of F_b, for j < 2^s (one thread each).
__global__ void eap_weights_kernel(Factors fs, uint32_t s, uint32_t* w /* [j][4] */) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (1u << s)) return;
  qm31 acc = qm_one();
  for (uint32_t b = 0; b < s; b++)
    if ((j >> b) & 1u) acc = qm_mul(acc, fs.f[b]);
  w[4 * j + 0] = acc.x.a; w[4 * j + 1] = acc.x.b; w[4 * j + 2] = acc.y.a; w[4 * j + 3] = acc.y.b;
}


// grid: (chunks per poly, n_polys). Each block handles one chunk of 2^s
// coefficients of one poly, 2^(s-8) per thread: products of M31 by the QM31
// weights accumulate in 64 bits, folded every third term (a folded value is
// below 2^34, a product below 2^62).
__global__ void __launch_bounds__(256) eap_chunk_kernel(const uint32_t* const* __restrict__ polys, uint32_t log_n,
                                                        uint32_t s, const uint32_t* __restrict__ w, Factors fs,
                                                        uint32_t* partials, bool vec) {
  __shared__ uint32_t red[4][256 / 32];
  const uint32_t poly = blockIdx.y;
  const uint32_t chunk = blockIdx.x;
  const uint32_t clen = 1u << s;
  const uint32_t* c = polys[poly] + ((size_t)chunk << s);
  uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  int cnt = 0;
  if (vec && clen >= 4 * blockDim.x) {
    // four consecutive coefficients per 16-byte load, two loads in flight
    for (uint32_t j0 = 4 * threadIdx.x; j0 < clen; j0 += 8 * blockDim.x) {
      uint4 v4[2];
      v4[0] = __ldg(reinterpret_cast<const uint4*>(c + j0));
      const bool two = j0 + 4 * blockDim.x < clen;
      if (two) v4[1] = __ldg(reinterpret_cast<const uint4*>(c + j0 + 4 * blockDim.x));
#pragma unroll
      for (int h = 0; h < 2; h++) {
        if (h == 1 && !two) break;
        const uint32_t jb = j0 + h * 4 * blockDim.x;
        const uint32_t vv[4] = {v4[h].x, v4[h].y, v4[h].z, v4[h].w};
#pragma unroll
        for (int e = 0; e < 4; e++) {
          uint4 wj = __ldg(reinterpret_cast<const uint4*>(w) + jb + e);
          const uint32_t v = vv[e];
          a0 += (uint64_t)wj.x * v; a1 += (uint64_t)wj.y * v; a2 += (uint64_t)wj.z * v; a3 += (uint64_t)wj.w * v;
          if (++cnt == 3) { a0 = fold64h(a0); a1 = fold64h(a1); a2 = fold64h(a2); a3 = fold64h(a3); cnt = 0; }
        }
      }
    }
  } else {
    for (uint32_t j = threadIdx.x; j < clen; j += blockDim.x) {
      uint32_t v = __ldg(c + j);
      uint4 wj = __ldg(reinterpret_cast<const uint4*>(w) + j);
      a0 += (uint64_t)wj.x * v; a1 += (uint64_t)wj.y * v; a2 += (uint64_t)wj.z * v; a3 += (uint64_t)wj.w * v;
      if (++cnt == 3) { a0 = fold64h(a0); a1 = fold64h(a1); a2 = fold64h(a2); a3 = fold64h(a3); cnt = 0; }
    }
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

// K polynomials per block for chunks of exactly 2^12 coefficients: each
// weight W[j] (16 bytes, read through L1) serves K coefficients, so L1
// traffic per coefficient drops from 20 to 4 + 16/K bytes (the one-polynomial
// kernel above is L1-bound). Thread t owns coefficients 4t + 1024q + e
// (q, e < 4): 16-byte coefficient loads, a warp reading 512 contiguous bytes
// per polynomial; the fold schedule is static (after every third
// coefficient: three products of < 2^62 on a folded value < 2^34 fit 64 bits).
constexpr uint32_t EAP_MULTI_LOG = 12;
template <int K>
__global__ void __launch_bounds__(256) eap_chunk_multi_kernel(const uint32_t* const* __restrict__ polys,
                                                              uint32_t n_polys, uint32_t log_n,
                                                              const uint32_t* __restrict__ w, Factors fs,
                                                              uint32_t* partials) {
  __shared__ uint32_t red[K][4][8];
  const uint32_t chunk = blockIdx.x, p0 = blockIdx.y * K;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint4* wv = reinterpret_cast<const uint4*>(w);
  const uint4* cp[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    const uint32_t p = p0 + k < n_polys ? p0 + k : n_polys - 1;  // tail rows recompute the last poly
    cp[k] = reinterpret_cast<const uint4*>(polys[p] + ((size_t)chunk << EAP_MULTI_LOG));
  }
  uint64_t acc[K][4];
#pragma unroll
  for (int k = 0; k < K; k++)
#pragma unroll
    for (int c = 0; c < 4; c++) acc[k][c] = 0;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const uint32_t j = 4 * threadIdx.x + 1024 * q;
    uint4 cv[K];
#pragma unroll
    for (int k = 0; k < K; k++) cv[k] = __ldg(cp[k] + (j >> 2));
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const uint4 wj = __ldg(wv + j + e);
#pragma unroll
      for (int k = 0; k < K; k++) {
        const uint32_t v = e == 0 ? cv[k].x : e == 1 ? cv[k].y : e == 2 ? cv[k].z : cv[k].w;
        acc[k][0] += (uint64_t)wj.x * v;
        acc[k][1] += (uint64_t)wj.y * v;
        acc[k][2] += (uint64_t)wj.z * v;
        acc[k][3] += (uint64_t)wj.w * v;
      }
      if ((4 * q + e) % 3 == 2)
#pragma unroll
        for (int k = 0; k < K; k++)
#pragma unroll
          for (int c = 0; c < 4; c++) acc[k][c] = fold64h(acc[k][c]);
    }
  }
#pragma unroll
  for (int k = 0; k < K; k++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      uint32_t r = reduce64(acc[k][c]);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) r = add(r, __shfl_down_sync(0xffffffffu, r, off));
      if (lane == 0) red[k][c][warp] = r;
    }
  __syncthreads();
  if (threadIdx.x < K && p0 + threadIdx.x < n_polys) {
    const uint32_t k = threadIdx.x;
    uint32_t t[4] = {0, 0, 0, 0};
#pragma unroll
    for (int c = 0; c < 4; c++)
#pragma unroll
      for (int q = 0; q < 8; q++) t[c] = add(t[c], red[k][c][q]);
    qm31 sum = qm_make(t[0], t[1], t[2], t[3]);
    for (uint32_t b = 0; EAP_MULTI_LOG + b < log_n; b++)
      if ((chunk >> b) & 1u) sum = qm_mul(sum, fs.f[EAP_MULTI_LOG + b]);
    uint32_t* o = partials + 4 * ((size_t)(p0 + k) * gridDim.x + chunk);
    o[0] = sum.x.a; o[1] = sum.x.b; o[2] = sum.y.a; o[3] = sum.y.b;
  }
}

// One block of 128 threads per polynomial: strided partial sums, then a
// shuffle and shared-memory reduction (field additions are exact, so the
// order does not change the result).
__global__ void __launch_bounds__(128) eap_finalize_kernel(const uint32_t* partials, uint32_t n_chunks, uint32_t n_polys,
                                                           uint32_t* out) {
  __shared__ uint4 red[4];
  const uint32_t poly = blockIdx.x;
  const uint4* p = reinterpret_cast<const uint4*>(partials) + (size_t)poly * n_chunks;
  uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0;
  for (uint32_t k = threadIdx.x; k < n_chunks; k += blockDim.x) {
    uint4 v = p[k];
    t0 = add(t0, v.x); t1 = add(t1, v.y); t2 = add(t2, v.z); t3 = add(t3, v.w);
  }
  for (int off = 16; off > 0; off >>= 1) {
    t0 = add(t0, __shfl_down_sync(0xffffffffu, t0, off));
    t1 = add(t1, __shfl_down_sync(0xffffffffu, t1, off));
    t2 = add(t2, __shfl_down_sync(0xffffffffu, t2, off));
    t3 = add(t3, __shfl_down_sync(0xffffffffu, t3, off));
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = make_uint4(t0, t1, t2, t3);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint4 r = red[0];
    for (uint32_t wv = 1; wv < blockDim.x / 32; wv++) {
      r.x = add(r.x, red[wv].x); r.y = add(r.y, red[wv].y); r.z = add(r.z, red[wv].z); r.w = add(r.w, red[wv].w);
    }
    out[4 * poly] = r.x; out[4 * poly + 1] = r.y; out[4 * poly + 2] = r.z; out[4 * poly + 3] = r.w;
  }
  (void)n_polys;
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

size_t eval_at_point_scratch_bytes(uint32_t n_polys, uint32_t log_n, uint32_t chunk_log) {
  uint32_t s = log_n < chunk_log ? log_n : chunk_log;
  size_t chunks = (size_t)1 << (log_n - s);
  return 16 * ((size_t)1 << s) + 16 * chunks * n_polys;
}

// out: 4 words per polynomial (device). scratch: eval_at_point_scratch_bytes()
// for the same chunk_log (coefficients per block, log 2).
int batch_eval_at_point(cudaStream_t st, const uint32_t* const* d_polys, uint32_t n_polys, uint32_t log_n, ptq point,
                        uint32_t* d_out, uint32_t* d_scratch, uint32_t chunk_log, bool vec) {
  GS_REQUIRE(log_n <= 30, "log size out of range");
  GS_REQUIRE(chunk_log >= 8 && chunk_log <= 14, "chunk log size out of range");
  if (n_polys == 0) return OK;
  Factors fs = eap_factors(point, log_n);
  uint32_t s = log_n < chunk_log ? log_n : chunk_log;
  uint32_t chunks = 1u << (log_n - s);
  GS_REQUIRE(chunks <= 65535 * 32768u, "too many chunks");
  uint32_t* w = d_scratch;
  uint32_t* partials = d_scratch + 4 * (1u << s);
  eap_weights_kernel<<<((1u << s) + 255) / 256, 256, 0, st>>>(fs, s, w);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  if (vec && s == EAP_MULTI_LOG) {
    // four polynomials per block (two: L1-bound again, 84 µs on the Poseidon2
    // 2^18 trace; eight: register-bound, 75 µs; four: 54 µs)
    dim3 grid(chunks, (n_polys + 3) / 4);
    eap_chunk_multi_kernel<4><<<grid, 256, 0, st>>>(d_polys, n_polys, log_n, w, fs, partials);
  } else {
    dim3 grid(chunks, n_polys);
    eap_chunk_kernel<<<grid, 256, 0, st>>>(d_polys, log_n, s, w, fs, partials, vec);
  }
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  eap_finalize_kernel<<<n_polys, 128, 0, st>>>(partials, chunks, n_polys, d_out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

// ------------------------------------------------------------ barycentric
// PolyOps::barycentric_weights for CanonicCoset(log) (crates/stwo/src/
// prover/backend/cpu/circle.rs:101-132): for the domain point q_i at
// bit-reversed position i,
//   w_i = V(p) / (s_i * v_i(p)),  V(p) = coset_vanishing(CanonicCoset(log), p),
//   s_i = -2 q_i.y * coset_vanishing_derivative(log, q_i)
//       = -2 * 4^(log-1) * q_i.y * prod_{j=1}^{log-1} pi^(j-1)(q_i.x),
//   v_i(p) = point_vanishing(q_i, p) = h.y / (1 + h.x),  h = p - q_i,
// because the vanishing polynomial of CanonicCoset(j) at a point is
// pi^(j-1) of its x (core/constraints.rs:12-55, 87-93). So
//   w_i = V(p) (1 + h.x) / (s_i h.y)
// with one QM31 inversion per point. c0 = -2 * 4^(log-1).
__global__ void barycentric_weights_kernel(DomainTables dt, uint32_t log_n, ptq p, qm31 vn_p, uint32_t c0,
                                           Planes out) {
  const size_t n = (size_t)1 << log_n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    pt31 q = domain_point_bitrev(dt, (uint32_t)i);
    uint32_t prod = 1, x = q.x;
    for (uint32_t j = 1; j < log_n; j++) {
      prod = mul(prod, x);
      x = double_x(x);
    }
    uint32_t si = mul(mul(c0, q.y), prod);
    // h = p + conj(q): (p.x q.x + p.y q.y, p.y q.x - p.x q.y)
    qm31 hx = qm_add(qm_mul_m31(p.x, q.x), qm_mul_m31(p.y, q.y));
    qm31 hy = qm_sub(qm_mul_m31(p.y, q.x), qm_mul_m31(p.x, q.y));
    qm31 w = qm_mul(qm_mul(vn_p, qm_add_m31(hx, 1)), qm_inv(qm_mul_m31(hy, si)));
    out.p[0][i] = w.x.a;
    out.p[1][i] = w.x.b;
    out.p[2][i] = w.y.a;
    out.p[3][i] = w.y.b;
  }
}

// PolyOps::barycentric_eval_at_point (cpu/circle.rs:134-141): sum_i evals[i]
// * w_i. Each block folds its rows into 64-bit accumulators (three products
// between folds) and writes one partial QM31; one block adds the partials.
constexpr int BARY_THREADS = 256;
__global__ void barycentric_dot_kernel(const uint32_t* __restrict__ evals, CPlanes w, size_t n, uint32_t* partials) {
  uint64_t acc[4] = {0, 0, 0, 0};
  int k = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t e = __ldg(evals + i);
#pragma unroll
    for (int q = 0; q < 4; q++) acc[q] += (uint64_t)e * __ldg(w.p[q] + i);
    if (++k == 3) {
#pragma unroll
      for (int q = 0; q < 4; q++) acc[q] = (acc[q] & P) + (acc[q] >> 31);
      k = 0;
    }
  }
  __shared__ uint32_t red[4][BARY_THREADS];
#pragma unroll
  for (int q = 0; q < 4; q++) red[q][threadIdx.x] = reduce64(acc[q]);
  __syncthreads();
  for (int half = BARY_THREADS / 2; half > 0; half >>= 1) {
    if ((int)threadIdx.x < half)
#pragma unroll
      for (int q = 0; q < 4; q++) red[q][threadIdx.x] = add(red[q][threadIdx.x], red[q][threadIdx.x + half]);
    __syncthreads();
  }
  if (threadIdx.x < 4) partials[4 * blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void barycentric_sum_kernel(const uint32_t* partials, uint32_t n_partials, uint32_t* out) {
  __shared__ uint32_t red[4][BARY_THREADS];
  uint32_t a[4] = {0, 0, 0, 0};
  for (uint32_t b = threadIdx.x; b < n_partials; b += blockDim.x)
#pragma unroll
    for (int q = 0; q < 4; q++) a[q] = add(a[q], partials[4 * b + q]);
#pragma unroll
  for (int q = 0; q < 4; q++) red[q][threadIdx.x] = a[q];
  __syncthreads();
  for (int half = BARY_THREADS / 2; half > 0; half >>= 1) {
    if ((int)threadIdx.x < half)
#pragma unroll
      for (int q = 0; q < 4; q++) red[q][threadIdx.x] = add(red[q][threadIdx.x], red[q][threadIdx.x + half]);
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = red[threadIdx.x][0];
}

int barycentric_weights(cudaStream_t st, const DomainTables& dt, ptq p, Planes out) {
  const uint32_t log_n = dt.lift;
  GS_REQUIRE(log_n >= 2 && log_n <= 30, "domain log size out of range");
  // V(p) = pi^(log-1)(p.x), c0 = -2 * 4^(log-1)
  qm31 vn = p.x;
  for (uint32_t j = 1; j < log_n; j++) vn = qm_double_x(vn);
  uint32_t c0 = neg(2);
  for (uint32_t j = 1; j < log_n; j++) c0 = mul(c0, 4);
  const size_t n = (size_t)1 << log_n;
  size_t blocks = (n + 255) / 256, cap = (size_t)num_sms() * 8;
  barycentric_weights_kernel<<<(unsigned)(blocks < cap ? blocks : cap), 256, 0, st>>>(dt, log_n, p, vn, c0, out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

size_t barycentric_scratch_words(size_t n) { return 4 * (size_t)num_sms() * 2 + 4; }

int barycentric_eval(cudaStream_t st, const uint32_t* d_evals, CPlanes w, size_t n, uint32_t* d_scratch,
                     uint32_t* d_out) {
  size_t blocks = (n + BARY_THREADS - 1) / BARY_THREADS, cap = (size_t)num_sms() * 2;
  if (blocks > cap) blocks = cap;
  if (blocks == 0) blocks = 1;
  barycentric_dot_kernel<<<(unsigned)blocks, BARY_THREADS, 0, st>>>(d_evals, w, n, d_scratch);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  barycentric_sum_kernel<<<1, BARY_THREADS, 0, st>>>(d_scratch, (uint32_t)blocks, d_out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

}  // namespace gs
