// FRI folds over QM31 columns stored as 4 coordinate planes.
//
// fold_line (crates/stwo/src/prover/backend/cpu/fri.rs:64-86):
//   for pair i of a line evaluation on half_odds(n) in bit-reversed order,
//   f0 = f(x) + f(-x), f1 = (f(x) - f(-x)) / x, out[i] = f0 + alpha f1,
//   with 1/x read from the itwiddle level of half_odds(n) (offset L - 2^n).
// fold_circle_into_line (cpu/fri.rs:88-113):
//   f0 = f(p) + f(-p), f1 = (f(p) - f(-p)) / p.y,
//   dst[i] = dst[i] alpha^2 + f0 + alpha f1,
//   with 1/p.y the circle-layer itwiddle of the domain (the same derivation
//   the interpolation's first layer uses).
//
// Fusion: when `leaf_out` is given, the thread that produced element i also
// hashes it as the Merkle leaf of the next FRI layer (Blake2s of the 4
// coordinates, one compression), so the folded layer is not read again for
// its leaf hashes.
#include "runtime.cuh"
#include "blake2s.cuh"
#include "channel.cuh"
#include "merkle_tail.cuh"

namespace gs {

__device__ __forceinline__ void leaf_hash4(uint32_t* leaf_out, size_t i, qm31 v) {
  uint32_t h[8], m[16];
  blake2s_init(h);
  m[0] = v.x.a; m[1] = v.x.b; m[2] = v.y.a; m[3] = v.y.b;
#pragma unroll
  for (int j = 4; j < 16; j++) m[j] = 0;
  blake2s_compress(h, m, 16, true);
  uint4* o = reinterpret_cast<uint4*>(leaf_out + 8 * i);
  o[0] = make_uint4(h[0], h[1], h[2], h[3]);
  o[1] = make_uint4(h[4], h[5], h[6], h[7]);
}

__device__ __forceinline__ void store_hash8(uint32_t* out, size_t i, const uint32_t h[8]) {
  uint4* o = reinterpret_cast<uint4*>(out + 8 * i);
  o[0] = make_uint4(h[0], h[1], h[2], h[3]);
  o[1] = make_uint4(h[4], h[5], h[6], h[7]);
}

__device__ __forceinline__ void load_pair(CPlanes s, size_t i, qm31& a, qm31& b) {
  uint2 p0 = __ldg(reinterpret_cast<const uint2*>(s.p[0]) + i);
  uint2 p1 = __ldg(reinterpret_cast<const uint2*>(s.p[1]) + i);
  uint2 p2 = __ldg(reinterpret_cast<const uint2*>(s.p[2]) + i);
  uint2 p3 = __ldg(reinterpret_cast<const uint2*>(s.p[3]) + i);
  a = qm_make(p0.x, p1.x, p2.x, p3.x);
  b = qm_make(p0.y, p1.y, p2.y, p3.y);
}

// d_alpha (optional): the challenge in device memory (4 words, then alpha^2),
// written by the device channel; overrides `alpha`.
__global__ void fold_line_kernel(CPlanes src, uint32_t log_n, qm31 alpha, Planes dst, const uint32_t* __restrict__ itw,
                                 uint32_t tw_len, uint32_t* leaf_out, const uint32_t* __restrict__ d_alpha) {
  const size_t half = (size_t)1 << (log_n - 1);
  if (d_alpha) alpha = qm_make(d_alpha[0], d_alpha[1], d_alpha[2], d_alpha[3]);
  const uint32_t* lvl = itw + (tw_len - (1u << log_n));
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < half; i += (size_t)gridDim.x * blockDim.x) {
    qm31 fx, fnx;
    load_pair(src, i, fx, fnx);
    uint32_t xinv = __ldg(lvl + i);
    qm31 f0 = qm_add(fx, fnx);
    qm31 f1 = qm_mul_m31(qm_sub(fx, fnx), xinv);
    qm31 r = qm_add(f0, qm_mul(alpha, f1));
    dst.p[0][i] = r.x.a; dst.p[1][i] = r.x.b; dst.p[2][i] = r.y.a; dst.p[3][i] = r.y.b;
    if (leaf_out) leaf_hash4(leaf_out, i, r);
  }
}

struct SmallInvY { uint32_t v[2]; };

__global__ void fold_circle_kernel(CPlanes src, uint32_t log_n, qm31 alpha, qm31 alpha_sq, Planes dst,
                                   const uint32_t* __restrict__ itw, uint32_t tw_len, SmallInvY small,
                                   uint32_t* leaf_out, const uint32_t* __restrict__ d_alpha) {
  const size_t half = (size_t)1 << (log_n - 1);
  if (d_alpha) {
    alpha = qm_make(d_alpha[0], d_alpha[1], d_alpha[2], d_alpha[3]);
    alpha_sq = qm_make(d_alpha[4], d_alpha[5], d_alpha[6], d_alpha[7]);
  }
  const uint32_t* t0 = log_n >= 3 ? itw + (tw_len - (1u << (log_n - 1))) : nullptr;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < half; i += (size_t)gridDim.x * blockDim.x) {
    qm31 fp, fnp;
    load_pair(src, i, fp, fnp);
    uint32_t yinv;
    if (t0) {
      uint32_t q = (uint32_t)(i >> 2), r = (uint32_t)(i & 3);
      uint32_t x = __ldg(t0 + 2 * q + (r < 2 ? 1u : 0u));
      yinv = (r == 1 || r == 2) ? neg(x) : x;
    } else {
      yinv = small.v[i];
    }
    qm31 f0 = qm_add(fp, fnp);
    qm31 f1 = qm_mul_m31(qm_sub(fp, fnp), yinv);
    qm31 fprime = qm_add(qm_mul(alpha, f1), f0);
    qm31 d = qm_make(dst.p[0][i], dst.p[1][i], dst.p[2][i], dst.p[3][i]);
    qm31 r = qm_add(qm_mul(d, alpha_sq), fprime);
    dst.p[0][i] = r.x.a; dst.p[1][i] = r.x.b; dst.p[2][i] = r.y.a; dst.p[3][i] = r.y.b;
    if (leaf_out) leaf_hash4(leaf_out, i, r);
  }
}

static unsigned grid_for(size_t n, int threads) {
  size_t b = (n + threads - 1) / threads;
  size_t cap = (size_t)num_sms() * 16;
  return (unsigned)(b < cap ? (b ? b : 1) : cap);
}

static int fold_line_launch(cudaStream_t st, CPlanes src, uint32_t log_n, qm31 alpha, Planes dst,
                            const uint32_t* d_itw, uint32_t tw_log, uint32_t* leaf_out, const uint32_t* d_alpha) {
  GS_REQUIRE(log_n >= 1 && log_n <= tw_log, "fold_line: line domain must fit the twiddle tree");
  size_t half = (size_t)1 << (log_n - 1);
  fold_line_kernel<<<grid_for(half, 256), 256, 0, st>>>(src, log_n, alpha, dst, d_itw, 1u << tw_log, leaf_out,
                                                        d_alpha);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

static pt31 host_point(uint32_t k) {
  pt31 r = {1u, 0u}, cur = {2u, 1268011823u};
  for (int b = 0; b < 31; b++) {
    if ((k >> b) & 1u) r = pt_add(r, cur);
    cur = pt_add(cur, cur);
  }
  return r;
}

int fold_line_fused(cudaStream_t st, CPlanes src, uint32_t log_n, qm31 alpha, Planes dst, const uint32_t* d_itw,
                    uint32_t tw_log, uint32_t* leaf_out) {
  return fold_line_launch(st, src, log_n, alpha, dst, d_itw, tw_log, leaf_out, nullptr);
}
int fold_line_dev_alpha(cudaStream_t st, CPlanes src, uint32_t log_n, const uint32_t* d_alpha, Planes dst,
                        const uint32_t* d_itw, uint32_t tw_log, uint32_t* leaf_out) {
  return fold_line_launch(st, src, log_n, qm_zero(), dst, d_itw, tw_log, leaf_out, d_alpha);
}

static int fold_circle_launch(cudaStream_t st, CPlanes src, uint32_t log_n, qm31 alpha, Planes dst,
                              const uint32_t* d_itw, uint32_t tw_log, uint32_t* leaf_out, const uint32_t* d_alpha) {
  GS_REQUIRE(log_n >= 1 && log_n <= tw_log + 1, "fold_circle_into_line: domain must fit the twiddle tree");
  SmallInvY small{{0, 0}};
  if (log_n < 3) {
    // CanonicCoset(n) half coset: initial index 2^(31-(n+1)), step 2^(31-(n-1)).
    uint32_t init = 1u << (31 - (log_n + 1)), step = log_n >= 2 ? 1u << (31 - (log_n - 1)) : 0u;
    for (uint32_t i = 0; i < (1u << (log_n - 1)); i++) {
      uint32_t j = (log_n - 1) ? ((i & 1) ? 1u : 0u) : 0u;  // bit-reverse over n-1 <= 1 bits
      pt31 p = host_point((init + j * step) & 0x7fffffffu);
      small.v[i] = inv(p.y);
    }
  }
  qm31 alpha_sq = qm_mul(alpha, alpha);
  size_t half = (size_t)1 << (log_n - 1);
  fold_circle_kernel<<<grid_for(half, 256), 256, 0, st>>>(src, log_n, alpha, alpha_sq, dst, d_itw, 1u << tw_log, small,
                                                          leaf_out, d_alpha);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}
int fold_circle_into_line_fused(cudaStream_t st, CPlanes src, uint32_t log_n, qm31 alpha, Planes dst,
                                const uint32_t* d_itw, uint32_t tw_log, uint32_t* leaf_out) {
  return fold_circle_launch(st, src, log_n, alpha, dst, d_itw, tw_log, leaf_out, nullptr);
}
int fold_circle_into_line_dev_alpha(cudaStream_t st, CPlanes src, uint32_t log_n, const uint32_t* d_alpha, Planes dst,
                                    const uint32_t* d_itw, uint32_t tw_log, uint32_t* leaf_out) {
  return fold_circle_launch(st, src, log_n, qm_zero(), dst, d_itw, tw_log, leaf_out, d_alpha);
}

// Fused tail of the FRI commit phase: every layer of log size <= 11 in one
// launch of one 1024-thread CTA. For layer k (log size log0 - k, leaves
// already hashed): its Merkle node levels (at most 1024 nodes each, one per
// thread), the channel step on its root (one thread), then fold_line into
// layer k + 1 with that layer's leaf hashes — the steps the per-layer kernels
// run, with the data in shared memory and `__syncthreads` between them. The
// tail is a chain of about a hundred dependent steps, most of them one
// Blake2s compression long; an earlier 8-CTA cluster version spent more on
// cluster barriers and L2 re-reads than it gained in width (164 µs against
// 132 µs for the Poseidon2 2^18 proof's tail).
// Shared memory (uint4): two node-hash buffers of 1024 hashes, the current
// layer's leaves (1024 hashes), the current and next layer values (1024
// QM31 each): 128 KiB.
constexpr uint32_t TAIL_CTA_SMEM = 8192 * 16;
__global__ void __launch_bounds__(1024) fri_tail_cta_kernel(FriTail a, uint32_t* state,
                                                            const uint32_t* __restrict__ itw, uint32_t tw_len) {
  extern __shared__ uint4 tsm[];
  __shared__ uint32_t alpha_s[4];
  uint4* nb[2] = {tsm, tsm + 2048};
  uint4* leaves = tsm + 4096;
  uint4* vals[2] = {tsm + 6144, tsm + 7168};
  const uint32_t tid = threadIdx.x;
  for (uint32_t k = 0; k < a.n; k++) {
    const uint32_t log = a.log0 - k;
    uint32_t* const* tree = a.tree[k];
    int cur = 0;
    for (int L = (int)log - 1; L >= 0; L--) {
      if (tid < (1u << L)) {
        uint4 c[4];
        if (L == (int)log - 1) {
          if (k == 0) {  // leaves hashed by the previous kernel
            const uint4* src = reinterpret_cast<const uint4*>(tree[log]) + 4 * (size_t)tid;
#pragma unroll
            for (int q = 0; q < 4; q++) c[q] = __ldg(src + q);
          } else {
#pragma unroll
            for (int q = 0; q < 4; q++) c[q] = leaves[4 * tid + q];
          }
        } else {
#pragma unroll
          for (int q = 0; q < 4; q++) c[q] = nb[cur ^ 1][4 * tid + q];
        }
        uint32_t h[8];
        hash_children16(c, h);
        tail_store_hash(tree[L], tid, h);
        nb[cur][2 * tid] = make_uint4(h[0], h[1], h[2], h[3]);
        nb[cur][2 * tid + 1] = make_uint4(h[4], h[5], h[6], h[7]);
      }
      __syncthreads();
      cur ^= 1;
    }
    if (tid == 0) {  // the root sits in the buffer of the last level
      const uint32_t* f = a.felts + 8 * k;
      channel_mix_root_draw_dev(state, reinterpret_cast<const uint32_t*>(nb[cur ^ 1]), a.roots + 8 * k,
                                a.felts + 8 * k);
#pragma unroll
      for (int j = 0; j < 4; j++) alpha_s[j] = f[j];
    }
    __syncthreads();
    const qm31 alpha = qm_make(alpha_s[0], alpha_s[1], alpha_s[2], alpha_s[3]);
    const uint32_t half = 1u << (log - 1);
    if (tid < half) {
      qm31 fx, fnx;
      if (k == 0) {  // layer 0's values come from the previous kernel
        uint32_t* const* sp = a.planes[0];
        fx = qm_make(__ldg(sp[0] + 2 * tid), __ldg(sp[1] + 2 * tid), __ldg(sp[2] + 2 * tid), __ldg(sp[3] + 2 * tid));
        fnx = qm_make(__ldg(sp[0] + 2 * tid + 1), __ldg(sp[1] + 2 * tid + 1), __ldg(sp[2] + 2 * tid + 1),
                      __ldg(sp[3] + 2 * tid + 1));
      } else {
        const uint4 u = vals[k & 1][2 * tid], v = vals[k & 1][2 * tid + 1];
        fx = qm_make(u.x, u.y, u.z, u.w);
        fnx = qm_make(v.x, v.y, v.z, v.w);
      }
      const uint32_t xinv = __ldg(itw + (tw_len - (1u << log)) + tid);
      const qm31 f0 = qm_add(fx, fnx);
      const qm31 f1 = qm_mul_m31(qm_sub(fx, fnx), xinv);
      const qm31 r = qm_add(f0, qm_mul(alpha, f1));
      uint32_t* const* dp = a.planes[k + 1];
      dp[0][tid] = r.x.a; dp[1][tid] = r.x.b; dp[2][tid] = r.y.a; dp[3][tid] = r.y.b;
      vals[(k + 1) & 1][tid] = make_uint4(r.x.a, r.x.b, r.y.a, r.y.b);
      if (k + 1 < a.n) {  // the next layer's leaf
        uint32_t h[8], m[16];
        blake2s_init(h);
        m[0] = r.x.a; m[1] = r.x.b; m[2] = r.y.a; m[3] = r.y.b;
#pragma unroll
        for (int j = 4; j < 16; j++) m[j] = 0;
        blake2s_compress(h, m, 16, true);
        tail_store_hash(a.tree[k + 1][log - 1], tid, h);
        leaves[2 * tid] = make_uint4(h[0], h[1], h[2], h[3]);
        leaves[2 * tid + 1] = make_uint4(h[4], h[5], h[6], h[7]);
      }
    }
    __syncthreads();
  }
}

int fri_tail(cudaStream_t st, const FriTail& a, uint32_t* d_state, const uint32_t* d_itw, uint32_t tw_log) {
  GS_REQUIRE(a.n >= 1 && a.n <= FRI_TAIL_MAX && a.log0 <= FRI_TAIL_MAX - 1 && a.log0 >= a.n,
             "FRI tail: layer sizes out of range");
  GS_REQUIRE(a.log0 <= tw_log, "FRI tail: line domain must fit the twiddle tree");
  static const cudaError_t attr =
      cudaFuncSetAttribute(fri_tail_cta_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TAIL_CTA_SMEM);
  GS_CUDA_TRY(attr);
  fri_tail_cta_kernel<<<1, 1024, TAIL_CTA_SMEM, st>>>(a, d_state, d_itw, 1u << tw_log);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

int fold_line(cudaStream_t st, CPlanes src, uint32_t log_n, qm31 alpha, Planes dst, const uint32_t* d_itwiddles,
              uint32_t tw_log) {
  return fold_line_fused(st, src, log_n, alpha, dst, d_itwiddles, tw_log, nullptr);
}
int fold_circle_into_line(cudaStream_t st, CPlanes src, uint32_t log_n, qm31 alpha, Planes dst,
                          const uint32_t* d_itwiddles, uint32_t tw_log) {
  return fold_circle_into_line_fused(st, src, log_n, alpha, dst, d_itwiddles, tw_log, nullptr);
}

}  // namespace gs
