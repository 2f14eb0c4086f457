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
// launch of one 8-CTA thread-block cluster. For layer k (log size log0 - k,
// leaves already hashed): its Merkle node layers (each CTA its eighth of the
// tree, then CTA 0 the last three levels), the channel step on its root (one
// thread), then fold_line into layer k + 1 with that layer's leaf hashes,
// split over the cluster — the same steps the per-layer kernels run, with
// cluster barriers in place of kernel boundaries. Data written inside the
// kernel by another CTA is read at L2 (__ldcg) after a cluster barrier.
__global__ void __cluster_dims__(8, 1, 1) __launch_bounds__(1024) fri_tail_kernel(FriTail a, uint32_t* state,
                                                                                  const uint32_t* __restrict__ itw,
                                                                                  uint32_t tw_len) {
  __shared__ uint4 buf[2][256];
  cg::cluster_group cluster = cg::this_cluster();
  const uint32_t gtid = cluster.block_rank() * blockDim.x + threadIdx.x;
  const uint32_t gthreads = 8 * blockDim.x;
  for (uint32_t k = 0; k < a.n; k++) {
    const uint32_t log = a.log0 - k;
    cluster_tree_levels(log, a.tree[k], k > 0, buf, cluster);
    if (cluster.block_rank() == 0 && threadIdx.x == 0)
      channel_mix_root_draw_dev(state, a.tree[k][0], a.roots + 8 * k, a.felts + 8 * k);
    cluster.sync();
    const uint32_t* f = a.felts + 8 * k;
    const qm31 alpha = qm_make(__ldcg(f), __ldcg(f + 1), __ldcg(f + 2), __ldcg(f + 3));
    const uint32_t half = 1u << (log - 1);
    const uint32_t* lvl = itw + (tw_len - (1u << log));
    uint32_t* const* sp = a.planes[k];
    uint32_t* const* dp = a.planes[k + 1];
    uint32_t* leaves = (k + 1 < a.n) ? a.tree[k + 1][log - 1] : nullptr;
    for (uint32_t i = gtid; i < half; i += gthreads) {
      // layer 0's planes come from the previous kernel; later ones from this one
      qm31 fx = qm_make(__ldcg(sp[0] + 2 * i), __ldcg(sp[1] + 2 * i), __ldcg(sp[2] + 2 * i), __ldcg(sp[3] + 2 * i));
      qm31 fnx = qm_make(__ldcg(sp[0] + 2 * i + 1), __ldcg(sp[1] + 2 * i + 1), __ldcg(sp[2] + 2 * i + 1),
                         __ldcg(sp[3] + 2 * i + 1));
      uint32_t xinv = __ldg(lvl + i);
      qm31 f0 = qm_add(fx, fnx);
      qm31 f1 = qm_mul_m31(qm_sub(fx, fnx), xinv);
      qm31 r = qm_add(f0, qm_mul(alpha, f1));
      dp[0][i] = r.x.a; dp[1][i] = r.x.b; dp[2][i] = r.y.a; dp[3][i] = r.y.b;
      if (leaves) leaf_hash4(leaves, i, r);
    }
    cluster.sync();
  }
}

int fri_tail(cudaStream_t st, const FriTail& a, uint32_t* d_state, const uint32_t* d_itw, uint32_t tw_log) {
  GS_REQUIRE(a.n >= 1 && a.n <= FRI_TAIL_MAX && a.log0 <= FRI_TAIL_MAX - 1 && a.log0 >= a.n,
             "FRI tail: layer sizes out of range");
  GS_REQUIRE(a.log0 <= tw_log, "FRI tail: line domain must fit the twiddle tree");
  fri_tail_kernel<<<8, 1024, 0, st>>>(a, d_state, d_itw, 1u << tw_log);
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
