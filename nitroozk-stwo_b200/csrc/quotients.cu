// DEEP quotients and lifted accumulation (QuotientOps / AccumulationOps).
//
// accumulate_numerators (crates/stwo/src/prover/backend/cpu/quotients.rs:21-45,
// core/pcs/quotients.rs:206-219): for one sample batch over columns of one
// log size,  partial[row] = sum_k c_k * col_k[row] - sum_k b_k   (QM31)
// with (a_k, b_k, c_k) the complex-conjugate line coefficients. The products
// c_k * v are accumulated lazily in 64-bit per coordinate and folded every
// two terms, so a term costs one wide multiply-add per coordinate.
//
// compute_quotients_and_combine (cpu/quotients.rs:47-75): for every row of
// the lifting domain (bit-reversed CanonicCoset(lift)),
//   q[row] = sum_a (partial_a[lift_idx_a(row)] - A_a * y) * den_a^-1,
//   den_a = (Re p_a.x - x) Im p_a.y - (Re p_a.y - y) Im p_a.x   (CM31)
// The CM31 denominators of R rows x K points of a thread are inverted with
// one field inversion (Montgomery's trick), instead of one inversion each.
//
// lift_and_accumulate (cpu/accumulation.rs:27-47): the chain of lifted adds
// collapses to res[i] = sum_c col_c[lift(i, L - L_c)] because lifted indices
// compose; one pass reads each column once.
#include "runtime.cuh"

namespace gs {

// ------------------------------------------------------------ numerators

// The batch's entries are staged in shared memory once per block. VEC: four
// consecutive rows per thread, each column read as one 16-byte load (all
// column pointers 16-byte aligned); otherwise one row per thread. Each step
// issues the column loads of 6 entries before using them (enough bytes in
// flight to cover DRAM latency), and the 64-bit accumulators are folded
// after every third product (a folded value is below 2^34, a product below
// 2^62).
constexpr uint32_t ACC_MAX_SMEM_ENTRIES = 512;

__device__ __forceinline__ void acc_term(uint64_t acc[4], const NumEntry& e, uint32_t v) {
  acc[0] += (uint64_t)e.c[0] * v;
  acc[1] += (uint64_t)e.c[1] * v;
  acc[2] += (uint64_t)e.c[2] * v;
  acc[3] += (uint64_t)e.c[3] * v;
}

template <int R>
__device__ __forceinline__ void load_rows(const uint32_t* col, size_t row0, uint32_t v[R]) {
  if (R == 4) {
    uint4 q = __ldg(reinterpret_cast<const uint4*>(col + row0));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
  } else {
    v[0] = __ldg(col + row0);
  }
}

template <int R>
__global__ void __launch_bounds__(256) accumulate_numerators_kernel(const NumEntry* __restrict__ entries,
                                                                    uint32_t n_entries, qm31 b_sum, uint32_t log_size,
                                                                    Planes out, const uint32_t* __restrict__ bsum_dev) {
  if (bsum_dev) b_sum = qm_make(bsum_dev[0], bsum_dev[1], bsum_dev[2], bsum_dev[3]);
  __shared__ NumEntry se[ACC_MAX_SMEM_ENTRIES];
  const bool staged = n_entries <= ACC_MAX_SMEM_ENTRIES;
  if (staged)
    for (uint32_t k = threadIdx.x; k < n_entries; k += blockDim.x) se[k] = entries[k];
  __syncthreads();
  const NumEntry* E = staged ? se : entries;
  const size_t n = (size_t)1 << log_size;
  for (size_t row0 = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) * R; row0 < n;
       row0 += (size_t)gridDim.x * blockDim.x * R) {
    uint64_t acc[R][4] = {};
    uint32_t k = 0;
    for (; k + 6 <= n_entries; k += 6) {
      uint32_t v[6][R];
#pragma unroll
      for (int j = 0; j < 6; j++) load_rows<R>(E[k + j].col, row0, v[j]);
#pragma unroll
      for (int j = 0; j < 6; j++) {
#pragma unroll
        for (int r = 0; r < R; r++) {
          acc_term(acc[r], E[k + j], v[j][r]);
          if (j == 2 || j == 5)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[r][q] = fold64h(acc[r][q]);
        }
      }
    }
    for (int cnt = 0; k < n_entries; k++) {
      uint32_t v[R];
      load_rows<R>(E[k].col, row0, v);
#pragma unroll
      for (int r = 0; r < R; r++) acc_term(acc[r], E[k], v[r]);
      if (++cnt == 3) {
        cnt = 0;
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
          for (int q = 0; q < 4; q++) acc[r][q] = fold64h(acc[r][q]);
      }
    }
    uint32_t o[4][R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      o[0][r] = sub(reduce64(acc[r][0]), b_sum.x.a);
      o[1][r] = sub(reduce64(acc[r][1]), b_sum.x.b);
      o[2][r] = sub(reduce64(acc[r][2]), b_sum.y.a);
      o[3][r] = sub(reduce64(acc[r][3]), b_sum.y.b);
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      if (R == 4)
        *reinterpret_cast<uint4*>(out.p[q] + row0) = make_uint4(o[q][0], o[q][1], o[q][2], o[q][3]);
      else
        out.p[q][row0] = o[q][0];
    }
  }
}

// Vector path with the entries split over the block's 8 warps: a block owns
// 128 rows (lane l: rows 4l..4l+3, one 16-byte word per column), warp w
// accumulates entries w, w + 8, ..., and the 8 partial sums meet in shared
// memory. Rounds of 6 entries stream through a per-warp double buffer with
// cp.async: round r + 1 is in flight while round r computes. Each lane copies
// exactly the 16 bytes it later reads, so its own cp.async.wait_group (a wait
// on its own copies) is the only synchronisation inside the entry loop.
constexpr int ACC_ROUND = 6;
constexpr size_t ACC_DYN_SMEM = sizeof(uint4) * 8 * 2 * ACC_ROUND * 32;  // 48 KiB; the partial sums reuse it

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// EG entry groups x (8 / EG) row groups: warp w = (entry group w / RG, row
// group w % RG); the block's tile is 128·RG rows, each warp 128 of them (lane
// l: 4 rows, one 16-byte word per column), and the entry groups split the
// entries (k = g, g + EG, ...). In a round the RG warps of an entry group
// read 512·RG contiguous bytes of one column, which keeps HBM pages open.
template <int EG>
__global__ void __launch_bounds__(256, 4) accumulate_numerators_split_kernel(const NumEntry* __restrict__ entries,
                                                                             uint32_t n_entries, qm31 b_sum,
                                                                             uint32_t log_size, Planes out,
                                                                             const uint32_t* __restrict__ bsum_dev) {
  if (bsum_dev) b_sum = qm_make(bsum_dev[0], bsum_dev[1], bsum_dev[2], bsum_dev[3]);
  constexpr uint32_t RG = 8 / EG, TILE = 128 * RG, STRIDE = EG * ACC_ROUND;
  extern __shared__ uint4 dyn[];  // [warp][slot][entry][lane] in the loop; part[group][q][row] after it
  uint32_t* part = reinterpret_cast<uint32_t*>(dyn);
  // entries are read where they lie (every thread of a warp reads the same
  // entry, an L1 broadcast): without a shared copy, 4 blocks fit on an SM
  const NumEntry* E = entries;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t eg = warp / RG, rg = warp % RG;
  uint4* wbuf = dyn + (size_t)warp * 2 * ACC_ROUND * 32;
  const size_t n = (size_t)1 << log_size;
  const uint32_t bs[4] = {b_sum.x.a, b_sum.x.b, b_sum.y.a, b_sum.y.b};
  // full rounds of this entry group: entries eg + STRIDE r + EG j, j < 6
  const uint32_t last = EG * (ACC_ROUND - 1);
  const uint32_t rounds = eg + last < n_entries ? (n_entries - 1 - last - eg) / STRIDE + 1 : 0;
  for (size_t tile = blockIdx.x; tile * TILE < n; tile += gridDim.x) {
    const size_t row0 = tile * TILE + 128 * rg + 4 * lane;
    auto issue = [&](uint32_t r) {
      uint4* b = wbuf + (r & 1) * ACC_ROUND * 32;
#pragma unroll
      for (int j = 0; j < ACC_ROUND; j++) cp_async16(b + j * 32 + lane, E[eg + STRIDE * r + EG * j].col + row0);
      cp_async_commit();
    };
    uint64_t acc[4][4] = {};
    if (rounds) issue(0);
    for (uint32_t r = 0; r < rounds; r++) {
      if (r + 1 < rounds) issue(r + 1);
      else cp_async_commit();  // an empty group keeps the count uniform
      cp_async_wait<1>();      // round r has landed (this lane's words)
      const uint4* b = wbuf + (r & 1) * ACC_ROUND * 32;
      const uint32_t k = eg + STRIDE * r;
#pragma unroll
      for (int j = 0; j < ACC_ROUND; j++) {
        const uint4 q4 = b[j * 32 + lane];
        const uint32_t v[4] = {q4.x, q4.y, q4.z, q4.w};
#pragma unroll
        for (int rr = 0; rr < 4; rr++) {
          acc_term(acc[rr], E[k + EG * j], v[rr]);
          if (j == 2 || j == 5)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[rr][q] = fold64h(acc[rr][q]);
        }
      }
    }
    // the group's remaining entries (fewer than 6), loaded directly
    for (uint32_t k = eg + STRIDE * rounds, cnt = 0; k < n_entries; k += EG) {
      uint32_t v[4];
      load_rows<4>(E[k].col, row0, v);
#pragma unroll
      for (int rr = 0; rr < 4; rr++) acc_term(acc[rr], E[k], v[rr]);
      if (++cnt == 3) {
        cnt = 0;
#pragma unroll
        for (int rr = 0; rr < 4; rr++)
#pragma unroll
          for (int q = 0; q < 4; q++) acc[rr][q] = fold64h(acc[rr][q]);
      }
    }
    if (EG == 1) {  // this warp holds its rows' whole sums
      cp_async_wait<0>();
#pragma unroll
      for (int q = 0; q < 4; q++)
        *reinterpret_cast<uint4*>(out.p[q] + row0) =
            make_uint4(sub(reduce64(acc[0][q]), bs[q]), sub(reduce64(acc[1][q]), bs[q]),
                       sub(reduce64(acc[2][q]), bs[q]), sub(reduce64(acc[3][q]), bs[q]));
      continue;
    }
    // every copy of every warp has landed before the buffers turn into part
    cp_async_wait<0>();
    __syncthreads();
#pragma unroll
    for (int rr = 0; rr < 4; rr++)
#pragma unroll
      for (int q = 0; q < 4; q++) part[(eg * 4 + q) * TILE + 128 * rg + 4 * lane + rr] = reduce64(acc[rr][q]);
    __syncthreads();
    for (uint32_t idx = threadIdx.x; idx < 4 * TILE; idx += blockDim.x) {
      const uint32_t q = idx / TILE, row = idx % TILE;
      uint32_t t = part[q * TILE + row];
#pragma unroll
      for (int g = 1; g < EG; g++) t = add(t, part[(g * 4 + q) * TILE + row]);
      if (tile * TILE + row < n) out.p[q][tile * TILE + row] = sub(t, bs[q]);
    }
    __syncthreads();
  }
}

int accumulate_numerators(cudaStream_t st, const void* d_entries, uint32_t n_entries, qm31 b_sum, uint32_t log_size,
                          Planes out, bool vec, const uint32_t* d_bsum) {
  GS_REQUIRE(log_size <= 30, "log size out of range");
  size_t n = (size_t)1 << log_size;
  int threads = 256;
  const uint32_t R = (vec && log_size >= 2) ? 4 : 1;
  if (R == 4)
    for (int q = 0; q < 4; q++) GS_REQUIRE(((uintptr_t)out.p[q] & 15) == 0, "vector path needs aligned planes");
  size_t blocks = (n / R + threads - 1) / threads;
  size_t cap = (size_t)num_sms() * 16;
  if (blocks > cap) blocks = cap;
  if (R == 4 && log_size >= 10) {
    // one entry group of 8 warps, 1024-row tiles (two groups of 4 warps on
    // 512-row tiles measured 104 µs against 95 µs on the Poseidon2 trace)
    const size_t tiles = n / 1024;
    const size_t cap2 = (size_t)num_sms() * 8;
    const unsigned grid = (unsigned)(tiles < cap2 ? tiles : cap2);
    static const cudaError_t attr = cudaFuncSetAttribute(
        accumulate_numerators_split_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ACC_DYN_SMEM);
    GS_CUDA_TRY(attr);
    accumulate_numerators_split_kernel<1><<<grid, 256, ACC_DYN_SMEM, st>>>((const NumEntry*)d_entries, n_entries,
                                                                         b_sum, log_size, out, d_bsum);
  } else if (R == 4)
    accumulate_numerators_kernel<4><<<(unsigned)blocks, threads, 0, st>>>((const NumEntry*)d_entries, n_entries,
                                                                         b_sum, log_size, out, d_bsum);
  else
    accumulate_numerators_kernel<1><<<(unsigned)blocks, threads, 0, st>>>((const NumEntry*)d_entries, n_entries,
                                                                         b_sum, log_size, out, d_bsum);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

// ------------------------------------------------------- line coefficients
__device__ __forceinline__ qm31 qm_pow_dev(qm31 x, uint32_t k) {
  qm31 r = qm_one();
  while (k) {
    if (k & 1u) r = qm_mul(r, x);
    x = qm_mul(x, x);
    k >>= 1;
  }
  return r;
}

__device__ __forceinline__ qm31 qm_ld(const uint32_t* p) { return qm_make(p[0], p[1], p[2], p[3]); }

__device__ __forceinline__ qm31 qm_shfl_down(qm31 v, int d) {
  return qm_make(__shfl_down_sync(0xffffffffu, v.x.a, d), __shfl_down_sync(0xffffffffu, v.x.b, d),
                 __shfl_down_sync(0xffffffffu, v.y.a, d), __shfl_down_sync(0xffffffffu, v.y.b, d));
}

__global__ void __launch_bounds__(512) quot_line_coeffs_kernel(const LineTerm* __restrict__ terms, uint32_t n_terms,
                                                               const uint32_t* __restrict__ vals,
                                                               const ptq* __restrict__ points, qm31 alpha,
                                                               NumEntry* entries, const uint32_t* batch_first,
                                                               const uint32_t* batch_point, uint32_t n_batches,
                                                               uint32_t* bsums, QuotAcc* accs, uint32_t n_points,
                                                               uint32_t* scratch) {
  __shared__ qm31 asum[QUOT_MAX_BATCHES];
  for (uint32_t i = threadIdx.x; i < n_terms; i += blockDim.x) {
    const LineTerm t = terms[i];
    const qm31 v = qm_ld(vals + t.val);
    const ptq p = points[t.point];
    const qm31 pw = qm_pow_dev(alpha, t.k);
    // complex_conjugate_line_coeffs: a = conj(v) - v, c = conj(p.y) - p.y,
    // b = v c - a p.y, all three times alpha^k
    const qm31 aa = qm_sub(qm_conj(v), v);
    const qm31 cc = qm_sub(qm_conj(p.y), p.y);
    const qm31 bb = qm_sub(qm_mul(v, cc), qm_mul(aa, p.y));
    const qm31 a = qm_mul(pw, aa), b = qm_mul(pw, bb), c = qm_mul(pw, cc);
    entries[i].c[0] = c.x.a; entries[i].c[1] = c.x.b; entries[i].c[2] = c.y.a; entries[i].c[3] = c.y.b;
    uint32_t* s = scratch + 8 * (size_t)i;
    s[0] = a.x.a; s[1] = a.x.b; s[2] = a.y.a; s[3] = a.y.b;
    s[4] = b.x.a; s[5] = b.x.b; s[6] = b.y.a; s[7] = b.y.b;
  }
  __syncthreads();
  // one warp per batch: the sums of a and b over its terms
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t bt = warp; bt < n_batches; bt += blockDim.x >> 5) {
    qm31 sa = qm_zero(), sb = qm_zero();
    for (uint32_t i = batch_first[bt] + lane; i < batch_first[bt + 1]; i += 32) {
      sa = qm_add(sa, qm_ld(scratch + 8 * (size_t)i));
      sb = qm_add(sb, qm_ld(scratch + 8 * (size_t)i + 4));
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
      sa = qm_add(sa, qm_shfl_down(sa, d));
      sb = qm_add(sb, qm_shfl_down(sb, d));
    }
    if (lane == 0) {
      asum[bt] = sa;
      bsums[4 * bt] = sb.x.a; bsums[4 * bt + 1] = sb.x.b; bsums[4 * bt + 2] = sb.y.a; bsums[4 * bt + 3] = sb.y.b;
    }
  }
  __syncthreads();
  // per sample point, its batches' a sums, in batch order
  for (uint32_t pt = threadIdx.x; pt < n_points; pt += blockDim.x) {
    qm31 f = qm_zero();
    for (uint32_t bt = 0; bt < n_batches; bt++)
      if (batch_point[bt] == pt) f = qm_add(f, asum[bt]);
    accs[pt].first_linear = f;
  }
}

int quot_line_coeffs(cudaStream_t st, const LineTerm* d_terms, uint32_t n_terms, const uint32_t* d_vals,
                     const ptq* d_points, qm31 alpha, NumEntry* d_entries, const uint32_t* d_batch_first,
                     const uint32_t* d_batch_point, uint32_t n_batches, uint32_t* d_bsums, QuotAcc* d_accs,
                     uint32_t n_points, uint32_t* d_scratch) {
  GS_REQUIRE(n_batches <= QUOT_MAX_BATCHES && n_points <= QUOT_MAX_POINTS, "too many quotient batches or points");
  GS_REQUIRE(n_terms == 0 || (d_terms && d_vals && d_points && d_entries && d_scratch), "null buffer");
  GS_REQUIRE(d_batch_first && d_batch_point && d_bsums && d_accs, "null buffer");
  quot_line_coeffs_kernel<<<1, 512, 0, st>>>(d_terms, n_terms, d_vals, d_points, alpha, d_entries, d_batch_first,
                                             d_batch_point, n_batches, d_bsums, d_accs, n_points, d_scratch);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

// ------------------------------------------------------------ quotients
constexpr int QUOT_ROWS = 2;   // rows per thread sharing one inversion
constexpr int QUOT_MAXK = 4;   // sample points per inversion chunk

__global__ void __launch_bounds__(128) quotients_kernel(const QuotAcc* __restrict__ accs, uint32_t n_accs,
                                                        DomainTables dt, Planes out) {
  const size_t n = (size_t)1 << dt.lift;
  const size_t n_groups = n / QUOT_ROWS;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < n_groups; g += (size_t)gridDim.x * blockDim.x) {
    // Rows g, g + n/R, ...: consecutive threads touch consecutive rows.
    pt31 dp[QUOT_ROWS];
    qm31 q[QUOT_ROWS];
#pragma unroll
    for (int r = 0; r < QUOT_ROWS; r++) {
      dp[r] = domain_point_bitrev(dt, (uint32_t)(g + r * n_groups));
      q[r] = qm_zero();
    }
    for (uint32_t a0 = 0; a0 < n_accs; a0 += QUOT_MAXK) {
      const uint32_t kc = n_accs - a0 < (uint32_t)QUOT_MAXK ? n_accs - a0 : (uint32_t)QUOT_MAXK;
      cm31 den[QUOT_ROWS][QUOT_MAXK];
      cm31 pref[QUOT_ROWS][QUOT_MAXK];
      cm31 run = {1, 0};
#pragma unroll
      for (int r = 0; r < QUOT_ROWS; r++) {
#pragma unroll
        for (int k = 0; k < QUOT_MAXK; k++) {
          if ((uint32_t)k < kc) {
            const QuotAcc& A = accs[a0 + k];
            cm31 d = cm_sub(cm_mul(cm_sub(A.prx, cm31{dp[r].x, 0}), A.piy),
                            cm_mul(cm_sub(A.pry, cm31{dp[r].y, 0}), A.pix));
            den[r][k] = d;
            pref[r][k] = run;
            run = cm_mul(run, d);
          }
        }
      }
      cm31 inv_run = cm_inv(run);
#pragma unroll
      for (int r = QUOT_ROWS - 1; r >= 0; r--) {
#pragma unroll
        for (int k = QUOT_MAXK - 1; k >= 0; k--) {
          if ((uint32_t)k < kc) {
            cm31 dinv = cm_mul(inv_run, pref[r][k]);
            inv_run = cm_mul(inv_run, den[r][k]);
            const QuotAcc& A = accs[a0 + k];
            uint32_t row = (uint32_t)(g + r * n_groups);
            uint32_t log_ratio = dt.lift - A.log_size;
            uint32_t li = ((row >> (log_ratio + 1)) << 1) + (row & 1u);
            qm31 pn = qm_make(__ldg(A.p[0] + li), __ldg(A.p[1] + li), __ldg(A.p[2] + li), __ldg(A.p[3] + li));
            qm31 full = qm_sub(pn, qm_mul_m31(A.first_linear, dp[r].y));
            q[r] = qm_add(q[r], qm_mul_cm31(full, dinv));
          }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < QUOT_ROWS; r++) {
      size_t row = g + r * n_groups;
      out.p[0][row] = q[r].x.a; out.p[1][row] = q[r].x.b; out.p[2][row] = q[r].y.a; out.p[3][row] = q[r].y.b;
    }
  }
}

// Point tables for the canonic half coset of log size lift-1:
// initial index 2^(31-(lift+1)), step 2^(31-(lift-1)).
__global__ void domain_tables_kernel(pt31* hi, pt31* lo, uint32_t s, uint32_t n_hi, uint32_t init, uint32_t step) {
  // circle generator powers, recomputed per thread (tiny tables)
  uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t n_lo = 1u << s;
  if (idx >= n_hi + n_lo) return;
  uint32_t k;
  if (idx < n_hi) k = (init + (uint32_t)(((uint64_t)idx << s) * step & 0x7fffffffu)) & 0x7fffffffu;
  else k = (uint32_t)(((uint64_t)(idx - n_hi) * step) & 0x7fffffffu);
  pt31 r = {1u, 0u}, cur = {2u, 1268011823u};
  for (int b = 0; b < 31; b++) {
    if ((k >> b) & 1u) r = pt_add(r, cur);
    cur = pt_add(cur, cur);
  }
  if (idx < n_hi) hi[idx] = r;
  else lo[idx - n_hi] = r;
}

int make_domain_tables(cudaStream_t st, uint32_t lift, pt31* d_buf /* n_hi + n_lo entries */, DomainTables* out) {
  GS_REQUIRE(lift >= 2 && lift <= 30, "lifting log size out of range");
  uint32_t half_log = lift - 1;
  uint32_t s = half_log / 2;
  uint32_t n_hi = 1u << (half_log - s), n_lo = 1u << s;
  uint32_t init = 1u << (31 - (lift + 1)), step = 1u << (31 - (lift - 1));
  uint32_t total = n_hi + n_lo;
  domain_tables_kernel<<<(total + 127) / 128, 128, 0, st>>>(d_buf, d_buf + n_hi, s, n_hi, init, step);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  *out = DomainTables{d_buf, d_buf + n_hi, s, lift};
  return OK;
}
size_t domain_tables_len(uint32_t lift) {
  uint32_t half_log = lift - 1, s = half_log / 2;
  return (size_t)(1u << (half_log - s)) + (1u << s);
}

int compute_quotients_and_combine(cudaStream_t st, const void* d_accs, uint32_t n_accs, const DomainTables& dt,
                                  Planes out) {
  size_t n = (size_t)1 << dt.lift;
  GS_REQUIRE(n >= QUOT_ROWS, "lifting domain too small");
  size_t groups = n / QUOT_ROWS;
  int threads = 128;
  size_t blocks = (groups + threads - 1) / threads;
  size_t cap = (size_t)num_sms() * 16;
  if (blocks > cap) blocks = cap;
  quotients_kernel<<<(unsigned)blocks, threads, 0, st>>>((const QuotAcc*)d_accs, n_accs, dt, out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

// ------------------------------------------------------------ accumulation
__global__ void lift_and_accumulate_kernel(const LiftCol* __restrict__ cols, uint32_t n_cols, uint32_t log_size,
                                           Planes out) {
  const size_t n = (size_t)1 << log_size;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (uint32_t c = 0; c < n_cols; c++) {
      const LiftCol& C = cols[c];
      uint32_t r = log_size - C.log_size;
      size_t li = ((i >> (r + 1)) << 1) + (i & 1);
      a0 = add(a0, __ldg(C.p[0] + li));
      a1 = add(a1, __ldg(C.p[1] + li));
      a2 = add(a2, __ldg(C.p[2] + li));
      a3 = add(a3, __ldg(C.p[3] + li));
    }
    out.p[0][i] = a0; out.p[1][i] = a1; out.p[2][i] = a2; out.p[3][i] = a3;
  }
}

int lift_and_accumulate(cudaStream_t st, const void* d_cols, uint32_t n_cols, uint32_t log_size, Planes out) {
  GS_REQUIRE(log_size >= 1 && log_size <= 30, "log size out of range");
  size_t n = (size_t)1 << log_size;
  size_t blocks = (n + 255) / 256;
  size_t cap = (size_t)num_sms() * 16;
  if (blocks > cap) blocks = cap;
  lift_and_accumulate_kernel<<<(unsigned)blocks, 256, 0, st>>>((const LiftCol*)d_cols, n_cols, log_size, out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

__global__ void accumulate_kernel(Planes a, CPlanes b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 4; c++) a.p[c][i] = add(a.p[c][i], __ldg(b.p[c] + i));
  }
}

int accumulate(cudaStream_t st, Planes a, CPlanes b, size_t n) {
  size_t blocks = (n + 255) / 256;
  size_t cap = (size_t)num_sms() * 16;
  if (blocks > cap) blocks = cap;
  if (blocks == 0) return OK;
  accumulate_kernel<<<(unsigned)blocks, 256, 0, st>>>(a, b, n);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

// AccumulationOps::generate_secure_powers (crates/stwo/src/prover/air/
// accumulation.rs:127-145; the reference's CUDA backend computes it on the
// host, prover/backend/cuda/accumulation.rs:20-22): out[i] = felt^i, i < n.
// Each thread raises felt to its index by squaring and multiplying.
__global__ void secure_powers_kernel(qm31 felt, size_t n, Planes out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    qm31 r = qm_one(), b = felt;
    for (size_t e = i; e; e >>= 1) {
      if (e & 1) r = qm_mul(r, b);
      b = qm_sqr(b);
    }
    out.p[0][i] = r.x.a;
    out.p[1][i] = r.x.b;
    out.p[2][i] = r.y.a;
    out.p[3][i] = r.y.b;
  }
}

int secure_powers(cudaStream_t st, qm31 felt, size_t n, Planes out) {
  if (n == 0) return OK;
  size_t blocks = (n + 255) / 256, cap = (size_t)num_sms() * 8;
  secure_powers_kernel<<<(unsigned)(blocks < cap ? blocks : cap), 256, 0, st>>>(felt, n, out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

}  // namespace gs
