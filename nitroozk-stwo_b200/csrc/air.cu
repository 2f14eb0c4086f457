// AIR kernels for the two benchmark components: trace generation, the
// Poseidon2 logup interaction column and the constraint quotients over the
// evaluation domain.
//
// Semantics follow the reference:
//   crates/examples/src/wide_fibonacci/mod.rs:48-58,86-130  (WideFibonacciEval, cuda trace: a=1, b=row)
//   crates/examples/src/poseidon/mod.rs:79-220,222-330      (Poseidon2 rounds, constraints, lookups, trace)
//   crates/constraint-framework/src/prover/component_prover.rs:177-280 (row_res * denom_inv[row >> trace_log])
//   crates/constraint-framework/src/prover/cpu_domain.rs:57-92 (offset rows, constraint powers)
//   crates/constraint-framework/src/lib.rs:218-262          (finalize_logup_in_pairs: one batch)
//   crates/constraint-framework/src/prover/logup.rs:100-140 (claimed sum, shifted prefix sum)
//   crates/stwo/src/prover/backend/simd/prefix_sum.rs:123-140 (prefix sum in coset order)
//
// Layout: a tree's columns are one contiguous buffer, column c at base + c * 2^log.
// Constraint values of the base-field constraints are accumulated as
// sum_k p_k * c_k with p_k in QM31 and c_k in M31: four wide products per term,
// folded every two terms (lazy reduction), one reduction per row.
#include "runtime.cuh"
#include "air.cuh"
#include <cub/device/device_scan.cuh>

namespace gs {

// ------------------------------------------------------------ seeded input
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// Uniform M31 for (seed, column, row): the first of mix64(seed ^ mix64(col *
// 0x100000001B3 + (row << 8) + k)) & (2^31 - 1), k = 0, 1, ..., below P.
__host__ __device__ __forceinline__ uint32_t seeded_m31(uint64_t seed, uint64_t col, uint64_t row) {
  for (uint64_t k = 0; k < 256; k++) {
    uint32_t v = (uint32_t)mix64(seed ^ mix64(col * 0x100000001B3ull + (row << 8) + k)) & 0x7fffffffu;
    if (v != P) return v;
  }
  return 0;  // unreachable in practice: 256 consecutive rejections of one value in 2^31
}

// ------------------------------------------------------------ wide fibonacci
__global__ void wf_trace_kernel(uint32_t* cols, uint32_t log_n, uint32_t n_cols, uint64_t seed, uint32_t mode) {
  const size_t n = (size_t)1 << log_n;
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
    // mode 0: the reference's inputs (a = 1, b = row); 1: seeded; 2: preloaded columns 0-1
    uint32_t a = mode == 2 ? cols[r] : (mode ? seeded_m31(seed, 0, r) : 1u);
    uint32_t b = mode == 2 ? cols[n + r] : (mode ? seeded_m31(seed, 1, r) : (uint32_t)(r % P));
    cols[r] = a;
    cols[n + r] = b;
    for (uint32_t k = 2; k < n_cols; k++) {
      uint32_t c = add(sqr(a), sqr(b));
      cols[(size_t)k * n + r] = c;
      a = b;
      b = c;
    }
  }
}


// Column access of the constraint kernels: a tree's columns as one
// contiguous buffer (the prover's layout: column c at base + c * n), or a
// device table of column pointers (callers of the C ABI, whose columns are
// separate allocations). cursor(c, r) walks row r of columns c, c+1, ...
struct ContigCols {
  const uint32_t* base;
  size_t n;
  struct Cursor {
    const uint32_t* p;
    size_t n;
    __device__ __forceinline__ uint32_t next() {
      uint32_t v = __ldg(p);
      p += n;
      return v;
    }
  };
  __device__ __forceinline__ const uint32_t* col(uint32_t c) const { return base + (size_t)c * n; }
  __device__ __forceinline__ Cursor cursor(uint32_t c, size_t r) const { return Cursor{col(c) + r, n}; }
};
struct TableCols {
  const uint32_t* const* tab;
  struct Cursor {
    const uint32_t* const* t;
    size_t r;
    __device__ __forceinline__ uint32_t next() { return __ldg(*t++ + r); }
  };
  __device__ __forceinline__ const uint32_t* col(uint32_t c) const { return tab[c]; }
  __device__ __forceinline__ Cursor cursor(uint32_t c, size_t r) const { return Cursor{tab + c, r}; }
};

// Writes (accumulate == 0) or adds to (accumulate != 0) the output planes.
__device__ __forceinline__ void store_quotient(const Planes& out, size_t r, const uint32_t v[4], uint32_t accumulate) {
#pragma unroll
  for (int q = 0; q < 4; q++) out.p[q][r] = accumulate ? add(out.p[q][r], v[q]) : v[q];
}

template <class Cols>
__global__ void __launch_bounds__(256) wf_constraints_kernel(Cols cols, uint32_t n_cols, uint32_t eval_log,
                                                             uint32_t trace_log, ConstraintParams prm, Planes out,
                                                             uint32_t accumulate) {
  const size_t n = (size_t)1 << eval_log;
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
    auto cur = cols.cursor(0, r);
    uint32_t a = cur.next(), b = cur.next();
    uint64_t acc[4] = {0, 0, 0, 0};
    for (uint32_t k = 2; k < n_cols; k++) {
      uint32_t c = cur.next();
      uint32_t cons = sub(c, add(sqr(a), sqr(b)));
      const uint32_t* p = prm.powers + 4 * (k - 2);
#pragma unroll
      for (int q = 0; q < 4; q++) acc[q] = fold64h(acc[q] + (uint64_t)p[q] * cons);
      a = b;
      b = c;
    }
    uint32_t dinv = prm.denom_inv[r >> trace_log];
    uint32_t v[4];
#pragma unroll
    for (int q = 0; q < 4; q++) v[q] = mul(reduce64(acc[q]), dinv);
    store_quotient(out, r, v, accumulate);
  }
}

// ------------------------------------------------------------ poseidon2
constexpr uint32_t PN_RC = 1234;  // the reference's placeholder round constants (poseidon/mod.rs:48-51)

__host__ __device__ __forceinline__ void p2_m4(uint32_t* x) {
  uint32_t t0 = add(x[0], x[1]);
  uint32_t t02 = add(t0, t0);
  uint32_t t1 = add(x[2], x[3]);
  uint32_t t12 = add(t1, t1);
  uint32_t t2 = add(add(x[1], x[1]), t1);
  uint32_t t3 = add(add(x[3], x[3]), t0);
  uint32_t t4 = add(add(t12, t12), t3);
  uint32_t t5 = add(add(t02, t02), t2);
  x[0] = add(t3, t5);
  x[1] = t5;
  x[2] = add(t2, t4);
  x[3] = t4;
}
__host__ __device__ __forceinline__ void p2_external(uint32_t* s) {
#pragma unroll
  for (int i = 0; i < 4; i++) p2_m4(s + 4 * i);
#pragma unroll
  for (int j = 0; j < 4; j++) {
    uint32_t t = add(add(s[j], s[j + 4]), add(s[j + 8], s[j + 12]));
#pragma unroll
    for (int i = 0; i < 4; i++) s[4 * i + j] = add(s[4 * i + j], t);
  }
}
// x * 2^k mod p for canonical x and 1 <= k <= 30: the 31-bit rotation of x
// left by k, which is canonical again (a rotation of a word that is not all
// ones is not all ones). On the device: one wide multiply by 2^(k+1), whose
// high word x >> (31 - k) and halved low word (x << k) mod 2^31 occupy
// disjoint bits, then one shift-add; no reduction step.
__host__ __device__ __forceinline__ uint32_t mul_pow2(uint32_t x, int k) {
#ifdef __CUDA_ARCH__
  uint64_t w = (uint64_t)x * (2u << k);
  return (uint32_t)(w >> 32) + ((uint32_t)w >> 1);
#else
  return ((x << k) & P) | (x >> (31 - k));
#endif
}
// The internal round matrix: s_i * 2^(i+1) + sum (the reference multiplies
// by the constant, poseidon/mod.rs:132-146).
__host__ __device__ __forceinline__ void p2_internal(uint32_t* s) {
  uint32_t sum = s[0];
#pragma unroll
  for (int i = 1; i < 16; i++) sum = add(sum, s[i]);
#pragma unroll
  for (int i = 0; i < 16; i++) s[i] = add(mul_pow2(s[i], i + 1), sum);
}
__host__ __device__ __forceinline__ uint32_t pow5(uint32_t x) { uint32_t x2 = sqr(x); return mul(sqr(x2), x); }

__global__ void poseidon_trace_kernel(uint32_t* cols, uint32_t log_n, uint64_t seed, uint32_t mode) {
  const size_t n = (size_t)1 << log_n;
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
    uint32_t s[16];
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) {
      // mode 0: the reference's inputs (row + i); 1: seeded; 2: preloaded columns 0-15
      s[i] = mode == 2 ? cols[(size_t)i * n + r] : (mode ? seeded_m31(seed, i, r) : (uint32_t)((r + i) % P));
      cols[(size_t)(c++) * n + r] = s[i];
    }
    for (int round = 0; round < 4; round++) {
#pragma unroll
      for (int i = 0; i < 16; i++) s[i] = add(s[i], PN_RC);
      p2_external(s);
#pragma unroll
      for (int i = 0; i < 16; i++) {
        s[i] = pow5(s[i]);
        cols[(size_t)(c++) * n + r] = s[i];
      }
    }
    for (int round = 0; round < 14; round++) {
      s[0] = add(s[0], PN_RC);
      p2_internal(s);
      s[0] = pow5(s[0]);
      cols[(size_t)(c++) * n + r] = s[0];
    }
    for (int round = 0; round < 4; round++) {
#pragma unroll
      for (int i = 0; i < 16; i++) s[i] = add(s[i], PN_RC);
      p2_external(s);
#pragma unroll
      for (int i = 0; i < 16; i++) {
        s[i] = pow5(s[i]);
        cols[(size_t)(c++) * n + r] = s[i];
      }
    }
  }
}

// LookupElements::combine of 16 columns (c0 .. c0 + 15) at row r.
template <class Cols>
__device__ __forceinline__ qm31 combine16(const LookupParams& lp, const Cols& cols, uint32_t c0, size_t r) {
  uint64_t acc[4] = {0, 0, 0, 0};
#pragma unroll
  for (int i = 0; i < 16; i++) {
    uint32_t x = __ldg(cols.col(c0 + i) + r);
    const uint32_t* a = lp.alpha_pow + 4 * i;
#pragma unroll
    for (int q = 0; q < 4; q++) acc[q] += (uint64_t)a[q] * x;
    // three products (< 2^62 each) and a folded accumulator (< 2^34) fit in 64 bits
    if (i % 3 == 2 || i == 15) {
#pragma unroll
      for (int q = 0; q < 4; q++) acc[q] = fold64h(acc[q]);
    }
  }
  qm31 s = qm_make(reduce64(acc[0]), reduce64(acc[1]), reduce64(acc[2]), reduce64(acc[3]));
  return qm_sub(s, qm_make(lp.z[0], lp.z[1], lp.z[2], lp.z[3]));
}

__device__ __forceinline__ uint32_t coset_index(uint32_t i, uint32_t log_n) {
  uint32_t n = 1u << log_n;
  uint32_t j = log_n ? (__brev(i) >> (32 - log_n)) : 0u;
  return j < n / 2 ? 2 * j : 2 * (n - 1 - j) + 1;
}

// Per row: (1/d0 - 1/d1) written at its coset-order position; d0 / d1 the
// lookup combination of the initial / final state (16 columns each, from
// column c_init of `init` and c_final of `fin`).
template <class InitCols, class FinalCols>
__global__ void logup_fraction_kernel(InitCols init, uint32_t c_init, FinalCols fin, uint32_t c_final, uint32_t log_n,
                                      LookupParams lp, uint4* __restrict__ coset_vals) {
  const size_t n = (size_t)1 << log_n;
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
    qm31 d0 = combine16(lp, init, c_init, r);
    qm31 d1 = combine16(lp, fin, c_final, r);
    qm31 v = qm_mul(qm_sub(d1, d0), qm_inv(qm_mul(d0, d1)));
    coset_vals[coset_index((uint32_t)r, log_n)] = make_uint4(v.x.a, v.x.b, v.y.a, v.y.b);
  }
}

struct AddQM {
  __device__ __forceinline__ uint4 operator()(const uint4& a, const uint4& b) const {
    return make_uint4(add(a.x, b.x), add(a.y, b.y), add(a.z, b.z), add(a.w, b.w));
  }
};

// out_c[i] = S_c[k] - (k + 1) * shift_c at k = coset position of storage row i,
// shift = S[n - 1] / n (the claimed sum over n, inv_n = 1/n mod p), read here
// so that the host need not wait for the sum first.
__global__ void logup_finalize_kernel(const uint4* __restrict__ scan, uint32_t log_n, uint32_t inv_n, Planes out) {
  const size_t n = (size_t)1 << log_n;
  const uint4 total = scan[n - 1];
  const qm31 shift = qm_mul_m31(qm_make(total.x, total.y, total.z, total.w), inv_n);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t k = coset_index((uint32_t)i, log_n);
    uint4 s = scan[k];
    uint32_t m = (k + 1) % P;
    out.p[0][i] = sub(s.x, mul(shift.x.a, m));
    out.p[1][i] = sub(s.y, mul(shift.x.b, m));
    out.p[2][i] = sub(s.z, mul(shift.y.a, m));
    out.p[3][i] = sub(s.w, mul(shift.y.b, m));
  }
}

// offset_bit_reversed_circle_domain_index(i, trace_log, eval_log, -1)
// (crates/stwo/src/core/utils.rs).
__device__ __forceinline__ uint32_t prev_row(uint32_t i, uint32_t trace_log, uint32_t eval_log) {
  uint32_t idx = __brev(i) >> (32 - eval_log);
  uint32_t half = 1u << (eval_log - 1);
  uint32_t step = 1u << (eval_log - trace_log - 1);
  if (idx < half) idx = (idx + half - step) & (half - 1);
  else idx = ((idx - half + step) & (half - 1)) + half;
  return __brev(idx) >> (32 - eval_log);
}

// Lazy accumulation: products are below 2^62 and a folded accumulator below
// 2^34, so three terms fit in 64 bits between folds; a fold follows every
// third term of a round and the round's last term. The round loops stay
// rolled: unrolled, the kernel outgrows the instruction cache. Registers are
// held to 72 (7 blocks of 128 per SM, no spills): 354 us per 2^20-row launch
// against 368 us at 96 registers (5 blocks) and 369 us at 64 (8 blocks).
template <class TraceCols, class InterCols>
__global__ void __launch_bounds__(128, 7) poseidon_constraints_kernel(TraceCols trace, InterCols inter, uint32_t eval_log,
                                                                   uint32_t trace_log, ConstraintParams prm,
                                                                   LookupParams lp, qm31 cumsum_shift, Planes out,
                                                                   uint32_t accumulate) {
  const size_t n = (size_t)1 << eval_log;
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
    uint64_t acc[4] = {0, 0, 0, 0};
    uint32_t k = 0;  // constraint index
    // term i of the current round; folds after every third term and the last
    auto add_cons = [&](uint32_t c, int i, int last) {
      const uint32_t* p = prm.powers + 4 * k;
#pragma unroll
      for (int q = 0; q < 4; q++) acc[q] += (uint64_t)p[q] * c;
      if (i % 3 == 2 || i == last) {
#pragma unroll
        for (int q = 0; q < 4; q++) acc[q] = fold64h(acc[q]);
      }
      k++;
    };
    auto col = trace.cursor(0, r);
    uint32_t s[16];
#pragma unroll
    for (int i = 0; i < 16; i++) s[i] = col.next();
#pragma unroll 1
    for (int round = 0; round < 4; round++) {
#pragma unroll
      for (int i = 0; i < 16; i++) s[i] = add(s[i], PN_RC);
      p2_external(s);
#pragma unroll
      for (int i = 0; i < 16; i++) {
        uint32_t m = col.next();
        add_cons(sub(pow5(s[i]), m), i, 15);
        s[i] = m;
      }
    }
#pragma unroll 1
    for (int round = 0; round < 14; round++) {
      s[0] = add(s[0], PN_RC);
      p2_internal(s);
      uint32_t m = col.next();
      add_cons(sub(pow5(s[0]), m), 0, 0);
      s[0] = m;
    }
#pragma unroll 1
    for (int round = 0; round < 4; round++) {
#pragma unroll
      for (int i = 0; i < 16; i++) s[i] = add(s[i], PN_RC);
      p2_external(s);
#pragma unroll
      for (int i = 0; i < 16; i++) {
        uint32_t m = col.next();
        add_cons(sub(pow5(s[i]), m), i, 15);
        s[i] = m;
      }
    }
    // logup: frac = 1/d0 - 1/d1 as (d1 - d0) / (d0 d1); constraint
    // (cur - prev + shift) * d0 d1 - (d1 - d0)
    qm31 d0 = combine16(lp, trace, 0, r);
    qm31 d1 = combine16(lp, trace, 158 - 16, r);
    uint32_t pr = prev_row((uint32_t)r, trace_log, eval_log);
    qm31 cur = qm_make(__ldg(inter.col(0) + r), __ldg(inter.col(1) + r), __ldg(inter.col(2) + r),
                       __ldg(inter.col(3) + r));
    qm31 prv = qm_make(__ldg(inter.col(0) + pr), __ldg(inter.col(1) + pr), __ldg(inter.col(2) + pr),
                       __ldg(inter.col(3) + pr));
    qm31 lc = qm_sub(qm_mul(qm_add(qm_sub(cur, prv), cumsum_shift), qm_mul(d0, d1)), qm_sub(d1, d0));
    qm31 pl = qm_make(prm.powers[4 * k], prm.powers[4 * k + 1], prm.powers[4 * k + 2], prm.powers[4 * k + 3]);
    qm31 res = qm_add(qm_make(reduce64(acc[0]), reduce64(acc[1]), reduce64(acc[2]), reduce64(acc[3])), qm_mul(pl, lc));
    uint32_t dinv = prm.denom_inv[r >> trace_log];
    uint32_t v[4] = {mul(res.x.a, dinv), mul(res.x.b, dinv), mul(res.y.a, dinv), mul(res.y.b, dinv)};
    store_quotient(out, r, v, accumulate);
  }
}

static unsigned grid_rows(size_t n, int threads) {
  size_t b = (n + threads - 1) / threads;
  size_t cap = (size_t)num_sms() * 32;
  return (unsigned)(b < cap ? (b ? b : 1) : cap);
}

int wf_trace(cudaStream_t st, uint32_t* cols, uint32_t log_n, uint32_t n_cols, uint64_t seed, uint32_t mode) {
  GS_REQUIRE(n_cols >= 2 && log_n <= 28, "bad wide fibonacci shape");
  wf_trace_kernel<<<grid_rows((size_t)1 << log_n, 256), 256, 0, st>>>(cols, log_n, n_cols, seed, mode);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

int wf_constraints(cudaStream_t st, const uint32_t* cols, uint32_t n_cols, uint32_t eval_log, uint32_t trace_log,
                   const ConstraintParams& prm, Planes out) {
  GS_REQUIRE(n_cols >= 3 && n_cols - 2 <= MAX_CONSTRAINTS, "bad wide fibonacci width");
  wf_constraints_kernel<<<grid_rows((size_t)1 << eval_log, 256), 256, 0, st>>>(
      ContigCols{cols, (size_t)1 << eval_log}, n_cols, eval_log, trace_log, prm, out, 0u);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

int wf_constraints_table(cudaStream_t st, const uint32_t* const* d_cols, uint32_t n_cols, uint32_t eval_log,
                         uint32_t trace_log, const ConstraintParams& prm, Planes out, bool accumulate) {
  GS_REQUIRE(n_cols >= 3 && n_cols - 2 <= MAX_CONSTRAINTS, "bad wide fibonacci width");
  GS_REQUIRE(eval_log > trace_log && eval_log - trace_log <= 3 && eval_log <= 30, "bad domain sizes");
  wf_constraints_kernel<<<grid_rows((size_t)1 << eval_log, 256), 256, 0, st>>>(
      TableCols{d_cols}, n_cols, eval_log, trace_log, prm, out, accumulate ? 1u : 0u);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

int poseidon_trace(cudaStream_t st, uint32_t* cols, uint32_t log_n, uint64_t seed, uint32_t mode) {
  GS_REQUIRE(log_n <= 28, "bad poseidon size");
  poseidon_trace_kernel<<<grid_rows((size_t)1 << log_n, 128), 128, 0, st>>>(cols, log_n, seed, mode);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

size_t logup_scratch_bytes(uint32_t log_n) {
  size_t n = (size_t)1 << log_n;
  size_t temp = 0;
  cub::DeviceScan::InclusiveScan(nullptr, temp, (const uint4*)nullptr, (uint4*)nullptr, AddQM(), (int)n);
  return 2 * n * sizeof(uint4) + ((temp + 255) & ~(size_t)255);
}

const void* logup_claimed_sum_ptr(const void* scratch, uint32_t log_n) {
  return (const uint4*)scratch + 2 * ((size_t)1 << log_n) - 1;
}

// The interaction trace from the 16 initial- and final-state columns (given
// as accessors), written to 4 planes, and the claimed sum (host; with
// claimed_sum null it is left on the device, at logup_claimed_sum_ptr).
// scratch: logup_scratch_bytes(log_n).
template <class InitCols, class FinalCols>
static int interaction_impl(cudaStream_t st, InitCols init, uint32_t c_init, FinalCols fin, uint32_t c_final,
                            uint32_t log_n, const LookupParams& lp, Planes out, void* scratch, qm31* claimed_sum,
                            void* h_pinned) {
  size_t n = (size_t)1 << log_n;
  uint4* vals = (uint4*)scratch;
  uint4* scan = vals + n;
  void* temp = (void*)(scan + n);
  size_t temp_bytes = 0;
  cub::DeviceScan::InclusiveScan(nullptr, temp_bytes, (const uint4*)nullptr, (uint4*)nullptr, AddQM(), (int)n);
  logup_fraction_kernel<<<grid_rows(n, 128), 128, 0, st>>>(init, c_init, fin, c_final, log_n, lp, vals);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  GS_CUDA_TRY(cub::DeviceScan::InclusiveScan(temp, temp_bytes, (const uint4*)vals, scan, AddQM(), (int)n, st));
  note_launch();
  logup_finalize_kernel<<<grid_rows(n, 256), 256, 0, st>>>(scan, log_n, inv((uint32_t)(n % P)), out);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  if (claimed_sum) {
    uint4 local;
    uint4* ht = h_pinned ? (uint4*)h_pinned : &local;  // pinned when the caller has a mailbox
    GS_CUDA_TRY(cudaMemcpyAsync(ht, scan + (n - 1), sizeof(uint4), cudaMemcpyDeviceToHost, st));
    GS_TRY(stream_sync(st));
    const uint4 total = *ht;
    *claimed_sum = qm_make(total.x, total.y, total.z, total.w);
  }
  return OK;
}

// Interaction column: writes the 4 coordinate columns (out, 4 x 2^log_n) and
// the claimed sum (host). scratch: logup_scratch_bytes(log_n).
int poseidon_interaction(cudaStream_t st, const uint32_t* trace, uint32_t log_n, const LookupParams& lp,
                         uint32_t* out, void* scratch, qm31* claimed_sum, void* h_pinned) {
  const size_t n = (size_t)1 << log_n;
  ContigCols t{trace, n};
  return interaction_impl(st, t, 0, t, 158 - 16, log_n, lp, Planes{{out, out + n, out + 2 * n, out + 3 * n}},
                          scratch, claimed_sum, h_pinned);
}

int poseidon_interaction_table(cudaStream_t st, const uint32_t* const* d_init, const uint32_t* const* d_final,
                               uint32_t log_n, const LookupParams& lp, Planes out, void* scratch,
                               qm31* claimed_sum) {
  GS_REQUIRE(log_n >= 1 && log_n <= 28, "bad poseidon size");
  return interaction_impl(st, TableCols{d_init}, 0, TableCols{d_final}, 0, log_n, lp, out, scratch, claimed_sum,
                          nullptr);
}

// generate_wide_fibonacci_trace / generate_poseidon_traces (the reference's
// CUDA trace generation, evaluate_wide_fibonacci.cu:127-179,
// evaluate_poseidon_constraint.cu:270-363) into columns given by device
// pointer tables: Wide-Fibonacci from the inputs a, b; Poseidon2 with the
// reference's input rule (row + i), also writing the 16 initial- and
// final-state lookup columns.
__global__ void wf_trace_table_kernel(const uint32_t* __restrict__ in_a, const uint32_t* __restrict__ in_b, size_t n,
                                      uint32_t* const* __restrict__ cols, uint32_t n_cols) {
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
    uint32_t a = __ldg(in_a + r), b = __ldg(in_b + r);
    cols[0][r] = a;
    cols[1][r] = b;
    for (uint32_t k = 2; k < n_cols; k++) {
      uint32_t c = add(sqr(a), sqr(b));
      cols[k][r] = c;
      a = b;
      b = c;
    }
  }
}

__global__ void poseidon_trace_table_kernel(uint32_t* const* __restrict__ cols, uint32_t* const* __restrict__ init,
                                            uint32_t* const* __restrict__ fin, size_t n) {
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
    uint32_t s[16];
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) {
      s[i] = (uint32_t)((r + i) % P);
      cols[c++][r] = s[i];
      init[i][r] = s[i];
    }
    for (int round = 0; round < 4; round++) {
#pragma unroll
      for (int i = 0; i < 16; i++) s[i] = add(s[i], PN_RC);
      p2_external(s);
#pragma unroll
      for (int i = 0; i < 16; i++) {
        s[i] = pow5(s[i]);
        cols[c++][r] = s[i];
      }
    }
    for (int round = 0; round < 14; round++) {
      s[0] = add(s[0], PN_RC);
      p2_internal(s);
      s[0] = pow5(s[0]);
      cols[c++][r] = s[0];
    }
    for (int round = 0; round < 4; round++) {
#pragma unroll
      for (int i = 0; i < 16; i++) s[i] = add(s[i], PN_RC);
      p2_external(s);
#pragma unroll
      for (int i = 0; i < 16; i++) {
        s[i] = pow5(s[i]);
        cols[c++][r] = s[i];
        if (round == 3) fin[i][r] = s[i];
      }
    }
  }
}

int wf_trace_table(cudaStream_t st, const uint32_t* in_a, const uint32_t* in_b, uint32_t log_n,
                   uint32_t* const* d_cols, uint32_t n_cols) {
  GS_REQUIRE(n_cols >= 2 && log_n <= 28, "bad wide fibonacci shape");
  const size_t n = (size_t)1 << log_n;
  wf_trace_table_kernel<<<grid_rows(n, 256), 256, 0, st>>>(in_a, in_b, n, d_cols, n_cols);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

int poseidon_trace_table(cudaStream_t st, uint32_t* const* d_cols, uint32_t* const* d_init, uint32_t* const* d_final,
                         uint32_t log_n) {
  GS_REQUIRE(log_n <= 28, "bad poseidon size");
  const size_t n = (size_t)1 << log_n;
  poseidon_trace_table_kernel<<<grid_rows(n, 128), 128, 0, st>>>(d_cols, d_init, d_final, n);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

int poseidon_constraints(cudaStream_t st, const uint32_t* trace, const uint32_t* inter, uint32_t eval_log,
                         uint32_t trace_log, const ConstraintParams& prm, const LookupParams& lp, qm31 cumsum_shift,
                         Planes out) {
  GS_REQUIRE(eval_log > trace_log, "poseidon constraints need an extended domain");
  const size_t n = (size_t)1 << eval_log;
  poseidon_constraints_kernel<<<grid_rows(n, 128), 128, 0, st>>>(ContigCols{trace, n}, ContigCols{inter, n}, eval_log,
                                                                  trace_log, prm, lp, cumsum_shift, out, 0u);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

int poseidon_constraints_table(cudaStream_t st, const uint32_t* const* d_trace, const uint32_t* const* d_inter,
                               uint32_t eval_log, uint32_t trace_log, const ConstraintParams& prm,
                               const LookupParams& lp, qm31 cumsum_shift, Planes out, bool accumulate) {
  GS_REQUIRE(eval_log > trace_log && eval_log - trace_log <= 3 && eval_log <= 30, "bad domain sizes");
  poseidon_constraints_kernel<<<grid_rows((size_t)1 << eval_log, 128), 128, 0, st>>>(
      TableCols{d_trace}, TableCols{d_inter}, eval_log, trace_log, prm, lp, cumsum_shift, out, accumulate ? 1u : 0u);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

}  // namespace gs
