// Batched circle FFT (interpolate / evaluate) over M31 columns.
//
// Semantics: crates/stwo/src/prover/backend/cpu/circle.rs:28-80 (interpolate)
// and :182-228 (evaluate). Layer i pairs index v with v + 2^i and uses the
// twiddle of group h = v >> (i + 1):
//   line layer i >= 1:  buf[L - 2^(n-i) + h]           (domain_line_twiddles_from_tree)
//   circle layer i = 0: from the first line slice T0,  h = 4q + r ->
//                       [T0[2q+1], -T0[2q+1], -T0[2q], T0[2q]][r]
// with buf = itwiddles for interpolation and twiddles for evaluation, L the
// twiddle buffer length. Interpolation runs layers 0..n-1 then scales by
// 1/2^n; evaluation runs layers n-1..0.
//
// Kernel design: a pass loads a tile of 2^(cnt+c) elements into shared
// memory, runs `cnt` consecutive layers there and writes the tile back. A
// tile keeps the c lowest index bits contiguous (64-byte runs with c = 4) so
// that strided passes still read whole DRAM sectors. Columns of one size are
// batched in a single launch (grid.y = column). The 1/2^n scale is fused
// into the store of the last interpolation pass.
//
// Low-degree extension (evaluate 2^m coefficients on a 2^n domain): the top
// n-m layers of the zero-padded forward FFT only copy (butterfly with a zero
// partner), so the first pass reads src[v mod 2^m] and only layers m-1..0
// are computed — the zero-extension pass of the reference disappears.
#include "runtime.cuh"
#include <algorithm>
#include <cstdlib>

namespace gs {

struct FftPass {
  uint32_t n;         // domain log size
  uint32_t lo, cnt;   // layers [lo, lo + cnt)
  uint32_t c;         // contiguous low index bits kept per tile (c <= lo)
  uint32_t src_mask;  // read src[v & src_mask] (LDE replication)
  uint32_t tw_len;    // twiddle buffer length
  uint32_t scale;     // multiply by scale on store when has_scale
  uint32_t has_scale;
};

__device__ __forceinline__ uint32_t fft_twiddle(const uint32_t* __restrict__ tw, uint32_t tw_len, uint32_t n,
                                                uint32_t i, uint32_t h) {
  if (i >= 1) return __ldg(tw + (tw_len - (1u << (n - i)) + h));
  uint32_t base = tw_len - (1u << (n - 1));
  uint32_t q = h >> 2, r = h & 3u;
  uint32_t x = __ldg(tw + base + 2 * q + (r < 2 ? 1u : 0u));
  return (r == 1 || r == 2) ? neg(x) : x;
}

template <bool INV>
__global__ void __launch_bounds__(512) fft_pass_kernel(const uint32_t* const* __restrict__ src_tab,
                                                       uint32_t* const* __restrict__ dst_tab,
                                                       const uint32_t* __restrict__ tw, FftPass a) {
  extern __shared__ uint32_t sm[];
  const uint32_t col = blockIdx.y;
  const uint32_t* __restrict__ src = src_tab[col];
  uint32_t* __restrict__ dst = dst_tab[col];
  const uint32_t t = a.cnt + a.c;
  const uint32_t tile = 1u << t;
  const uint32_t ml_bits = a.lo - a.c;
  const uint32_t midlow = blockIdx.x & ((1u << ml_bits) - 1u);
  const uint32_t hi = blockIdx.x >> ml_bits;
  const uint32_t cmask = (1u << a.c) - 1u;
  const uint32_t base = (hi << (a.lo + a.cnt)) | (midlow << a.c);

  for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) {
    uint32_t v = base | ((e >> a.c) << a.lo) | (e & cmask);
    sm[e] = src[v & a.src_mask];
  }
  __syncthreads();

  for (uint32_t k = 0; k < a.cnt; k++) {
    const uint32_t li = INV ? k : (a.cnt - 1 - k);
    const uint32_t i = a.lo + li;
    const uint32_t s = li + a.c;
    const uint32_t smask = (1u << s) - 1u;
    for (uint32_t b = threadIdx.x; b < (tile >> 1); b += blockDim.x) {
      uint32_t e0 = ((b & ~smask) << 1) | (b & smask);
      uint32_t e1 = e0 | (1u << s);
      uint32_t v0 = base | ((e0 >> a.c) << a.lo) | (e0 & cmask);
      uint32_t w = fft_twiddle(tw, a.tw_len, a.n, i, v0 >> (i + 1));
      uint32_t x0 = sm[e0], x1 = sm[e1];
      if (INV) {
        sm[e0] = add(x0, x1);
        sm[e1] = mul(sub(x0, x1), w);
      } else {
        uint32_t tmp = mul(x1, w);
        sm[e0] = add(x0, tmp);
        sm[e1] = sub(x0, tmp);
      }
    }
    __syncthreads();
  }

  for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) {
    uint32_t v = base | ((e >> a.c) << a.lo) | (e & cmask);
    uint32_t x = sm[e];
    if (a.has_scale) x = mul(x, a.scale);
    dst[v] = x;
  }
}

// Domains of log size 1 and 2: closed forms of cpu/circle.rs:37-60 and
// :193-208, with constants precomputed on the host.
struct SmallFft {
  uint32_t n;
  uint32_t inverse;
  uint32_t k[4];
  uint32_t src_mask;
};
__global__ void fft_small_kernel(const uint32_t* const* src_tab, uint32_t* const* dst_tab, SmallFft a, uint32_t n_cols) {
  uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n_cols) return;
  const uint32_t* s = src_tab[col];
  uint32_t* d = dst_tab[col];
  if (a.n == 1) {
    uint32_t v0 = s[0], v1 = s[1 & a.src_mask];
    if (a.inverse) {  // k = {y_inv, n_inv}
      uint32_t r0 = add(v0, v1), r1 = mul(sub(v0, v1), a.k[0]);
      d[0] = mul(r0, a.k[1]);
      d[1] = mul(r1, a.k[1]);
    } else {  // k = {y}
      uint32_t tmp = mul(v1, a.k[0]);
      d[0] = add(v0, tmp);
      d[1] = sub(v0, tmp);
    }
  } else {
    uint32_t v0 = s[0], v1 = s[1 & a.src_mask], v2 = s[2 & a.src_mask], v3 = s[3 & a.src_mask];
    if (a.inverse) {  // k = {x_inv, y_inv, n_inv}
      auto ib = [](uint32_t& p, uint32_t& q, uint32_t w) { uint32_t t0 = p; p = add(t0, q); q = mul(sub(t0, q), w); };
      ib(v0, v1, a.k[1]);
      ib(v2, v3, neg(a.k[1]));
      ib(v0, v2, a.k[0]);
      ib(v1, v3, a.k[0]);
      d[0] = mul(v0, a.k[2]); d[1] = mul(v1, a.k[2]); d[2] = mul(v2, a.k[2]); d[3] = mul(v3, a.k[2]);
    } else {  // k = {x, y}
      auto fb = [](uint32_t& p, uint32_t& q, uint32_t w) { uint32_t t0 = mul(q, w); q = sub(p, t0); p = add(p, t0); };
      fb(v0, v2, a.k[0]);
      fb(v1, v3, a.k[0]);
      fb(v0, v1, a.k[1]);
      fb(v2, v3, neg(a.k[1]));
      d[0] = v0; d[1] = v1; d[2] = v2; d[3] = v3;
    }
  }
}

// Host-side circle point at a circle index (double-and-add on the host).
static pt31 host_index_to_point(uint32_t k) {
  pt31 r = {1u, 0u}, cur = {2u, 1268011823u};
  for (int b = 0; b < 31; b++) {
    if ((k >> b) & 1u) r = pt_add(r, cur);
    cur = pt_add(cur, cur);
  }
  return r;
}
// Initial point of the half coset of CanonicCoset(n): index 2^(31 - (n + 1)).
static pt31 canonic_half_coset_initial(uint32_t n) { return host_index_to_point(1u << (31 - (n + 1))); }

static int launch_small(cudaStream_t st, const uint32_t* const* src, uint32_t* const* dst, uint32_t n_cols, uint32_t n,
                        bool inverse, uint32_t src_mask) {
  pt31 p = canonic_half_coset_initial(n);
  SmallFft a{};
  a.n = n;
  a.inverse = inverse;
  a.src_mask = src_mask;
  if (n == 1) {
    if (inverse) {
      uint32_t yn_inv = inv(mul(p.y, 2));
      a.k[0] = mul(yn_inv, 2);     // y_inv
      a.k[1] = mul(yn_inv, p.y);   // n_inv
    } else {
      a.k[0] = p.y;
    }
  } else {
    if (inverse) {
      uint32_t xyn_inv = inv(mul(mul(p.x, p.y), 4));
      a.k[0] = mul(mul(xyn_inv, p.y), 4);  // x_inv
      a.k[1] = mul(mul(xyn_inv, p.x), 4);  // y_inv
      a.k[2] = mul(mul(xyn_inv, p.x), p.y);  // n_inv
    } else {
      a.k[0] = p.x;
      a.k[1] = p.y;
    }
  }
  uint32_t threads = 128;
  fft_small_kernel<<<(n_cols + threads - 1) / threads, threads, 0, st>>>(src, dst, a, n_cols);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

struct FftTuning {
  uint32_t tile_log = 12;      // log2 of shared-memory tile (elements)
  uint32_t coalesce_bits = 4;  // contiguous low bits per strided tile row
};
static FftTuning g_fft_tuning;

static void fft_partition(uint32_t layers, std::vector<std::pair<uint32_t, uint32_t>>& parts) {
  // Splits layers [0, layers) into passes (lo, cnt): the first pass keeps the
  // whole tile for layers; later ones reserve `coalesce_bits` of the tile.
  const uint32_t T = g_fft_tuning.tile_log, C = g_fft_tuning.coalesce_bits;
  uint32_t lo = 0;
  while (lo < layers) {
    uint32_t c = std::min(C, lo);
    uint32_t cnt = std::min(layers - lo, T - c);
    parts.push_back({lo, cnt});
    lo += cnt;
  }
}

template <bool INV>
static int run_passes(cudaStream_t st, const uint32_t* const* src, uint32_t* const* dst, uint32_t n_cols, uint32_t n,
                      uint32_t layers, uint32_t src_mask, const uint32_t* tw, uint32_t tw_len) {
  std::vector<std::pair<uint32_t, uint32_t>> parts;
  fft_partition(layers, parts);
  if (!INV) std::reverse(parts.begin(), parts.end());
  for (size_t p = 0; p < parts.size(); p++) {
    FftPass a{};
    a.n = n;
    a.lo = parts[p].first;
    a.cnt = parts[p].second;
    a.c = std::min(g_fft_tuning.coalesce_bits, a.lo);
    a.src_mask = (p == 0) ? src_mask : 0xffffffffu;
    a.tw_len = tw_len;
    a.has_scale = (INV && p + 1 == parts.size()) ? 1u : 0u;
    a.scale = a.has_scale ? inv(1u << n) : 1u;
    uint32_t t = a.cnt + a.c;
    uint32_t tiles = 1u << (n - t);
    uint32_t threads = std::min<uint32_t>(512, std::max<uint32_t>(32, 1u << (t - 1)));
    size_t smem = sizeof(uint32_t) << t;
    dim3 grid(tiles, n_cols);
    const uint32_t* const* s = (p == 0) ? src : (const uint32_t* const*)dst;
    fft_pass_kernel<INV><<<grid, threads, smem, st>>>(s, dst, tw, a);
    note_launch();
    GS_CUDA_TRY(cudaGetLastError());
  }
  return OK;
}

int interpolate_columns(cudaStream_t st, uint32_t* const* d_cols, uint32_t n_cols, uint32_t log_n,
                        const uint32_t* d_itwiddles, uint32_t tw_log) {
  if (n_cols == 0) return OK;
  GS_REQUIRE(log_n >= 1 && log_n <= 30, "log_n out of range");
  GS_REQUIRE(n_cols <= 65535, "too many columns in one call");
  if (log_n <= 2) return launch_small(st, (const uint32_t* const*)d_cols, d_cols, n_cols, log_n, true, 0xffffffffu);
  GS_REQUIRE(tw_log + 1 >= log_n, "twiddle tree too small for the domain");
  return run_passes<true>(st, (const uint32_t* const*)d_cols, d_cols, n_cols, log_n, log_n, 0xffffffffu, d_itwiddles,
                          1u << tw_log);
}

int evaluate_columns(cudaStream_t st, const uint32_t* const* d_src, uint32_t coeff_log, uint32_t* const* d_dst,
                     uint32_t n_cols, uint32_t log_n, const uint32_t* d_twiddles, uint32_t tw_log) {
  if (n_cols == 0) return OK;
  GS_REQUIRE(log_n >= 1 && log_n <= 30, "log_n out of range");
  GS_REQUIRE(coeff_log >= 1 && coeff_log <= log_n, "coefficient log size must be in [1, log_n]");
  GS_REQUIRE(n_cols <= 65535, "too many columns in one call");
  uint32_t src_mask = (1u << coeff_log) - 1u;
  if (log_n <= 2) return launch_small(st, d_src, d_dst, n_cols, log_n, false, src_mask);
  GS_REQUIRE(tw_log + 1 >= log_n, "twiddle tree too small for the domain");
  return run_passes<false>(st, d_src, d_dst, n_cols, log_n, coeff_log, src_mask, d_twiddles, 1u << tw_log);
}

void set_fft_tuning(uint32_t tile_log, uint32_t coalesce_bits) {
  if (tile_log >= 4 && tile_log <= 13) g_fft_tuning.tile_log = tile_log;
  if (coalesce_bits <= 6 && coalesce_bits + 2 <= g_fft_tuning.tile_log) g_fft_tuning.coalesce_bits = coalesce_bits;
}

// In-place bit reversal of one column (ColumnOps::bit_reverse_column).
__global__ void bit_reverse_kernel(uint32_t* d, uint32_t log_n) {
  uint32_t n = 1u << log_n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t j = __brev(i) >> (32 - log_n);
    if (j > i) {
      uint32_t a = d[i];
      d[i] = d[j];
      d[j] = a;
    }
  }
}
int bit_reverse(cudaStream_t st, uint32_t* d, uint32_t log_n) {
  GS_REQUIRE(log_n <= 31, "log_n out of range");
  if (log_n == 0) return OK;
  uint32_t n = 1u << log_n;
  int blocks = (int)std::min<uint32_t>((n + 255) / 256, (uint32_t)num_sms() * 16);
  bit_reverse_kernel<<<blocks, 256, 0, st>>>(d, log_n);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

}  // namespace gs
