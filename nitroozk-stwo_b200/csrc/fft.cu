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
// Kernel design (radix-2^R in registers): a pass covers L consecutive layers
// on tiles of 2^t = 2^(c+L) elements. Each thread holds 2^R elements (R = 5:
// 32 registers) whose tile indices differ in an R-bit window and runs up to R
// layers on them with compile-time indexing; stages exchange data through
// shared memory with an XOR swizzle (bank = e[0:5] ^ e[5:10]) that keeps
// every access pattern bank-conflict free. The twiddles a thread needs for
// one layer are consecutive and aligned in the tree, so they arrive as a few
// 16-byte loads. A tile keeps its c lowest index bits contiguous in global
// memory (64-byte runs with c = 4) so strided passes read whole sectors.
// Columns of one size are batched in one launch (grid.y = column). The 1/2^n
// scale is fused into the final store of the interpolation.
//
// Low-degree extension (evaluate 2^m coefficients on a 2^n domain): the top
// n-m layers of the zero-padded forward FFT only copy (butterfly with a zero
// partner), so the first pass reads src[v mod 2^m] and only layers m-1..0
// are computed — no zero-extension pass.
#include "runtime.cuh"
#include <algorithm>
#include <vector>
#include <iterator>
#include <cstdlib>

namespace gs {

struct FftPass {
  uint32_t n;           // domain log size
  uint32_t lo, L;       // layers [lo, lo + L)
  uint32_t c;           // contiguous low index bits kept per tile (c <= lo)
  uint32_t t;           // tile log size = c + L
  uint32_t K;           // register stages
  uint32_t tile_shift;  // log2(tiles per block)
  uint32_t src_mask;    // read src[v & src_mask] (LDE replication)
  uint32_t tw_len;      // twiddle buffer length
  uint32_t scale;       // multiply by scale on the final store when has_scale
  uint32_t has_scale;
  uint32_t vec_ok;      // all column pointers 16-byte aligned: vector loads/stores allowed
};

__device__ __forceinline__ uint32_t circle_twiddle(const uint32_t* __restrict__ tw, uint32_t tw_len, uint32_t n,
                                                   uint32_t h) {
  uint32_t base = tw_len - (1u << (n - 1));
  uint32_t q = h >> 2, r = h & 3u;
  uint32_t x = __ldg(tw + base + 2 * q + (r < 2 ? 1u : 0u));
  return (r == 1 || r == 2) ? neg(x) : x;
}

// COUNT consecutive twiddles of layer i starting at group hth (aligned to COUNT).
template <int COUNT>
__device__ __forceinline__ void load_twiddles(uint32_t* w, const uint32_t* __restrict__ tw, uint32_t tw_len,
                                              uint32_t n, uint32_t i, uint32_t hth) {
  if (i >= 1) {
    const uint32_t* p = tw + (tw_len - (1u << (n - i)) + hth);
    if (COUNT >= 4) {
#pragma unroll
      for (int g = 0; g < COUNT / 4; g++) {
        uint4 v = __ldg(reinterpret_cast<const uint4*>(p) + g);
        w[4 * g] = v.x; w[4 * g + 1] = v.y; w[4 * g + 2] = v.z; w[4 * g + 3] = v.w;
      }
    } else if (COUNT == 2) {
      uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
      w[0] = v.x; w[1] = v.y;
    } else {
      w[0] = __ldg(p);
    }
  } else {
    if (COUNT >= 4) {
      const uint32_t* t0 = tw + (tw_len - (1u << (n - 1)));
#pragma unroll
      for (int g = 0; g < COUNT / 4; g++) {
        uint2 xy = __ldg(reinterpret_cast<const uint2*>(t0) + (hth >> 2) + g);
        w[4 * g] = xy.y; w[4 * g + 1] = neg(xy.y); w[4 * g + 2] = neg(xy.x); w[4 * g + 3] = xy.x;
      }
    } else {
#pragma unroll
      for (int g = 0; g < COUNT; g++) w[g] = circle_twiddle(tw, tw_len, n, hth + g);
    }
  }
}

template <bool INV>
__device__ __forceinline__ void bfly(uint32_t& a, uint32_t& b, uint32_t w) {
  if (INV) {
    uint32_t t0 = a;
    a = add(t0, b);
    b = mul(sub(t0, b), w);
  } else {
    uint32_t t0 = mul(b, w);
    b = sub(a, t0);
    a = add(a, t0);
  }
}

// XOR swizzle over the block's shared-memory index (tile offset included, so
// blocks holding several small tiles stay conflict free as well).
__device__ __forceinline__ uint32_t swz(uint32_t e) { return e ^ ((e >> 5) & 31u); }

template <bool INV, int R>
__global__ void __launch_bounds__(256) fft_pass_kernel(const uint32_t* const* __restrict__ src_tab,
                                                       uint32_t* const* __restrict__ dst_tab,
                                                       const uint32_t* __restrict__ tw, FftPass a) {
  extern __shared__ uint32_t sm[];
  constexpr int NQ = 1 << R;
  const uint32_t col = blockIdx.y;
  const uint32_t* __restrict__ src = src_tab[col];
  uint32_t* __restrict__ dst = dst_tab[col];
  const uint32_t tpt_log = a.t - R;
  const uint32_t ltid = threadIdx.x & ((1u << tpt_log) - 1u);
  const uint32_t sub_tile = threadIdx.x >> tpt_log;
  const uint32_t tile = (blockIdx.x << a.tile_shift) | sub_tile;
  const uint32_t smbase = sub_tile << a.t;  // swizzled together with the tile index
  const uint32_t ml = a.lo - a.c;
  const uint32_t midlow = tile & ((1u << ml) - 1u);
  const uint32_t hi = tile >> ml;
  const uint32_t cmask = (1u << a.c) - 1u;
  const uint32_t basev = (hi << (a.lo + a.L)) | (midlow << a.c);
  uint32_t x[NQ];

  for (uint32_t k = 0; k < a.K; k++) {
    uint32_t s0, ja, jb;
    if (INV) {
      if (k + 1 < a.K) { s0 = a.c + k * R; ja = 0; jb = R; }
      else { s0 = a.t - R; ja = a.c + k * R - s0; jb = R; }
    } else {
      if (k + 1 < a.K) { s0 = a.t - (k + 1) * R; ja = 0; jb = R; }
      else { s0 = a.c; ja = 0; jb = a.t - k * R - a.c; }
    }
    const uint32_t ebase = ((ltid >> s0) << (s0 + R)) | (ltid & ((1u << s0) - 1u));
    if (k == 0) {
      // the tile's elements are contiguous only when it starts at layer 0
      if (a.vec_ok && s0 == 0 && a.c == 0 && a.lo == 0 && a.src_mask == 0xffffffffu && NQ >= 4) {
        const uint4* p = reinterpret_cast<const uint4*>(src + (basev | ebase));
#pragma unroll
        for (int g = 0; g < NQ / 4; g++) {
          uint4 v = __ldg(p + g);
          x[4 * g] = v.x; x[4 * g + 1] = v.y; x[4 * g + 2] = v.z; x[4 * g + 3] = v.w;
        }
      } else {
#pragma unroll
        for (int q = 0; q < NQ; q++) {
          uint32_t e = ebase | ((uint32_t)q << s0);
          uint32_t v = basev | ((e >> a.c) << a.lo) | (e & cmask);
          x[q] = __ldg(src + (v & a.src_mask));
        }
      }
    } else {
      __syncthreads();
#pragma unroll
      for (int q = 0; q < NQ; q++) x[q] = sm[swz(smbase | ebase | ((uint32_t)q << s0))];
      __syncthreads();
    }
    const uint32_t vth = basev | ((ebase >> a.c) << a.lo) | (ebase & cmask);
#pragma unroll
    for (int jj = 0; jj < R; jj++) {
      const int j = INV ? jj : (R - 1 - jj);
      if ((uint32_t)j < ja || (uint32_t)j >= jb) continue;
      const uint32_t i = a.lo + s0 + (uint32_t)j - a.c;
      const uint32_t hth = vth >> (i + 1);
      constexpr int MAXW = NQ / 2;
      uint32_t w[MAXW];
      // COUNT = 2^(R-1-j), resolved at compile time after unrolling
      switch (R - 1 - j) {
        case 0: load_twiddles<1>(w, tw, a.tw_len, a.n, i, hth); break;
        case 1: load_twiddles<2>(w, tw, a.tw_len, a.n, i, hth); break;
        case 2: load_twiddles<4>(w, tw, a.tw_len, a.n, i, hth); break;
        case 3: load_twiddles<8>(w, tw, a.tw_len, a.n, i, hth); break;
        default: load_twiddles<16>(w, tw, a.tw_len, a.n, i, hth); break;
      }
#pragma unroll
      for (int q = 0; q < NQ; q++) {
        if (q & (1 << j)) continue;
        bfly<INV>(x[q], x[q | (1 << j)], w[q >> (j + 1)]);
      }
    }
    if (k + 1 < a.K) {
#pragma unroll
      for (int q = 0; q < NQ; q++) sm[swz(smbase | ebase | ((uint32_t)q << s0))] = x[q];
    } else {
      if (a.has_scale) {
#pragma unroll
        for (int q = 0; q < NQ; q++) x[q] = mul(x[q], a.scale);
      }
      if (a.vec_ok && s0 == 0 && a.c == 0 && a.lo == 0 && NQ >= 4) {
        uint4* p = reinterpret_cast<uint4*>(dst + (basev | ebase));
#pragma unroll
        for (int g = 0; g < NQ / 4; g++) p[g] = make_uint4(x[4 * g], x[4 * g + 1], x[4 * g + 2], x[4 * g + 3]);
      } else {
#pragma unroll
        for (int q = 0; q < NQ; q++) {
          uint32_t e = ebase | ((uint32_t)q << s0);
          uint32_t v = basev | ((e >> a.c) << a.lo) | (e & cmask);
          dst[v] = x[q];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Geometry-specialised pass: the same index mapping as fft_pass_kernel with
// L (layers) and C (contiguous low bits) fixed at compile time, so every
// stage's window, shift and shared-memory offset is a constant:
//  * shared memory is padded (word e at e + e/32) instead of XOR-swizzled;
//    for disjoint bit fields the padding is additive, so the offset of
//    element q folds into the load/store's immediate and each access costs
//    no address arithmetic — and every access pattern of the pass stays
//    bank-conflict free (bank = lane);
//  * the first add of every field add/sub is an IMAD with a runtime 1 / -1
//    (the integer ALU pipe is the bottleneck of the butterfly; IMAD runs on
//    the FMA pipe), leaving one add-then-min (VIADDMNMX) per add/sub on the
//    ALU pipe.
// ---------------------------------------------------------------------------
// (imad_u32, add_f, sub_f: m31.cuh)
template <bool INV>
__device__ __forceinline__ void bfly_f(uint32_t& a, uint32_t& b, uint32_t w, uint32_t one, uint32_t neg1) {
  if (INV) {
    uint32_t t0 = a;
    a = add_f(t0, b, one);
    b = mul(sub_f(t0, b, neg1), w);
  } else {
    uint32_t t0 = mul(b, w);
    b = sub_f(a, t0, neg1);
    a = add_f(a, t0, one);
  }
}
__host__ __device__ constexpr uint32_t padw(uint32_t e) { return e + (e >> 5); }

template <bool INV, int L, int C>
__global__ void __launch_bounds__(256) fft_tile_kernel(const uint32_t* const* __restrict__ src_tab,
                                                       uint32_t* const* __restrict__ dst_tab,
                                                       const uint32_t* __restrict__ tw, FftPass a, uint32_t one,
                                                       uint32_t neg1) {
  extern __shared__ uint32_t sm[];
  constexpr int R = 5, NQ = 32;
  constexpr int T = L + C;
  constexpr int K = (L + R - 1) / R;
  constexpr int TPT_LOG = T - R;
  constexpr uint32_t CMASK = (1u << C) - 1u;
  const uint32_t col = blockIdx.y;
  const uint32_t* __restrict__ src = src_tab[col];
  uint32_t* __restrict__ dst = dst_tab[col];
  const uint32_t ltid = threadIdx.x & ((1u << TPT_LOG) - 1u);
  const uint32_t sub_tile = threadIdx.x >> TPT_LOG;
  const uint32_t tile = (blockIdx.x << a.tile_shift) | sub_tile;
  const uint32_t ml = a.lo - C;
  const uint32_t midlow = tile & ((1u << ml) - 1u);
  const uint32_t hi = tile >> ml;
  const uint32_t basev = (hi << (a.lo + L)) | (midlow << C);
  const uint32_t tile_pad = padw(sub_tile << T);
  uint32_t x[NQ];

#pragma unroll
  for (int k = 0; k < K; k++) {
    const int s0 = INV ? ((k + 1 < K) ? C + k * R : T - R) : ((k + 1 < K) ? T - (k + 1) * R : C);
    const int ja = INV ? ((k + 1 < K) ? 0 : C + k * R - s0) : 0;
    const int jb = INV ? R : ((k + 1 < K) ? R : T - k * R - C);
    const uint32_t ebase = ((ltid >> s0) << (s0 + R)) | (ltid & ((1u << s0) - 1u));
    const uint32_t pbase = tile_pad + padw(ebase);
    // global offset of element q relative to q = 0 (bits of q << s0 above C
    // move up to the pass's layer bits)
    const uint32_t gbase = basev | ((ebase >> C) << a.lo) | (ebase & CMASK);
    if (k == 0) {
      // contiguous only when the tile starts at layer 0 (C == 0 with lo > 0
      // spaces the elements 2^lo apart)
      if (C == 0 && s0 == 0 && a.lo == 0 && a.vec_ok && a.src_mask == 0xffffffffu) {
        const uint4* p = reinterpret_cast<const uint4*>(src + gbase);
#pragma unroll
        for (int g = 0; g < NQ / 4; g++) {
          uint4 v = __ldg(p + g);
          x[4 * g] = v.x; x[4 * g + 1] = v.y; x[4 * g + 2] = v.z; x[4 * g + 3] = v.w;
        }
      } else {
        // s0 >= C in every stage, so element q sits at gbase + q * 2^(s0-C+lo);
        // with the LDE mask, (gbase | off) & mask = (gbase & mask) + (off & mask)
        const uint32_t* p0 = src + (gbase & a.src_mask);
        const uint32_t stride = 1u << (s0 - C + a.lo);
        if (a.src_mask == 0xffffffffu) {
#pragma unroll
          for (int q = 0; q < NQ; q++) x[q] = __ldg(p0 + (size_t)((uint32_t)q * stride));
        } else {
#pragma unroll
          for (int q = 0; q < NQ; q++) x[q] = __ldg(p0 + (((uint32_t)q * stride) & a.src_mask));
        }
      }
    } else {
      __syncthreads();
#pragma unroll
      for (int q = 0; q < NQ; q++) x[q] = sm[pbase + padw((uint32_t)q << s0)];
      __syncthreads();
    }
#pragma unroll
    for (int jj = 0; jj < R; jj++) {
      const int j = INV ? jj : (R - 1 - jj);
      if (j < ja || j >= jb) continue;
      const uint32_t i = a.lo + (uint32_t)(s0 + j - C);
      const uint32_t hth = gbase >> (i + 1);
      uint32_t w[NQ / 2];
      switch (R - 1 - j) {
        case 0: load_twiddles<1>(w, tw, a.tw_len, a.n, i, hth); break;
        case 1: load_twiddles<2>(w, tw, a.tw_len, a.n, i, hth); break;
        case 2: load_twiddles<4>(w, tw, a.tw_len, a.n, i, hth); break;
        case 3: load_twiddles<8>(w, tw, a.tw_len, a.n, i, hth); break;
        default: load_twiddles<16>(w, tw, a.tw_len, a.n, i, hth); break;
      }
#pragma unroll
      for (int q = 0; q < NQ; q++) {
        if (q & (1 << j)) continue;
        bfly_f<INV>(x[q], x[q | (1 << j)], w[q >> (j + 1)], one, neg1);
      }
    }
    if (k + 1 < K) {
#pragma unroll
      for (int q = 0; q < NQ; q++) sm[pbase + padw((uint32_t)q << s0)] = x[q];
    } else {
      if (a.has_scale) {
#pragma unroll
        for (int q = 0; q < NQ; q++) x[q] = mul(x[q], a.scale);
      }
      if (C == 0 && s0 == 0 && a.lo == 0 && a.vec_ok) {
        uint4* p = reinterpret_cast<uint4*>(dst + gbase);
#pragma unroll
        for (int g = 0; g < NQ / 4; g++) p[g] = make_uint4(x[4 * g], x[4 * g + 1], x[4 * g + 2], x[4 * g + 3]);
      } else {
        uint32_t* p0 = dst + gbase;
        const uint32_t stride = 1u << (s0 - C + a.lo);
#pragma unroll
        for (int q = 0; q < NQ; q++) p0[(size_t)((uint32_t)q * stride)] = x[q];
      }
    }
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
    // coefficients beyond 2^coeff_log are zero: these closed forms run every
    // butterfly, so the padding is explicit (the pass kernels skip the copy
    // layers and replicate instead)
    uint32_t v0 = s[0], v1 = 1 <= a.src_mask ? s[1] : 0u;
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
    uint32_t v0 = s[0], v1 = 1 <= a.src_mask ? s[1] : 0u, v2 = 2 <= a.src_mask ? s[2] : 0u,
             v3 = 3 <= a.src_mask ? s[3] : 0u;
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
  uint32_t tile_log = 13;      // log2 of the shared-memory tile (elements), <= 13
  uint32_t coalesce_bits = 4;  // contiguous low bits per strided tile row
};
// Per number of computed layers (an FFT of 2^n, or an LDE from 2^n
// coefficients, computes n layers) and extension (domain log size minus
// layers: 0 for an FFT, the blowup for an LDE; capped at FFT_MAX_EXT). Written
// at set-up (set_fft_tuning, fft_autotune), read by every launch.
constexpr uint32_t FFT_MAX_EXT = 3;
static FftTuning g_fft_tuning[32][FFT_MAX_EXT + 1];
static uint32_t ext_slot(uint32_t layers, uint32_t n) {
  return n - layers < FFT_MAX_EXT ? n - layers : FFT_MAX_EXT;
}
static FftTuning tuning_for(uint32_t layers, uint32_t n) {
  return g_fft_tuning[layers < 32 ? layers : 31][ext_slot(layers, n)];
}

// Splits layers [0, layers) into balanced passes (lo, L): the first pass has
// the whole tile for layers, later ones reserve `coalesce_bits` of it.
static void fft_partition(uint32_t layers, uint32_t n, std::vector<std::pair<uint32_t, uint32_t>>& parts) {
  const FftTuning tn = tuning_for(layers, n);
  const uint32_t T = tn.tile_log, C = tn.coalesce_bits;
  if (layers <= T) {
    parts.push_back({0, layers});
    return;
  }
  uint32_t np = 1 + (layers - T + (T - C) - 1) / (T - C);
  uint32_t lr = std::min(T - C, (layers + np - 1) / np);
  uint32_t l0 = layers - lr * (np - 1);
  parts.push_back({0, l0});
  uint32_t lo = l0;
  for (uint32_t p = 1; p < np; p++) {
    parts.push_back({lo, lr});
    lo += lr;
  }
}

template <bool INV, int R>
static void launch_pass(cudaStream_t st, dim3 grid, uint32_t threads, size_t smem, const uint32_t* const* s,
                        uint32_t* const* d, const uint32_t* tw, const FftPass& a) {
  fft_pass_kernel<INV, R><<<grid, threads, smem, st>>>(s, d, tw, a);
  note_launch();
}

template <bool INV, int L, int C>
static void launch_tile(cudaStream_t st, dim3 grid, uint32_t threads, const uint32_t* const* s, uint32_t* const* d,
                        const uint32_t* tw, const FftPass& a) {
  const uint32_t words = 1u << (a.t + a.tile_shift);
  const size_t smem = (size_t)4 * (words + (words >> 5));
  fft_tile_kernel<INV, L, C><<<grid, threads, smem, st>>>(s, d, tw, a, 1u, 0xffffffffu);
  note_launch();
}

// The specialised kernel covers first passes (C = 0, 5..13 layers) and later
// passes with 16 or 32 contiguous words per tile row (C = 4 with 5..9 layers,
// C = 5 with 5..8); anything else runs the generic pass. GS_FFT_GENERIC=1 forces the generic
// pass (for comparisons).
template <bool INV>
static bool launch_tile_any(cudaStream_t st, dim3 grid, uint32_t threads, const uint32_t* const* s,
                            uint32_t* const* d, const uint32_t* tw, const FftPass& a) {
  static const bool generic = [] {
    const char* e = getenv("GS_FFT_GENERIC");
    return e && e[0] == '1';
  }();
  if (generic) return false;
#define GS_TILE(LL, CC) \
  case LL: launch_tile<INV, LL, CC>(st, grid, threads, s, d, tw, a); return true;
  if (a.c == 0) {
    switch (a.L) { GS_TILE(5, 0) GS_TILE(6, 0) GS_TILE(7, 0) GS_TILE(8, 0) GS_TILE(9, 0) GS_TILE(10, 0)
                   GS_TILE(11, 0) GS_TILE(12, 0) GS_TILE(13, 0) default: return false; }
  }
  if (a.c == 4) {
    switch (a.L) { GS_TILE(5, 4) GS_TILE(6, 4) GS_TILE(7, 4) GS_TILE(8, 4) GS_TILE(9, 4) default: return false; }
  }
  if (a.c == 5) {
    switch (a.L) { GS_TILE(5, 5) GS_TILE(6, 5) GS_TILE(7, 5) GS_TILE(8, 5) default: return false; }
  }
#undef GS_TILE
  return false;
}

// Column pointers of the current call are 16-byte aligned (checked by the
// callers that know them on the host; the device tables are opaque here).
static thread_local bool g_cols_aligned = true;
void fft_set_columns_aligned(bool aligned) { g_cols_aligned = aligned; }

template <bool INV>
static int run_passes(cudaStream_t st, const uint32_t* const* src, uint32_t* const* dst, uint32_t n_cols, uint32_t n,
                      uint32_t layers, uint32_t src_mask, const uint32_t* tw, uint32_t tw_len) {
  std::vector<std::pair<uint32_t, uint32_t>> parts;
  fft_partition(layers, n, parts);
  if (!INV) std::reverse(parts.begin(), parts.end());
  for (size_t p = 0; p < parts.size(); p++) {
    FftPass a{};
    a.n = n;
    a.lo = parts[p].first;
    a.L = parts[p].second;
    a.c = std::min(tuning_for(layers, n).coalesce_bits, a.lo);
    a.t = a.c + a.L;
    const uint32_t R = std::min<uint32_t>(5, a.L);
    a.K = (a.L + R - 1) / R;
    a.src_mask = (p == 0) ? src_mask : 0xffffffffu;
    a.tw_len = tw_len;
    a.has_scale = (INV && p + 1 == parts.size()) ? 1u : 0u;
    a.scale = a.has_scale ? inv(1u << n) : 1u;
    a.vec_ok = g_cols_aligned ? 1u : 0u;
    const uint32_t tpt_log = a.t - R;
    const uint32_t tiles_log = n - a.t;
    uint32_t tile_shift = tpt_log < 7 ? 7 - tpt_log : 0;
    if (tile_shift > tiles_log) tile_shift = tiles_log;
    a.tile_shift = tile_shift;
    const uint32_t threads = 1u << (tpt_log + tile_shift);
    const size_t smem = (size_t)4 << (a.t + tile_shift);
    dim3 grid(1u << (tiles_log - tile_shift), n_cols);
    const uint32_t* const* s = (p == 0) ? src : (const uint32_t* const*)dst;
    if (R == 5 && launch_tile_any<INV>(st, grid, threads, s, dst, tw, a)) {
      GS_CUDA_TRY(cudaGetLastError());
      continue;
    }
    switch (R) {
      case 1: launch_pass<INV, 1>(st, grid, threads, smem, s, dst, tw, a); break;
      case 2: launch_pass<INV, 2>(st, grid, threads, smem, s, dst, tw, a); break;
      case 3: launch_pass<INV, 3>(st, grid, threads, smem, s, dst, tw, a); break;
      case 4: launch_pass<INV, 4>(st, grid, threads, smem, s, dst, tw, a); break;
      default: launch_pass<INV, 5>(st, grid, threads, smem, s, dst, tw, a); break;
    }
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

// Out-of-place interpolation (src and dst tables may differ).
int interpolate_columns_to(cudaStream_t st, const uint32_t* const* d_src, uint32_t* const* d_dst, uint32_t n_cols,
                           uint32_t log_n, const uint32_t* d_itwiddles, uint32_t tw_log) {
  if (n_cols == 0) return OK;
  GS_REQUIRE(log_n >= 1 && log_n <= 30, "log_n out of range");
  GS_REQUIRE(n_cols <= 65535, "too many columns in one call");
  if (log_n <= 2) return launch_small(st, d_src, d_dst, n_cols, log_n, true, 0xffffffffu);
  GS_REQUIRE(tw_log + 1 >= log_n, "twiddle tree too small for the domain");
  return run_passes<true>(st, d_src, d_dst, n_cols, log_n, log_n, 0xffffffffu, d_itwiddles, 1u << tw_log);
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

// ------------------------------------------------------------- work-list
// Device form of an item: the host adds the 1/2^log scale of an
// interpolation.
struct FftWlItem {
  const uint32_t* src;
  uint32_t* dst;
  uint32_t log, coeff_log, inverse, scale;
};

// Persistent grid: block b takes items b, b + gridDim.x, ... of a list sorted
// by decreasing size, so the large items start first. Each item runs whole in
// shared memory: load (an evaluation replicates its 2^coeff_log
// coefficients over the domain, the top layers of the zero-padded FFT being
// copies), the layers with the twiddle rule of the pass kernels (line layer
// i >= 1: tw[tw_len - 2^(log - i) + h]; circle layer 0: circle_twiddle), one
// block barrier per layer, then the store (scaled for an interpolation).
__global__ void __launch_bounds__(256) fft_worklist_kernel(const FftWlItem* __restrict__ items, uint32_t n_items,
                                                           const uint32_t* __restrict__ tw,
                                                           const uint32_t* __restrict__ itw, uint32_t tw_len) {
  extern __shared__ uint32_t sm[];
  for (uint32_t it = blockIdx.x; it < n_items; it += gridDim.x) {
    const FftWlItem w = items[it];
    const uint32_t n = w.log, N = 1u << n;
    const uint32_t cmask = w.inverse ? N - 1u : (1u << w.coeff_log) - 1u;
    for (uint32_t v = threadIdx.x; v < N; v += blockDim.x) sm[v] = __ldg(w.src + (v & cmask));
    __syncthreads();
    const uint32_t* t = w.inverse ? itw : tw;
    const uint32_t layers = w.inverse ? n : w.coeff_log;
    for (uint32_t k = 0; k < layers; k++) {
      const uint32_t i = w.inverse ? k : layers - 1 - k;
      for (uint32_t j = threadIdx.x; j < N / 2; j += blockDim.x) {
        const uint32_t h = j >> i;
        const uint32_t v = (h << (i + 1)) | (j & ((1u << i) - 1u));
        const uint32_t u = v + (1u << i);
        const uint32_t tw_h = i == 0 ? circle_twiddle(t, tw_len, n, h) : __ldg(t + tw_len - (1u << (n - i)) + h);
        const uint32_t a = sm[v], b = sm[u];
        if (w.inverse) {
          sm[v] = add(a, b);
          sm[u] = mul(sub(a, b), tw_h);
        } else {
          const uint32_t p = mul(b, tw_h);
          sm[v] = add(a, p);
          sm[u] = sub(a, p);
        }
      }
      __syncthreads();
    }
    for (uint32_t v = threadIdx.x; v < N; v += blockDim.x) w.dst[v] = w.inverse ? mul(sm[v], w.scale) : sm[v];
    __syncthreads();  // the next item reuses the shared buffer
  }
}

int fft_worklist(Context& ctx, const FftItem* items, uint32_t n_items, const uint32_t* d_twiddles,
                 const uint32_t* d_itwiddles, uint32_t tw_log) {
  if (n_items == 0) return OK;
  GS_REQUIRE(items != nullptr, "null item list");
  GS_REQUIRE(tw_log <= 30, "twiddle log size out of range");
  cudaStream_t st = ctx.stream;
  // 1/2^log for every log, once; the items bucketed by size, largest first
  static const std::vector<uint32_t> inv_pow2 = [] {
    std::vector<uint32_t> t(31);
    for (uint32_t k = 0; k <= 30; k++) t[k] = inv(1u << k);
    return t;
  }();
  uint32_t count[FFT_WL_MAX_LOG + 1] = {0};
  for (uint32_t k = 0; k < n_items; k++) {
    const FftItem& x = items[k];
    GS_REQUIRE(x.src && x.dst, "null column in a work-list item");
    GS_REQUIRE(x.log >= 1 && x.log <= 30 && tw_log + 1 >= x.log, "work-list item size out of range");
    GS_REQUIRE(x.inverse || (x.coeff_log >= 1 && x.coeff_log <= x.log), "coefficient log size must be in [1, log]");
    GS_REQUIRE(x.inverse ? d_itwiddles != nullptr : d_twiddles != nullptr, "null twiddle tree");
    if (x.log >= FFT_WL_MIN_LOG && x.log <= FFT_WL_MAX_LOG) count[x.log]++;
  }
  uint32_t first[FFT_WL_MAX_LOG + 2] = {0}, total = 0;
  for (int lg = (int)FFT_WL_MAX_LOG; lg >= (int)FFT_WL_MIN_LOG; lg--) {
    first[lg] = total;
    total += count[lg];
  }
  std::vector<FftWlItem> wl(total);
  for (uint32_t k = 0; k < n_items; k++) {
    const FftItem& x = items[k];
    if (x.log < FFT_WL_MIN_LOG || x.log > FFT_WL_MAX_LOG) continue;
    wl[first[x.log]++] = FftWlItem{x.src, x.dst, x.log, x.inverse ? x.log : x.coeff_log, x.inverse ? 1u : 0u,
                                   x.inverse ? inv_pow2[x.log] : 1u};
  }
  // the items outside the shared-memory range, one call each
  for (uint32_t k = 0; k < n_items; k++) {
    const FftItem& x = items[k];
    if (x.log >= FFT_WL_MIN_LOG && x.log <= FFT_WL_MAX_LOG) continue;
    const void* const* ts = nullptr;
    const void* const* td = nullptr;
    GS_TRY(ctx.stage_ptrs((const void* const*)&x.src, 1, &ts));
    GS_TRY(ctx.stage_ptrs((const void* const*)&x.dst, 1, &td));
    if (x.inverse)
      GS_TRY(interpolate_columns_to(st, (const uint32_t* const*)ts, (uint32_t* const*)td, 1, x.log, d_itwiddles,
                                    tw_log));
    else
      GS_TRY(evaluate_columns(st, (const uint32_t* const*)ts, x.coeff_log, (uint32_t* const*)td, 1, x.log,
                              d_twiddles, tw_log));
  }
  if (wl.empty()) return OK;
  const void* d = nullptr;
  void* owned = nullptr;  // a list too long for the staging ring: a buffer of its own
  const size_t bytes = wl.size() * sizeof(FftWlItem);
  if (bytes <= ctx.ring_cap / 2) {
    GS_TRY(ctx.stage_bytes(wl.data(), bytes, &d));
  } else {
    GS_TRY(ctx.alloc_async(bytes, &owned));
    GS_CUDA_TRY(cudaMemcpyAsync(owned, wl.data(), bytes, cudaMemcpyHostToDevice, st));
    d = owned;
  }
  const size_t smem = (size_t)4 << wl.front().log;
  static const cudaError_t attr = cudaFuncSetAttribute(fft_worklist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       4 << FFT_WL_MAX_LOG);
  GS_CUDA_TRY(attr);
  const uint32_t per_sm = (uint32_t)std::min<size_t>(8, (200u << 10) / smem);
  const uint32_t grid = (uint32_t)std::min<size_t>(wl.size(), (size_t)num_sms() * (per_sm ? per_sm : 1));
  fft_worklist_kernel<<<grid, 256, smem, st>>>((const FftWlItem*)d, (uint32_t)wl.size(), d_twiddles, d_itwiddles,
                                               1u << tw_log);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  if (owned) GS_CUDA_TRY(cudaFreeAsync(owned, st));  // stream-ordered: after the kernel
  return OK;
}

// Installs the tuning for FFTs computing `layers` layers (0: every size) on
// a domain `ext` log sizes larger (ext > FFT_MAX_EXT: every extension). A
// tile holds 2^tile_log words (at most 2^13, 32 KiB of shared memory), of
// which 2^coalesce_bits are contiguous in memory; a pass needs room for 5
// layers besides them.
int set_fft_tuning(uint32_t layers, uint32_t ext, uint32_t tile_log, uint32_t coalesce_bits) {
  GS_REQUIRE(layers < 32, "log size out of range");
  GS_REQUIRE(tile_log >= 6 && tile_log <= 13, "tile log must be in [6, 13]");
  GS_REQUIRE(coalesce_bits <= 5 && coalesce_bits + 5 <= tile_log, "coalesced bits must be <= min(5, tile_log - 5)");
  for (uint32_t l = layers; l < (layers ? layers + 1 : 32u); l++)
    for (uint32_t e = 0; e <= FFT_MAX_EXT; e++)
      if (ext > FFT_MAX_EXT || e == ext) g_fft_tuning[l][e] = FftTuning{tile_log, coalesce_bits};
  return OK;
}

// Picks, for every FFT log size n in [lo, hi] and extension e in [0,
// max_ext], the tile size and coalesced row width whose pass split is
// fastest, and installs it. e = 0 times an evaluate + interpolate round trip
// of 2^n-word columns in place; e > 0 an LDE of 2^n coefficients onto 2^(n+e)
// points, the shape of a commitment's or constraint domain's extension.
// Scratch columns fill 2^24 output words (or one column when larger); sizes
// whose output exceeds the scratch keep their tuning. Each split is timed with
// CUDA events as the best of 3 trials of 3 runs; the installed split (first
// in the list) is replaced only by one at least 2% faster, so timing noise
// does not move it. Candidates that give the same pass split as an earlier
// one are not timed again. Every candidate computes the same values; only the
// split, and so the speed, differ. Not thread-safe against concurrent
// launches (a set-up step). Outputs: (hi - lo + 1) x (max_ext + 1), by size.
int fft_autotune(cudaStream_t st, uint32_t lo, uint32_t hi, uint32_t max_ext, const uint32_t* tw, const uint32_t* itw,
                 uint32_t tw_log, uint32_t* out_tile, uint32_t* out_coalesce) {
  GS_REQUIRE(lo >= 3 && hi <= 27 && lo <= hi && max_ext <= FFT_MAX_EXT && tw_log + 1 >= hi,
             "autotune range out of bounds");
  static const FftTuning fixed[] = {{13, 4}, {12, 4}, {11, 4}, {10, 4}, {13, 5}, {12, 5}, {11, 5}, {13, 3}};
  const uint32_t w_log = hi > 24 ? hi : 24;
  const size_t words = (size_t)1 << w_log;
  uint32_t* buf = nullptr;  // outputs (and in-place round trips)
  uint32_t* src = nullptr;  // LDE inputs
  uint32_t** tab = nullptr;
  uint32_t** stab = nullptr;
  const uint32_t max_cols = 32768;
  GS_CUDA_TRY(cudaMallocAsync((void**)&buf, 4 * words, st));
  GS_CUDA_TRY(cudaMallocAsync((void**)&src, 2 * words, st));
  GS_CUDA_TRY(cudaMallocAsync((void**)&tab, sizeof(void*) * max_cols, st));
  GS_CUDA_TRY(cudaMallocAsync((void**)&stab, sizeof(void*) * max_cols, st));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = OK;
  if (cudaMemsetAsync(buf, 0, 4 * words, st) != cudaSuccess || cudaMemsetAsync(src, 0, 2 * words, st) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    rc = ERR_CUDA;
  const bool aligned = g_cols_aligned;
  g_cols_aligned = true;
  std::vector<uint32_t*> h, hs;
  for (uint32_t n = lo; n <= hi && rc == OK; n++) {
    for (uint32_t e = 0; e <= max_ext && rc == OK; e++) {
      const uint32_t dn = n + e;  // domain log size
      const size_t slot = (size_t)(n - lo) * (max_ext + 1) + e;
      if (dn > w_log || tw_log + 1 < dn) {
        if (out_tile) out_tile[slot] = g_fft_tuning[n][e].tile_log;
        if (out_coalesce) out_coalesce[slot] = g_fft_tuning[n][e].coalesce_bits;
        continue;
      }
      const uint32_t cols = (uint32_t)std::min<size_t>(words >> dn, max_cols);
      h.resize(cols);
      hs.resize(cols);
      for (uint32_t c = 0; c < cols; c++) {
        h[c] = buf + ((size_t)c << dn);
        hs[c] = src + ((size_t)c << n);
      }
      if (cudaMemcpyAsync(tab, h.data(), sizeof(void*) * cols, cudaMemcpyHostToDevice, st) != cudaSuccess ||
          cudaMemcpyAsync(stab, hs.data(), sizeof(void*) * cols, cudaMemcpyHostToDevice, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess) {
        rc = ERR_CUDA;
        break;
      }
      const FftTuning keep = g_fft_tuning[n][e];
      float best = 1e30f, keep_ms = 1e30f;
      FftTuning pick = keep;
      std::vector<std::vector<std::pair<uint32_t, uint32_t>>> seen;
      std::vector<FftTuning> cand(1, keep);
      cand.insert(cand.end(), std::begin(fixed), std::end(fixed));
      for (size_t ci = 0; ci < cand.size() && rc == OK; ci++) {
        const FftTuning c = cand[ci];
        g_fft_tuning[n][e] = c;
        std::vector<std::pair<uint32_t, uint32_t>> parts;
        fft_partition(n, dn, parts);
        for (auto& pr : parts) pr.first = std::min(c.coalesce_bits, pr.first) | (pr.first << 8);
        if (std::find(seen.begin(), seen.end(), parts) != seen.end()) continue;
        seen.push_back(parts);
        float ms = 1e30f;
        for (int trial = 0; trial < 4 && rc == OK; trial++) {  // trial 0 warms up
          for (int rep = 0; rep < 3 && rc == OK; rep++) {
            if (rep == 0 && cudaEventRecord(e0, st) != cudaSuccess) rc = ERR_CUDA;
            if (rc != OK) break;
            if (e == 0) {
              rc = run_passes<false>(st, (const uint32_t* const*)tab, tab, cols, n, n, 0xffffffffu, tw, 1u << tw_log);
              if (rc == OK)
                rc = run_passes<true>(st, (const uint32_t* const*)tab, tab, cols, n, n, 0xffffffffu, itw,
                                      1u << tw_log);
            } else {
              rc = run_passes<false>(st, (const uint32_t* const*)stab, tab, cols, dn, n, (1u << n) - 1u, tw,
                                     1u << tw_log);
            }
          }
          float t = 0;
          if (rc == OK && (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                           cudaEventElapsedTime(&t, e0, e1) != cudaSuccess))
            rc = ERR_CUDA;
          if (rc == OK && trial > 0) ms = std::min(ms, t);
        }
        if (rc != OK) break;
        if (ci == 0) keep_ms = ms;
        if (ms < best) {
          best = ms;
          pick = c;
        }
      }
      if (best > 0.98f * keep_ms) pick = keep;
      g_fft_tuning[n][e] = rc == OK ? pick : keep;
      if (out_tile) out_tile[slot] = g_fft_tuning[n][e].tile_log;
      if (out_coalesce) out_coalesce[slot] = g_fft_tuning[n][e].coalesce_bits;
    }
  }
  g_cols_aligned = aligned;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFreeAsync(stab, st);
  cudaFreeAsync(tab, st);
  cudaFreeAsync(src, st);
  cudaFreeAsync(buf, st);
  if (rc == ERR_CUDA) set_error(std::string("fft autotune: ") + cudaGetErrorString(cudaGetLastError()));
  return rc;
}

void get_fft_tuning(uint32_t layers, uint32_t ext, uint32_t* tile_log, uint32_t* coalesce_bits) {
  const FftTuning t = g_fft_tuning[layers < 32 ? layers : 31][ext < FFT_MAX_EXT ? ext : FFT_MAX_EXT];
  *tile_log = t.tile_log;
  *coalesce_bits = t.coalesce_bits;
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
