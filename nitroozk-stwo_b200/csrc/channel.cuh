// Device-side Fiat-Shamir step of the Blake2s channel (Blake2sChannel::
// mix_root followed by draw_secure_felt, crates/stwo/src/core/channel/
// blake2s.rs), shared by the stand-alone channel kernel and the fused FRI
// tail kernel. Run by one thread.
//
//   mix_root:    digest <- Blake2s(digest || root), n_draws <- 0
//   draw_u32s:   Blake2s(digest || n_draws (LE u32) || 0x00), n_draws += 1
//   draw_felt:   repeat draw_u32s until all 8 words are < 2p; the secure
//                field element is the first 4 words reduced mod p.
//
// state: 8 digest words, n_draws, status (set nonzero when no challenge was
// found within the draw bound). felt_out: the challenge, then its square.
#pragma once
#include "runtime.cuh"
#include "blake2s.cuh"

namespace gs {

__device__ __forceinline__ void channel_mix_root_draw_dev(uint32_t* state, const uint32_t* root, uint32_t* root_copy,
                                                          uint32_t* felt_out) {
  uint32_t m[16], d[8];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    m[j] = state[j];
    m[8 + j] = root[j];
  }
  blake2s_init(d);
  blake2s_compress(d, m, 64, true);
  if (root_copy)
    for (int j = 0; j < 8; j++) root_copy[j] = root[j];
  uint32_t n_draws = 0;
  // A draw is rejected with probability < 2^-27; 64 rejections in a row do
  // not happen for a hash, and running out is reported, never looped on.
  for (int attempt = 0; attempt < 64; attempt++) {
    uint32_t h[8];
#pragma unroll
    for (int j = 0; j < 8; j++) m[j] = d[j];
    m[8] = n_draws;
#pragma unroll
    for (int j = 9; j < 16; j++) m[j] = 0;
    blake2s_init(h);
    blake2s_compress(h, m, 37, true);
    n_draws++;
    bool ok = true;
#pragma unroll
    for (int j = 0; j < 8; j++) ok = ok && h[j] < 2u * P;
    if (ok) {
      qm31 a = qm_make(h[0] >= P ? h[0] - P : h[0], h[1] >= P ? h[1] - P : h[1], h[2] >= P ? h[2] - P : h[2],
                       h[3] >= P ? h[3] - P : h[3]);
      qm31 a2 = qm_mul(a, a);
      felt_out[0] = a.x.a; felt_out[1] = a.x.b; felt_out[2] = a.y.a; felt_out[3] = a.y.b;
      felt_out[4] = a2.x.a; felt_out[5] = a2.x.b; felt_out[6] = a2.y.a; felt_out[7] = a2.y.b;
      for (int j = 0; j < 8; j++) state[j] = d[j];
      state[8] = n_draws;
      return;
    }
  }
  for (int j = 0; j < 8; j++) state[j] = d[j];
  state[8] = n_draws;
  state[9] = 1;
}

}  // namespace gs
