// Fiat-Shamir steps of the Blake2s channel on the device
// (Blake2sChannel::mix_root + draw_secure_felt, crates/stwo/src/core/channel/
// blake2s.rs), so that the FRI commit phase chains layer after layer — Merkle
// root, folding challenge, fold — with no host round trip in between.
//
//   mix_root:    digest <- Blake2s(digest || root), n_draws <- 0
//   draw_u32s:   Blake2s(digest || n_draws (LE u32) || 0x00), n_draws += 1
//   draw_felt:   repeat draw_u32s until all 8 words are < 2p; the secure
//                field element is the first 4 words reduced mod p.
//
// The host replays the same steps on the roots read back at the end of the
// phase and checks every challenge against the device's.
#include "channel.cuh"

namespace gs {

__global__ void channel_mix_root_draw_kernel(uint32_t* state, const uint32_t* root, uint32_t* root_copy,
                                             uint32_t* felt_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  channel_mix_root_draw_dev(state, root, root_copy, felt_out);
}

int channel_mix_root_draw(cudaStream_t st, uint32_t* d_state, const uint32_t* d_root, uint32_t* d_root_copy,
                          uint32_t* d_felt) {
  channel_mix_root_draw_kernel<<<1, 32, 0, st>>>(d_state, d_root, d_root_copy, d_felt);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

}  // namespace gs
