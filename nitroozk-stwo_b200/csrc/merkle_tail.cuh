// Merkle node levels of a small tree by one 8-CTA thread-block cluster
// (shared by the Merkle tail kernel and the fused FRI tail).
#pragma once
#include <cooperative_groups.h>
#include "runtime.cuh"
#include "blake2s.cuh"

namespace gs {

namespace cg = cooperative_groups;

__device__ __forceinline__ void tail_store_hash(uint32_t* out, size_t i, const uint32_t h[8]) {
  uint4* o = reinterpret_cast<uint4*>(out + 8 * i);
  o[0] = make_uint4(h[0], h[1], h[2], h[3]);
  o[1] = make_uint4(h[4], h[5], h[6], h[7]);
}

__device__ __forceinline__ void hash_children16(const uint4* c, uint32_t h[8]) {
  uint32_t m[16];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    m[4 * q] = c[q].x; m[4 * q + 1] = c[q].y; m[4 * q + 2] = c[q].z; m[4 * q + 3] = c[q].w;
  }
  blake2s_init(h);
  blake2s_compress(h, m, 64, true);
}

// The subtree part for a tree with `top` <= 11, run by every CTA of the
// cluster, then the cluster barrier, then CTA 0's last layers. `fresh_top`:
// the top layer was written earlier in the same kernel by other CTAs (read
// at L2, not through the non-coherent path).
__device__ __forceinline__ void cluster_tree_levels(uint32_t top, uint32_t* const* layer, bool fresh_top, uint4 (*buf)[256],
                                    cg::cluster_group& cluster) {
  const uint32_t rank = cluster.block_rank();
  const uint32_t tid = threadIdx.x;
  const int split = top >= 4 ? 3 : (int)top;
  int cur = 0;
  for (int L = (int)top - 1; L >= split; L--) {
    const uint32_t per = 1u << (L - 3);
    const uint32_t base = rank * per;
    for (uint32_t j = tid; j < per; j += blockDim.x) {
      uint4 c[4];
      if (L == (int)top - 1) {
        const uint4* src = reinterpret_cast<const uint4*>(layer[L + 1]) + 4 * (size_t)(base + j);
#pragma unroll
        for (int q = 0; q < 4; q++) c[q] = fresh_top ? __ldcg(src + q) : __ldg(src + q);
      } else {
#pragma unroll
        for (int q = 0; q < 4; q++) c[q] = buf[cur ^ 1][4 * j + q];
      }
      uint32_t h[8];
      hash_children16(c, h);
      tail_store_hash(layer[L], base + j, h);
      buf[cur][2 * j] = make_uint4(h[0], h[1], h[2], h[3]);
      buf[cur][2 * j + 1] = make_uint4(h[4], h[5], h[6], h[7]);
    }
    __syncthreads();
    cur ^= 1;
  }
  cluster.sync();
  if (rank == 0) {
    for (int L = split - 1; L >= 0; L--) {
      for (uint32_t i = tid; i < (1u << L); i += blockDim.x) {
        const uint4* src = reinterpret_cast<const uint4*>(layer[L + 1]) + 4 * (size_t)i;
        uint4 c[4];
#pragma unroll
        for (int q = 0; q < 4; q++) c[q] = __ldcg(src + q);
        uint32_t h[8];
        hash_children16(c, h);
        tail_store_hash(layer[L], i, h);
      }
      __syncthreads();
    }
  }
}

}  // namespace gs
