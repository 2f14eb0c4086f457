// Blake2s Merkle layer: MerkleOps<Blake2sMerkleHasher>::commit_on_layer.
//
// Node i of a layer of log size L is
//   Blake2s-256( prev[2i] || prev[2i+1] || col_0[i] || ... || col_{k-1}[i] )
// with the children only when a previous (larger) layer exists and each
// column value as 4 little-endian bytes (crates/stwo/src/core/vcs/
// blake2_merkle.rs:18-39, cpu/blake2s.rs:13-26).
//
// One thread hashes one node: its message block is built directly in
// registers from coalesced column reads (consecutive threads read
// consecutive rows of a column) and compressed in place; the children are
// read as 4 x 16-byte vector loads. No byte-wise buffering.
#include "runtime.cuh"
#include "blake2s.cuh"
#include "merkle_tail.cuh"
#include "channel.cuh"
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>

namespace gs {

__device__ __forceinline__ void store_hash(uint32_t* out, size_t i, const uint32_t h[8]) {
  uint4* o = reinterpret_cast<uint4*>(out + 8 * i);
  o[0] = make_uint4(h[0], h[1], h[2], h[3]);
  o[1] = make_uint4(h[4], h[5], h[6], h[7]);
}

// FMA: adds of the compression on the FMA pipe (blake2s_compress_f).
template <bool FMA>
__global__ void __launch_bounds__(256) merkle_layer_kernel(uint32_t log_size, const uint32_t* __restrict__ prev,
                                                           const uint32_t* const* __restrict__ cols, uint32_t n_cols,
                                                           uint32_t* __restrict__ out, uint32_t one) {
  const size_t n = (size_t)1 << log_size;
  const uint32_t prev_words = prev ? 16u : 0u;
  const uint32_t total_words = prev_words + n_cols;
  const uint32_t total_bytes = 4u * total_words;
  const uint32_t n_blocks = total_words == 0 ? 1u : (total_words + 15u) / 16u;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t h[8];
    blake2s_init(h);
    uint32_t m[16];
    uint32_t blk = 0;
    uint32_t col = 0;
    if (prev) {
      const uint4* p = reinterpret_cast<const uint4*>(prev + 16 * i);
      uint4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
      m[0] = a.x; m[1] = a.y; m[2] = a.z; m[3] = a.w;
      m[4] = b.x; m[5] = b.y; m[6] = b.z; m[7] = b.w;
      m[8] = c.x; m[9] = c.y; m[10] = c.z; m[11] = c.w;
      m[12] = d.x; m[13] = d.y; m[14] = d.z; m[15] = d.w;
      blk = 1;
      uint32_t t = total_bytes < 64u ? total_bytes : 64u;
      if (FMA) blake2s_compress_f(h, m, t, n_blocks == 1, one);
      else blake2s_compress(h, m, t, n_blocks == 1);
    }
    for (; blk < n_blocks; blk++) {
#pragma unroll
      for (int j = 0; j < 16; j++) {
        uint32_t c = col + j;
        m[j] = c < n_cols ? __ldg(cols[c] + i) : 0u;
      }
      col += 16;
      uint32_t t = 64u * (blk + 1);
      if (t > total_bytes) t = total_bytes;
      if (FMA) blake2s_compress_f(h, m, t, blk + 1 == n_blocks, one);
      else blake2s_compress(h, m, t, blk + 1 == n_blocks);
    }
    store_hash(out, i, h);
  }
}

// Lifted Merkle leaves (MerkleOpsLifted::build_leaves, crates/stwo/src/
// prover/backend/cpu/merkle_lifted.rs:12-77): leaf i of 2^lift hashes every
// column's value at its lifted index ((i >> (lift - log + 1)) << 1) + (i & 1),
// columns in increasing size order (the caller sorts, stably). One leaf per
// thread; message blocks are filled straight from the column loads.
__global__ void __launch_bounds__(256) merkle_lifted_leaves_kernel(uint32_t lift, const uint32_t* const* __restrict__ cols,
                                                                   const uint8_t* __restrict__ shifts, uint32_t n_cols,
                                                                   uint32_t* __restrict__ out, uint32_t one) {
  const size_t n = (size_t)1 << lift;
  const uint32_t total_bytes = 4u * n_cols;
  const uint32_t n_blocks = (n_cols + 15u) / 16u;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t h[8], m[16];
    blake2s_init(h);
    uint32_t col = 0;
    for (uint32_t blk = 0; blk < n_blocks; blk++) {
#pragma unroll
      for (int j = 0; j < 16; j++) {
        uint32_t c = col + j;
        uint32_t v = 0;
        if (c < n_cols) {
          const uint32_t s = shifts[c];  // lift - log
          const size_t idx = ((i >> (s + 1)) << 1) + (i & 1);
          v = __ldg(cols[c] + idx);
        }
        m[j] = v;
      }
      col += 16;
      uint32_t t = 64u * (blk + 1);
      if (t > total_bytes) t = total_bytes;
      blake2s_compress_f(h, m, t, blk + 1 == n_blocks, one);
    }
    store_hash(out, i, h);
  }
}

int lifted_leaves(cudaStream_t st, uint32_t lift, const uint32_t* const* d_cols, const uint8_t* d_shifts,
                  uint32_t n_cols, uint32_t* d_out) {
  GS_REQUIRE(lift <= 30 && n_cols >= 1, "bad lifted leaf layer");
  GS_REQUIRE(((uintptr_t)d_out & 15) == 0, "hash buffers must be 16-byte aligned");
  size_t n = (size_t)1 << lift;
  size_t blocks = (n + 255) / 256;
  size_t cap = (size_t)num_sms() * 8;
  if (blocks > cap) blocks = cap;
  merkle_lifted_leaves_kernel<<<(unsigned)blocks, 256, 0, st>>>(lift, d_cols, d_shifts, n_cols, d_out, 1u);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

int commit_on_layer(cudaStream_t st, uint32_t log_size, const uint32_t* d_prev, const uint32_t* const* d_cols,
                    uint32_t n_cols, uint32_t* d_out) {
  GS_REQUIRE(log_size <= 30, "layer log size out of range");
  GS_REQUIRE(d_out != nullptr, "null output");
  GS_REQUIRE(n_cols == 0 || d_cols != nullptr, "null column table");
  GS_REQUIRE(((uintptr_t)d_out & 15) == 0 && ((uintptr_t)d_prev & 15) == 0, "hash buffers must be 16-byte aligned");
  size_t n = (size_t)1 << log_size;
  int threads = 256;
  size_t blocks = (n + threads - 1) / threads;
  size_t cap = (size_t)num_sms() * 8;
  if (blocks > cap) blocks = cap;
  static const bool alu_only = [] {
    const char* e = getenv("GS_BLAKE_ALU");
    return e && e[0] == '1';
  }();
  if (alu_only)
    merkle_layer_kernel<false><<<(unsigned)blocks, threads, 0, st>>>(log_size, d_prev, d_cols, n_cols, d_out, 1u);
  else
    merkle_layer_kernel<true><<<(unsigned)blocks, threads, 0, st>>>(log_size, d_prev, d_cols, n_cols, d_out, 1u);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

// Node-only layers of a small tree in one launch of one 8-CTA thread-block
// cluster: starting from the layer of log size `top` (<= MERKLE_TAIL_LOG,
// already in memory), every layer down to the root, node = Blake2s(left ||
// right). Each CTA first computes its own eighth of the tree (layers top-1
// down to 3) with block barriers only, passing each level to the next through
// shared memory (and writing it to its global layer); after one cluster
// barrier, CTA 0 computes the last 3 layers from the 8 subtree roots. Below
// 2^11 nodes a per-layer launch is latency-bound; 8 SMs give the first levels
// enough throughput.
struct LayerPtrs { uint32_t* p[12]; };

// With `state`, the channel step (mix_root + draw_secure_felt) on the new
// root follows in the same launch (FRI layers).
__global__ void __cluster_dims__(8, 1, 1) __launch_bounds__(1024) merkle_tail_kernel(uint32_t top, LayerPtrs layers,
                                                                                    uint32_t* state, uint32_t* root_copy,
                                                                                    uint32_t* felt) {
  __shared__ uint4 buf[2][256];
  cg::cluster_group cluster = cg::this_cluster();
  cluster_tree_levels(top, layers.p, false, buf, cluster);
  if (state && cluster.block_rank() == 0 && threadIdx.x == 0)
    channel_mix_root_draw_dev(state, layers.p[0], root_copy, felt);
}

// Every node layer of a tree in one launch. A unit is a 512-child subtree:
// a block of 128 threads hashes its 256 parents, then each level above
// through shared memory, down to the unit's root (9 levels), writing every
// level to its global layer. Stage 1 has one block per unit of the input
// layer. The block that finishes last among the units under one next-stage
// unit goes on to hash that unit from the global layer; it learns that it is
// last from a ticket (atomicInc after __threadfence, the counter wrapping
// back to 0 for the next launch). No block waits for another, so there is no
// spinning and nothing to bound. The block that writes the root runs the
// optional channel step. Critical path: one compression per level, against
// one launch per level before.
struct TreePtrs { uint32_t* p[TREE_MAX_LOG + 1]; };
// Threads per 512-child unit: 128, each hashing two nodes of the unit's first
// level (452 us of tree kernels per Poseidon2 2^18 proof, against 464 us
// with 256 threads and 568 us with 64): half the warps wait at the barriers
// of the upper levels, and twice as many units fit on an SM.
constexpr int TREE_THREADS = 128;

template <int U, int TH>
__global__ void __launch_bounds__(TH, TH >= 256 ? 4 : 8)
    merkle_tree_kernel(uint32_t top, TreePtrs layers, uint32_t* counters, uint32_t* state, uint32_t* root_copy,
                       uint32_t* felt) {
  __shared__ uint4 buf[2][1 << U];
  __shared__ uint32_t last;
  const uint32_t tid = threadIdx.x;
  uint32_t in_log = top;
  uint32_t u = blockIdx.x;
  uint32_t cnt_off = 0;
  for (;;) {
    const uint32_t out_log = in_log > U ? in_log - U : 0;
    int cur = 0;
    for (int L = (int)in_log - 1; L >= (int)out_log; L--) {
      const uint32_t n = 1u << (L - (int)out_log);  // this unit's nodes on level L (<= 2^(U-1))
      for (uint32_t i = tid; i < n; i += TH) {
        const size_t node = ((size_t)u << (L - (int)out_log)) + i;
        uint4 c[4];
        if (L == (int)in_log - 1) {
          // written before the launch, or by other blocks of this launch:
          // read at L2, not through the non-coherent path
          const uint4* src = reinterpret_cast<const uint4*>(layers.p[L + 1]) + 4 * node;
#pragma unroll
          for (int q = 0; q < 4; q++) c[q] = __ldcg(src + q);
        } else {
#pragma unroll
          for (int q = 0; q < 4; q++) c[q] = buf[cur ^ 1][4 * i + q];
        }
        uint32_t h[8];
        hash_children16(c, h);
        tail_store_hash(layers.p[L], node, h);
        buf[cur][2 * i] = make_uint4(h[0], h[1], h[2], h[3]);
        buf[cur][2 * i + 1] = make_uint4(h[4], h[5], h[6], h[7]);
      }
      __syncthreads();
      cur ^= 1;
    }
    if (out_log == 0) break;  // this block wrote the root
    const uint32_t group_log = out_log > U ? (uint32_t)U : out_log;
    const uint32_t next_u = u >> group_log;
    if (tid == 0) {
      __threadfence();  // this unit's root (written by thread 0) before the ticket
      const uint32_t ticket = atomicInc(counters + cnt_off + next_u, (1u << group_log) - 1u);
      last = ticket == (1u << group_log) - 1u;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    cnt_off += 1u << (out_log - group_log);
    u = next_u;
    in_log = out_log;
  }
  if (tid == 0) {
    if (state) {
      channel_mix_root_draw_dev(state, layers.p[0], root_copy, felt);
    } else if (root_copy) {
#pragma unroll
      for (int j = 0; j < 8; j++) root_copy[j] = layers.p[0][j];
    }
  }
}

int commit_node_layers_ch(cudaStream_t st, uint32_t top_log, uint32_t* const* layers, uint32_t* d_counters,
                          uint32_t* d_state, uint32_t* d_root_copy, uint32_t* d_felt);

// ------------------------------------------------------------- work-list
// A tree of the work-list on the device: its columns and layers as offsets
// into one pointer pool.
struct MerkleWlItem {
  uint32_t col_off, n_cols, layer_off, log;
};

// Persistent grid: block b takes trees b, b + gridDim.x, ... of a list
// bucketed by decreasing size. Leaf i hashes the columns' values at row i
// (commit_on_layer without a previous layer: 16 column words per message
// block, the last block final); each node layer hashes pairs of the layer
// below from shared memory (two buffers: 2^log and 2^(log-1) hashes), every
// layer also stored to its global buffer.
__global__ void __launch_bounds__(256) merkle_worklist_kernel(const MerkleWlItem* __restrict__ items, uint32_t n_items,
                                                              void* const* __restrict__ pool, uint32_t max_log) {
  extern __shared__ uint4 sb[];
  uint4* const buf0 = sb;
  uint4* const buf1 = sb + 2 * (1u << max_log);
  for (uint32_t it = blockIdx.x; it < n_items; it += gridDim.x) {
    const MerkleWlItem w = items[it];
    const uint32_t* const* cols = reinterpret_cast<const uint32_t* const*>(pool + w.col_off);
    uint32_t* const* layers = reinterpret_cast<uint32_t* const*>(pool + w.layer_off);
    const uint32_t n = 1u << w.log;
    const uint32_t total_bytes = 4u * w.n_cols;
    const uint32_t n_blocks = (w.n_cols + 15u) / 16u;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      uint32_t h[8], m[16];
      blake2s_init(h);
      for (uint32_t blk = 0; blk < n_blocks; blk++) {
#pragma unroll
        for (int j = 0; j < 16; j++) {
          const uint32_t c = 16 * blk + j;
          m[j] = c < w.n_cols ? __ldg(cols[c] + i) : 0u;
        }
        uint32_t t = 64u * (blk + 1);
        if (t > total_bytes) t = total_bytes;
        blake2s_compress(h, m, t, blk + 1 == n_blocks);
      }
      store_hash(layers[w.log], i, h);
      buf0[2 * i] = make_uint4(h[0], h[1], h[2], h[3]);
      buf0[2 * i + 1] = make_uint4(h[4], h[5], h[6], h[7]);
    }
    __syncthreads();
    bool in0 = true;  // the layer below sits in buf0
    for (int L = (int)w.log - 1; L >= 0; L--) {
      const uint4* in = in0 ? buf0 : buf1;
      uint4* out = in0 ? buf1 : buf0;
      for (uint32_t j = threadIdx.x; j < (1u << L); j += blockDim.x) {
        uint4 c[4];
#pragma unroll
        for (int q = 0; q < 4; q++) c[q] = in[4 * j + q];
        uint32_t h[8];
        hash_children16(c, h);
        store_hash(layers[L], j, h);
        out[2 * j] = make_uint4(h[0], h[1], h[2], h[3]);
        out[2 * j + 1] = make_uint4(h[4], h[5], h[6], h[7]);
      }
      __syncthreads();
      in0 = !in0;
    }
    __syncthreads();  // the next tree reuses the buffers
  }
}

int merkle_worklist(Context& ctx, const MerkleItem* items, uint32_t n_items) {
  if (n_items == 0) return OK;
  GS_REQUIRE(items != nullptr, "null tree list");
  cudaStream_t st = ctx.stream;
  uint32_t count[MERKLE_WL_MAX_LOG + 1] = {0};
  for (uint32_t k = 0; k < n_items; k++) {
    const MerkleItem& x = items[k];
    GS_REQUIRE(x.cols && x.layers && x.n_cols >= 1, "a work-list tree needs columns and layers");
    GS_REQUIRE(x.log <= 30, "tree log size out of range");
    for (uint32_t c = 0; c < x.n_cols; c++) GS_REQUIRE(x.cols[c] != nullptr, "null column");
    for (uint32_t L = 0; L <= x.log; L++)
      GS_REQUIRE(x.layers[L] && ((uintptr_t)x.layers[L] & 15) == 0, "layer buffers must be 16-byte aligned");
    if (x.log <= MERKLE_WL_MAX_LOG) count[x.log]++;
  }
  // larger trees: the per-tree path
  for (uint32_t k = 0; k < n_items; k++) {
    const MerkleItem& x = items[k];
    if (x.log <= MERKLE_WL_MAX_LOG) continue;
    const void* const* d = nullptr;
    GS_TRY(ctx.stage_ptrs((const void* const*)x.cols, x.n_cols, &d));
    GS_TRY(commit_on_layer(st, x.log, nullptr, (const uint32_t* const*)d, x.n_cols, x.layers[x.log]));
    GS_TRY(commit_node_layers(st, x.log, x.layers, ctx.tree_counters));
  }
  uint32_t first[MERKLE_WL_MAX_LOG + 1] = {0}, total = 0, max_log = 0;
  for (int lg = (int)MERKLE_WL_MAX_LOG; lg >= 0; lg--) {
    first[lg] = total;
    total += count[lg];
    if (count[lg] && max_log == 0) max_log = (uint32_t)lg;
  }
  if (total == 0) return OK;
  // one upload: the items, then the pointer pool (columns and layers)
  std::vector<MerkleWlItem> wl(total);
  std::vector<void*> pool;  // column pointers are only read
  for (uint32_t k = 0; k < n_items; k++) {
    const MerkleItem& x = items[k];
    if (x.log > MERKLE_WL_MAX_LOG) continue;
    MerkleWlItem w{(uint32_t)pool.size(), x.n_cols, 0, x.log};
    for (uint32_t c = 0; c < x.n_cols; c++) pool.push_back(const_cast<uint32_t*>(x.cols[c]));
    w.layer_off = (uint32_t)pool.size();
    for (uint32_t L = 0; L <= x.log; L++) pool.push_back(x.layers[L]);
    wl[first[x.log]++] = w;
  }
  const size_t o_pool = (wl.size() * sizeof(MerkleWlItem) + 15) & ~(size_t)15;
  const size_t bytes = o_pool + pool.size() * sizeof(void*);
  std::vector<uint8_t> up(bytes);
  memcpy(up.data(), wl.data(), wl.size() * sizeof(MerkleWlItem));
  memcpy(up.data() + o_pool, pool.data(), pool.size() * sizeof(void*));
  const void* d = nullptr;
  void* owned = nullptr;
  if (bytes <= ctx.ring_cap / 2) {
    GS_TRY(ctx.stage_bytes(up.data(), bytes, &d));
  } else {
    GS_TRY(ctx.alloc_async(bytes, &owned));
    GS_CUDA_TRY(cudaMemcpyAsync(owned, up.data(), bytes, cudaMemcpyHostToDevice, st));
    d = owned;
  }
  const size_t smem = (size_t)3 * 16 << max_log;  // 2^max_log + 2^(max_log - 1) hashes, reserved as 3 * 2^max_log uint4
  static const cudaError_t attr = cudaFuncSetAttribute(
      merkle_worklist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(((size_t)3 * 16) << MERKLE_WL_MAX_LOG));
  GS_CUDA_TRY(attr);
  const uint32_t per_sm = (uint32_t)std::min<size_t>(8, ((size_t)200 << 10) / smem);
  const uint32_t grid = (uint32_t)std::min<size_t>(wl.size(), (size_t)num_sms() * (per_sm ? per_sm : 1));
  merkle_worklist_kernel<<<grid, 256, smem, st>>>((const MerkleWlItem*)d, (uint32_t)wl.size(),
                                                  (void* const*)((const uint8_t*)d + o_pool), max_log);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  if (owned) GS_CUDA_TRY(cudaFreeAsync(owned, st));  // stream-ordered: after the kernel
  return OK;
}

int commit_node_layers(cudaStream_t st, uint32_t top_log, uint32_t* const* layers, uint32_t* d_counters) {
  return commit_node_layers_ch(st, top_log, layers, d_counters, nullptr, nullptr, nullptr);
}

static bool merkle_legacy() {
  static const bool legacy = [] {
    const char* e = getenv("GS_MERKLE_LEGACY");
    return e && e[0] == '1';
  }();
  return legacy;
}

int commit_node_layers_to(cudaStream_t st, uint32_t top_log, uint32_t* const* layers, uint32_t* d_counters,
                          uint32_t* root_out) {
  GS_REQUIRE(root_out != nullptr, "null root output");
  if (top_log == 0 || merkle_legacy()) {  // no tree kernel writes the root
    GS_TRY(commit_node_layers(st, top_log, layers, d_counters));
    GS_CUDA_TRY(cudaMemcpyAsync(root_out, layers[0], 32, cudaMemcpyDefault, st));
    return OK;
  }
  return commit_node_layers_ch(st, top_log, layers, d_counters, nullptr, root_out, nullptr);
}

// A tree of top_log <= TREE_MAX_LOG uses at most 2^(27 - 2U) + 2^(27 - 3U) + 1
// ticket counters for units of 2^U children (checked against TREE_COUNTERS).
int commit_node_layers_ch(cudaStream_t st, uint32_t top_log, uint32_t* const* layers, uint32_t* d_counters,
                          uint32_t* d_state, uint32_t* d_root_copy, uint32_t* d_felt) {
  GS_REQUIRE(top_log <= 30, "layer log size out of range");
  const bool legacy = merkle_legacy();
  if (!legacy) {
    uint32_t top = top_log;
    while (top > TREE_MAX_LOG) {  // layers above 2^27 nodes: one launch each
      GS_TRY(commit_on_layer(st, top - 1, layers[top], nullptr, 0, layers[top - 1]));
      top--;
    }
    if (top == 0) {
      GS_REQUIRE(d_state == nullptr, "channel step needs a tree of at least two leaves");
      return OK;
    }
    GS_REQUIRE(d_counters != nullptr, "tree kernel needs its counters");
    TreePtrs tp{};
    for (uint32_t k = 0; k <= top; k++) {
      GS_REQUIRE(((uintptr_t)layers[k] & 15) == 0, "hash buffers must be 16-byte aligned");
      tp.p[k] = layers[k];
    }
    // units of 2^9 children (256 threads): 2^8 (440 -> 464 us of tree
    // kernels per Poseidon2 2^18 proof), 2^7 (854 us) and 2^10 (449 us) were
    // slower
    constexpr int unit = 9;
    {  // ticket counters the continuation stages use
      size_t need = 0;
      for (uint32_t in = top; in > (uint32_t)unit;) {
        const uint32_t out = in - unit, g = out > (uint32_t)unit ? (uint32_t)unit : out;
        need += (size_t)1 << (out - g);
        in = out;
      }
      GS_REQUIRE(need <= TREE_COUNTERS, "tree too large for the ticket counters");
    }
    const uint32_t blocks = top > (uint32_t)unit ? 1u << (top - unit) : 1u;
    merkle_tree_kernel<unit, TREE_THREADS><<<blocks, TREE_THREADS, 0, st>>>(top, tp, d_counters, d_state,
                                                                           d_root_copy, d_felt);
    note_launch();
    GS_CUDA_TRY(cudaGetLastError());
    return OK;
  }
  // Layers of 2^11 nodes and more: one full-GPU launch each; the rest in
  // one cluster launch.
  uint32_t top = top_log;
  while (top > MERKLE_TAIL_LOG) {
    GS_TRY(commit_on_layer(st, top - 1, layers[top], nullptr, 0, layers[top - 1]));
    top--;
  }
  int L = (int)top - 1;
  uint32_t tail_top = (uint32_t)(L + 1);
  if (tail_top == 0) {  // a single node: it is the root already
    GS_REQUIRE(d_state == nullptr, "channel step needs a tree of at least two leaves");
    return OK;
  }
  LayerPtrs lp{};
  for (uint32_t k = 0; k <= tail_top && k < 12; k++) {
    GS_REQUIRE(((uintptr_t)layers[k] & 15) == 0, "hash buffers must be 16-byte aligned");
    lp.p[k] = layers[k];
  }
  merkle_tail_kernel<<<8, 1024, 0, st>>>(tail_top, lp, d_state, d_root_copy, d_felt);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  return OK;
}

}  // namespace gs
