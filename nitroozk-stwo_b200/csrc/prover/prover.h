// GPU prover: prove() for the two benchmark components, all column data
// resident on the device, only roots, OODS values, the last FRI layer and the
// decommitted values crossing to the host.
//
// Control flow follows the reference's unchanged generic prover:
//   crates/stwo/src/prover/mod.rs:37-150            (prove_ex)
//   crates/stwo/src/prover/pcs/mod.rs:57-494        (commitment scheme, prove_values, decommit)
//   crates/stwo/src/prover/pcs/quotient_ops.rs:45-145 (FRI quotients)
//   crates/stwo/src/prover/fri.rs:85-330            (FRI commit / decommit)
//   crates/stwo/src/prover/vcs/prover.rs:50-210     (Merkle decommit)
//   crates/examples/src/{wide_fibonacci,poseidon}/mod.rs (the drivers)
#pragma once
#include <map>
#include <set>
#include "../air.cuh"
#include "host.h"

namespace gs {
namespace prover {

struct PcsConfig {
  uint32_t pow_bits = 10, log_blowup = 1, log_last_layer = 0, n_queries = 70, fold_step = 1;
};

// Stream-ordered device allocations released together.
struct Arena {
  cudaStream_t st = nullptr;
  cudaMemPool_t pool = nullptr;  // the context's pool (default pool if null)
  std::vector<void*> ptrs;
  int alloc(size_t bytes, void** out) {
    void* p = nullptr;
    cudaError_t e = pool ? cudaMallocFromPoolAsync(&p, bytes ? bytes : 16, pool, st)
                         : cudaMallocAsync(&p, bytes ? bytes : 16, st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error(std::string("device allocation failed: ") + cudaGetErrorString(e));
      return ERR_OOM;
    }
    ptrs.push_back(p);
    *out = p;
    return OK;
  }
  template <class T> int alloc_n(size_t n, T** out) { return alloc(n * sizeof(T), (void**)out); }
  void release() {
    for (void* p : ptrs) cudaFreeAsync(p, st);
    ptrs.clear();
  }
  ~Arena() { release(); }
};

// A committed tree whose columns all have one size (true for every tree of
// the two components). Columns are contiguous: column c at base + c * 2^log.
struct Tree {
  uint32_t n_cols = 0;
  uint32_t coeff_log = 0, eval_log = 0;
  const uint32_t* const* coeff_tab = nullptr;  // device pointer tables
  uint32_t* evals = nullptr;
  std::vector<const uint32_t*> coeff_ptrs;    // host copies of the column pointers
  std::vector<uint32_t*> layers;              // layers[L]: 2^L hashes; empty tree: none
  host::Hash root{};
  uint32_t max_log() const { return layers.empty() ? 0 : (uint32_t)layers.size() - 1; }
  const uint32_t* eval_col(uint32_t c) const { return evals + ((size_t)c << eval_log); }
};

// Batched device gathers for decommitments: column values are described per
// (column set, sorted positions) block and expanded on the device; hash
// witnesses are (layer, index) items. One launch per kind, one read-back.
struct GatherPlan {
  std::vector<ColGather> blocks;
  std::vector<uint32_t> positions;
  std::vector<GatherItem> hashes;
  size_t n_words = 0;
  uint32_t max_items = 0;
  std::vector<uint32_t> word_out, hash_out;
  // Values of `cols` at `pos`, position-major; returns the first output word.
  // More than 4 columns must be equally spaced (one tree's columns are).
  int add_cols(const std::vector<const uint32_t*>& cols, const std::vector<size_t>& pos, size_t* first) {
    ColGather b{};
    b.n_cols = (uint32_t)cols.size();
    b.n_pos = (uint32_t)pos.size();
    b.pos_off = positions.size();
    b.out_off = n_words;
    if (b.n_cols <= 4) {
      for (uint32_t c = 0; c < b.n_cols; c++) b.cols[c] = cols[c];
    } else {
      b.base = cols[0];
      b.stride = (uint64_t)(cols[1] - cols[0]);
      for (uint32_t c = 2; c < b.n_cols; c++)
        GS_REQUIRE((uint64_t)(cols[c] - cols[0]) == c * b.stride, "decommitted columns are not equally spaced");
    }
    for (size_t p : pos) positions.push_back((uint32_t)p);
    *first = n_words;
    n_words += (size_t)b.n_cols * b.n_pos;
    max_items = std::max<uint32_t>(max_items, b.n_cols * b.n_pos);
    if (b.n_cols && b.n_pos) blocks.push_back(b);
    return OK;
  }
  size_t add_hash(const uint32_t* src, size_t idx) { hashes.push_back({src, idx}); return hashes.size() - 1; }
  template <class T>
  static int upload(Context& ctx, T* dst, const std::vector<T>& v) {
    const size_t bytes = v.size() * sizeof(T);
    if (!bytes) return OK;
    if (bytes <= ctx.ring_cap / 2) {  // through the pinned staging ring
      const void* d = nullptr;
      GS_TRY(ctx.stage_bytes(v.data(), bytes, &d));
      GS_CUDA_TRY(cudaMemcpyAsync(dst, d, bytes, cudaMemcpyDeviceToDevice, ctx.stream));
    } else {
      GS_CUDA_TRY(cudaMemcpyAsync(dst, v.data(), bytes, cudaMemcpyHostToDevice, ctx.stream));
    }
    return OK;
  }
  int run(Context& ctx, Arena& A) {
    cudaStream_t st = ctx.stream;
    const size_t nh = hashes.size();
    ColGather* d_blocks = nullptr;
    uint32_t* d_pos = nullptr;
    GatherItem* d_items = nullptr;
    uint32_t* d_out = nullptr;
    // hashes are written as 16-byte vectors: their region starts at a
    // multiple of 4 words
    const size_t hbase = (n_words + 3) & ~(size_t)3;
    GS_TRY(A.alloc_n(blocks.size() + 1, &d_blocks));
    GS_TRY(A.alloc_n(positions.size() + 1, &d_pos));
    GS_TRY(A.alloc_n(nh + 1, &d_items));
    GS_TRY(A.alloc_n(hbase + 8 * nh + 4, &d_out));
    GS_TRY(upload(ctx, d_blocks, blocks));
    GS_TRY(upload(ctx, d_pos, positions));
    GS_TRY(upload(ctx, d_items, hashes));
    GS_TRY(gather_cols(st, d_blocks, (uint32_t)blocks.size(), max_items, d_pos, d_out));
    GS_TRY(gather_hashes(st, d_items, nh, d_out + hbase));
    const size_t out_words = hbase + 8 * nh;
    void* hr = nullptr;
    GS_TRY(ctx.read_buffer(out_words * 4, &hr));
    if (out_words) GS_CUDA_TRY(cudaMemcpyAsync(hr, d_out, out_words * 4, cudaMemcpyDeviceToHost, st));
    GS_TRY(stream_sync(st));
    const uint32_t* o = (const uint32_t*)hr;
    word_out.assign(o, o + n_words);
    hash_out.assign(o + hbase, o + out_words);
    return OK;
  }
  host::Hash hash(size_t slot) const { return host::hash_from_words(hash_out.data() + 8 * slot); }
};

// Merkle decommitment of a tree whose columns all sit at the leaf layer
// (MerkleProver::decommit, prover/vcs/prover.rs:50-210, specialised):
// queried values are node-major / column-minor at the leaves, the hash witness
// lists, layer by layer from the leaves up, the children that the verifier
// cannot recompute. Pass 1 queues the gathers, pass 2 assembles.
struct MerkleDecommitPlan {
  std::vector<size_t> positions;
  size_t value_base = 0, n_cols = 0;
  std::vector<size_t> hash_slots;
  // with_values = false: the caller gathers the queried values itself.
  int plan(GatherPlan& g, const std::vector<uint32_t*>& layers, const std::vector<const uint32_t*>& cols,
           const std::vector<size_t>& pos, bool with_values = true) {
    positions = pos;
    n_cols = with_values ? cols.size() : 0;
    if (with_values) GS_TRY(g.add_cols(cols, pos, &value_base));
    // positions are sorted and unique at every layer, so membership of a
    // sibling is a linear merge against the previous layer's list
    std::vector<size_t> prev = pos, merged;
    for (int L = (int)layers.size() - 2; L >= 0; L--) {
      merged.clear();
      for (size_t q : prev)
        if (merged.empty() || merged.back() != q / 2) merged.push_back(q / 2);
      size_t ip = 0;
      for (size_t node : merged)
        for (size_t ch = 2 * node; ch <= 2 * node + 1; ch++) {
          while (ip < prev.size() && prev[ip] < ch) ip++;
          if (ip == prev.size() || prev[ip] != ch) hash_slots.push_back(g.add_hash(layers[L + 1], ch));
        }
      prev.swap(merged);
    }
    return OK;
  }
  void assemble(const GatherPlan& g, std::vector<uint32_t>& queried, host::Decommitment& d) const {
    queried.assign(g.word_out.begin() + value_base, g.word_out.begin() + value_base + positions.size() * n_cols);
    d.hash_witness.reserve(d.hash_witness.size() + hash_slots.size());
    for (size_t s : hash_slots) {
      d.hash_witness.emplace_back();
      memcpy(d.hash_witness.back().data(), g.hash_out.data() + 8 * s, 32);
    }
  }
};

}  // namespace prover
}  // namespace gs
