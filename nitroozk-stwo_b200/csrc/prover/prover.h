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
  std::vector<void*> ptrs;
  int alloc(size_t bytes, void** out) {
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes ? bytes : 16, st);
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

// Batched device gathers for decommitments: items are queued on the host,
// fetched with one launch per kind and read back with one copy.
struct GatherPlan {
  std::vector<GatherItem> words, hashes;
  std::vector<uint32_t> word_out, hash_out;
  size_t add_word(const uint32_t* src, size_t idx) { words.push_back({src, idx}); return words.size() - 1; }
  size_t add_hash(const uint32_t* src, size_t idx) { hashes.push_back({src, idx}); return hashes.size() - 1; }
  int run(Context& ctx, Arena& A) {
    cudaStream_t st = ctx.stream;
    size_t nw = words.size(), nh = hashes.size();
    GatherItem *d_items = nullptr;
    uint32_t* d_out = nullptr;
    // hashes are written as 16-byte vectors: their region starts at a
    // multiple of 4 words
    const size_t hbase = (nw + 3) & ~(size_t)3;
    GS_TRY(A.alloc_n(nw + nh + 1, &d_items));
    GS_TRY(A.alloc_n(hbase + 8 * nh + 4, &d_out));
    std::vector<GatherItem> all(words);
    all.insert(all.end(), hashes.begin(), hashes.end());
    if (!all.empty())
      GS_CUDA_TRY(cudaMemcpyAsync(d_items, all.data(), all.size() * sizeof(GatherItem), cudaMemcpyHostToDevice, st));
    GS_TRY(gather_words(st, d_items, nw, d_out));
    GS_TRY(gather_hashes(st, d_items + nw, nh, d_out + hbase));
    std::vector<uint32_t> out(hbase + 8 * nh);
    if (!out.empty()) GS_CUDA_TRY(cudaMemcpyAsync(out.data(), d_out, out.size() * 4, cudaMemcpyDeviceToHost, st));
    GS_CUDA_TRY(cudaStreamSynchronize(st));
    word_out.assign(out.begin(), out.begin() + nw);
    hash_out.assign(out.begin() + hbase, out.end());
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
  void plan(GatherPlan& g, const std::vector<uint32_t*>& layers, const std::vector<const uint32_t*>& cols,
            const std::vector<size_t>& pos) {
    positions = pos;
    n_cols = cols.size();
    value_base = g.words.size();
    for (size_t node : pos)
      for (auto* c : cols) g.add_word(c, node);
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
  }
  void assemble(const GatherPlan& g, std::vector<uint32_t>& queried, host::Decommitment& d) const {
    queried.assign(g.word_out.begin() + value_base, g.word_out.begin() + value_base + positions.size() * n_cols);
    for (size_t s : hash_slots) d.hash_witness.push_back(g.hash(s));
  }
};

}  // namespace prover
}  // namespace gs
