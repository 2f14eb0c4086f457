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
  std::vector<void*> ptrs;       // pool allocations, freed (or kept) by release()
  std::vector<size_t> sizes;     // their sizes
  // previous allocations of the same context to take back first (null: none)
  std::vector<std::pair<size_t, void*>>* spare = nullptr;
  // Requests below SMALL bytes are carved, 256-byte aligned, from chunks of
  // the pool (2 MiB, doubling to 16 MiB): a proof makes a few hundred small
  // allocations (every level of every Merkle tree), and one pool call each
  // costs host time on every proof.
  static constexpr size_t SMALL = (size_t)1 << 20;
  uint8_t* chunk = nullptr;
  size_t chunk_left = 0, next_chunk = (size_t)2 << 20;
  int pool_alloc(size_t bytes, void** out) {
    if (spare)
      for (size_t i = 0; i < spare->size(); i++)
        if ((*spare)[i].first == bytes) {
          *out = (*spare)[i].second;
          (*spare)[i] = spare->back();
          spare->pop_back();
          ptrs.push_back(*out);
          sizes.push_back(bytes);
          return OK;
        }
    void* p = nullptr;
    cudaError_t e = pool ? cudaMallocFromPoolAsync(&p, bytes, pool, st) : cudaMallocAsync(&p, bytes, st);
    if (e != cudaSuccess && spare && !spare->empty()) {  // give the kept buffers back and retry
      cudaGetLastError();
      for (auto& b : *spare) cudaFreeAsync(b.second, st);
      spare->clear();
      e = pool ? cudaMallocFromPoolAsync(&p, bytes, pool, st) : cudaMallocAsync(&p, bytes, st);
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error(std::string("device allocation failed: ") + cudaGetErrorString(e));
      return ERR_OOM;
    }
    ptrs.push_back(p);
    sizes.push_back(bytes);
    *out = p;
    return OK;
  }
  size_t n_requests = 0;
  int alloc(size_t bytes, void** out) {
    n_requests++;
    const size_t need = ((bytes ? bytes : 16) + 255) & ~(size_t)255;
    if (need >= SMALL) return pool_alloc(need, out);
    if (need > chunk_left) {
      void* c = nullptr;
      GS_TRY(pool_alloc(next_chunk, &c));
      chunk = (uint8_t*)c;
      chunk_left = next_chunk;
      if (next_chunk < ((size_t)16 << 20)) next_chunk *= 2;
    }
    *out = chunk;
    chunk += need;
    chunk_left -= need;
    return OK;
  }
  template <class T> int alloc_n(size_t n, T** out) { return alloc(n * sizeof(T), (void**)out); }
  // With a spare list: the spare buffers not taken back are freed and this
  // arena's allocations become the spare list; else every allocation is freed.
  void release() {
    if (spare) {
      for (auto& b : *spare) cudaFreeAsync(b.second, st);
      spare->clear();
      for (size_t i = 0; i < ptrs.size(); i++) spare->push_back({sizes[i], ptrs[i]});
    } else {
      for (void* p : ptrs) cudaFreeAsync(p, st);
    }
    ptrs.clear();
    sizes.clear();
    chunk = nullptr;
    chunk_left = 0;
    next_chunk = (size_t)2 << 20;
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
  // evaluations on the constraint domain (2^ext_log rows per column), filled
  // column range by column range as the prover finds idle device time
  uint32_t* ext = nullptr;
  uint32_t ext_log = 0;
  uint32_t ext_done = 0;  // columns [0, ext_done) extended
  uint32_t max_log() const { return layers.empty() ? 0 : (uint32_t)layers.size() - 1; }
  const uint32_t* eval_col(uint32_t c) const { return evals + ((size_t)c << eval_log); }
};

// Results of one launched gather, in the context's pinned read-back buffer
// (valid until its next read-back): gathered words, then 8 words per hash.
struct GatherOut {
  const uint32_t* word_out = nullptr;
  const uint32_t* hash_out = nullptr;
  int wait(Context& ctx) { return stream_sync(ctx.stream); }
};

// Batched device gathers for decommitments: column values are described per
// (column set, sorted positions) block and expanded on the device; hash
// witnesses are (layer, index) items. One launch per kind, one read-back.
struct GatherPlan {
  std::vector<ColGather> blocks;
  std::vector<uint32_t> positions;
  std::vector<HashRun> runs;
  std::vector<uint32_t> hidx;    // hash index of every witness, in output order
  std::vector<uint8_t> packed;   // the upload: blocks | positions | runs | hidx
  size_t n_words = 0;
  size_t n_hash_out = 0;         // hashes the runs write, in run order
  uint32_t max_items = 0;
  // Empties the plan, keeping its capacity (one plan serves many proofs).
  void clear() {
    blocks.clear();
    positions.clear();
    runs.clear();
    hidx.clear();
    n_words = 0;
    n_hash_out = 0;
    max_items = 0;
  }
  size_t n_hashes() const { return n_hash_out; }
  // Values of `cols` at `pos`, position-major; returns the first output word.
  // More than 4 columns must be equally spaced (one tree's columns are).
  int add_cols(const std::vector<const uint32_t*>& cols, const std::vector<size_t>& pos, size_t* first) {
    return add_cols(cols.data(), cols.size(), pos, first);
  }
  int add_cols(const uint32_t* const* cols, size_t n_cols, const std::vector<size_t>& pos, size_t* first) {
    ColGather b{};
    b.n_cols = (uint32_t)n_cols;
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
    const size_t p0 = positions.size();
    positions.resize(p0 + pos.size());
    for (size_t i = 0; i < pos.size(); i++) positions[p0 + i] = (uint32_t)pos[i];
    *first = n_words;
    n_words += (size_t)b.n_cols * b.n_pos;
    max_items = std::max<uint32_t>(max_items, b.n_cols * b.n_pos);
    if (b.n_cols && b.n_pos) blocks.push_back(b);
    return OK;
  }
  // Witnesses hidx[first, first + count) read from the layer at `src`; they
  // take the next `count` output hashes.
  void add_run(const uint32_t* src, size_t first, size_t count) {
    runs.push_back(HashRun{src, (uint32_t)first, (uint32_t)count, (uint32_t)n_hash_out, 0});
    n_hash_out += count;
  }
  // The upload, both gathers and the read-back, enqueued on the context's
  // stream; `out` is valid after GatherOut::wait. The plan itself may be
  // cleared and reused once launch returns (the upload has been taken).
  int launch(Context& ctx, Arena& A, GatherOut* out) {
    cudaStream_t st = ctx.stream;
    const size_t nh = hidx.size();
    auto al = [](size_t b) { return (b + 15) & ~(size_t)15; };
    const size_t o_pos = al(blocks.size() * sizeof(ColGather));
    const size_t o_runs = o_pos + al(positions.size() * 4);
    const size_t o_idx = o_runs + al(runs.size() * sizeof(HashRun));
    const size_t total = o_idx + al(nh * 4);
    packed.resize(total);
    if (!blocks.empty()) memcpy(packed.data(), blocks.data(), blocks.size() * sizeof(ColGather));
    if (!positions.empty()) memcpy(packed.data() + o_pos, positions.data(), positions.size() * 4);
    if (!runs.empty()) memcpy(packed.data() + o_runs, runs.data(), runs.size() * sizeof(HashRun));
    if (nh) memcpy(packed.data() + o_idx, hidx.data(), nh * 4);
    // kernels read the upload where it lands: the staging ring when it fits
    const uint8_t* d_in = nullptr;
    if (total == 0) {
    } else if (total <= ctx.ring_cap / 2) {
      const void* d = nullptr;
      GS_TRY(ctx.stage_bytes(packed.data(), total, &d));
      d_in = (const uint8_t*)d;
    } else {
      uint8_t* d = nullptr;
      GS_TRY(A.alloc_n(total, &d));
      GS_CUDA_TRY(cudaMemcpyAsync(d, packed.data(), total, cudaMemcpyHostToDevice, st));
      d_in = d;
    }
    // hashes are written as 16-byte vectors: their region starts at a
    // multiple of 4 words
    const size_t hbase = (n_words + 3) & ~(size_t)3;
    const size_t out_words = hbase + 8 * n_hash_out;
    // one launch writes both gathers straight into the mapped read buffer
    // (or into device memory, published after, where it has no alias)
    void* hr = nullptr;
    GS_TRY(ctx.read_buffer(out_words * 4 + 16, &hr));
    uint32_t* d_out = (uint32_t*)ctx.d_read;
    if (!d_out) GS_TRY(A.alloc_n(out_words + 4, &d_out));
    GS_TRY(gather_all(st, (const ColGather*)d_in, (uint32_t)blocks.size(), max_items, (const uint32_t*)(d_in + o_pos),
                      d_out, (const HashRun*)(d_in + o_runs), (uint32_t)runs.size(), (const uint32_t*)(d_in + o_idx),
                      d_out + hbase));
    if (!ctx.d_read) {
      const void* h = nullptr;
      GS_TRY(ctx.publish(d_out, out_words * 4, &h));
      hr = (void*)h;
    }
    out->word_out = (const uint32_t*)hr;
    out->hash_out = out->word_out + hbase;
    return OK;
  }
};

// Merkle decommitment of a tree whose columns all sit at the leaf layer
// (MerkleProver::decommit, prover/vcs/prover.rs:50-210, specialised):
// queried values are node-major / column-minor at the leaves, the hash witness
// lists, layer by layer from the leaves up, the children that the verifier
// cannot recompute. Pass 1 queues the gathers, pass 2 assembles.
struct SharedWitness;

struct MerkleDecommitPlan {
  size_t n_positions = 0;
  size_t value_base = 0, n_cols = 0;
  size_t hash_begin = 0, n_hashes = 0;  // this plan's witnesses: consecutive gather slots
  // with_values = false: the caller gathers the queried values itself.
  int plan(GatherPlan& g, const std::vector<uint32_t*>& layers, const std::vector<const uint32_t*>& cols,
           const std::vector<size_t>& pos, bool with_values = true) {
    n_positions = pos.size();
    n_cols = with_values ? cols.size() : 0;
    if (with_values) GS_TRY(g.add_cols(cols, pos, &value_base));
    // Positions are sorted and unique on every layer, so a node's sibling is
    // known exactly when it is the neighbour in the list; otherwise the
    // sibling is a witness. Witnesses come out parent by parent, left child
    // first, as the verifier consumes them.
    // The loop body has no data-dependent branch: every position writes its
    // sibling and its parent, and the counts advance only for a missing
    // sibling and for a new parent.
    hash_begin = g.n_hashes();
    static thread_local std::vector<size_t> prev, next;
    prev.assign(pos.begin(), pos.end());
    for (int L = (int)layers.size() - 2; L >= 0; L--) {
      const size_t n = prev.size();
      const size_t base = g.hidx.size();
      g.hidx.resize(base + n);  // at most one witness per position
      uint32_t* w = g.hidx.data() + base;
      next.resize(n);
      size_t nw = 0, nn = 0, last_parent = ~(size_t)0;
      for (size_t i = 0; i < n; i++) {
        const size_t q = prev[i];
        // the sibling q ^ 1 can only be the left (odd q) or the right (even q)
        // neighbour in the sorted list: compare both, without a branch
        const size_t left = i > 0 ? prev[i - 1] : ~(size_t)0;
        const size_t right = i + 1 < n ? prev[i + 1] : ~(size_t)0;
        const bool sib = (left == (q ^ 1)) | (right == (q ^ 1));
        w[nw] = (uint32_t)(q ^ 1);
        nw += sib ? 0 : 1;
        const size_t par = q >> 1;
        next[nn] = par;
        nn += par != last_parent ? 1 : 0;
        last_parent = par;
      }
      g.hidx.resize(base + nw);
      if (nw) g.add_run(layers[L + 1], base, nw);
      next.resize(nn);
      prev.swap(next);
    }
    n_hashes = g.n_hashes() - hash_begin;
    return OK;
  }
  // The same plan from shared witness lists: the tree's level just above
  // layers[top_L + 1] holds the positions S_m0, the next S_(m0 + 1), and so
  // on (top_L = layers.size() - 2 when the leaves are S_0; a FRI layer's
  // leaves are the complete pairs of S_i, which reveal no hash, so it starts
  // one level up with top_L = layers.size() - 3 and m0 = i + 1).
  int plan_shared(GatherPlan& g, const std::vector<uint32_t*>& layers, const std::vector<const uint32_t*>& cols,
                  const std::vector<size_t>& pos, const SharedWitness& sw, int top_L, size_t m0,
                  bool with_values = true);
  // The hash witnesses alone, for n_positions leaf positions.
  int plan_shared_hashes(GatherPlan& g, const std::vector<uint32_t*>& layers, size_t n_positions,
                         const SharedWitness& sw, int top_L, size_t m0);
  // Serialised MerkleDecommitment (hash witnesses, no column witness) and
  // the queried values: gathered bytes, written by the writer's gathered pass.
  void write_decommitment(host::Writer& w, const GatherOut& g) const {
    w.u64(n_hashes);
    w.put_gathered(w.gathered ? g.hash_out + 8 * hash_begin : nullptr, 32 * n_hashes);
    w.u64(0);
  }
  void write_queried(host::Writer& w, const GatherOut& g) const {
    w.u64(n_positions * n_cols);
    w.put_gathered(w.gathered ? g.word_out + value_base : nullptr, 4 * n_positions * n_cols);
  }
};

// Witness index lists shared by every tree decommitted at the same query
// positions. Level m of the query set is S_m = {q >> m} (sorted, unique); at a
// Merkle level whose positions are S_m a decommitment reveals W(S_m), the
// siblings that are not in S_m, in order. The trees with leaves at S_0 (every
// tree of the lifting size) and every FRI layer (leaves = the pairs of S_i,
// level above = S_(i+1)) reveal W(S_m) at their levels, so each list is
// computed and uploaded once and read by one hash run per tree.
struct SharedWitness {
  std::vector<size_t> s0;            // S_0
  std::vector<size_t> first, count;  // W(S_m) = g.hidx[first[m], first[m] + count[m])
  void build(GatherPlan& g, const std::vector<size_t>& queries, size_t levels) {
    s0 = queries;
    first.assign(levels, 0);
    count.assign(levels, 0);
    static thread_local std::vector<size_t> prev, next;
    prev.assign(queries.begin(), queries.end());
    for (size_t m = 0; m < levels; m++) {
      const size_t n = prev.size();
      const size_t base = g.hidx.size();
      g.hidx.resize(base + n);
      uint32_t* w = g.hidx.data() + base;
      next.resize(n);
      size_t nw = 0, nn = 0, last_parent = ~(size_t)0;
      for (size_t i = 0; i < n; i++) {
        const size_t q = prev[i];
        // the sibling q ^ 1 can only be the left (odd q) or the right (even q)
        // neighbour in the sorted list: compare both, without a branch
        const size_t left = i > 0 ? prev[i - 1] : ~(size_t)0;
        const size_t right = i + 1 < n ? prev[i + 1] : ~(size_t)0;
        const bool sib = (left == (q ^ 1)) | (right == (q ^ 1));
        w[nw] = (uint32_t)(q ^ 1);
        nw += sib ? 0 : 1;
        const size_t par = q >> 1;
        next[nn] = par;
        nn += par != last_parent ? 1 : 0;
        last_parent = par;
      }
      g.hidx.resize(base + nw);
      first[m] = base;
      count[m] = nw;
      next.resize(nn);
      prev.swap(next);
    }
  }
};

inline int MerkleDecommitPlan::plan_shared(GatherPlan& g, const std::vector<uint32_t*>& layers,
                                           const std::vector<const uint32_t*>& cols, const std::vector<size_t>& pos,
                                           const SharedWitness& sw, int top_L, size_t m0, bool with_values) {
  if (with_values) GS_TRY(g.add_cols(cols, pos, &value_base));
  GS_TRY(plan_shared_hashes(g, layers, pos.size(), sw, top_L, m0));
  n_cols = with_values ? cols.size() : 0;
  return OK;
}

inline int MerkleDecommitPlan::plan_shared_hashes(GatherPlan& g, const std::vector<uint32_t*>& layers,
                                                  size_t n_pos, const SharedWitness& sw, int top_L, size_t m0) {
  GS_REQUIRE(top_L < (int)layers.size() - 1 && m0 + (size_t)(top_L + 1) <= sw.first.size(),
             "shared witness lists too short for the tree");
  n_positions = n_pos;
  n_cols = 0;
  hash_begin = g.n_hashes();
  size_t m = m0;
  for (int L = top_L; L >= 0; L--, m++)
    if (sw.count[m]) g.add_run(layers[L + 1], sw.first[m], sw.count[m]);
  n_hashes = g.n_hashes() - hash_begin;
  return OK;
}

}  // namespace prover
}  // namespace gs
