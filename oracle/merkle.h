// ORACLE — test infrastructure only (see fields.h).
// Merkle tree (Blake2s or Poseidon252 hashes): commit_on_layer, commit, decommit.
// Follows:
//   crates/stwo/src/core/vcs/blake2_merkle.rs:18-39       (hash_node)
//   crates/stwo/src/prover/backend/cpu/blake2s.rs:13-26   (commit_on_layer)
//   crates/stwo/src/prover/backend/cpu/poseidon252.rs:11-24 (the same with Poseidon252MerkleHasher)
//   crates/stwo/src/prover/vcs/prover.rs:22-48            (commit: sort by length desc, stable)
//   crates/stwo/src/prover/vcs/prover.rs:50-210           (decommit: witness order)
//   crates/stwo/src/prover/backend/mod.rs:70-86           (batch_at_multi row-major order)
//   crates/stwo/src/prover/backend/cpu/merkle_lifted.rs:12-88 (lifted leaves, next layer)
#pragma once
#include "blake2s.h"
#include "channel.h"
#include "fields.h"
#include "circle.h"
#include <algorithm>
#include <map>
#include <set>

namespace orc {

inline Hash32 hash_node(const Hash32* left, const Hash32* right, const M31* vals, size_t n,
                        MerkleHash kind = MerkleHash::Blake2s) {
  if (kind == MerkleHash::Poseidon252)
    return p252::hash_node(left ? left->data() : nullptr, right ? right->data() : nullptr, vals, n);
  Blake2s s;
  if (left) { s.update(left->data(), 32); s.update(right->data(), 32); }
  for (size_t i = 0; i < n; i++) s.update_u32(vals[i].v);
  return s.finalize();
}

inline std::vector<Hash32> commit_on_layer(uint32_t log_size, const std::vector<Hash32>* prev,
                                           const std::vector<const std::vector<M31>*>& cols,
                                           MerkleHash kind = MerkleHash::Blake2s) {
  size_t n = (size_t)1 << log_size;
  std::vector<Hash32> out(n);
#pragma omp parallel for schedule(static)
  for (long long ii = 0; ii < (long long)n; ii++) {
    size_t i = (size_t)ii;
    std::vector<M31> vals(cols.size());
    for (size_t c = 0; c < cols.size(); c++) vals[c] = (*cols[c])[i];
    if (prev) out[i] = hash_node(&(*prev)[2 * i], &(*prev)[2 * i + 1], vals.data(), vals.size(), kind);
    else out[i] = hash_node(nullptr, nullptr, vals.data(), vals.size(), kind);
  }
  return out;
}

// Lifted Merkle leaves (MerkleOpsLifted::build_leaves, crates/stwo/src/
// prover/backend/cpu/merkle_lifted.rs:12-77): columns sorted by increasing
// length (stable); leaf i of 2^lift hashes, in that order, every column's
// value at the lifted index ((i >> (lift - log + 1)) << 1) + (i & 1). The
// reference shares hasher prefixes between sizes; the byte stream hashed per
// leaf is the same. No columns: the single leaf is the hash of nothing.
inline std::vector<Hash32> lifted_leaves(const std::vector<const std::vector<M31>*>& columns_in, uint32_t lift) {
  if (columns_in.empty()) {
    Blake2s s;
    return {s.finalize()};
  }
  std::vector<size_t> order(columns_in.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t a, size_t b) { return columns_in[a]->size() < columns_in[b]->size(); });
  size_t n = (size_t)1 << lift;
  std::vector<Hash32> out(n);
#pragma omp parallel for schedule(static)
  for (long long ii = 0; ii < (long long)n; ii++) {
    size_t i = (size_t)ii;
    Blake2s s;
    for (size_t k : order) {
      const auto& c = *columns_in[k];
      uint32_t lg = 0;
      while (((size_t)1 << lg) < c.size()) lg++;
      size_t idx = ((i >> (lift - lg + 1)) << 1) + (i & 1);
      s.update_u32(c[idx].v);
    }
    out[i] = s.finalize();
  }
  return out;
}

struct MerkleDecommitment {
  std::vector<Hash32> hash_witness;
  std::vector<M31> column_witness;
};

struct MerkleProver {
  std::vector<std::vector<Hash32>> layers;  // layers[i] has 2^i nodes; layers[0] = root

  static MerkleProver commit(const std::vector<const std::vector<M31>*>& columns_in,
                             MerkleHash kind = MerkleHash::Blake2s) {
    MerkleProver mp;
    if (columns_in.empty()) {
      mp.layers.push_back(commit_on_layer(0, nullptr, {}, kind));
      return mp;
    }
    std::vector<const std::vector<M31>*> cols(columns_in);
    std::stable_sort(cols.begin(), cols.end(), [](auto a, auto b) { return a->size() > b->size(); });
    uint32_t max_log = ilog2(cols[0]->size());
    std::vector<std::vector<Hash32>> rev;
    size_t ci = 0;
    for (int ls = (int)max_log; ls >= 0; ls--) {
      std::vector<const std::vector<M31>*> lc;
      while (ci < cols.size() && ilog2(cols[ci]->size()) == (uint32_t)ls) lc.push_back(cols[ci++]);
      rev.push_back(commit_on_layer((uint32_t)ls, rev.empty() ? nullptr : &rev.back(), lc, kind));
    }
    mp.layers.assign(rev.rbegin(), rev.rend());
    return mp;
  }
  const Hash32& root() const { return layers[0][0]; }

  // Returns (queried_values, decommitment); queries_per_log_size maps a layer
  // log size to its sorted, deduplicated queried node indices.
  std::pair<std::vector<M31>, MerkleDecommitment> decommit(
      const std::map<uint32_t, std::vector<size_t>>& queries_per_log_size,
      const std::vector<const std::vector<M31>*>& columns_in) const {
    std::vector<M31> queried_values;
    MerkleDecommitment dec;
    std::vector<const std::vector<M31>*> cols(columns_in);
    std::stable_sort(cols.begin(), cols.end(), [](auto a, auto b) { return a->size() > b->size(); });
    size_t ci = 0;
    std::vector<size_t> last_layer_queries;
    for (int ls = (int)layers.size() - 1; ls >= 0; ls--) {
      bool has_prev = (size_t)ls + 1 < layers.size();
      std::set<size_t> prev_set(last_layer_queries.begin(), last_layer_queries.end());
      std::set<size_t> merged;
      for (size_t q : last_layer_queries) merged.insert(q / 2);
      std::set<size_t> col_q;
      auto it = queries_per_log_size.find((uint32_t)ls);
      if (it != queries_per_log_size.end()) col_q.insert(it->second.begin(), it->second.end());
      merged.insert(col_q.begin(), col_q.end());
      std::vector<const std::vector<M31>*> lc;
      while (ci < cols.size() && ilog2(cols[ci]->size()) == (uint32_t)ls) lc.push_back(cols[ci++]);
      std::vector<size_t> queried_nodes, witness_nodes;
      for (size_t node : merged) {
        if (has_prev) {
          const auto& prev = layers[ls + 1];
          if (!prev_set.count(2 * node)) dec.hash_witness.push_back(prev[2 * node]);
          if (!prev_set.count(2 * node + 1)) dec.hash_witness.push_back(prev[2 * node + 1]);
        }
        if (col_q.count(node)) queried_nodes.push_back(node);
        else witness_nodes.push_back(node);
      }
      if (!lc.empty()) {
        for (size_t node : queried_nodes)
          for (auto* c : lc) queried_values.push_back((*c)[node]);
        for (size_t node : witness_nodes)
          for (auto* c : lc) dec.column_witness.push_back((*c)[node]);
      }
      last_layer_queries.assign(merged.begin(), merged.end());
    }
    return {queried_values, dec};
  }
};

}  // namespace orc
