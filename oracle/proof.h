// ORACLE — test infrastructure only (see fields.h).
// Proof structures and their byte serialisation.
// Field order follows the reference's serde-derived structs:
//   crates/stwo/src/core/pcs/quotients.rs:29-38  (CommitmentSchemeProof)
//   crates/stwo/src/core/pcs/mod.rs:31-36        (PcsConfig), core/fri.rs:32-37 (FriConfig)
//   crates/stwo/src/core/vcs/verifier.rs:13-22   (MerkleDecommitment)
//   crates/stwo/src/core/fri.rs:363-398          (FriProof, FriLayerProof), core/poly/line.rs:96-101 (LinePoly)
// Encoding: bincode-1.x style fixed-width little endian, u64 sequence lengths,
// Option as a 1-byte tag, a hash as 32 raw bytes, M31 as u32, QM31 as 4 x u32.
#pragma once
#include "merkle.h"
#include <string>

namespace orc {

struct PcsConfig {
  uint32_t pow_bits = 10;
  uint32_t log_blowup = 1;
  uint32_t log_last_layer = 0;
  uint32_t n_queries = 70;
  uint32_t fold_step = 1;
  bool has_lifting = false;
  uint32_t lifting = 0;
};

struct FriLayerProof {
  std::vector<QM31> fri_witness;
  MerkleDecommitment decommitment;
  Hash32 commitment{};
};

struct FriProof {
  FriLayerProof first;
  std::vector<FriLayerProof> inner;
  std::vector<QM31> last_layer_coeffs;  // LinePoly internal (bit-reversed) order
  uint32_t last_layer_log = 0;
};

struct StarkProof {
  PcsConfig config;
  std::vector<Hash32> commitments;
  std::vector<std::vector<std::vector<QM31>>> sampled_values;
  std::vector<MerkleDecommitment> decommitments;
  std::vector<std::vector<M31>> queried_values;
  uint64_t proof_of_work = 0;
  FriProof fri;
};

struct ByteWriter {
  std::string b;
  void u8(uint8_t v) { b.push_back((char)v); }
  void u32(uint32_t v) { for (int i = 0; i < 4; i++) b.push_back((char)(v >> (8 * i))); }
  void u64(uint64_t v) { for (int i = 0; i < 8; i++) b.push_back((char)(v >> (8 * i))); }
  void hash(const Hash32& h) { b.append((const char*)h.data(), 32); }
  void qm(const QM31& q) { for (int i = 0; i < 4; i++) u32(q.coord(i)); }
  void decommitment(const MerkleDecommitment& d) {
    u64(d.hash_witness.size());
    for (auto& h : d.hash_witness) hash(h);
    u64(d.column_witness.size());
    for (auto& v : d.column_witness) u32(v.v);
  }
  void fri_layer(const FriLayerProof& l) {
    u64(l.fri_witness.size());
    for (auto& q : l.fri_witness) qm(q);
    decommitment(l.decommitment);
    hash(l.commitment);
  }
};

inline std::string serialize(const StarkProof& p) {
  ByteWriter w;
  w.u32(p.config.pow_bits);
  w.u32(p.config.log_blowup);
  w.u32(p.config.log_last_layer);
  w.u64(p.config.n_queries);
  w.u32(p.config.fold_step);
  if (p.config.has_lifting) { w.u8(1); w.u32(p.config.lifting); } else { w.u8(0); }
  w.u64(p.commitments.size());
  for (auto& h : p.commitments) w.hash(h);
  w.u64(p.sampled_values.size());
  for (auto& tree : p.sampled_values) {
    w.u64(tree.size());
    for (auto& col : tree) {
      w.u64(col.size());
      for (auto& q : col) w.qm(q);
    }
  }
  w.u64(p.decommitments.size());
  for (auto& d : p.decommitments) w.decommitment(d);
  w.u64(p.queried_values.size());
  for (auto& t : p.queried_values) {
    w.u64(t.size());
    for (auto& v : t) w.u32(v.v);
  }
  w.u64(p.proof_of_work);
  w.fri_layer(p.fri.first);
  w.u64(p.fri.inner.size());
  for (auto& l : p.fri.inner) w.fri_layer(l);
  w.u64(p.fri.last_layer_coeffs.size());
  for (auto& q : p.fri.last_layer_coeffs) w.qm(q);
  w.u32(p.fri.last_layer_log);
  return w.b;
}

}  // namespace orc
