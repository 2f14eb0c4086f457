// Request/response of the GPU prover driver.
#pragma once
#include <string>
#include "prover.h"

namespace gs {
namespace prover {

struct ProveRequest {
  uint32_t air = 0;          // 0 = wide fibonacci, 1 = poseidon2
  uint32_t log_n = 0;        // trace rows (log)
  uint32_t n_cols = 100;     // wide fibonacci width
  uint64_t seed = 0;
  uint32_t input_mode = 0;   // 0 reference rule, 1 seeded, 2 host inputs
  const uint32_t* host_inputs = nullptr;  // mode 2: WF a,b columns; Poseidon 16 state columns
  uint32_t split_log = 1;    // composition split
  uint32_t merkle_channel = 0;  // 0 Blake2sMerkleChannel, 1 Poseidon252MerkleChannel
  PcsConfig cfg;
  // Optional caller buffer: when the proof fits, it is serialised straight
  // into it (ProveStats::in_out_buf) and the string stays untouched.
  uint8_t* out_buf = nullptr;
  size_t out_cap = 0;
};

struct ProveStats {
  double constraint_check = 0;  // 1 if the composition sanity check passed
  size_t proof_len = 0;         // serialised proof bytes
  bool in_out_buf = false;      // written to ProveRequest::out_buf
};

struct Prover;
struct AirHost;
// The checks every proof request passes before any device work (direct
// gs_prove_* calls and proof-server submissions alike): component, channel,
// input mode, PcsConfig ranges, Wide-Fibonacci width. ERR_INVALID otherwise.
int validate_request(const ProveRequest& r);
int prove_component(Context& ctx, const ProveRequest& req, std::string* proof_bytes, ProveStats* stats);
int prove_tail(Prover& pv, AirHost& air, uint32_t split, std::string* proof_bytes, ProveStats* stats,
               uint8_t* out_buf = nullptr, size_t out_cap = 0);

// Batched commitment of columns of mixed sizes (commit.cpp).
struct CommitPlan;
int plan_create(Context& ctx, const uint32_t* log_sizes, uint32_t n, uint32_t blowup, bool use_graph,
                CommitPlan** out);
int plan_run(CommitPlan* p, const uint32_t* const* inputs, uint32_t root[8]);
int plan_extended(CommitPlan* p, uint32_t column, const uint32_t** out);
int plan_layer(CommitPlan* p, uint32_t log_size, const uint32_t** out);
void plan_destroy(CommitPlan* p);

}  // namespace prover
}  // namespace gs
