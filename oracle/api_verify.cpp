// ORACLE — test infrastructure only (see fields.h).
// C entry points of the verifier (verifier.h) and of the statement data a
// Poseidon2 verifier needs besides the proof: the lookup elements, drawn from
// the channel after the trace commitment, and the logup claimed sum of the
// trace (crates/examples/src/poseidon/mod.rs:305-335: the sum over rows of
// 1/combine(initial state) - 1/combine(final state)).
#include "verifier.h"
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace orc;

static void qm_out(const QM31& q, uint32_t* o) {
  for (int k = 0; k < 4; k++) o[k] = q.coord(k);
}
static QM31 qm_in(const uint32_t* w) { return QM31::from_m31(M31(w[0]), M31(w[1]), M31(w[2]), M31(w[3])); }

extern "C" {

// air: 0 = wide fibonacci (n_cols columns), 1 = poseidon2; claimed_sum: 4
// words (poseidon2 only; may be NULL for wide fibonacci); merkle_channel: 0 =
// Blake2sMerkleChannel, 1 = Poseidon252MerkleChannel; config: the verifier's
// PcsConfig as 5 words (pow_bits, log_blowup, log_last_layer, n_queries,
// line_fold_step), or NULL to take the one serialised in the proof (as the
// reference's Poseidon2 test does with proof.config). Returns 0 when the
// proof is accepted, else the error class (verifier.h Code) with a message.
int oracle_verify(uint32_t air, uint32_t log_n, uint32_t n_cols, uint32_t split_log, const uint32_t* claimed_sum,
                  uint32_t merkle_channel, const uint32_t* config, const uint8_t* proof, size_t proof_len, char* msg,
                  size_t msg_cap) {
  ver::Statement st;
  st.kind = air == 0 ? ver::Air::WideFibonacci : ver::Air::Poseidon;
  st.log_n = log_n;
  st.n_cols = n_cols;
  st.split_log = split_log;
  if (claimed_sum) st.claimed_sum = qm_in(claimed_sum);
  st.hash = merkle_channel ? MerkleHash::Poseidon252 : MerkleHash::Blake2s;
  ver::Result r;
  StarkProof p;
  if (!ver::deserialize(proof, proof_len, p)) r = ver::fail(ver::INVALID_STRUCTURE, "proof bytes do not parse");
  else if (st.kind == ver::Air::WideFibonacci && (n_cols < 3 || log_n < 1)) r = ver::fail(ver::INVALID_STRUCTURE, "statement");
  else {
    PcsConfig cfg = p.config;
    if (config) {
      cfg = PcsConfig{};
      cfg.pow_bits = config[0];
      cfg.log_blowup = config[1];
      cfg.log_last_layer = config[2];
      cfg.n_queries = config[3];
      cfg.fold_step = config[4];
    }
    r = ver::verify(st, p, cfg);
  }
  if (msg && msg_cap) {
    strncpy(msg, r.msg.c_str(), msg_cap - 1);
    msg[msg_cap - 1] = 0;
  }
  return r.code;
}

// The Poseidon2 lookup elements (z, alpha) a verifier draws from the proof's
// first two commitments (poseidon/mod.rs:913-917). Returns 0, or 1 when the
// bytes do not parse.
int oracle_verify_lookup_elements(uint32_t merkle_channel, const uint8_t* proof, size_t proof_len, uint32_t* z4,
                                  uint32_t* alpha4) {
  StarkProof p;
  if (!ver::deserialize(proof, proof_len, p) || p.commitments.size() < 2) return 1;
  Channel ch(merkle_channel ? MerkleHash::Poseidon252 : MerkleHash::Blake2s);
  ch.mix_root(p.commitments[0]);
  ch.mix_root(p.commitments[1]);
  auto zs = ch.draw_secure_felts(2);
  qm_out(zs[0], z4);
  qm_out(zs[1], alpha4);
  return 0;
}

// The logup claimed sum of a Poseidon2 trace: input_mode 0 = the reference's
// inputs (row + i), 1 = seeded (the provers' seeded rule), 2 = host_inputs
// (16 columns of 2^log_n words).
uint32_t oracle_seeded_m31(uint64_t seed, uint64_t col, uint64_t row);
void oracle_poseidon_claimed_sum(uint32_t log_n, uint64_t seed, uint32_t input_mode, const uint32_t* host_inputs,
                                 const uint32_t* z4, const uint32_t* alpha4, uint32_t* out4) {
  LookupElements16 le;
  le.z = qm_in(z4);
  le.alpha = qm_in(alpha4);
  QM31 cur(M31(1));
  for (int i = 0; i < 16; i++) {
    le.alpha_powers[i] = cur;
    cur = cur * le.alpha;
  }
  size_t n = (size_t)1 << log_n;
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  std::vector<QM31> partial(nt);
#pragma omp parallel
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    QM31 acc;
#pragma omp for schedule(static)
    for (long long rr = 0; rr < (long long)n; rr++) {
      size_t r = (size_t)rr;
      M31 s[16], cols[PN_COLUMNS], f[16];
      for (int i = 0; i < 16; i++) {
        if (input_mode == 0) s[i] = M31((uint32_t)((r + i) % P));
        else if (input_mode == 1) s[i] = M31(oracle_seeded_m31(seed, i, r));
        else s[i] = M31(host_inputs[(size_t)i * n + r]);
      }
      poseidon_trace_row(s, cols, f);
      acc += inv(combine16(le, s)) - inv(combine16(le, f));
    }
    partial[tid] = acc;
  }
  QM31 total;
  for (auto& q : partial) total += q;
  qm_out(total, out4);
}

}  // extern "C"
