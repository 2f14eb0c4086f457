// ORACLE — test infrastructure only (see fields.h).
// Full proofs of the two benchmark AIRs on the CPU restatement.
// Follows the example drivers:
//   crates/examples/src/wide_fibonacci/mod.rs:140-184   (cuda_prove_wide_fibonacci, input a=1, b=row)
//   crates/examples/src/poseidon/mod.rs:222-335,617-700 (trace, interaction trace, cuda_prove_poseidon)
//   crates/constraint-framework/src/prover/logup.rs     (LogupTraceGenerator: fractions, claimed sum,
//                                                        shifted inclusive prefix sum in coset order)
//   crates/stwo/src/prover/backend/simd/prefix_sum.rs:123-140 (coset-order prefix sum)
#include "prover.h"
#include <cstring>

using namespace orc;

// Seeded uniform M31 input (the "seeded" input mode): for column c and row r,
// the first value v = mix64(seed ^ mix64(c * 0x100000001B3 + (r << 8) + k)) & (2^31 - 1)
// over k = 0, 1, ... that is below P (SplitMix64 finalizer).
static inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static inline uint32_t seeded_m31(uint64_t seed, uint64_t col, uint64_t row) {
  for (uint64_t k = 0;; k++) {
    uint32_t v = (uint32_t)mix64(seed ^ mix64(col * 0x100000001B3ull + (row << 8) + k)) & 0x7fffffffu;
    if (v != P) return v;
  }
}

static size_t coset_index_of_storage(size_t i, uint32_t log_n) {
  size_t n = (size_t)1 << log_n;
  size_t j = bit_reverse_index(i, log_n);
  return j < n / 2 ? 2 * j : 2 * (n - 1 - j) + 1;
}

extern "C" {

uint32_t oracle_seeded_m31(uint64_t seed, uint64_t col, uint64_t row) { return seeded_m31(seed, col, row); }

// air: 0 = wide fibonacci (n_cols columns), 1 = poseidon2.
// input_mode: 0 = the reference examples' inputs, 1 = seeded uniform M31.
// Returns 0 on success (proof bytes in out, length in *out_len), 1 if the
// composition sanity check fails, 2 if the buffer is too small.
// split_log: composition split (1 = the reference's fixed split).
// merkle_channel: 0 = Blake2sMerkleChannel, 1 = Poseidon252MerkleChannel
// (wide_fibonacci/mod.rs:335-379, poseidon/mod.rs:702-785).
int oracle_prove(uint32_t air, uint32_t log_n, uint32_t n_cols, uint64_t seed, uint32_t input_mode, uint32_t pow_bits,
                 uint32_t n_queries, uint32_t log_blowup, uint32_t log_last_layer, uint32_t split_log,
                 uint32_t merkle_channel, void* out, size_t cap, size_t* out_len) {
  PcsConfig cfg;
  cfg.log_last_layer = log_last_layer;
  cfg.pow_bits = pow_bits;
  cfg.n_queries = n_queries;
  cfg.log_blowup = log_blowup;
  CommitmentScheme cs;
  cs.config = cfg;
  Channel ch(merkle_channel ? MerkleHash::Poseidon252 : MerkleHash::Blake2s);
  cs.commit_evals({}, ch);  // empty preprocessed tree
  size_t n = (size_t)1 << log_n;
  AirSpec spec;
  spec.log_n = log_n;
  if (air == 0) {
    spec.kind = AirKind::WideFibonacci;
    spec.n_cols = n_cols;
    std::vector<std::vector<M31>> cols(n_cols, std::vector<M31>(n));
#pragma omp parallel for schedule(static)
    for (long long rr = 0; rr < (long long)n; rr++) {
      size_t r = (size_t)rr;
      M31 a = input_mode ? M31(seeded_m31(seed, 0, r)) : M31(1);
      M31 b = input_mode ? M31(seeded_m31(seed, 1, r)) : M31((uint32_t)r);
      cols[0][r] = a;
      cols[1][r] = b;
      for (uint32_t k = 2; k < n_cols; k++) {
        M31 c = a * a + b * b;
        cols[k][r] = c;
        a = b;
        b = c;
      }
    }
    cs.commit_evals(cols, ch);
  } else {
    spec.kind = AirKind::Poseidon;
    std::vector<std::vector<M31>> cols(PN_COLUMNS, std::vector<M31>(n));
    std::vector<std::array<M31, 16>> init(n), fin(n);
#pragma omp parallel for schedule(static)
    for (long long rr = 0; rr < (long long)n; rr++) {
      size_t r = (size_t)rr;
      M31 s[16], row_cols[PN_COLUMNS], f[16];
      for (int i = 0; i < 16; i++) s[i] = input_mode ? M31(seeded_m31(seed, i, r)) : M31((uint32_t)(r + i));
      poseidon_trace_row(s, row_cols, f);
      for (int c = 0; c < PN_COLUMNS; c++) cols[c][r] = row_cols[c];
      for (int i = 0; i < 16; i++) { init[r][i] = s[i]; fin[r][i] = f[i]; }
    }
    cs.commit_evals(cols, ch);
    // lookup elements and the logup interaction column
    auto zs = ch.draw_secure_felts(2);
    spec.le.z = zs[0];
    spec.le.alpha = zs[1];
    QM31 cur(M31(1));
    for (int i = 0; i < 16; i++) { spec.le.alpha_powers[i] = cur; cur = cur * spec.le.alpha; }
    std::vector<QM31> val(n);
#pragma omp parallel for schedule(static)
    for (long long rr = 0; rr < (long long)n; rr++) {
      QM31 d0 = combine16(spec.le, init[rr].data()), d1 = combine16(spec.le, fin[rr].data());
      val[rr] = (d1 - d0) * inv(d0 * d1);
    }
    QM31 claimed;
    for (auto& v : val) claimed += v;
    spec.claimed_sum = claimed;
    QM31 shift = claimed / M31((uint32_t)n);
    std::vector<QM31> by_coset(n);
    for (size_t i = 0; i < n; i++) by_coset[coset_index_of_storage(i, log_n)] = val[i] - shift;
    for (size_t k = 1; k < n; k++) by_coset[k] = by_coset[k - 1] + by_coset[k];
    std::vector<std::vector<M31>> icols(4, std::vector<M31>(n));
    for (size_t i = 0; i < n; i++) {
      QM31 v = by_coset[coset_index_of_storage(i, log_n)];
      for (int c = 0; c < 4; c++) icols[c][i] = M31(v.coord(c));
    }
    cs.commit_evals(icols, ch);
  }
  ProveResult R = prove(cs, ch, spec, split_log);
  std::string bytes = serialize(R.proof);
  *out_len = bytes.size();
  if (!R.constraints_ok) return 1;
  if (bytes.size() > cap) return 2;
  memcpy(out, bytes.data(), bytes.size());
  return 0;
}

}  // extern "C"
