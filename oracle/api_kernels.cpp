// ORACLE — test infrastructure only (see fields.h).
// extern "C" surface of the CPU restatement used by the parity tests (via
// ctypes) and by bench.py's CPU baseline. QM31 columns cross this boundary as
// 4 coordinate planes, QM31 scalars as uint32[4], hashes as 32 bytes.
#include "fri_ops.h"
#include "merkle.h"
#include "channel.h"
#include <omp.h>

using namespace orc;

static QM31 q_in(const uint32_t* v) { return QM31::u(v[0], v[1], v[2], v[3]); }
static void q_out(QM31 q, uint32_t* o) { for (int i = 0; i < 4; i++) o[i] = q.coord(i); }
static std::vector<QM31> planes_in(const uint32_t* const* p, size_t n) {
  std::vector<QM31> r(n);
  for (size_t i = 0; i < n; i++) r[i] = QM31::u(p[0][i], p[1][i], p[2][i], p[3][i]);
  return r;
}
static void planes_out(const std::vector<QM31>& v, uint32_t* const* p) {
  for (size_t i = 0; i < v.size(); i++) for (int c = 0; c < 4; c++) p[c][i] = v[i].coord(c);
}
static std::vector<M31> col_in(const uint32_t* p, size_t n) {
  std::vector<M31> r(n);
  for (size_t i = 0; i < n; i++) r[i] = M31(p[i]);
  return r;
}

extern "C" {

void oracle_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int oracle_max_threads(void) { return omp_get_max_threads(); }

// M31 helpers (fields/m31.rs) for known-answer checks.
uint32_t oracle_m31_reduce(uint64_t v) { return reduce64(v); }
uint32_t oracle_m31_partial_reduce(uint32_t v) { return partial_reduce(v); }
uint32_t oracle_m31_mul(uint32_t a, uint32_t b) { return (M31(a) * M31(b)).v; }
uint32_t oracle_m31_inv(uint32_t a) { return inv(M31(a)).v; }
void oracle_qm31_mul(const uint32_t* a, const uint32_t* b, uint32_t* out) { q_out(q_in(a) * q_in(b), out); }
void oracle_qm31_inv(const uint32_t* a, uint32_t* out) { q_out(inv(q_in(a)), out); }

// Point of the M31 circle at a CirclePointIndex.
void oracle_index_to_point(uint64_t index, uint32_t* xy) {
  auto p = CPI{index}.reduce().to_point();
  xy[0] = p.x.v; xy[1] = p.y.v;
}
// Order check of the secure-field generator: out = GEN * scalar (scalar as lo/hi u64).
void oracle_secure_gen_mul(uint64_t lo, uint64_t hi, uint32_t* out8) {
  unsigned __int128 s = ((unsigned __int128)hi << 64) | lo;
  auto p = mul_scalar(SECURE_FIELD_CIRCLE_GEN, s);
  q_out(p.x, out8); q_out(p.y, out8 + 4);
}

void oracle_blake2s(const uint8_t* data, size_t len, uint8_t* out32) {
  Hash32 h = Blake2s::hash(data, len);
  memcpy(out32, h.data(), 32);
}

// Twiddle tree of the coset half_odds(log_size) (the coset prove() uses).
void oracle_twiddles_half_odds(uint32_t log_size, uint32_t* tw, uint32_t* itw) {
  TwiddleTree t = precompute_twiddles(Coset::half_odds(log_size));
  for (size_t i = 0; i < t.twiddles.size(); i++) { tw[i] = t.twiddles[i].v; itw[i] = t.itwiddles[i].v; }
}

// Interpolate bit-reversed evaluations on CanonicCoset(log_n) in place, using
// the twiddle tree of half_odds(root_log) (root_log >= log_n - 1).
void oracle_interpolate(uint32_t* values, uint32_t log_n, uint32_t root_log) {
  TwiddleTree t = precompute_twiddles(Coset::half_odds(root_log));
  auto v = col_in(values, (size_t)1 << log_n);
  interpolate(v, CanonicCoset::make(log_n).circle_domain(), t);
  for (size_t i = 0; i < v.size(); i++) values[i] = v[i].v;
}
// Batched variant for many columns of one size (threads over columns).
void oracle_interpolate_columns(uint32_t** cols, uint32_t n_cols, uint32_t log_n, uint32_t root_log) {
  TwiddleTree t = precompute_twiddles(Coset::half_odds(root_log));
  CircleDomain d = CanonicCoset::make(log_n).circle_domain();
#pragma omp parallel for schedule(dynamic)
  for (long long c = 0; c < (long long)n_cols; c++) {
    auto v = col_in(cols[c], (size_t)1 << log_n);
    interpolate(v, d, t);
    for (size_t i = 0; i < v.size(); i++) cols[c][i] = v[i].v;
  }
}
// Evaluate `coeff_len` coefficients on CanonicCoset(log_n), bit-reversed order.
void oracle_evaluate(const uint32_t* coeffs, size_t coeff_len, uint32_t log_n, uint32_t root_log, uint32_t* out) {
  TwiddleTree t = precompute_twiddles(Coset::half_odds(root_log));
  auto v = evaluate(col_in(coeffs, coeff_len), CanonicCoset::make(log_n).circle_domain(), t);
  for (size_t i = 0; i < v.size(); i++) out[i] = v[i].v;
}
void oracle_evaluate_columns(const uint32_t* const* coeffs, uint32_t n_cols, size_t coeff_len, uint32_t log_n,
                             uint32_t root_log, uint32_t* const* out) {
  TwiddleTree t = precompute_twiddles(Coset::half_odds(root_log));
  CircleDomain d = CanonicCoset::make(log_n).circle_domain();
#pragma omp parallel for schedule(dynamic)
  for (long long c = 0; c < (long long)n_cols; c++) {
    auto v = evaluate(col_in(coeffs[c], coeff_len), d, t);
    for (size_t i = 0; i < v.size(); i++) out[c][i] = v[i].v;
  }
}

void oracle_bit_reverse(uint32_t* values, uint32_t log_n) {
  std::vector<uint32_t> v(values, values + ((size_t)1 << log_n));
  bit_reverse(v);
  memcpy(values, v.data(), v.size() * 4);
}

// One Merkle layer (commit_on_layer). prev may be NULL (leaf layer).
void oracle_commit_on_layer(uint32_t log_size, const uint8_t* prev, uint32_t n_cols, const uint32_t* const* cols, uint8_t* out) {
  size_t n = (size_t)1 << log_size;
  std::vector<std::vector<M31>> cv(n_cols);
  std::vector<const std::vector<M31>*> cp;
  for (uint32_t c = 0; c < n_cols; c++) { cv[c] = col_in(cols[c], n); cp.push_back(&cv[c]); }
  std::vector<Hash32> pv;
  if (prev) { pv.resize(2 * n); memcpy(pv.data(), prev, 64 * n); }
  auto r = commit_on_layer(log_size, prev ? &pv : nullptr, cp);
  memcpy(out, r.data(), 32 * n);
}

// Lifted Merkle leaves (2^lift hashes, or 1 for no columns).
void oracle_lifted_leaves(uint32_t n_cols, const uint32_t* const* cols, const uint32_t* log_sizes, uint32_t lift,
                          uint8_t* out) {
  std::vector<std::vector<M31>> cv(n_cols);
  std::vector<const std::vector<M31>*> cp;
  for (uint32_t c = 0; c < n_cols; c++) { cv[c] = col_in(cols[c], (size_t)1 << log_sizes[c]); cp.push_back(&cv[c]); }
  auto r = lifted_leaves(cp, lift);
  memcpy(out, r.data(), 32 * r.size());
}

// Full Merkle commit of columns with the given log sizes; writes the root.
void oracle_merkle_root(uint32_t n_cols, const uint32_t* const* cols, const uint32_t* log_sizes, uint8_t* root) {
  std::vector<std::vector<M31>> cv(n_cols);
  std::vector<const std::vector<M31>*> cp;
  for (uint32_t c = 0; c < n_cols; c++) { cv[c] = col_in(cols[c], (size_t)1 << log_sizes[c]); cp.push_back(&cv[c]); }
  auto mp = MerkleProver::commit(cp);
  memcpy(root, mp.root().data(), 32);
}

// Channel known-answer checks: start from the default channel, run a script.
void oracle_channel_mix_u32s(const uint32_t* words, size_t n, uint8_t* digest_out) {
  Channel ch;
  ch.mix_u32s(std::vector<uint32_t>(words, words + n));
  memcpy(digest_out, ch.digest.data(), 32);
}
void oracle_channel_mix_u64(uint64_t v, uint8_t* digest_out) {
  Channel ch;
  ch.mix_u64(v);
  memcpy(digest_out, ch.digest.data(), 32);
}
// Draws n secure felts from a channel whose digest is `digest`; out = 4n u32.
uint32_t oracle_channel_draw_secure_felts(const uint8_t* digest, size_t n, uint32_t* out) {
  Channel ch;
  memcpy(ch.digest.data(), digest, 32);
  auto f = ch.draw_secure_felts(n);
  for (size_t i = 0; i < n; i++) q_out(f[i], out + 4 * i);
  return ch.n_draws;
}

uint64_t oracle_grind(const uint8_t* digest, uint32_t pow_bits) {
  Channel ch;
  memcpy(ch.digest.data(), digest, 32);
  return ch.grind(pow_bits);
}
int oracle_verify_pow(const uint8_t* digest, uint32_t pow_bits, uint64_t nonce) {
  Channel ch;
  memcpy(ch.digest.data(), digest, 32);
  return ch.verify_pow_nonce(pow_bits, nonce) ? 1 : 0;
}

// ---- Poseidon252 (felt252 values as 32 big-endian bytes)
// MerkleOps<Poseidon252MerkleHasher>::commit_on_layer; prev may be NULL.
void oracle_p252_commit_on_layer(uint32_t log_size, const uint8_t* prev, uint32_t n_cols, const uint32_t* const* cols,
                                 uint8_t* out) {
  size_t n = (size_t)1 << log_size;
  std::vector<std::vector<M31>> cv(n_cols);
  std::vector<const std::vector<M31>*> cp;
  for (uint32_t c = 0; c < n_cols; c++) { cv[c] = col_in(cols[c], n); cp.push_back(&cv[c]); }
  std::vector<Hash32> pv;
  if (prev) { pv.resize(2 * n); memcpy(pv.data(), prev, 64 * n); }
  auto r = commit_on_layer(log_size, prev ? &pv : nullptr, cp, MerkleHash::Poseidon252);
  memcpy(out, r.data(), 32 * n);
}
// The Hades permutation of n states (3 felts each, reduced mod p on input).
void oracle_p252_permute(const uint8_t* in, size_t n, uint8_t* out) {
  for (size_t k = 0; k < n; k++) {
    std::array<p252::Fe, 3> s;
    for (int j = 0; j < 3; j++) s[j] = p252::from_int(p252::reduce_be(in + 96 * k + 32 * j));
    p252::permute(s);
    for (int j = 0; j < 3; j++) memcpy(out + 96 * k + 32 * j, p252::to_hash(s[j]).data(), 32);
  }
}
static p252::Channel p252_channel(const uint8_t* digest, uint32_t n_draws) {
  p252::Channel ch;
  ch.digest = p252::from_hash(digest);
  ch.n_draws = n_draws;
  return ch;
}
// One channel operation from the state (digest, n_draws); writes the new
// digest and returns the new n_draws. op 0: mix_root(bytes), 1: mix_u64(v),
// 2: mix_u32s(words, n), 3: mix_felts(n QM31 as 4n words), 4: draw n secure
// felts into out (4n words), 5: draw_u32s n times into out (7n words).
uint32_t oracle_p252_channel_op(const uint8_t* digest, uint32_t n_draws, uint32_t op, const uint8_t* bytes, uint64_t v,
                                const uint32_t* words, size_t n, uint32_t* out, uint8_t* digest_out) {
  p252::Channel ch = p252_channel(digest, n_draws);
  if (op == 0) ch.mix_root(bytes);
  else if (op == 1) ch.mix_u64(v);
  else if (op == 2) ch.mix_u32s(std::vector<uint32_t>(words, words + n));
  else if (op == 3) {
    std::vector<std::array<uint32_t, 4>> f(n);
    for (size_t i = 0; i < n; i++) for (int c = 0; c < 4; c++) f[i][c] = words[4 * i + c];
    ch.mix_felts(f);
  } else if (op == 4) {
    Channel full(MerkleHash::Poseidon252);
    full.pc = ch;
    auto f = full.draw_secure_felts(n);
    for (size_t i = 0; i < n; i++) q_out(f[i], out + 4 * i);
    ch = full.pc;
  } else if (op == 5) {
    for (size_t i = 0; i < n; i++) {
      auto w = ch.draw_u32s();
      memcpy(out + 7 * i, w.data(), 28);
    }
  }
  memcpy(digest_out, p252::to_hash(ch.digest).data(), 32);
  return ch.n_draws;
}
uint64_t oracle_p252_grind(const uint8_t* digest, uint32_t pow_bits) { return p252_channel(digest, 0).grind(pow_bits); }
int oracle_p252_verify_pow(const uint8_t* digest, uint32_t pow_bits, uint64_t nonce) {
  return p252_channel(digest, 0).verify_pow_nonce(pow_bits, nonce) ? 1 : 0;
}

// fold_line on LineDomain(half_odds(log_n)); eval/out are QM31 planes.
void oracle_fold_line(const uint32_t* const* eval, uint32_t log_n, const uint32_t* alpha, uint32_t* const* out) {
  auto v = planes_in(eval, (size_t)1 << log_n);
  auto r = fold_line(v, Coset::half_odds(log_n), q_in(alpha));
  planes_out(r, out);
}
// fold_circle_into_line from CanonicCoset(log_n) into dst of size 2^(log_n-1).
void oracle_fold_circle_into_line(uint32_t* const* dst, const uint32_t* const* src, uint32_t log_n, const uint32_t* alpha) {
  auto s = planes_in(src, (size_t)1 << log_n);
  auto d = planes_in((const uint32_t* const*)dst, (size_t)1 << (log_n - 1));
  fold_circle_into_line(d, s, CanonicCoset::make(log_n).circle_domain(), q_in(alpha));
  planes_out(d, dst);
}

// One sample batch: out = Σ_k c_k·col[idx_k][row] − b_k (line coeffs from the
// sample point/value/random coeff), first linear term Σ a_k.
void oracle_accumulate_numerators(uint32_t log_size, uint32_t n_cols, const uint32_t* const* cols,
                                  const uint32_t* point8, uint32_t n_entries, const uint32_t* col_idx,
                                  const uint32_t* values4, const uint32_t* rand4,
                                  uint32_t* const* out, uint32_t* first_linear4) {
  size_t n = (size_t)1 << log_size;
  std::vector<std::vector<M31>> cv(n_cols);
  std::vector<const std::vector<M31>*> cp;
  for (uint32_t c = 0; c < n_cols; c++) { cv[c] = col_in(cols[c], n); cp.push_back(&cv[c]); }
  ColumnSampleBatch b;
  b.point = {q_in(point8), q_in(point8 + 4)};
  for (uint32_t k = 0; k < n_entries; k++) b.entries.push_back({col_idx[k], q_in(values4 + 4 * k), q_in(rand4 + 4 * k)});
  std::vector<AccumulatedNumerators> accs;
  accumulate_numerators(cp, {b}, accs);
  planes_out(accs[0].partial, out);
  q_out(accs[0].first_linear_term, first_linear4);
}

void oracle_compute_quotients_and_combine(uint32_t n_accs, const uint32_t* const* partial_planes /* 4*n_accs */,
                                          const uint32_t* log_sizes, const uint32_t* first_linear4,
                                          const uint32_t* points8, uint32_t lifting_log_size, uint32_t* const* out) {
  std::vector<AccumulatedNumerators> accs(n_accs);
  for (uint32_t a = 0; a < n_accs; a++) {
    accs[a].partial = planes_in(partial_planes + 4 * a, (size_t)1 << log_sizes[a]);
    accs[a].first_linear_term = q_in(first_linear4 + 4 * a);
    accs[a].sample_point = {q_in(points8 + 8 * a), q_in(points8 + 8 * a + 4)};
  }
  planes_out(compute_quotients_and_combine(accs, lifting_log_size), out);
}

// lift_and_accumulate over columns given in increasing size order.
void oracle_lift_and_accumulate(uint32_t n, const uint32_t* const* planes, const uint32_t* log_sizes, uint32_t* const* out) {
  std::vector<std::vector<QM31>> cols;
  for (uint32_t i = 0; i < n; i++) cols.push_back(planes_in(planes + 4 * i, (size_t)1 << log_sizes[i]));
  planes_out(lift_and_accumulate(cols), out);
}

void oracle_eval_at_point(const uint32_t* coeffs, uint32_t log_n, const uint32_t* point8, uint32_t* out4) {
  auto c = col_in(coeffs, (size_t)1 << log_n);
  q_out(eval_at_point(c, {q_in(point8), q_in(point8 + 4)}), out4);
}

}  // extern "C"
