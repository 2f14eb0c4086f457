// gpustark runtime: execution context, error reporting and the internal
// (C++) launch interface shared by the kernels, the C ABI and the host prover.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>
#include "m31.cuh"

namespace gs {

enum Status : int {
  OK = 0,
  ERR_INVALID = 1,    // bad argument (size, alignment, null pointer)
  ERR_CUDA = 2,       // CUDA runtime / launch failure
  ERR_OOM = 3,        // device allocation failed
  ERR_UNSUPPORTED = 4,
  ERR_PROOF = 5,      // proving failed (constraints not satisfied)
  ERR_TIMEOUT = 6,    // a bounded device wait ran out
};

void set_error(const std::string& msg);
const char* last_error();

#define GS_CUDA_TRY(expr)                                                                 \
  do {                                                                                    \
    cudaError_t _e = (expr);                                                              \
    if (_e != cudaSuccess) {                                                              \
      ::gs::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e) + " @" __FILE__); \
      return ::gs::ERR_CUDA;                                                              \
    }                                                                                     \
  } while (0)
#define GS_REQUIRE(cond, msg)                     \
  do {                                            \
    if (!(cond)) {                                \
      ::gs::set_error(std::string("invalid: ") + (msg)); \
      return ::gs::ERR_INVALID;                   \
    }                                             \
  } while (0)
#define GS_TRY(expr)                      \
  do {                                    \
    int _s = (expr);                      \
    if (_s != ::gs::OK) return _s;        \
  } while (0)

// A QM31 column as 4 coordinate planes, passed by value to kernels.
struct Planes { uint32_t* p[4]; };
struct CPlanes { const uint32_t* p[4]; };

// Count of kernel launches issued by this library (for launch accounting).
void note_launch(unsigned n = 1);
unsigned long long launch_count();

// Point tables of a canonic circle domain of log size `lift`: natural-order
// half-coset point j is hi[j >> s] + lo[j & (2^s - 1)]; the other half are the
// conjugates (used to get domain points from bit-reversed row indices).
struct DomainTables {
  const pt31* hi;
  const pt31* lo;
  uint32_t s;
  uint32_t lift;
};

#ifdef __CUDACC__
__device__ __forceinline__ pt31 ld_pt(const pt31* p) {
  uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
  return {v.x, v.y};
}
// CanonicCoset(lift).circle_domain().at(bit_reverse(row)).
__device__ __forceinline__ pt31 domain_point_bitrev(const DomainTables& t, uint32_t row) {
  uint32_t j = __brev(row) >> (32 - t.lift);
  uint32_t half = 1u << (t.lift - 1);
  bool second = j >= half;
  if (second) j -= half;
  pt31 p = pt_add(ld_pt(t.hi + (j >> t.s)), ld_pt(t.lo + (j & ((1u << t.s) - 1))));
  return second ? pt_conj(p) : p;
}
#endif

// Waits for `st`. By default CUDA's own stream synchronisation (the lowest
// latency for one proof at a time). A thread that installs a blocking-sync
// event (the proof server's workers, many threads sharing one device and the
// host cores) records it, polls it for a short window (GS_WAIT_SPIN_US,
// default 50 µs: most waits are short read-backs, which a sleep and wake-up
// would lengthen), then sleeps on it.
int stream_sync(cudaStream_t st);
// Waits for an event recorded earlier (through the thread's hook if one is set).
int event_sync(cudaEvent_t ev);
void set_thread_wait_event(cudaEvent_t ev);
// Replaces stream_sync's wait on the calling thread (the proof server's
// fiber scheduler installs one; nullptr restores the default).
void set_thread_sync_hook(int (*hook)(cudaStream_t, cudaEvent_t));

// Number of SMs of the current device (cached).
int num_sms();

// Execution context: one CUDA stream plus a device-side ring for the column
// pointer tables that the C ABI receives as host arrays.
struct Context {
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;
  // A proof runs on `work`, a stream of the device's greatest priority
  // (ordered after the caller's stream on entry); `side`, of the lowest
  // priority, carries work that the protocol's next steps do not need yet,
  // so its blocks take only the SMs that latency-bound work on `work`
  // leaves idle. Both are created on first use (begin_proof).
  cudaStream_t work = nullptr, side = nullptr;
  cudaStream_t caller = nullptr;  // may be the legacy default stream (null)
  bool in_proof = false;
  cudaEvent_t ev_enter = nullptr, ev_fork = nullptr, ev_join = nullptr;
  bool side_pending = false;
  int begin_proof();  // stream := work, after the caller's stream
  int end_proof();    // the caller's stream after work; stream := caller
  int fork_side();    // side waits for the work enqueued on `stream` so far
  int join_side();    // `stream` waits for the side work enqueued so far
  // pointer-table staging: pinned host ring -> device ring, stream ordered
  uint8_t* h_ring = nullptr;
  uint8_t* d_ring = nullptr;
  size_t ring_cap = 0, ring_off = 0;
  // small device scratch for results (grind, reductions)
  uint8_t* d_small = nullptr;
  uint8_t* h_small = nullptr;  // pinned mirror
  size_t small_cap = 0;
  // ticket counters of the one-launch Merkle tree kernel (TREE_COUNTERS words)
  uint32_t* tree_counters = nullptr;

  // Stream-ordered memory pool owned by this context. Contexts that run
  // concurrently (the proof server's workers) do not share a pool, so
  // reusing freed memory never inserts a dependency on another stream.
  cudaMemPool_t pool = nullptr;
  int alloc_async(size_t bytes, void** out);
  // The last proof's pool allocations (size, pointer), kept for the next
  // proof on this context: a proof of the same shape makes the same requests
  // and takes them back in stream order without a pool call, and the last
  // proof's frees do not delay its return. Buffers the next proof does not
  // take are freed when it ends. Off (keep_buffers = false) for the proof
  // server's contexts, whose HBM budget counts only the proofs in flight.
  bool keep_buffers = true;
  std::vector<std::pair<size_t, void*>> spare;
  // Small device-to-host read through the pinned mailbox, then synchronise.
  int read_back(const void* d_src, size_t bytes, void* host_dst);
  // Reads that the host waits for later: mail_start enqueues a copy of at
  // most MAIL_BYTES into slot `slot` of a pinned area of its own and records
  // the slot's event; work enqueued after it runs on meanwhile, and
  // mail_wait(slot) waits for that event only (not for the stream).
  static constexpr int MAIL_SLOTS = 4;
  static constexpr size_t MAIL_BYTES = 256;
  uint8_t* h_mail = nullptr;
  // The slots' device alias (the area is mapped pinned memory), or null: a
  // kernel that writes its result there directly needs no copy, only
  // mail_record(slot) after it.
  uint8_t* d_mail = nullptr;
  cudaEvent_t mail_ev[MAIL_SLOTS] = {nullptr};
  int mail_start(int slot, const void* d_src, size_t bytes);
  int mail_record(int slot);
  int mail_wait(int slot, const void** host);
  // growable pinned host buffer for read-backs (decommitment values), and
  // its device alias (mapped pinned memory), or null
  uint8_t* h_read = nullptr;
  void* d_read = nullptr;
  size_t read_cap = 0;
  int read_buffer(size_t bytes, void** out);
  // Stores `bytes` (a multiple of 4) from device memory into the read
  // buffer with a kernel on the context's stream (no copy-engine step
  // between the producing kernels and the host), or with a copy where the
  // buffer has no device alias; *host points to them once the stream has
  // reached this point.
  int publish(const void* d_src, size_t bytes, const void** host);
  // read_back through publish: the same result.
  int read_back_published(const void* d_src, size_t bytes, void* host_dst);
  // growable device scratch (stream ordered)
  void* scratch = nullptr;
  size_t scratch_cap = 0;
  // cached domain point tables per lifting log size
  void* dom_buf[31] = {nullptr};
  DomainTables dom[31];

  int init(void* user_stream);
  int stage_bytes(const void* host, size_t bytes, const void** out);
  int get_scratch(size_t bytes, void** out);
  int domain_tables(uint32_t lift, DomainTables* out);
  // device-resident twiddle trees of half_odds(root_log), kept across calls
  uint32_t* tw_buf[31] = {nullptr};
  uint32_t* itw_buf[31] = {nullptr};
  int twiddles(uint32_t root_log, const uint32_t** tw, const uint32_t** itw);
  void destroy();
  // Copies `n` host pointers into device memory usable by kernels launched on
  // `stream` after this call; returns the device address.
  int stage_ptrs(const void* const* host_ptrs, size_t n, const void* const** out);
  int sync();
};

// ------------------------------------------------------------ launch API
// All functions enqueue work on `st` and return a Status.

// twiddles.cu
int precompute_twiddles(cudaStream_t st, uint32_t initial_index, uint32_t step_index, uint32_t log_size,
                        uint32_t* d_twiddles, uint32_t* d_itwiddles);
int batch_inverse(cudaStream_t st, const uint32_t* d_in, uint32_t* d_out, size_t n);

// fft.cu (columns given by a device table of pointers)
int interpolate_columns(cudaStream_t st, uint32_t* const* d_cols, uint32_t n_cols, uint32_t log_n,
                        const uint32_t* d_itwiddles, uint32_t tw_log);
// One FFT of a work-list: interpolate (inverse != 0) 2^log evaluations, or
// evaluate 2^coeff_log coefficients on the domain of 2^log; src and dst are
// device columns (the same column for an in-place interpolation).
struct FftItem {
  const uint32_t* src;
  uint32_t* dst;
  uint32_t log, coeff_log, inverse, pad;
};
constexpr uint32_t FFT_WL_MIN_LOG = 3, FFT_WL_MAX_LOG = 13;
// Many FFTs of uneven sizes: every item of log size in [FFT_WL_MIN_LOG,
// FFT_WL_MAX_LOG] in one launch of a persistent grid whose blocks walk the
// list (largest first), each item whole in shared memory; the others through
// interpolate_columns / evaluate_columns, one call each. Twiddle trees as for
// those (tw_log + 1 >= every log).
int fft_worklist(Context& ctx, const FftItem* items, uint32_t n_items, const uint32_t* d_twiddles,
                 const uint32_t* d_itwiddles, uint32_t tw_log);
int evaluate_columns(cudaStream_t st, const uint32_t* const* d_src, uint32_t coeff_log, uint32_t* const* d_dst,
                     uint32_t n_cols, uint32_t log_n, const uint32_t* d_twiddles, uint32_t tw_log);
int bit_reverse(cudaStream_t st, uint32_t* d, uint32_t log_n);
// Pass-split tuning per number of computed layers and extension (domain log
// size minus layers), process-wide, written at set-up time.
int set_fft_tuning(uint32_t layers, uint32_t ext, uint32_t tile_log, uint32_t coalesce_bits);
void get_fft_tuning(uint32_t layers, uint32_t ext, uint32_t* tile_log, uint32_t* coalesce_bits);
int fft_autotune(cudaStream_t st, uint32_t lo, uint32_t hi, uint32_t max_ext, const uint32_t* tw, const uint32_t* itw,
                 uint32_t tw_log, uint32_t* out_tile, uint32_t* out_coalesce);

// merkle.cu
int commit_on_layer(cudaStream_t st, uint32_t log_size, const uint32_t* d_prev, const uint32_t* const* d_cols,
                    uint32_t n_cols, uint32_t* d_out);
// All node-only layers below `top_log` (layers[L] has 2^L hashes, layers[top_log] given),
// in one launch up to TREE_MAX_LOG. d_counters: TREE_COUNTERS zeroed words
// owned by the calling stream (left zeroed); no two launches that share them
// may run at the same time.
constexpr uint32_t TREE_MAX_LOG = 27;
constexpr uint32_t TREE_COUNTERS = 1024;
int commit_node_layers(cudaStream_t st, uint32_t top_log, uint32_t* const* layers, uint32_t* d_counters);
// One tree of a Merkle work-list: n_cols >= 1 device columns of 2^log words
// (host array of pointers) and log + 1 device layers (host array; layers[L]
// holds 2^L hashes, 16-byte aligned), the leaves hashing the columns.
struct MerkleItem {
  const uint32_t* const* cols;
  uint32_t n_cols, log;
  uint32_t* const* layers;
};
constexpr uint32_t MERKLE_WL_MAX_LOG = 10;
// Many trees: every tree of log <= MERKLE_WL_MAX_LOG whole (leaves and every
// node layer) in one launch of a persistent grid walking the list, largest
// first, each tree in one block through shared memory; larger trees through
// commit_on_layer + commit_node_layers, one tree at a time.
int merkle_worklist(Context& ctx, const MerkleItem* items, uint32_t n_items);
// The same, with the root also written to root_out (8 words, e.g. mapped
// host memory) by the launch that computes it (or copied there when no tree
// kernel runs).
int commit_node_layers_to(cudaStream_t st, uint32_t top_log, uint32_t* const* layers, uint32_t* d_counters,
                          uint32_t* root_out);
// The same, followed by the Fiat-Shamir channel step on the root in the same
// launch (the FRI commit phase).
int commit_node_layers_ch(cudaStream_t st, uint32_t top_log, uint32_t* const* layers, uint32_t* d_counters,
                          uint32_t* d_state, uint32_t* d_root_copy, uint32_t* d_felt);
// Lifted Merkle leaves; d_shifts[c] = lift - log size of column c (columns in
// increasing size order).
int lifted_leaves(cudaStream_t st, uint32_t lift, const uint32_t* const* d_cols, const uint8_t* d_shifts,
                  uint32_t n_cols, uint32_t* d_out);

// poseidon252.cu: Poseidon252 Merkle layers and permutations; hashes are
// felt252 values as 32 big-endian bytes.
int poseidon252_commit_on_layer(cudaStream_t st, uint32_t log_size, const uint8_t* d_prev,
                                const uint32_t* const* d_cols, uint32_t n_cols, uint8_t* d_out);
int poseidon252_permute(cudaStream_t st, const uint8_t* d_in, uint32_t n, uint8_t* d_out);
// d_scratch: 48 bytes of device memory; h_word: 8 bytes of pinned host memory.
// digest_is_prefixed: d_digest already holds poseidon_hash_many([POW_PREFIX,
// digest, pow_bits]) (computed by a host that has the channel).
int poseidon252_grind(cudaStream_t st, const uint8_t* d_digest, uint32_t pow_bits, uint8_t* d_scratch,
                      uint32_t* h_word, uint64_t* nonce_out, bool digest_is_prefixed = false);

// FRI layers of log size <= 11 in one launch (fri.cu): layer k has log size
// log0 - k; layers 0..n-1 are committed (tree[k][L] = their Merkle layers,
// leaves of layer 0 already hashed), layer n is the last layer.
constexpr uint32_t FRI_TAIL_MAX = 12;
// Largest layer (log size) handled by the cluster tails: Merkle node layers
// below it, and the fused FRI tail from it down.
constexpr uint32_t MERKLE_TAIL_LOG = 11;
constexpr uint32_t FRI_TAIL_LOG = 11;
struct FriTail {
  uint32_t n = 0, log0 = 0;
  uint32_t* planes[FRI_TAIL_MAX + 1][4] = {};
  uint32_t* tree[FRI_TAIL_MAX][FRI_TAIL_MAX] = {};
  uint32_t* roots = nullptr;  // 8 words per committed layer
  uint32_t* felts = nullptr;  // 8 words per committed layer (challenge, square)
};
int fri_tail(cudaStream_t st, const FriTail& a, uint32_t* d_state, const uint32_t* d_itw, uint32_t tw_log);

// fri.cu
int fold_line(cudaStream_t st, CPlanes src, uint32_t log_n, qm31 alpha, Planes dst, const uint32_t* d_itwiddles,
              uint32_t tw_log);
int fold_circle_into_line(cudaStream_t st, CPlanes src, uint32_t log_n, qm31 alpha, Planes dst,
                          const uint32_t* d_itwiddles, uint32_t tw_log);

// quotients.cu
// vec: every column pointer and output plane is 16-byte aligned (4 rows per
// thread with vector loads).
// d_bsum (optional): b_sum as 4 words in device memory, written by an earlier
// kernel of the stream (quot_line_coeffs); the b_sum argument is then unused.
int accumulate_numerators(cudaStream_t st, const void* d_entries, uint32_t n_entries, qm31 b_sum, uint32_t log_size,
                          Planes out, bool vec = false, const uint32_t* d_bsum = nullptr);
int compute_quotients_and_combine(cudaStream_t st, const void* d_accs, uint32_t n_accs, const DomainTables& dt,
                                  Planes out);
int lift_and_accumulate(cudaStream_t st, const void* d_cols, uint32_t n_cols, uint32_t log_size, Planes out);
int accumulate(cudaStream_t st, Planes a, CPlanes b, size_t n);
int make_domain_tables(cudaStream_t st, uint32_t lift, pt31* d_buf, DomainTables* out);
size_t domain_tables_len(uint32_t lift);
// entry layouts shared with the host side
struct NumEntry { const uint32_t* col; uint32_t c[4]; };
struct QuotAcc {
  const uint32_t* p[4];
  uint32_t log_size;
  uint32_t pad;
  qm31 first_linear;
  cm31 prx, pry, pix, piy;
};
struct LiftCol { const uint32_t* p[4]; uint32_t log_size; uint32_t pad; };
// One term of the DEEP quotients: a column's value at a sample point.
// val: word offset of the value (4 words) in the sampled values; point: its
// sample point; k: the power of the random coefficient it takes.
struct LineTerm { uint32_t val, point, k, pad; };
constexpr uint32_t QUOT_MAX_BATCHES = 32, QUOT_MAX_POINTS = 16;
// The line coefficients of every term (complex_conjugate_line_coeffs with
// alpha^k, core/constraints.rs:119-134), in one block: c into entries[i] (the
// entries of batch b are [batch_first[b], batch_first[b + 1])), the batch's
// sum of b into d_bsums[4b, 4b + 4), and per sample point the sum of a over
// its batches (batch_point[b]) into accs[point].first_linear. d_scratch: 8
// words per term. points: ptq per sample point.
int quot_line_coeffs(cudaStream_t st, const LineTerm* d_terms, uint32_t n_terms, const uint32_t* d_vals,
                     const ptq* d_points, qm31 alpha, NumEntry* d_entries, const uint32_t* d_batch_first,
                     const uint32_t* d_batch_point, uint32_t n_batches, uint32_t* d_bsums, QuotAcc* d_accs,
                     uint32_t n_points, uint32_t* d_scratch);

// eval_at_point.cu
size_t eval_at_point_scratch_bytes(uint32_t n_polys, uint32_t log_n, uint32_t chunk_log = 12);
int batch_eval_at_point(cudaStream_t st, const uint32_t* const* d_polys, uint32_t n_polys, uint32_t log_n, ptq point,
                        uint32_t* d_out, uint32_t* d_scratch, uint32_t chunk_log = 12, bool vec = false);

// barycentric weights on CanonicCoset(dt.lift) (4 planes) and evaluation
// (d_scratch: barycentric_scratch_words(n) words; d_out: 4 words)
int barycentric_weights(cudaStream_t st, const DomainTables& dt, ptq p, Planes out);
size_t barycentric_scratch_words(size_t n);
int barycentric_eval(cudaStream_t st, const uint32_t* d_evals, CPlanes w, size_t n, uint32_t* d_scratch,
                     uint32_t* d_out);
// quotients.cu: out[i] = felt^i
int secure_powers(cudaStream_t st, qm31 felt, size_t n, Planes out);
// gather.cu: Column::batch_at_multi (row-major) and hashes of one layer
int gather_multi(cudaStream_t st, const uint32_t* const* d_cols, uint32_t n_cols, const uint32_t* d_idx,
                 uint32_t n_idx, uint32_t* d_out);
int gather_hashes(cudaStream_t st, const uint32_t* d_layer, const uint32_t* d_idx, uint32_t n_idx, uint32_t* d_out);

// grind.cu
// hi0: the first high word searched (a search whose chunk hi = 0 already ran
// on the device, as fri_last_layer_pow does, continues at 1)
int grind_blake2s(cudaStream_t st, const uint32_t prefixed_digest[8], uint32_t pow_bits, uint32_t* d_scratch,
                  uint64_t* nonce_out, uint32_t* h_word = nullptr, uint32_t hi0 = 0);
// The Blake2s channel's steps between the last FRI layer and the queries, on
// the device: the last layer (4 planes of 2^log values at d_last) into its
// LinePoly coefficients, mixed into the channel digest d_state[0, 8); the
// proof of work's prefixed digest; and the grind's first chunk (nonces below
// 2^20). d_out receives the 4 * 2^bound_log coefficient words, the mixed
// digest (8 words), the prefixed digest (8 words) and the smallest passing
// nonce of the chunk (1 word, all ones when none passed). Layers of at most
// FRI_POW_MAX_LOG values' log and bound_log <= 3; the host checks every word.
constexpr uint32_t FRI_POW_MAX_LOG = 5;
size_t fri_last_layer_pow_words(uint32_t bound_log);
int fri_last_layer_pow(cudaStream_t st, const uint32_t* d_last, uint32_t log, uint32_t bound_log, uint32_t pow_bits,
                       const uint32_t* d_state, uint32_t* d_out);

}  // namespace gs
