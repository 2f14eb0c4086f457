// gpustark runtime: context, error state, pointer-table staging.
#include "runtime.cuh"
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <atomic>

namespace gs {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

static std::atomic<unsigned long long> g_launches{0};
void note_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

static thread_local cudaEvent_t g_wait_ev = nullptr;
void set_thread_wait_event(cudaEvent_t ev) { g_wait_ev = ev; }
static double wait_spin_us() {
  static const double us = [] {
    const char* e = getenv("GS_WAIT_SPIN_US");
    return e ? atof(e) : 50.0;
  }();
  return us;
}
static thread_local int (*g_sync_hook)(cudaStream_t, cudaEvent_t) = nullptr;
void set_thread_sync_hook(int (*hook)(cudaStream_t, cudaEvent_t)) { g_sync_hook = hook; }

// Polls ev for the spin time, then blocks on it.
static int spin_then_wait(cudaEvent_t ev) {
  const double limit = wait_spin_us();
  const auto t0 = std::chrono::steady_clock::now();
  while (limit > 0) {
    const cudaError_t q = cudaEventQuery(ev);
    if (q == cudaSuccess) return OK;
    if (q != cudaErrorNotReady) GS_CUDA_TRY(q);
    if (std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count() > limit) break;
  }
  GS_CUDA_TRY(cudaEventSynchronize(ev));
  return OK;
}

int stream_sync(cudaStream_t st) {
  if (g_sync_hook) return g_sync_hook(st, nullptr);
  if (g_wait_ev) {
    GS_CUDA_TRY(cudaEventRecord(g_wait_ev, st));
    return spin_then_wait(g_wait_ev);
  }
  GS_CUDA_TRY(cudaStreamSynchronize(st));
  return OK;
}

int event_sync(cudaEvent_t ev) {
  if (g_sync_hook) return g_sync_hook(nullptr, ev);
  if (g_wait_ev) return spin_then_wait(ev);
  GS_CUDA_TRY(cudaEventSynchronize(ev));
  return OK;
}

int num_sms() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (!cached[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cached[dev] = n;
  }
  return cached[dev];
}

int Context::init(void* user_stream) {
  GS_CUDA_TRY(cudaGetDevice(&device));
  // The given stream is always used as is; NULL is CUDA's default stream
  // (the stream torch reports as 0), so work stays ordered with the caller's.
  stream = (cudaStream_t)user_stream;
  own_stream = false;
  {
    // A pool of this context's own; freed memory stays in it between proofs.
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    GS_CUDA_TRY(cudaMemPoolCreate(&pool, &props));
    uint64_t threshold = UINT64_MAX;
    GS_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
  }
  ring_cap = 4 << 20;
  ring_off = 0;
  GS_CUDA_TRY(cudaMallocHost((void**)&h_ring, ring_cap));
  GS_CUDA_TRY(cudaMalloc((void**)&d_ring, ring_cap));
  small_cap = 4096;
  GS_CUDA_TRY(cudaMalloc((void**)&d_small, small_cap));
  GS_CUDA_TRY(cudaMallocHost((void**)&h_small, small_cap + MAIL_SLOTS * MAIL_BYTES));
  h_mail = h_small + small_cap;
  {
    void* dm = nullptr;
    if (cudaHostGetDevicePointer(&dm, h_mail, 0) == cudaSuccess) {
      d_mail = (uint8_t*)dm;
    } else {
      cudaGetLastError();
      d_mail = nullptr;
    }
  }
  for (int i = 0; i < MAIL_SLOTS; i++) GS_CUDA_TRY(cudaEventCreateWithFlags(&mail_ev[i], cudaEventDisableTiming));
  GS_CUDA_TRY(cudaMalloc((void**)&tree_counters, 4 * TREE_COUNTERS));
  GS_CUDA_TRY(cudaMemsetAsync(tree_counters, 0, 4 * TREE_COUNTERS, stream));
  return OK;
}

void Context::destroy() {
  if (stream) cudaStreamSynchronize(stream);
  for (auto& b : spare) cudaFreeAsync(b.second, stream);
  spare.clear();
  if (stream) cudaStreamSynchronize(stream);
  if (work) {
    cudaStreamSynchronize(work);
    cudaStreamSynchronize(side);
    cudaStreamDestroy(work);
    cudaStreamDestroy(side);
    cudaEventDestroy(ev_enter);
    cudaEventDestroy(ev_fork);
    cudaEventDestroy(ev_join);
    work = side = nullptr;
    ev_enter = ev_fork = ev_join = nullptr;
  }
  if (scratch) {
    cudaFreeAsync(scratch, stream);
    cudaStreamSynchronize(stream);
  }
  scratch = nullptr;
  for (int i = 0; i < 31; i++) {
    if (dom_buf[i]) cudaFree(dom_buf[i]);
    if (tw_buf[i]) cudaFree(tw_buf[i]);
    if (itw_buf[i]) cudaFree(itw_buf[i]);
    dom_buf[i] = nullptr;
    tw_buf[i] = itw_buf[i] = nullptr;
  }
  if (h_ring) cudaFreeHost(h_ring);
  if (d_ring) cudaFree(d_ring);
  if (d_small) cudaFree(d_small);
  if (tree_counters) cudaFree(tree_counters);
  tree_counters = nullptr;
  if (h_small) cudaFreeHost(h_small);
  for (int i = 0; i < MAIL_SLOTS; i++) {
    if (mail_ev[i]) cudaEventDestroy(mail_ev[i]);
    mail_ev[i] = nullptr;
  }
  h_mail = nullptr;
  d_mail = nullptr;
  if (h_read) cudaFreeHost(h_read);
  h_read = nullptr;
  d_read = nullptr;
  read_cap = 0;
  if (pool) cudaMemPoolDestroy(pool);  // released once its last allocation is freed
  pool = nullptr;
  if (own_stream && stream) cudaStreamDestroy(stream);
  h_ring = d_ring = d_small = h_small = nullptr;
  stream = nullptr;
}

int Context::begin_proof() {
  if (!work) {
    int least = 0, greatest = 0;
    GS_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    GS_CUDA_TRY(cudaStreamCreateWithPriority(&work, cudaStreamNonBlocking, greatest));
    GS_CUDA_TRY(cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, least));
    GS_CUDA_TRY(cudaEventCreateWithFlags(&ev_enter, cudaEventDisableTiming));
    GS_CUDA_TRY(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    GS_CUDA_TRY(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
  }
  GS_REQUIRE(!in_proof, "proof already in progress on this context");
  GS_CUDA_TRY(cudaEventRecord(ev_enter, stream));
  GS_CUDA_TRY(cudaStreamWaitEvent(work, ev_enter, 0));
  caller = stream;
  stream = work;
  in_proof = true;
  return OK;
}

int Context::end_proof() {
  if (!in_proof) return OK;
  // the caller's stream is restored on every path, also when a wait fails
  int rc = OK;
  if (side_pending) rc = join_side();
  if (rc == OK && cudaEventRecord(ev_enter, work) == cudaSuccess &&
      cudaStreamWaitEvent(caller, ev_enter, 0) == cudaSuccess) {
  } else {
    cudaStreamSynchronize(side);
    cudaStreamSynchronize(work);
  }
  stream = caller;
  caller = nullptr;
  in_proof = false;
  return rc;
}

int Context::fork_side() {
  GS_REQUIRE(side != nullptr, "side stream outside a proof");
  GS_CUDA_TRY(cudaEventRecord(ev_fork, stream));
  GS_CUDA_TRY(cudaStreamWaitEvent(side, ev_fork, 0));
  side_pending = true;
  return OK;
}

int Context::join_side() {
  if (!side_pending) return OK;
  GS_CUDA_TRY(cudaEventRecord(ev_join, side));
  GS_CUDA_TRY(cudaStreamWaitEvent(stream, ev_join, 0));
  side_pending = false;
  return OK;
}

int Context::stage_bytes(const void* host, size_t len, const void** out) {
  size_t bytes = (len + 255) & ~(size_t)255;
  GS_REQUIRE(bytes <= ring_cap, "staged argument block too large");
  if (ring_off + bytes > ring_cap) {
    // Wrap: earlier copies out of the pinned ring, and the kernels reading
    // their device copies (on either stream), must have completed before
    // their slots are rewritten.
    GS_CUDA_TRY(cudaStreamSynchronize(stream));
    if (side_pending) GS_CUDA_TRY(cudaStreamSynchronize(side));
    ring_off = 0;
  }
  memcpy(h_ring + ring_off, host, len);
  GS_CUDA_TRY(cudaMemcpyAsync(d_ring + ring_off, h_ring + ring_off, len, cudaMemcpyHostToDevice, stream));
  *out = (const void*)(d_ring + ring_off);
  ring_off += bytes;
  return OK;
}

int Context::stage_ptrs(const void* const* host_ptrs, size_t n, const void* const** out) {
  const void* d = nullptr;
  GS_TRY(stage_bytes(host_ptrs, n * sizeof(void*), &d));
  *out = (const void* const*)d;
  return OK;
}

int Context::alloc_async(size_t bytes, void** out) {
  cudaError_t e = pool ? cudaMallocFromPoolAsync(out, bytes ? bytes : 16, pool, stream)
                       : cudaMallocAsync(out, bytes ? bytes : 16, stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(std::string("device allocation failed: ") + cudaGetErrorString(e));
    return ERR_OOM;
  }
  return OK;
}

int Context::read_back(const void* d_src, size_t bytes, void* host_dst) {
  if (bytes == 0) return OK;
  void* h = nullptr;
  if (bytes <= small_cap) {
    h = h_small;
  } else {
    GS_TRY(read_buffer(bytes, &h));
  }
  GS_CUDA_TRY(cudaMemcpyAsync(h, d_src, bytes, cudaMemcpyDeviceToHost, stream));
  GS_TRY(stream_sync(stream));
  memcpy(host_dst, h, bytes);
  return OK;
}

int Context::mail_start(int slot, const void* d_src, size_t bytes) {
  GS_REQUIRE(slot >= 0 && slot < MAIL_SLOTS && bytes <= MAIL_BYTES, "mailbox read out of range");
  GS_CUDA_TRY(cudaMemcpyAsync(h_mail + slot * MAIL_BYTES, d_src, bytes, cudaMemcpyDeviceToHost, stream));
  GS_CUDA_TRY(cudaEventRecord(mail_ev[slot], stream));
  return OK;
}

int Context::mail_record(int slot) {
  GS_REQUIRE(slot >= 0 && slot < MAIL_SLOTS, "mailbox slot out of range");
  GS_CUDA_TRY(cudaEventRecord(mail_ev[slot], stream));
  return OK;
}

int Context::mail_wait(int slot, const void** host) {
  GS_REQUIRE(slot >= 0 && slot < MAIL_SLOTS, "mailbox slot out of range");
  GS_TRY(event_sync(mail_ev[slot]));
  *host = h_mail + slot * MAIL_BYTES;
  return OK;
}

int Context::read_buffer(size_t bytes, void** out) {
  if (bytes > read_cap) {
    if (h_read) {
      GS_CUDA_TRY(cudaStreamSynchronize(stream));
      cudaFreeHost(h_read);
    }
    h_read = nullptr;
    read_cap = 0;
    size_t cap = bytes < (1u << 20) ? (1u << 20) : bytes + bytes / 2;
    GS_CUDA_TRY(cudaMallocHost((void**)&h_read, cap));
    read_cap = cap;
    d_read = nullptr;
    void* dm = nullptr;
    if (cudaHostGetDevicePointer(&dm, h_read, 0) == cudaSuccess) d_read = dm;
    else cudaGetLastError();
  }
  *out = h_read;
  return OK;
}

// Device words into mapped pinned memory: 16-byte stores where source and
// destination allow, single words for the rest.
__global__ void publish_kernel(const uint32_t* __restrict__ src, uint32_t* dst, size_t n_words) {
  const size_t n16 = n_words / 4;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (size_t i = t0; i < n16; i += stride)
    reinterpret_cast<uint4*>(dst)[i] = __ldg(reinterpret_cast<const uint4*>(src) + i);
  for (size_t i = 4 * n16 + t0; i < n_words; i += stride) dst[i] = src[i];
}

int Context::publish(const void* d_src, size_t bytes, const void** host) {
  GS_REQUIRE(bytes % 4 == 0, "published reads are whole words");
  void* h = nullptr;
  GS_TRY(read_buffer(bytes ? bytes : 4, &h));
  if (bytes && d_read && ((uintptr_t)d_src & 15) == 0) {
    const size_t n16 = bytes / 16;
    size_t blocks = (n16 + 255) / 256;
    const size_t cap = (size_t)num_sms() * 4;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    publish_kernel<<<(unsigned)blocks, 256, 0, stream>>>((const uint32_t*)d_src, (uint32_t*)d_read, bytes / 4);
    note_launch();
    GS_CUDA_TRY(cudaGetLastError());
  } else if (bytes) {
    GS_CUDA_TRY(cudaMemcpyAsync(h, d_src, bytes, cudaMemcpyDeviceToHost, stream));
  }
  *host = h;
  return OK;
}

int Context::read_back_published(const void* d_src, size_t bytes, void* host_dst) {
  if (bytes == 0) return OK;
  const void* h = nullptr;
  GS_TRY(publish(d_src, bytes, &h));
  GS_TRY(stream_sync(stream));
  memcpy(host_dst, h, bytes);
  return OK;
}

int Context::get_scratch(size_t bytes, void** out) {
  if (bytes > scratch_cap) {
    if (scratch) GS_CUDA_TRY(cudaFreeAsync(scratch, stream));
    scratch = nullptr;
    size_t cap = bytes < (1u << 20) ? (1u << 20) : bytes;
    if (alloc_async(cap, &scratch) != OK) {
      scratch_cap = 0;
      set_error("scratch allocation failed");
      return ERR_OOM;
    }
    scratch_cap = cap;
  }
  *out = scratch;
  return OK;
}

int Context::domain_tables(uint32_t lift, DomainTables* out) {
  GS_REQUIRE(lift >= 2 && lift <= 30, "lifting log size out of range");
  if (!dom_buf[lift]) {
    void* buf = nullptr;
    GS_CUDA_TRY(cudaMalloc(&buf, domain_tables_len(lift) * sizeof(pt31)));
    GS_TRY(make_domain_tables(stream, lift, (pt31*)buf, &dom[lift]));
    dom_buf[lift] = buf;
  }
  *out = dom[lift];
  return OK;
}

int Context::twiddles(uint32_t root_log, const uint32_t** tw, const uint32_t** itw) {
  GS_REQUIRE(root_log >= 1 && root_log <= 29, "twiddle root log size out of range");
  if (!tw_buf[root_log]) {
    size_t n = (size_t)1 << root_log;
    GS_CUDA_TRY(cudaMalloc((void**)&tw_buf[root_log], 4 * n));
    GS_CUDA_TRY(cudaMalloc((void**)&itw_buf[root_log], 4 * n));
    uint32_t initial = 1u << (31 - (root_log + 2)), step = 1u << (31 - root_log);
    GS_TRY(precompute_twiddles(stream, initial, step, root_log, tw_buf[root_log], itw_buf[root_log]));
  }
  *tw = tw_buf[root_log];
  *itw = itw_buf[root_log];
  return OK;
}

int Context::sync() {
  GS_TRY(stream_sync(stream));
  return OK;
}

}  // namespace gs
