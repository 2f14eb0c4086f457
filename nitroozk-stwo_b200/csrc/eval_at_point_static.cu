// Allocation-free batch_eval_at_point: the same kernels as
// gs_batch_eval_at_point (eval_at_point.cu), with every device word the call
// needs taken from one file-scope __device__ array instead of a context's
// scratch pool and pinned staging ring.
//
// Layout of the static array (all offsets 256-byte aligned):
//   [0, 2 KiB)         polynomial pointer table, written by a 1-block kernel
//                      from a by-value kernel parameter (no host->device copy)
//   [2 KiB, 6 KiB)     results, 16 bytes per polynomial
//   [6 KiB, end)       eval_at_point scratch: 2^s weights, then the per-chunk
//                      partial sums (eval_at_point_scratch_bytes)
// Every word a kernel reads is written earlier in the same call on the same
// stream, so nothing needs clearing between calls.
//
// The array's device address belongs to a CUDA context. It is looked up with
// cudaGetSymbolAddress the first time a call runs under a context (for the
// usual case, the device's primary context, once per device; that first call
// also loads this library's kernels onto the device) and cached per context.
// The current context is read through the runtime's driver entry point for
// cuCtxGetCurrent, so the library does not link the driver library; should
// that entry point be unavailable, every call looks the address up again.
// There is one array per context: calls that overlap in time under one
// context race on it, whatever their streams or threads.
#include <cuda.h>
#include <mutex>
#include <utility>
#include <vector>
#include "../../include/gpustark.h"
#include "runtime.cuh"

namespace gs {

constexpr uint32_t EAPS_MAX_POLYS = 256;
constexpr uint32_t EAPS_CHUNK_LOG = 10;                                 // 2^10 coefficients per chunk
constexpr size_t EAPS_TABLE_BYTES = EAPS_MAX_POLYS * sizeof(void*);    // 2 KiB
constexpr size_t EAPS_OUT_BYTES = 16 * (size_t)EAPS_MAX_POLYS;         // 4 KiB
constexpr size_t EAPS_WORK_BYTES = (16u << 10) + (4u << 20);           // 2^10 weights + 2^18 partials
constexpr size_t EAPS_TOTAL_BYTES = EAPS_TABLE_BYTES + EAPS_OUT_BYTES + EAPS_WORK_BYTES;

static __device__ __align__(256) uint8_t g_eap_static[EAPS_TOTAL_BYTES];

struct PolyTable { const uint32_t* p[EAPS_MAX_POLYS]; };

__global__ void eaps_table_kernel(PolyTable t, uint32_t n, const uint32_t** dst) {
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = t.p[i];
}

static std::mutex g_eaps_mu;
static std::vector<std::pair<CUcontext, void*>> g_eaps_addr;  // address of the array per context

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
static CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (CtxGetCurrentFn)p;
    else
      cudaGetLastError();
  });
  return fn;
}

static int eaps_base(uint8_t** out) {
  CtxGetCurrentFn fn = ctx_get_current();
  CUcontext ctx = nullptr;
  if (fn && fn(&ctx) != CUDA_SUCCESS) ctx = nullptr;
  std::lock_guard<std::mutex> lk(g_eaps_mu);
  if (ctx)
    for (auto& e : g_eaps_addr)
      if (e.first == ctx) {
        *out = (uint8_t*)e.second;
        return OK;
      }
  // the lookup makes the device's primary context current when no context is
  void* a = nullptr;
  GS_CUDA_TRY(cudaGetSymbolAddress(&a, g_eap_static));
  if (fn && !ctx && fn(&ctx) != CUDA_SUCCESS) ctx = nullptr;
  if (ctx) g_eaps_addr.push_back({ctx, a});
  *out = (uint8_t*)a;
  return OK;
}

}  // namespace gs

using namespace gs;

extern "C" int gs_batch_eval_at_point_noalloc(void* stream, const uint32_t* const* polys, uint32_t n_polys,
                                              uint32_t log_size, gs_point_qm31 point, gs_qm31* out) {
  if (n_polys == 0) return OK;
  GS_REQUIRE(polys && out, "null argument");
  GS_REQUIRE(n_polys <= EAPS_MAX_POLYS, "more than 256 polynomials");
  GS_REQUIRE(log_size <= 30, "log size out of range");
  GS_REQUIRE(eval_at_point_scratch_bytes(n_polys, log_size, EAPS_CHUNK_LOG) <= EAPS_WORK_BYTES,
             "n_polys * 2^(log_size - 10) exceeds 2^18 chunks");
  PolyTable t;
  for (uint32_t i = 0; i < n_polys; i++) {
    GS_REQUIRE(polys[i] != nullptr, "null polynomial");
    t.p[i] = polys[i];
  }
  uint8_t* base = nullptr;
  GS_TRY(eaps_base(&base));
  cudaStream_t st = (cudaStream_t)stream;
  const uint32_t** d_table = (const uint32_t**)base;
  uint32_t* d_out = (uint32_t*)(base + EAPS_TABLE_BYTES);
  uint32_t* d_work = (uint32_t*)(base + EAPS_TABLE_BYTES + EAPS_OUT_BYTES);
  eaps_table_kernel<<<1, 256, 0, st>>>(t, n_polys, d_table);
  note_launch();
  GS_CUDA_TRY(cudaGetLastError());
  ptq p = {qm_make(point.x.a, point.x.b, point.x.c, point.x.d), qm_make(point.y.a, point.y.b, point.y.c, point.y.d)};
  GS_TRY(batch_eval_at_point(st, (const uint32_t* const*)d_table, n_polys, log_size, p, d_out, d_work,
                             EAPS_CHUNK_LOG));
  GS_CUDA_TRY(cudaMemcpyAsync(out, d_out, 16 * (size_t)n_polys, cudaMemcpyDeviceToHost, st));
  GS_CUDA_TRY(cudaStreamSynchronize(st));
  return OK;
}
