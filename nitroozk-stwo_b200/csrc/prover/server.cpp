// Proof server: continuous batching of independent proof jobs on one GPU.
//
// Worker threads each own an execution context (a non-blocking CUDA stream);
// a job is admitted when the estimated device footprint of the jobs in flight
// plus its own fits the HBM budget. While one proof waits on a host step
// (Merkle roots into the channel, FRI alphas, the proof of work, the
// decommitment read-back), the other workers' kernels keep the GPU busy.
// Every job runs the same prove() as a single proof, so its result is
// identical alone and in the mix.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <set>
#include <cstring>
#include <mutex>
#include <thread>
#include "../../../include/gpustark.h"
#include "fiber.h"
#include "prove_api.h"

namespace gs {
namespace prover {

struct Job {
  uint64_t id;
  ProveRequest req;
  size_t footprint;
  std::chrono::steady_clock::time_point submitted;
};
struct Done {
  int status = OK;
  std::string proof, error;
  double latency_ms = 0, service_ms = 0;
};

// Device bytes a proof holds at its peak (trace, coefficients, LDEs, the
// constraint-domain extension, composition, Merkle layers), with headroom.
size_t proof_footprint(const ProveRequest& r) {
  const size_t n = (size_t)1 << r.log_n;
  const size_t b = (size_t)1 << r.cfg.log_blowup;
  const size_t cols = r.air == 0 ? r.n_cols : 162;
  const size_t ext = r.air == 0 ? 2 : 4;
  size_t words = cols * n * (2 + b + ext) + 16 * n * ext + 64 * n * b;
  return words * 4 + (64u << 20);
}

struct Server {
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_jobs, cv_done;
  std::deque<Job> queue;
  std::map<uint64_t, Done> done;
  std::set<uint64_t> fetched;  // results already handed out
  size_t budget = 0, in_flight = 0;
  uint64_t next_id = 1;
  bool stopping = false;
  int device = 0;
  uint32_t fibers = 1;  // proofs per host thread (fiber mode when > 1)

  bool admissible() const {
    return !queue.empty() && (in_flight == 0 || in_flight + queue.front().footprint <= budget);
  }

  // Proves one job on a context and publishes the result.
  void serve(Context& ctx, cudaStream_t st, int init, Job& job) {
    Done d;
    auto t0 = std::chrono::steady_clock::now();
    if (init != OK) {
      d.status = init;
      d.error = "context initialisation failed";
    } else {
      d.status = prove_component(ctx, job.req, &d.proof, nullptr);
      if (d.status != OK) d.error = last_error();
      stream_sync(st);
    }
    auto t1 = std::chrono::steady_clock::now();
    d.service_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    d.latency_ms = std::chrono::duration<double, std::milli>(t1 - job.submitted).count();
    {
      std::lock_guard<std::mutex> lk(mu);
      in_flight -= job.footprint;
      done[job.id] = std::move(d);
    }
    cv_done.notify_all();
    cv_jobs.notify_all();
  }

  // Fiber mode: `fibers` proof loops on this host thread, each with its own
  // stream and context; a loop with no admissible job yields, and the thread
  // sleeps on the job queue only when every loop is idle.
  void fiber_worker() {
    cudaSetDevice(device);
    std::vector<std::function<void()>> bodies;
    for (uint32_t k = 0; k < fibers; k++) {
      bodies.push_back([this] {
        cudaStream_t st;
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        Context ctx;
        int init = ctx.init(st);
        ctx.keep_buffers = false;
        for (;;) {
          Job job;
          bool got = false, quit = false;
          {
            std::lock_guard<std::mutex> lk(mu);
            if (admissible()) {
              job = std::move(queue.front());
              queue.pop_front();
              in_flight += job.footprint;
              got = true;
            } else if (stopping && queue.empty()) {
              quit = true;
            }
          }
          if (quit) break;
          if (!got) {
            FiberScheduler::yield_idle();
            continue;
          }
          serve(ctx, st, init, job);
        }
        ctx.destroy();
        cudaStreamDestroy(st);
      });
    }
    FiberScheduler sched;
    sched.run(std::move(bodies), [this] {
      std::unique_lock<std::mutex> lk(mu);
      cv_jobs.wait_for(lk, std::chrono::milliseconds(2), [&] { return stopping || admissible(); });
    });
  }

  void worker() {
    if (fibers > 1) return fiber_worker();
    cudaSetDevice(device);
    cudaStream_t st;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    Context ctx;
    int init = ctx.init(st);
    ctx.keep_buffers = false;
    // waits of this worker: poll briefly, then sleep
    cudaEvent_t wait_ev = nullptr;
    if (cudaEventCreateWithFlags(&wait_ev, cudaEventBlockingSync | cudaEventDisableTiming) == cudaSuccess)
      set_thread_wait_event(wait_ev);
    for (;;) {
      Job job;
      {
        std::unique_lock<std::mutex> lk(mu);
        // admission by footprint holds while the server drains at shutdown too
        cv_jobs.wait(lk, [&] { return (stopping && queue.empty()) || admissible(); });
        if (queue.empty()) break;
        job = std::move(queue.front());
        queue.pop_front();
        in_flight += job.footprint;
      }
      serve(ctx, st, init, job);
    }
    set_thread_wait_event(nullptr);
    ctx.destroy();
    if (wait_ev) cudaEventDestroy(wait_ev);
    cudaStreamDestroy(st);
  }
};

}  // namespace prover
}  // namespace gs

using namespace gs;
using namespace gs::prover;

struct gs_server {
  Server s;
};

extern "C" {

int gs_server_create(uint32_t n_workers, size_t hbm_budget_bytes, gs_server** out) {
  return gs_server_create_fibers(n_workers, 1, hbm_budget_bytes, out);
}

int gs_server_create_fibers(uint32_t n_threads, uint32_t fibers_per_thread, size_t hbm_budget_bytes,
                            gs_server** out) {
  GS_REQUIRE(out != nullptr && n_threads >= 1 && n_threads <= 64, "bad server arguments");
  GS_REQUIRE(fibers_per_thread >= 1 && fibers_per_thread <= 64, "fibers per thread must be in [1, 64]");
  gs_server* sv = new gs_server();
  sv->s.budget = hbm_budget_bytes;
  sv->s.fibers = fibers_per_thread;
  cudaGetDevice(&sv->s.device);
  for (uint32_t i = 0; i < n_threads; i++) sv->s.workers.emplace_back([sv] { sv->s.worker(); });
  *out = sv;
  return OK;
}

static int submit_job(gs_server* sv, uint32_t air, uint32_t log_n, uint32_t n_columns, uint64_t seed,
                      uint32_t composition_log_split, const gs_pcs_config* config, uint32_t merkle_channel,
                      uint64_t* job_id) {
  GS_REQUIRE(sv && job_id, "null argument");
  Job j;
  j.req.air = air;
  j.req.merkle_channel = merkle_channel;
  j.req.log_n = log_n;
  j.req.n_cols = n_columns;
  j.req.seed = seed;
  j.req.input_mode = GS_INPUT_SEEDED;
  j.req.split_log = composition_log_split;
  if (config) {
    j.req.cfg.pow_bits = config->pow_bits;
    j.req.cfg.log_blowup = config->log_blowup_factor;
    j.req.cfg.log_last_layer = config->log_last_layer_degree_bound;
    j.req.cfg.n_queries = config->n_queries;
    j.req.cfg.fold_step = config->line_fold_step;
  }
  GS_TRY(validate_request(j.req));
  j.footprint = proof_footprint(j.req);
  j.submitted = std::chrono::steady_clock::now();
  {
    std::lock_guard<std::mutex> lk(sv->s.mu);
    j.id = sv->s.next_id++;
    *job_id = j.id;
    sv->s.queue.push_back(std::move(j));
  }
  sv->s.cv_jobs.notify_one();
  return OK;
}

int gs_server_submit(gs_server* sv, uint32_t air, uint32_t log_n, uint32_t n_columns, uint64_t seed,
                     uint32_t composition_log_split, const gs_pcs_config* config, uint64_t* job_id) {
  return submit_job(sv, air, log_n, n_columns, seed, composition_log_split, config, 0, job_id);
}
int gs_server_submit_poseidon252(gs_server* sv, uint32_t air, uint32_t log_n, uint32_t n_columns, uint64_t seed,
                                 uint32_t composition_log_split, const gs_pcs_config* config, uint64_t* job_id) {
  return submit_job(sv, air, log_n, n_columns, seed, composition_log_split, config, 1, job_id);
}

int gs_server_wait(gs_server* sv, uint64_t job_id, uint8_t* proof, size_t capacity, size_t* proof_len,
                   double* latency_ms) {
  GS_REQUIRE(sv && proof_len, "null argument");
  std::unique_lock<std::mutex> lk(sv->s.mu);
  GS_REQUIRE(job_id >= 1 && job_id < sv->s.next_id, "unknown job id");
  GS_REQUIRE(!sv->s.fetched.count(job_id), "job result already fetched");
  sv->s.cv_done.wait(lk, [&] { return sv->s.done.count(job_id) != 0; });
  Done& d = sv->s.done[job_id];
  *proof_len = d.proof.size();
  if (latency_ms) *latency_ms = d.latency_ms;
  if (d.status != OK) {
    int st = d.status;
    set_error(d.error);
    sv->s.done.erase(job_id);
    sv->s.fetched.insert(job_id);
    return st;
  }
  if (!proof || capacity < d.proof.size()) {  // the result stays available for a retry
    set_error("proof buffer too small");
    return ERR_INVALID;
  }
  memcpy(proof, d.proof.data(), d.proof.size());
  sv->s.done.erase(job_id);
  sv->s.fetched.insert(job_id);
  return OK;
}

int gs_server_destroy(gs_server* sv) {
  if (!sv) return OK;
  {
    std::lock_guard<std::mutex> lk(sv->s.mu);
    sv->s.stopping = true;
  }
  sv->s.cv_jobs.notify_all();
  for (auto& t : sv->s.workers) t.join();
  delete sv;
  return OK;
}

}  // extern "C"
