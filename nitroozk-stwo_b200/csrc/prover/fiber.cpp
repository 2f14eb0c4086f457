// Cooperative fiber scheduler (fiber.h).
#include "fiber.h"
#include <thread>
#include "../runtime.cuh"

namespace gs {
namespace prover {

static thread_local FiberScheduler* t_sched = nullptr;
static thread_local void* t_current = nullptr;  // the running Fiber, null on the scheduler's own stack
static thread_local ucontext_t* t_main = nullptr;

void FiberScheduler::entry() {
  Fiber* f = (Fiber*)t_current;
  f->body();
  f->state = DONE;
  // returning switches to uc_link, the scheduler
}

void FiberScheduler::yield_idle() {
  Fiber* f = (Fiber*)t_current;
  if (!f) {
    std::this_thread::yield();
    return;
  }
  f->state = IDLE;
  swapcontext(&f->uc, t_main);
}

int FiberScheduler::wait_device(cudaStream_t st, cudaEvent_t ev) {
  Fiber* f = (Fiber*)t_current;
  if (!f) {
    if (ev) GS_CUDA_TRY(cudaEventSynchronize(ev));
    else GS_CUDA_TRY(cudaStreamSynchronize(st));
    return OK;
  }
  if (!ev) {
    GS_CUDA_TRY(cudaEventRecord(f->ev, st));
    ev = f->ev;
  }
  f->waiting_on = ev;
  f->state = WAITING;
  swapcontext(&f->uc, t_main);
  if (f->status != OK) {
    set_error("stream wait failed in a proof fiber");
    return ERR_CUDA;
  }
  return OK;
}

void FiberScheduler::run(std::vector<std::function<void()>> bodies, const std::function<void()>& idle_wait,
                         size_t stack_bytes) {
  fibers_.clear();
  for (auto& b : bodies) {
    auto f = std::make_unique<Fiber>();
    f->body = std::move(b);
    f->stack.reset(new char[stack_bytes]);
    cudaEventCreateWithFlags(&f->ev, cudaEventDisableTiming);
    getcontext(&f->uc);
    f->uc.uc_stack.ss_sp = f->stack.get();
    f->uc.uc_stack.ss_size = stack_bytes;
    f->uc.uc_link = &main_uc_;
    makecontext(&f->uc, (void (*)())entry, 0);
    fibers_.push_back(std::move(f));
  }
  FiberScheduler* prev_sched = t_sched;
  ucontext_t* prev_main = t_main;
  t_sched = this;
  t_main = &main_uc_;
  set_thread_sync_hook(&FiberScheduler::wait_device);
  size_t live = fibers_.size();
  while (live > 0) {
    bool progress = false, waiting = false;
    for (auto& fp : fibers_) {
      Fiber* f = fp.get();
      if (f->state == DONE) continue;
      if (f->state == WAITING) {
        const cudaError_t q = cudaEventQuery(f->waiting_on);
        if (q == cudaErrorNotReady) {
          waiting = true;
          continue;
        }
        f->status = q == cudaSuccess ? OK : ERR_CUDA;
        if (q != cudaSuccess) cudaGetLastError();
        f->state = READY;
      }
      const bool was_idle = f->state == IDLE;
      f->state = READY;
      t_current = f;
      swapcontext(&main_uc_, &f->uc);
      t_current = nullptr;
      if (f->state == DONE) live--;
      if (!was_idle || f->state != IDLE) progress = true;
    }
    if (!progress && live > 0) {
      if (waiting) std::this_thread::yield();
      else idle_wait();
    }
  }
  set_thread_sync_hook(nullptr);
  t_sched = prev_sched;
  t_main = prev_main;
  for (auto& f : fibers_)
    if (f->ev) cudaEventDestroy(f->ev);
  fibers_.clear();
}

}  // namespace prover
}  // namespace gs
