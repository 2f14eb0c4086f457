// Cooperative fibers: many proofs driven by one host thread.
//
// A proof waits on its CUDA stream at every host round trip of the protocol
// (a Merkle root into the channel, the logup claimed sum, the proof-of-work
// word, the decommitment read-back). With one host thread per proof those
// waits leave threads idle and the threads contend for the driver while they
// launch. Here each proof runs in a fiber (its own stack, switched with
// swapcontext): a wait records an event on the proof's stream and yields; the
// scheduler resumes the fiber once the event has completed and meanwhile runs
// the host steps and launches of the other fibers, so one thread keeps the
// work of many proofs queued on their streams. The prover code is unchanged:
// its waits all go through stream_sync, which calls the hook the scheduler
// installs for its thread.
#pragma once
#include <cuda_runtime.h>
#include <ucontext.h>
#include <functional>
#include <memory>
#include <vector>

namespace gs {
namespace prover {

class FiberScheduler {
 public:
  // Runs every body as a fiber on the calling thread and returns when all
  // have returned. idle_wait is called when every live fiber is idle (no
  // work to take) and none waits on the device; it should block briefly.
  void run(std::vector<std::function<void()>> bodies, const std::function<void()>& idle_wait,
           size_t stack_bytes = 1u << 20);
  // Inside a fiber: there is no work now; resume me on the next round.
  static void yield_idle();
  // The stream_sync / event_sync hook: inside a fiber, yield until `ev` (or,
  // when ev is null, an event recorded now on st) has completed; elsewhere,
  // synchronise the stream or the event.
  static int wait_device(cudaStream_t st, cudaEvent_t ev);

 private:
  enum State { READY, WAITING, IDLE, DONE };
  struct Fiber {
    ucontext_t uc;
    std::unique_ptr<char[]> stack;
    std::function<void()> body;
    State state = READY;
    cudaEvent_t ev = nullptr;       // the fiber's own event, recorded on its stream
    cudaEvent_t waiting_on = nullptr;  // the event the fiber waits for
    int status = 0;
  };
  static void entry();
  ucontext_t main_uc_;
  std::vector<std::unique_ptr<Fiber>> fibers_;
};

}  // namespace prover
}  // namespace gs
