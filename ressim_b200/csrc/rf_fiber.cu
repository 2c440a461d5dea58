// rf_fiber.cu — the ensemble's batched stepping: many variants per host thread, one launch per
// level-scheduled kernel kind per group.
//
// A variant's report step (the reference's controller, fim/timestep.rs:989-1848) is a host loop
// that launches short kernels and now and then waits for a scalar read back from its stream.  In a
// batch step the variants are split into groups; each group has one host thread and one CUDA
// stream that all its variants use.  Every variant's rf_step runs as a fiber (its own stack,
// ucontext switches) on the group's thread:
//   - a wait on the stream (stream_wait / d2h_wait) records an event and suspends the fiber; the
//     thread resumes other fibers and picks the fiber up once the event has completed;
//   - a level-scheduled kernel (the ILU0 factorisation, the pressure BiCGStab, the block-ILU0
//     sweep) is not launched directly: the fiber files its arguments with the group and suspends.  When every unfinished
//     fiber of the group is waiting for such a launch, the thread launches one kernel per kind
//     whose thread block b runs item b, and resumes the fibers.
// So the device runs the pressure solves of a whole group as one launch, and the groups' launches
// overlap on their own streams: far more solves run at once than there are hardware queues.  The
// fibers of a group advance from one batched launch to the next together; the arithmetic of every
// solve is the one of its single launch, so a variant's results do not depend on its batch.
#include <ucontext.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "rf_fiber.hpp"

namespace rf {

namespace {

struct Fiber {
  ucontext_t uc;
  void (*fn)(void*) = nullptr;
  void* arg = nullptr;
  int state = 0;  // 0 runnable, 1 waiting for an event, 2 waiting for a batched launch, 3 done
  cudaEvent_t ev = nullptr;
  long long order = 0;  // when it started waiting (the group's stream completes in order)
};

struct GroupRun {
  ucontext_t main;
  Fiber* cur = nullptr;
  BatchGroup* g = nullptr;
  long long tick = 0;
};

thread_local GroupRun* tl_run = nullptr;

void fiber_trampoline(unsigned lo, unsigned hi) {
  Fiber* f = reinterpret_cast<Fiber*>((uintptr_t(hi) << 32) | uintptr_t(lo));
  f->fn(f->arg);  // rf_step: errors come back as status codes, never as exceptions
  f->state = 3;
  // returning continues at uc_link, the group thread's scheduler
}

void suspend(int state) {
  GroupRun* r = tl_run;
  Fiber* f = r->cur;
  f->state = state;
  f->order = r->tick++;
  swapcontext(&f->uc, &r->main);
}

// One launch per kind and value type over the filed items, in chunks of kBatchItems.
void launch_pending(BatchGroup& g) {
  std::vector<BatchItem>& items = g.pending;
  for (int kind = 0; kind < kBatchKinds; ++kind)
    for (int type = 0; type < 2; ++type) {
      std::vector<const BatchItem*> sel;
      for (const BatchItem& it : items)
        if (it.kind == kind && it.type == type) sel.push_back(&it);
      for (size_t off = 0; off < sel.size(); off += kBatchItems) {
        const int count = int(std::min<size_t>(kBatchItems, sel.size() - off));
        cudaEvent_t a = nullptr;
        if (g.profiling) {
          a = g.timing_event();
          cudaEventRecord(a, g.stream);
        }
        if (!launch_batch_items(kind, type, sel.data() + off, count, g.stream)) g.failed = true;
        if (g.profiling) {
          cudaEvent_t b = g.timing_event();
          cudaEventRecord(b, g.stream);
          g.timed.push_back({kind, {a, b}});
        }
        g.launches[kind]++;
        g.items[kind] += count;
      }
    }
  items.clear();
}

}  // namespace

bool fiber_active() { return tl_run != nullptr && tl_run->cur != nullptr; }

void fiber_wait_event(cudaEvent_t ev) {
  if (!fiber_active()) return;
  tl_run->cur->ev = ev;
  suspend(1);
}

bool fiber_submit(const BatchItem& item) {
  if (!fiber_active()) return false;
  tl_run->g->pending.push_back(item);
  suspend(2);
  return true;
}

bool fiber_file(int kind, int type, const void* args, size_t bytes, int threads, size_t smem) {
  if (!fiber_active() || bytes > kBatchArgBytes) return false;
  BatchItem it;
  it.kind = kind;
  it.type = type;
  it.threads = threads;
  it.smem = smem;
  std::memcpy(it.args, args, bytes);
  return fiber_submit(it);
}

cudaEvent_t BatchGroup::timing_event() {
  if (ev_used == ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    ev_pool.push_back(e);
  }
  return ev_pool[ev_used++];
}

void BatchGroup::resolve_timing() {
  if (timed.empty()) return;
  cudaStreamSynchronize(stream);
  for (auto& t : timed) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, t.second.first, t.second.second) == cudaSuccess) ms_by_kind[t.first] += ms;
  }
  timed.clear();
  ev_used = 0;
}

void BatchGroup::reset_stats() {
  for (int k = 0; k < kBatchKinds; ++k) {
    launches[k] = items[k] = 0;
    ms_by_kind[k] = 0.0;
  }
}

BatchGroup::~BatchGroup() {
  for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
}

// Runs fn(args[i]) for every i as fibers on the calling thread, with stacks of `stack_bytes`.
void run_fibers(BatchGroup& g, void (*fn)(void*), void* const* args, int count, size_t stack_bytes) {
  std::vector<Fiber> fibers(count);
  GroupRun run;
  run.g = &g;
  if (g.stacks.size() < size_t(count) * stack_bytes) g.stacks.assign(size_t(count) * stack_bytes, 0);
  for (int i = 0; i < count; ++i) {
    Fiber& f = fibers[i];
    f.fn = fn;
    f.arg = args[i];
    getcontext(&f.uc);
    f.uc.uc_stack.ss_sp = g.stacks.data() + size_t(i) * stack_bytes;
    f.uc.uc_stack.ss_size = stack_bytes;
    f.uc.uc_link = &run.main;
    const uintptr_t p = reinterpret_cast<uintptr_t>(&f);
    makecontext(&f.uc, reinterpret_cast<void (*)()>(fiber_trampoline), 2, unsigned(p & 0xffffffffu),
                unsigned(p >> 32));
    f.state = 0;
  }
  tl_run = &run;
  for (;;) {
    bool ran = false, all_done = true;
    Fiber* oldest = nullptr;
    for (Fiber& f : fibers) {
      if (f.state == 3) continue;
      all_done = false;
      if (f.state == 1) {
        const cudaError_t e = cudaEventQuery(f.ev);
        if (e == cudaErrorNotReady) {
          if (!oldest || f.order < oldest->order) oldest = &f;
          continue;
        }
        f.state = 0;  // complete, or failed: the fiber's own check of the event reports it
      }
      if (f.state == 0) {
        run.cur = &f;
        swapcontext(&run.main, &f.uc);
        run.cur = nullptr;
        ran = true;
      }
    }
    if (all_done) break;
    if (ran) continue;
    if (oldest) {
      // nothing runnable: wait for the wait filed first (the group's stream completes in order),
      // yielding the core meanwhile (many group threads share the host's cores, and the driver's
      // own wait spins)
      while (cudaEventQuery(oldest->ev) == cudaErrorNotReady) std::this_thread::yield();
      continue;
    }
    // every unfinished fiber waits for a batched launch
    launch_pending(g);
    for (Fiber& f : fibers)
      if (f.state == 2) f.state = 0;
  }
  tl_run = nullptr;
}

}  // namespace rf
