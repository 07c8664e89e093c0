// Block/thread scheduler of the CPU kernel emulation (TEST INFRASTRUCTURE
// ONLY).  run_grid() calls a kernel body once per (block, thread).  Without
// barriers the threads of a block simply run in order.  With barriers each
// thread is a ucontext fiber: __syncthreads() switches back to the scheduler,
// which resumes the next unfinished thread; a barrier is complete when every
// live thread has reached it, exactly the semantics the kernels rely on
// (threads that returned early no longer take part).
#include <ucontext.h>

#include <cstdlib>
#include <functional>
#include <vector>

#include "prelude.h"

namespace refshim {
Idx g_thread{0, 0, 0}, g_block{0, 0, 0}, g_bdim{1, 1, 1}, g_gdim{1, 1, 1};

namespace {
constexpr size_t kStack = 64 * 1024;
struct Fiber {
  ucontext_t ctx;
  std::vector<char> stack;
  bool done = false;
  unsigned tid = 0;
};
ucontext_t g_sched;
std::vector<Fiber>* g_fibers = nullptr;
int g_cur = -1;
const std::function<void()>* g_body = nullptr;

void fiber_entry() {
  (*g_body)();
  (*g_fibers)[g_cur].done = true;
  // returning resumes uc_link (the scheduler)
}
}  // namespace

void sync() {
  if (g_cur < 0) return;                 // no fibers: barrier-free launch
  swapcontext(&(*g_fibers)[g_cur].ctx, &g_sched);
}

// Runs body for every thread of a gx x bx launch (1-D, as the reference's
// kernels are launched).
void run_grid(unsigned gx, unsigned bx, bool barriers, const std::function<void()>& body) {
  g_gdim = {gx, 1, 1};
  g_bdim = {bx, 1, 1};
  if (!barriers) {
    g_cur = -1;
    for (unsigned b = 0; b < gx; ++b) {
      g_block = {b, 0, 0};
      for (unsigned t = 0; t < bx; ++t) {
        g_thread = {t, 0, 0};
        body();
      }
    }
    return;
  }
  std::vector<Fiber> fibers(bx);
  for (auto& f : fibers) f.stack.resize(kStack);
  g_fibers = &fibers;
  g_body = &body;
  for (unsigned b = 0; b < gx; ++b) {
    g_block = {b, 0, 0};
    for (unsigned t = 0; t < bx; ++t) {
      Fiber& f = fibers[t];
      f.done = false;
      f.tid = t;
      getcontext(&f.ctx);
      f.ctx.uc_stack.ss_sp = f.stack.data();
      f.ctx.uc_stack.ss_size = kStack;
      f.ctx.uc_link = &g_sched;
      makecontext(&f.ctx, fiber_entry, 0);
    }
    bool live = true;
    while (live) {
      live = false;
      for (unsigned t = 0; t < bx; ++t) {
        if (fibers[t].done) continue;
        g_cur = (int)t;
        g_thread = {t, 0, 0};
        swapcontext(&g_sched, &fibers[t].ctx);
        if (!fibers[t].done) live = true;
      }
    }
  }
  g_cur = -1;
  g_fibers = nullptr;
}
}  // namespace refshim
