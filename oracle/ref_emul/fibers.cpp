// Cooperative-fiber emulation of a CUDA thread block (test infrastructure; see
// cuda_host_shim.h).  Single OS thread; not re-entrant.
#include "cuda_host_shim.h"
#include <ucontext.h>
#include <vector>

agdref_dim3 threadIdx = {0, 0, 0}, blockIdx = {0, 0, 0}, blockDim = {1, 1, 1}, gridDim = {1, 1, 1};

namespace {
const size_t kStack = 256 * 1024;
struct Fiber {
    ucontext_t ctx;
    std::vector<char> stack;
    bool done;
};
ucontext_t g_main;
std::vector<Fiber> g_fibers;
int g_n = 0, g_cur = 0;
void (*g_body)(void *) = nullptr;
void *g_arg = nullptr;

void switch_next() {
    const int prev = g_cur;
    for (int k = 1; k <= g_n; ++k) {
        const int c = (prev + k) % g_n;
        if (!g_fibers[c].done) {
            if (c == prev) return;  // only fiber left: a barrier is a no-op
            g_cur = c;
            threadIdx.x = c;
            swapcontext(&g_fibers[prev].ctx, &g_fibers[c].ctx);
            threadIdx.x = prev;  // resumed: restore our identity
            g_cur = prev;
            return;
        }
    }
    swapcontext(&g_fibers[prev].ctx, &g_main);  // every fiber finished
}

void fiber_entry() {
    g_body(g_arg);
    g_fibers[g_cur].done = true;
    switch_next();
    std::abort();  // unreachable: a finished fiber is never resumed
}
}  // namespace

void __syncthreads() { switch_next(); }

void agdref_run_block(void (*body)(void *), void *arg, int nthreads, int block_index) {
    if ((int)g_fibers.size() < nthreads) g_fibers.resize(nthreads);
    g_n = nthreads;
    g_body = body;
    g_arg = arg;
    blockIdx.x = block_index;
    blockDim.x = nthreads;
    for (int t = 0; t < nthreads; ++t) {
        Fiber &f = g_fibers[t];
        if (f.stack.size() != kStack) f.stack.assign(kStack, 0);
        f.done = false;
        getcontext(&f.ctx);
        f.ctx.uc_stack.ss_sp = f.stack.data();
        f.ctx.uc_stack.ss_size = kStack;
        f.ctx.uc_link = nullptr;
        makecontext(&f.ctx, fiber_entry, 0);
    }
    g_cur = 0;
    threadIdx.x = 0;
    swapcontext(&g_main, &g_fibers[0].ctx);
}
