// CPU emulation of the small CUDA runtime subset that the reference's live
// engine (src/mm.cu) uses, so that its own kernels and host code can run on
// the host as a parity pin for the oracle. Test infrastructure only: nothing
// in the product links this.
//
// What is emulated, and how:
//  * `__global__` kernels are plain functions; a launch `k<<<g, b>>>(args)`
//    becomes `shim_launch(g, b, k, args)` (a mechanical rewrite of the launch
//    syntax done when the reference file is compiled, see rewrite_launches.py).
//  * Grid blocks run one after the other. The threads of a block run as
//    cooperative fibers (ucontext) on one OS thread: a fiber runs until it
//    reaches __syncthreads() or returns, and when every live fiber has
//    arrived, all of them are resumed again. Within each phase the fibers run
//    in DESCENDING threadIdx order. That order reproduces the lock-step
//    execution a single-warp block has on the GPU: binGEMM (src/mm.cu:288-312,
//    32 threads) rewrites its shared `offset` from thread 0 at the top of the
//    next loop iteration with no barrier after the previous iteration's
//    stores, which is only correct if every other thread finished those
//    stores first -- as a converged warp does, and as thread 0 running last
//    does here.
//  * `__shared__` variables are function-level statics: one copy shared by
//    the fibers of the running block, as blocks never overlap.
//  * Atomics are plain read-modify-writes (one OS thread). Overload
//    resolution is the CUDA one: atomicAdd(int*, float) picks
//    atomicAdd(int*, int) and truncates the float, as the reference's int
//    dense accumulator does (src/mm.cu:33, 386).
//  * Device memory is host memory. cudaMalloc zero-fills and pads every
//    allocation with SHIM_PAD zero bytes, so the reference's reads past the
//    ends of its arrays (mergeGEMM's row loop, src/mm.cu:374-383, reads up to
//    ~2*gridDim rows past c_ptr_base / c_ptr_nnz and writes c_ptr_nnz there;
//    inspectGEMM reads a_ptr[n+1] / b_ptr[n+1], src/mm.cu:200-202) land in
//    owned memory. The uninitialised arrays the reference accumulates into
//    (ptr in cudaCOO2CM, c_ptr_base in cudaInitGEMM, src/mm.cu:89, 111, 164)
//    therefore start at zero.
#pragma once

#include <ucontext.h>

#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <tuple>
#include <utility>
#include <vector>

#define __global__
#define __device__
#define __host__
#define __shared__ static

struct dim3 {
  unsigned x, y, z;
};
inline dim3 threadIdx = {0, 0, 0};
inline dim3 blockIdx = {0, 0, 0};
inline dim3 blockDim = {1, 1, 1};
inline dim3 gridDim = {1, 1, 1};

typedef int cudaError;
typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
enum cudaMemcpyKind {
  cudaMemcpyHostToHost = 0,
  cudaMemcpyHostToDevice = 1,
  cudaMemcpyDeviceToHost = 2,
  cudaMemcpyDeviceToDevice = 3
};

constexpr size_t SHIM_PAD = 1 << 20;

inline std::map<void*, size_t>& shim_allocs() {
  static std::map<void*, size_t> m;
  return m;
}

inline cudaError_t cudaMalloc(void** p, size_t bytes) {
  void* q = std::calloc(1, bytes + SHIM_PAD);
  if (!q) return cudaErrorMemoryAllocation;
  shim_allocs()[q] = bytes;
  *p = q;
  return cudaSuccess;
}
inline cudaError_t cudaFree(void* p) {
  if (!p) return cudaSuccess;
  auto it = shim_allocs().find(p);
  if (it != shim_allocs().end()) {  // only memory this shim handed out
    shim_allocs().erase(it);
    std::free(p);
  }
  return cudaSuccess;
}
inline cudaError_t cudaMemcpy(void* dst, const void* src, size_t bytes, cudaMemcpyKind) {
  if (bytes) std::memmove(dst, src, bytes);
  return cudaSuccess;
}
inline cudaError_t cudaMemset(void* dst, int v, size_t bytes) {
  if (bytes) std::memset(dst, v, bytes);
  return cudaSuccess;
}
template <class T>
inline cudaError_t cudaMemcpyToSymbol(T& sym, const void* src, size_t bytes, size_t offset = 0,
                                      cudaMemcpyKind = cudaMemcpyHostToDevice) {
  std::memcpy(reinterpret_cast<char*>(&sym) + offset, src, bytes);
  return cudaSuccess;
}
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
inline cudaError_t cudaGetLastError() { return cudaSuccess; }
inline const char* cudaGetErrorString(cudaError_t) { return "no error"; }

inline int atomicAdd(int* a, int v) {
  const int old = *a;
  *a = old + v;
  return old;
}
inline unsigned atomicAdd(unsigned* a, unsigned v) {
  const unsigned old = *a;
  *a = old + v;
  return old;
}
inline float atomicAdd(float* a, float v) {
  const float old = *a;
  *a = old + v;
  return old;
}
inline int atomicExch(int* a, int v) {
  const int old = *a;
  *a = v;
  return old;
}
inline float atomicExch(float* a, float v) {
  const float old = *a;
  *a = v;
  return old;
}

// ---- block scheduler (fibers) ----
namespace shim {

enum State { READY, AT_BARRIER, DONE };

struct Block {
  ucontext_t sched;
  std::vector<ucontext_t> ctx;
  std::vector<std::vector<char>> stacks;
  std::vector<int> state;
  int cur = -1;
  void (*body)(void*) = nullptr;
  void* arg = nullptr;
};

inline Block& block() {
  static Block b;
  return b;
}

inline void fiber_entry() {
  Block& b = block();
  b.body(b.arg);
  b.state[b.cur] = DONE;  // returns to b.sched through uc_link
}

constexpr size_t STACK_BYTES = 256 * 1024;

// Runs body(arg) as the `nthreads` threads of one block.
inline void run_block(unsigned nthreads, void (*body)(void*), void* arg) {
  Block& b = block();
  if (b.stacks.size() < nthreads) b.stacks.resize(nthreads);
  b.ctx.assign(nthreads, ucontext_t{});
  b.state.assign(nthreads, READY);
  b.body = body;
  b.arg = arg;
  for (unsigned t = 0; t < nthreads; ++t) {
    if (b.stacks[t].size() < STACK_BYTES) b.stacks[t].resize(STACK_BYTES);
    getcontext(&b.ctx[t]);
    b.ctx[t].uc_stack.ss_sp = b.stacks[t].data();
    b.ctx[t].uc_stack.ss_size = STACK_BYTES;
    b.ctx[t].uc_link = &b.sched;
    makecontext(&b.ctx[t], fiber_entry, 0);
  }
  for (;;) {
    bool any = false;
    for (int t = (int)nthreads - 1; t >= 0; --t) {  // descending: thread 0 last
      if (b.state[t] != READY) continue;
      any = true;
      b.cur = t;
      threadIdx = dim3{(unsigned)t, 0, 0};
      swapcontext(&b.sched, &b.ctx[t]);
    }
    if (!any) break;
    bool waiting = false;
    for (unsigned t = 0; t < nthreads; ++t)
      if (b.state[t] == AT_BARRIER) { b.state[t] = READY; waiting = true; }
    if (!waiting) break;
  }
  b.cur = -1;
}

}  // namespace shim

inline void __syncthreads() {
  shim::Block& b = shim::block();
  const int me = b.cur;
  b.state[me] = shim::AT_BARRIER;
  swapcontext(&b.ctx[me], &b.sched);
  threadIdx = dim3{(unsigned)me, 0, 0};
}

template <class K, class Tup>
struct LaunchArg {
  K kernel;
  Tup* args;
};

template <class K, class Tup>
inline void launch_body(void* p) {
  auto* la = static_cast<LaunchArg<K, Tup>*>(p);
  std::apply(la->kernel, *la->args);
}

// k<<<grid, block>>>(args...) for 1-D launches.
template <class... P, class... A>
inline void shim_launch(long long grid, long long blk, void (*k)(P...), A&&... a) {
  using Tup = std::tuple<P...>;
  Tup args(static_cast<P>(a)...);
  LaunchArg<void (*)(P...), Tup> la{k, &args};
  gridDim = dim3{(unsigned)grid, 1, 1};
  blockDim = dim3{(unsigned)blk, 1, 1};
  for (long long g = 0; g < grid; ++g) {
    blockIdx = dim3{(unsigned)g, 0, 0};
    shim::run_block((unsigned)blk, launch_body<void (*)(P...), Tup>, &la);
  }
}
