// Host-side stand-ins for the CUDA language features used by the reference's
// eikonal kernels, so that those kernels (header sources kept where they lie in
// the reference tree) can be compiled by g++ and executed on the CPU.
//
// This is TEST INFRASTRUCTURE ONLY (the "reference run here" that pins the
// oracle).  Nothing in the product path links it.
//
// Execution model: one CUDA thread block is emulated by `blockDim.x` cooperative
// fibers (ucontext) on a single OS thread.  `__syncthreads()` is a round-robin
// yield: fiber k runs until its next barrier, then fiber k+1, ..., and after
// the last fiber the first resumes past the barrier.  `__shared__` locals become
// function statics, which every fiber of the (single, sequential) block shares,
// exactly like shared memory.  Blocks of a grid run one after the other.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstdint>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__ static
#define __forceinline__ inline
// C99-style `T a[__restrict__ n]` parameters are not C++: drop the hint.
#define __restrict__

struct agdref_dim3 { int x, y, z; };
extern agdref_dim3 threadIdx, blockIdx, blockDim, gridDim;

void __syncthreads();

// CUDA integer intrinsics used by the reference headers.
inline int __clz(int x) { return x == 0 ? 32 : __builtin_clz((unsigned)x); }
inline int __ffs(int x) { return __builtin_ffs(x); }

// CUDA's min/max overloads: floating point versions have fmin/fmax semantics
// (a NaN operand yields the other operand); integer versions are plain.
inline float  max(float a, float b)   { return std::fmax(a, b); }
inline double max(double a, double b) { return std::fmax(a, b); }
inline double max(double a, float b)  { return std::fmax(a, (double)b); }
inline double max(float a, double b)  { return std::fmax((double)a, b); }
inline int    max(int a, int b)       { return a > b ? a : b; }
inline long long max(long long a, long long b) { return a > b ? a : b; }
inline float  min(float a, float b)   { return std::fmin(a, b); }
inline double min(double a, double b) { return std::fmin(a, b); }
inline double min(double a, float b)  { return std::fmin(a, (double)b); }
inline double min(float a, double b)  { return std::fmin((double)a, b); }
inline int    min(int a, int b)       { return a < b ? a : b; }
inline long long min(long long a, long long b) { return a < b ? a : b; }
using std::abs;
using std::sqrt;
using std::floor;
using std::round;
using std::isnan;

// Fiber-emulated launch of one block of `nthreads` threads running `body(arg)`.
void agdref_run_block(void (*body)(void *), void *arg, int nthreads, int block_index);
