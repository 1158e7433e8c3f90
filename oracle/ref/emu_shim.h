// emu_shim.h -- force-included (g++ -include) ahead of every reference
// source compiled by oracle/ref/Makefile.refemu.
//
// TEST INFRASTRUCTURE ONLY.  It lets the reference's own CUDA sources
// (collision/lbvh, collision/bvtt_front, collision/auxiliary,
// collision/narrow_phase, utility) compile unmodified as host C++ and run
// every kernel one thread at a time, in thread-index order, on the CPU:
//   * device memory is host memory (cudaMalloc/cudaMemcpy/cudaMemset/...
//     are renamed to the emu_* functions of emu_runtime.cpp);
//   * thrust runs on its sequential CPP system;
//   * the launcher of Mine/system/CudaDevice/CudaKernelLauncher.cu, the only
//     reference file with a <<<grid, block>>> launch, is replaced by one that
//     loops over blocks and threads with the same signatures;
//   * atomics, bit intrinsics and the warp intrinsics of atomicAggInc
//     (Mine/utility/CudaDeviceUtils.cu:57-80) act on one thread at a time --
//     every warp holds exactly one active lane;
//   * Logger (Mine/system/Log/Logger.hpp) is silent.
// None of the reference's kernels uses shared memory, __syncthreads or a
// spin-wait, so a sequential schedule is one of the schedules a GPU may run;
// results that depend on the schedule (the order of front entries within a
// node, the order of emitted pairs) are compared as sets.
#pragma once

#define __STORAGE__ extern
#define __CUDA_LAUNCHER_H_
#define __LOGGER_HPP_

#define cudaMalloc emu_cudaMalloc
#define cudaFree emu_cudaFree
#define cudaMemcpy emu_cudaMemcpy
#define cudaMemset emu_cudaMemset
#define cudaMemGetInfo emu_cudaMemGetInfo
#define cudaDeviceSynchronize emu_cudaDeviceSynchronize
#define cudaGetLastError emu_cudaGetLastError
#define cudaPeekAtLastError emu_cudaPeekAtLastError

#include <cuda_runtime.h>
#include <device_launch_parameters.h>

#include <math.h>
#include <cstdint>
#include <cstring>
#include <string>
#include <iostream>
#include <thrust/system_error.h>

// ---- intrinsics, one thread at a time ------------------------------------
inline int atomicAdd(int *a, int v) { int o = *a; *a = o + v; return o; }
inline unsigned atomicAdd(unsigned *a, unsigned v) { unsigned o = *a; *a = o + v; return o; }
inline unsigned long long atomicAdd(unsigned long long *a, unsigned long long v) {
    unsigned long long o = *a; *a = o + v; return o;
}
inline float atomicAdd(float *a, float v) { float o = *a; *a = o + v; return o; }
inline double atomicAdd(double *a, double v) { double o = *a; *a = o + v; return o; }
inline int atomicSub(int *a, int v) { int o = *a; *a = o - v; return o; }
inline unsigned atomicSub(unsigned *a, unsigned v) { unsigned o = *a; *a = o - v; return o; }
inline int atomicMin(int *a, int v) { int o = *a; if (v < o) *a = v; return o; }
inline unsigned atomicMin(unsigned *a, unsigned v) { unsigned o = *a; if (v < o) *a = v; return o; }
inline int atomicMax(int *a, int v) { int o = *a; if (v > o) *a = v; return o; }
inline unsigned atomicMax(unsigned *a, unsigned v) { unsigned o = *a; if (v > o) *a = v; return o; }
inline int atomicOr(int *a, int v) { int o = *a; *a = o | v; return o; }
inline unsigned atomicOr(unsigned *a, unsigned v) { unsigned o = *a; *a = o | v; return o; }
inline int atomicAnd(int *a, int v) { int o = *a; *a = o & v; return o; }
inline unsigned atomicAnd(unsigned *a, unsigned v) { unsigned o = *a; *a = o & v; return o; }
inline int atomicExch(int *a, int v) { int o = *a; *a = v; return o; }
inline unsigned atomicExch(unsigned *a, unsigned v) { unsigned o = *a; *a = v; return o; }
inline float atomicExch(float *a, float v) { float o = *a; *a = v; return o; }
inline int atomicCAS(int *a, int c, int v) { int o = *a; if (o == c) *a = v; return o; }
inline unsigned atomicCAS(unsigned *a, unsigned c, unsigned v) { unsigned o = *a; if (o == c) *a = v; return o; }
inline unsigned long long atomicCAS(unsigned long long *a, unsigned long long c, unsigned long long v) {
    unsigned long long o = *a; if (o == c) *a = v; return o;
}

inline int __clz(int x) { return x == 0 ? 32 : __builtin_clz((unsigned)x); }
inline int __clzll(long long x) { return x == 0 ? 64 : __builtin_clzll((unsigned long long)x); }
inline int __popc(unsigned x) { return __builtin_popcount(x); }
inline int __popcll(unsigned long long x) { return __builtin_popcountll(x); }
inline int __ffs(int x) { return __builtin_ffs(x); }
inline int __float_as_int(float f) { int i; std::memcpy(&i, &f, 4); return i; }
inline float __int_as_float(int i) { float f; std::memcpy(&f, &i, 4); return f; }
inline unsigned __float_as_uint(float f) { unsigned i; std::memcpy(&i, &f, 4); return i; }
inline float __uint_as_float(unsigned i) { float f; std::memcpy(&f, &i, 4); return f; }
inline long long __double_as_longlong(double d) { long long i; std::memcpy(&i, &d, 8); return i; }
inline double __longlong_as_double(long long i) { double d; std::memcpy(&d, &i, 8); return d; }
// Only normalize() in Mine/utility/CudaDeviceUtils.cu calls rsqrt, and nothing
// on the collision path calls normalize().
inline float rsqrt(float x) { return 1.0f / sqrtf(x); }
inline double rsqrt(double x) { return 1.0 / sqrt(x); }
inline void __threadfence() {}
inline unsigned __activemask() { return 1u << (threadIdx.x & 31u); }
inline unsigned __ballot_sync(unsigned mask, int pred) { return pred ? (mask & __activemask()) : 0u; }
template <typename T>
inline T __shfl_sync(unsigned, T v, int, int = 32) { return v; }

// ---- silent logger (same interface as Mine/system/Log/Logger.hpp) --------
#include "base/Singleton.h"
namespace mn {
enum class TimerType { CPU, GPU };
class Logger : public ManagedSingleton<Logger> {
  public:
    template <TimerType> static void tick() {}
    template <TimerType> static void tock() {}
    template <TimerType> static void tock(std::string) {}
    template <TimerType> static void blankLine() {}
    template <TimerType> static void recordSection(std::string) {}
    static void message(const std::string &) {}
    static void record(const std::string &) {}
    static void insertRecord(const std::string &) {}
};
}  // namespace mn

// ---- sequential launcher (same signatures as CudaKernelLauncher.cu) ------
#include "utility/CudaExecutionPolicy.h"
namespace mn {
template <typename... Arguments>
void emu_grid(int gs, int bs, void (*f)(Arguments...), Arguments... args) {
    gridDim = dim3(gs > 0 ? gs : 0, 1, 1);
    blockDim = dim3(bs, 1, 1);
    for (int b = 0; b < gs; b++) {
        blockIdx = make_uint3(b, 0, 0);
        for (int t = 0; t < bs; t++) {
            threadIdx = make_uint3(t, 0, 0);
            f(args...);
        }
    }
}
constexpr int kEmuBlock = 256;
template <typename... Arguments>
void debugLaunch(int gs, int bs, void (*f)(Arguments...), Arguments... args) { emu_grid(gs, bs, f, args...); }
template <typename... Arguments>
void recordLaunch(std::string, int gs, int bs, size_t, void (*f)(Arguments...), Arguments... args) {
    emu_grid(gs, bs, f, args...);
}
template <typename... Arguments>
void recordLaunch(const char *, int gs, int bs, size_t, void (*f)(Arguments...), Arguments... args) {
    emu_grid(gs, bs, f, args...);
}
template <typename... Arguments>
void cleanLaunch(int gs, int bs, void (*f)(Arguments...), Arguments... args) { emu_grid(gs, bs, f, args...); }
template <typename... Arguments>
void configuredLaunch(LaunchInput instr, void (*f)(Arguments...), Arguments... args) {
    const int n = instr.threads();
    if (n <= 0) return;
    emu_grid((n + kEmuBlock - 1) / kEmuBlock, kEmuBlock, f, args...);
}
}  // namespace mn
