// TEST INFRASTRUCTURE ONLY.  Lets g++ compile the library's device sources
// (dazi_current_release_b200/csrc/*.cu) as host code so that the CPU test
// suite can check the device arithmetic against the oracle without a GPU.
// CUDA qualifiers become plain C++, the round-to-nearest intrinsics become
// the corresponding IEEE operations, and the warp primitives act on one
// lane.  Nothing in the shipped library includes this file.
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#undef __device__
#undef __host__
#undef __global__
#undef __forceinline__
#undef __noinline__
#undef __constant__
#undef __launch_bounds__
#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __noinline__
#define __constant__
#define __launch_bounds__(...)
using std::isfinite;
using std::max;
using std::min;
using std::signbit;
static inline float __fmul_rn(float a, float b) { return a * b; }
static inline float __fadd_rn(float a, float b) { return a + b; }
static inline float __fsub_rn(float a, float b) { return a - b; }
static inline float __fdiv_rn(float a, float b) { return a / b; }
static inline float __fsqrt_rn(float a) { return std::sqrt(a); }
static inline double __dmul_rn(double a, double b) { return a * b; }
static inline double __dadd_rn(double a, double b) { return a + b; }
static inline double __dsub_rn(double a, double b) { return a - b; }
static inline double __ddiv_rn(double a, double b) { return a / b; }
static inline double __dsqrt_rn(double a) { return std::sqrt(a); }
static inline float __double2float_rn(double a) { return (float)a; }
static inline int __double2hiint(double a)
{
    uint64_t u;
    std::memcpy(&u, &a, 8);
    return (int)(uint32_t)(u >> 32);
}
static inline double __hiloint2double(int hi, int lo)
{
    const uint64_t u = ((uint64_t)(uint32_t)hi << 32) | (uint32_t)lo;
    double d;
    std::memcpy(&d, &u, 8);
    return d;
}
static inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
static inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }
static inline void __syncthreads() {}
// CUDA's fast single-precision exponential (device approximation); the host
// build uses the libm function (one translation unit includes this file)
extern "C" float __expf(float x) noexcept { return expf(x); }
extern "C" float __fdividef(float a, float b) noexcept { return a / b; }
extern "C" void __sincosf(float x, float* s, float* c) noexcept { sincosf(x, s, c); }
struct EmuDim { unsigned x = 0, y = 0, z = 0; };
static EmuDim threadIdx, blockIdx, blockDim, gridDim;
static inline unsigned atomicAdd(unsigned* p, unsigned v) { unsigned o = *p; *p += v; return o; }
static inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v)
{
    unsigned long long o = *p;
    *p += v;
    return o;
}
static inline int atomicAdd(int* p, int v) { int o = *p; *p += v; return o; }
static inline int atomicCAS(int* p, int cmp, int v) { int o = *p; if (o == cmp) *p = v; return o; }
static inline void __syncwarp(unsigned = 0xffffffffu) {}
static inline int atomicOr(int* p, int v) { int o = *p; *p |= v; return o; }
template <class T> static inline T __shfl_sync(unsigned, T v, int) { return v; }
template <class T> static inline T __shfl_xor_sync(unsigned, T v, int) { return v; }
static inline float __int_as_float(int i) { float f; std::memcpy(&f, &i, 4); return f; }
static inline unsigned __reduce_add_sync(unsigned, unsigned v) { return v; }
static inline bool __any_sync(unsigned, bool v) { return v; }
