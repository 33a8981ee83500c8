// Reciprocal and square root for the sweeps whose results are held to a
// tolerance rather than to bit parity (the Gc/Gs and adjoint kernels): the
// hardware approximations (rcp.approx / rsqrt.approx, about 22 correct
// bits) refined by two Newton-Raphson steps, each of which squares the
// relative error (below 2^-52 after two).  A few fused multiply-adds, with
// no branch and no slow path, where an IEEE division or sqrt inlines both.
// Arguments are finite and normal where these are used; a zero divisor
// gives inf/NaN as a division would.  The root search keeps IEEE division.
#pragma once
#include <cuda_runtime.h>

namespace dk {

__device__ __forceinline__ double fast_rcp(double x)
{
#ifdef __CUDA_ARCH__
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
#else
    return 1.0 / x;
#endif
}

// sqrt(x), x >= 0: x / sqrt(x) by the refined reciprocal square root
// (y <- y (3 - x y^2) / 2, twice).
__device__ __forceinline__ double fast_sqrt(double x)
{
#ifdef __CUDA_ARCH__
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double h = 0.5 * x;
    y = y * fma(-h * y, y, 1.5);
    y = y * fma(-h * y, y, 1.5);
    return x > 0.0 ? x * y : 0.0;
#else
    return sqrt(x);
#endif
}

}  // namespace dk
