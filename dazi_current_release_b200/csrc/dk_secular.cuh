// Rayleigh and Love secular functions and the reference's root search, in
// FP64 on the CUDA cores.
//
//   dltar4 + var + dnka + normc   surfdisp96.f:767-865, 868-985, 1018-1062, 989-1014
//   dltar1 (Love)                 surfdisp96.f:704-763
//   getsol (bracket)              surfdisp96.f:384-476
//   nevill + half (refine)        surfdisp96.f:551-680
//   surfdisp96 period loop        surfdisp96.f:52-354 (mode 1; phase, or
//                                 group velocity by the second root at
//                                 period t/(1-h), :226-233, 276-303)
//
// Optional FP32 coarse scan (DAZI_FORM_SCAN_FP32): the getsol
// scan steps evaluate the secular function in FP32 and use only its sign;
// values below kScanTrust32 are re-evaluated in FP64, and both ends of a
// detected bracket are evaluated in FP64 before nevill() (whose steps are
// FP64), so the values nevill() sees are the reference's.  A bracket end
// whose FP64 sign contradicts its FP32 sign restarts the period in FP64.
// A warp step runs in FP32 only when all its waiting lanes scan.  The root
// search is latency-bound (each lane a chain of dependent operations), so
// FP32 evaluations are not much cheaper than FP64 ones here: the scan runs
// in FP64 unless this flag asks otherwise.
//
// The layer chain is a sequential product of 5x5 Dunkin compound matrices,
// one model per thread; the tensor cores have no role here.  The root search
// is written as a state machine that performs exactly one secular-function
// evaluation per step, so all lanes of a warp run the layer chain together
// (lock-step over the layers, broadcast shared-memory reads) even though
// each lane's bracket and Neville sequence are its own.  The sequence of
// evaluation points is the reference's, step for step.
#pragma once
#include "dk_model.cuh"
#include <type_traits>
#include <utility>

namespace dk {

constexpr double TWOPI = 2.0 * 3.141592653589793;

__device__ __forceinline__ double fsign1(double x) { return signbit(x) ? -1.0 : 1.0; }

// normc() between layers: the reference divides the vector by its largest
// component t1 (unless t1 < 1e-40).  The value returned is the top layer's
// f0 / max|f|, which any exact positive rescaling of the intermediate
// vectors leaves unchanged, so the intermediate layers are scaled by
// 2^-e (e the exponent of max|f|, read from the bits; exact, no rounding)
// and only the last vector is divided by its largest component.  The
// result differs from the reference's per-layer divisions only in rounding.
__device__ __forceinline__ void normc_pow2(double& e0, double& e1, double& e2, double& e3, double& e4)
{
    // high words of |e_i|: ordered as the magnitudes (to 2^-20)
    const int h = max(max(max(__double2hiint(e0) & 0x7fffffff, __double2hiint(e1) & 0x7fffffff),
                          max(__double2hiint(e2) & 0x7fffffff, __double2hiint(e3) & 0x7fffffff)),
                      __double2hiint(e4) & 0x7fffffff);
    // below 1e-40 (high word 0x37a16c26) the reference leaves the vector
    // as it is
    if (h < 0x37a16c26) return;
    const int ex = min((h >> 20) - 1023, 1022);
    const double sc = __hiloint2double((1023 - ex) << 20, 0);   // 2^-ex
    e0 *= sc; e1 *= sc; e2 *= sc; e3 *= sc; e4 *= sc;
}

// Secular-function value at wavenumber wvno, angular frequency omega.
// Each layer product is rescaled (normc_pow2); the factors are discarded,
// as in the reference, since they do not move roots.
template <class M>
__device__ __forceinline__ double dltar4(const M& mdl, int mmax, double wvno, double omega)
{
    if (omega < 1.0e-4) omega = 1.0e-4;
    const double wvno2 = wvno * wvno;
    const double iom = 1.0 / omega;
    const double tio2 = 2.0 * iom * iom;
    LayerD L = mdl.layer(mmax - 1);
    double xka = omega * L.ia, xkb = omega * L.ib;
    double ra = sqrt((wvno + xka) * fabs(wvno - xka));
    double rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
    double gammk = L.b2 * tio2;
    double gam = gammk * wvno2;
    double gamm1 = gam - 1.0;
    double rho1 = L.rho;
    double e0 = rho1 * rho1 * (gamm1 * gamm1 - gam * gammk * ra * rb);
    double e1 = -rho1 * ra;
    double e2 = rho1 * (gamm1 - gammk * ra * rb);
    double e3 = rho1 * rb;
    double e4 = wvno2 - ra * rb;
    // the next layer's record is loaded one step ahead: the loads of a
    // column's table come from L2/DRAM (the resident columns' tables exceed
    // L2) and a layer step is long enough to cover that latency
    LayerD Ln = mdl.layer(mmax >= 2 ? mmax - 2 : 0);
#pragma unroll 1
    for (int m = mmax - 2; m >= 0; --m) {
        L = Ln;
        Ln = mdl.layer(m > 0 ? m - 1 : 0);
        const double dpth = L.d;
        xka = omega * L.ia; xkb = omega * L.ib;
        gammk = L.b2 * tio2;
        gam = gammk * wvno2;
        const double pa = (wvno + xka) * fabs(wvno - xka);
        const double pb = (wvno + xkb) * fabs(wvno - xkb);
        const double ira = rsqrt(pa), irb = rsqrt(pb);
        ra = pa * ira; rb = pb * irb;
        const double p = ra * dpth, q = rb * dpth;
        // var(): cos/sin (oscillatory) or scaled cosh/sinh (evanescent)
        double w, x, cosp, y, z, cosq, ep = 1.0, eq = 1.0;
        bool evp = false, evq = false;
        if (wvno < xka) {
            double sp, cp;
            sincos(p, &sp, &cp);
            w = sp * ira; x = -ra * sp; cosp = cp;
        } else if (wvno == xka) {
            cosp = 1.0; w = dpth; x = 0.0;
        } else {
            evp = true;
            ep = exp(-p);
            const double fac = (p < 16.0) ? ep * ep : 0.0;
            cosp = (1.0 + fac) * 0.5;
            const double sinp = (1.0 - fac) * 0.5;
            w = sinp * ira; x = ra * sinp;
        }
        if (wvno < xkb) {
            double sq, cq;
            sincos(q, &sq, &cq);
            y = sq * irb; z = -rb * sq; cosq = cq;
        } else if (wvno == xkb) {
            cosq = 1.0; y = dpth; z = 0.0;
        } else {
            evq = true;
            eq = exp(-q);
            const double fac = (q < 16.0) ? eq * eq : 0.0;
            cosq = (1.0 + fac) * 0.5;
            const double sinq = (1.0 - fac) * 0.5;
            y = sinq * irb; z = rb * sinq;
        }
        // a0 = exp(-(pex + sex)), 0 once the exponent reaches 60
        const double exa = (evp ? p : 0.0) + (evq ? q : 0.0);
        const double a0 = (exa < 60.0) ? ep * eq : 0.0;
        const double cpcq = cosp * cosq, cpy = cosp * y, cpz = cosp * z;
        const double cqw = cosq * w, cqx = cosq * x;
        const double xy = x * y, xz = x * z, wy = w * y, wz = w * z;
        // dnka(): Dunkin compound matrix
        rho1 = L.rho;
        const double rinv = L.irho, rho2 = rho1 * rho1, r2inv = rinv * rinv;
        const double gamm1l = gam - 1.0, twgm1 = gam + gamm1l, gmgmk = gam * gammk;
        const double gmgm1 = gam * gamm1l, gm1sq = gamm1l * gamm1l;
        const double a0pq = a0 - cpcq;
        const double c11 = cpcq - 2.0 * gmgm1 * a0pq - gmgmk * xz - wvno2 * gm1sq * wy;
        const double c12 = (wvno2 * cpy - cqx) * rinv;
        const double c13 = -(twgm1 * a0pq + gammk * xz + wvno2 * gamm1l * wy) * rinv;
        const double c14 = (cpz - wvno2 * cqw) * rinv;
        const double c15 = -(2.0 * wvno2 * a0pq + xz + wvno2 * wvno2 * wy) * r2inv;
        const double c21 = (gmgmk * cpz - gm1sq * cqw) * rho1;
        const double c22 = cpcq;
        const double c23 = gammk * cpz - gamm1l * cqw;
        const double c24 = -wz;
        const double c41 = (gm1sq * cpy - gmgmk * cqx) * rho1;
        const double c42 = -xy;
        const double c43 = gamm1l * cpy - gammk * cqx;
        const double c51 = -(2.0 * gmgmk * gm1sq * a0pq + gmgmk * gmgmk * xz + gm1sq * gm1sq * wy) * rho2;
        const double c53 = -(gammk * gamm1l * twgm1 * a0pq + gam * gammk * gammk * xz + gamm1l * gm1sq * wy) * rho1;
        const double tt = -2.0 * wvno2;
        const double c31 = tt * c53, c32 = tt * c43;
        const double c33 = a0 + 2.0 * (cpcq - c11);
        const double c34 = tt * c23, c35 = tt * c13;
        // ee(i) = sum_j e(j) * ca(j,i), using ca's symmetries
        //   ca(2,5)=ca(1,4) ca(4,4)=ca(2,2) ca(4,5)=ca(1,2) ca(5,2)=ca(4,1)
        //   ca(5,4)=ca(2,1) ca(5,5)=ca(1,1)
        const double f0 = e0 * c11 + e1 * c21 + e2 * c31 + e3 * c41 + e4 * c51;
        const double f1 = e0 * c12 + e1 * c22 + e2 * c32 + e3 * c42 + e4 * c41;
        const double f2 = e0 * c13 + e1 * c23 + e2 * c33 + e3 * c43 + e4 * c53;
        const double f3 = e0 * c14 + e1 * c24 + e2 * c34 + e3 * c22 + e4 * c21;
        const double f4 = e0 * c15 + e1 * c14 + e2 * c35 + e3 * c12 + e4 * c11;
        e0 = f0; e1 = f1; e2 = f2; e3 = f3; e4 = f4;
        normc_pow2(e0, e1, e2, e3, e4);
    }
    if (mmax < 2) return e0;   // no layer above the half-space: no normc
    // the top layer's normc(): e0 / max|e|
    double t1 = fmax(fmax(fmax(fabs(e0), fabs(e1)), fmax(fabs(e2), fabs(e3))), fabs(e4));
    if (t1 < 1.0e-40) t1 = 1.0;
    return e0 / t1;
}

// Love-wave secular function, surfdisp96.f:704-763: the Haskell-Thomson
// SH product from the half-space to the surface, each step rescaled by its
// larger component.  Reads the real*4 layer values (d, Vp, Vs, rho) and
// promotes them, as dble(b(m)) does; every operation is rounded on its own
// (no fused multiply-add), in the reference's order.
template <class M>
__device__ __forceinline__ double dltar1(const M& mdl, int mmax, double wvno, double omega)
{
    float4 L = mdl.layerf(mmax - 1);
    double beta1 = (double)L.z, rho1 = (double)L.w;
    double xkb = __ddiv_rn(omega, beta1);
    double rb = __dsqrt_rn(__dmul_rn(__dadd_rn(wvno, xkb), fabs(__dsub_rn(wvno, xkb))));
    double e1 = __dmul_rn(rho1, rb);
    double e2 = __ddiv_rn(1.0, __dmul_rn(beta1, beta1));
#pragma unroll 1
    for (int m = mmax - 2; m >= 0; --m) {
        L = mdl.layerf(m);
        beta1 = (double)L.z;
        rho1 = (double)L.w;
        const double dm = (double)L.x;
        const double xmu = __dmul_rn(__dmul_rn(rho1, beta1), beta1);
        xkb = __ddiv_rn(omega, beta1);
        rb = __dsqrt_rn(__dmul_rn(__dadd_rn(wvno, xkb), fabs(__dsub_rn(wvno, xkb))));
        const double q = __dmul_rn(dm, rb);
        double y, z, cosq;
        if (wvno < xkb) {
            double sinq;
            sincos(q, &sinq, &cosq);
            y = __ddiv_rn(sinq, rb);
            z = __dmul_rn(-rb, sinq);
        } else if (wvno == xkb) {
            cosq = 1.0; y = dm; z = 0.0;
        } else {
            const double fac = (q < 16.0) ? exp(__dmul_rn(-2.0, q)) : 0.0;
            cosq = __dmul_rn(__dadd_rn(1.0, fac), 0.5);
            const double sinq = __dmul_rn(__dsub_rn(1.0, fac), 0.5);
            y = __ddiv_rn(sinq, rb);
            z = __dmul_rn(rb, sinq);
        }
        const double e10 = __dadd_rn(__dmul_rn(e1, cosq), __dmul_rn(__dmul_rn(e2, xmu), z));
        const double e20 = __dadd_rn(__ddiv_rn(__dmul_rn(e1, y), xmu), __dmul_rn(e2, cosq));
        // normalise by xnor = max(|e10|, |e20|) (1 below 1e-40): the larger
        // component's quotient is exactly +-1, so one division gives the
        // reference's two quotients bit for bit
        const double xnor = fabs(e10), ynor = fabs(e20);
        if (fmax(xnor, ynor) < 1.0e-40) {
            e1 = e10;
            e2 = e20;
        } else if (ynor > xnor) {
            e1 = __ddiv_rn(e10, ynor);
            e2 = copysign(1.0, e20);
        } else {
            e1 = copysign(1.0, e10);
            e2 = __ddiv_rn(e20, xnor);
        }
    }
    return e1;
}

// The same secular function in FP32, for the coarse trial-velocity scan.
// Reads the flattened layer table (d, Vp, Vs, rho) directly; exponentials,
// reciprocals and square roots in single precision.  Only the sign of the
// result is used, and only where its magnitude exceeds kScanTrust32 (on the
// normalised scale of F, |F| <= 1; the FP32 error measured on the uneven
// batch stays below 7e-4, on high-contrast random columns below 0.15 at
// |F| ~ 0.6); smaller values and every bracket end point are re-evaluated
// in FP64.  The fast intrinsics (__sincosf, __expf, __fdividef) are enough
// for a sign that is verified.
constexpr float kScanTrust32 = 0.05f;

template <class LayerF>
__device__ __forceinline__ float dltar4_f32(LayerF layerf, int mmax, float wvno, float omega)
{
    if (omega < 1.0e-4f) omega = 1.0e-4f;
    const float wvno2 = wvno * wvno;
    const float iom = 1.0f / omega;
    const float tio2 = 2.0f * iom * iom;
    float4 L = layerf(mmax - 1);
    float xka = __fdividef(omega, L.y), xkb = __fdividef(omega, L.z);
    float ra = sqrtf((wvno + xka) * fabsf(wvno - xka));
    float rb = sqrtf((wvno + xkb) * fabsf(wvno - xkb));
    float gammk = L.z * L.z * tio2;
    float gam = gammk * wvno2;
    float gamm1 = gam - 1.0f;
    float rho1 = L.w;
    float e0 = rho1 * rho1 * (gamm1 * gamm1 - gam * gammk * ra * rb);
    float e1 = -rho1 * ra;
    float e2 = rho1 * (gamm1 - gammk * ra * rb);
    float e3 = rho1 * rb;
    float e4 = wvno2 - ra * rb;
#pragma unroll 1
    for (int m = mmax - 2; m >= 0; --m) {
        L = layerf(m);
        const float dpth = L.x;
        xka = __fdividef(omega, L.y); xkb = __fdividef(omega, L.z);
        gammk = L.z * L.z * tio2;
        gam = gammk * wvno2;
        const float pa = (wvno + xka) * fabsf(wvno - xka);
        const float pb = (wvno + xkb) * fabsf(wvno - xkb);
        const float ira = rsqrtf(pa), irb = rsqrtf(pb);
        ra = pa * ira; rb = pb * irb;
        const float p = ra * dpth, q = rb * dpth;
        float w, x, cosp, y, z, cosq, ep = 1.0f, eq = 1.0f;
        bool evp = false, evq = false;
        if (wvno < xka) {
            float sp, cp;
            __sincosf(p, &sp, &cp);
            w = sp * ira; x = -ra * sp; cosp = cp;
        } else if (wvno == xka) {
            cosp = 1.0f; w = dpth; x = 0.0f;
        } else {
            evp = true;
            ep = __expf(-p);
            const float fac = (p < 16.0f) ? ep * ep : 0.0f;
            cosp = (1.0f + fac) * 0.5f;
            const float sinp = (1.0f - fac) * 0.5f;
            w = sinp * ira; x = ra * sinp;
        }
        if (wvno < xkb) {
            float sq, cq;
            __sincosf(q, &sq, &cq);
            y = sq * irb; z = -rb * sq; cosq = cq;
        } else if (wvno == xkb) {
            cosq = 1.0f; y = dpth; z = 0.0f;
        } else {
            evq = true;
            eq = __expf(-q);
            const float fac = (q < 16.0f) ? eq * eq : 0.0f;
            cosq = (1.0f + fac) * 0.5f;
            const float sinq = (1.0f - fac) * 0.5f;
            y = sinq * irb; z = rb * sinq;
        }
        const float exa = (evp ? p : 0.0f) + (evq ? q : 0.0f);
        const float a0 = (exa < 60.0f) ? ep * eq : 0.0f;
        const float cpcq = cosp * cosq, cpy = cosp * y, cpz = cosp * z;
        const float cqw = cosq * w, cqx = cosq * x;
        const float xy = x * y, xz = x * z, wy = w * y, wz = w * z;
        rho1 = L.w;
        const float rinv = __fdividef(1.0f, rho1), rho2 = rho1 * rho1, r2inv = rinv * rinv;
        const float gamm1l = gam - 1.0f, twgm1 = gam + gamm1l, gmgmk = gam * gammk;
        const float gmgm1 = gam * gamm1l, gm1sq = gamm1l * gamm1l;
        const float a0pq = a0 - cpcq;
        const float c11 = cpcq - 2.0f * gmgm1 * a0pq - gmgmk * xz - wvno2 * gm1sq * wy;
        const float c12 = (wvno2 * cpy - cqx) * rinv;
        const float c13 = -(twgm1 * a0pq + gammk * xz + wvno2 * gamm1l * wy) * rinv;
        const float c14 = (cpz - wvno2 * cqw) * rinv;
        const float c15 = -(2.0f * wvno2 * a0pq + xz + wvno2 * wvno2 * wy) * r2inv;
        const float c21 = (gmgmk * cpz - gm1sq * cqw) * rho1;
        const float c22 = cpcq;
        const float c23 = gammk * cpz - gamm1l * cqw;
        const float c24 = -wz;
        const float c41 = (gm1sq * cpy - gmgmk * cqx) * rho1;
        const float c42 = -xy;
        const float c43 = gamm1l * cpy - gammk * cqx;
        const float c51 = -(2.0f * gmgmk * gm1sq * a0pq + gmgmk * gmgmk * xz + gm1sq * gm1sq * wy) * rho2;
        const float c53 = -(gammk * gamm1l * twgm1 * a0pq + gam * gammk * gammk * xz + gamm1l * gm1sq * wy) * rho1;
        const float tt = -2.0f * wvno2;
        const float c31 = tt * c53, c32 = tt * c43;
        const float c33 = a0 + 2.0f * (cpcq - c11);
        const float c34 = tt * c23, c35 = tt * c13;
        const float f0 = e0 * c11 + e1 * c21 + e2 * c31 + e3 * c41 + e4 * c51;
        const float f1 = e0 * c12 + e1 * c22 + e2 * c32 + e3 * c42 + e4 * c41;
        const float f2 = e0 * c13 + e1 * c23 + e2 * c33 + e3 * c43 + e4 * c53;
        const float f3 = e0 * c14 + e1 * c24 + e2 * c34 + e3 * c22 + e4 * c21;
        const float f4 = e0 * c15 + e1 * c14 + e2 * c35 + e3 * c12 + e4 * c11;
        float t1 = fmaxf(fmaxf(fmaxf(fabsf(f0), fabsf(f1)), fmaxf(fabsf(f2), fabsf(f3))), fabsf(f4));
        if (!(t1 > 1.0e-30f)) t1 = 1.0f;
        const float tinv = __fdividef(1.0f, t1);
        e0 = f0 * tinv; e1 = f1 * tinv; e2 = f2 * tinv; e3 = f3 * tinv; e4 = f4 * tinv;
    }
    return e0;
}

// ------------------------------------------------------------------------
// Root search state machine.  One instance per model; `next()` consumes the
// secular value of the last requested point and advances to the next point
// to evaluate (or to the end of the model).
//
// GROUP (igr > 0, surfdisp96.f:226-233, 276-303): each period k solves at
// t1a = t/(1+h) (the phase root c(k), which also seeds period k+1), then
// runs getsol again at t1b = t/(1-h) from c(k) - 1.5 dc with floor
// cb(k) + 0.01 dc (cb(k) = 0 for the fundamental mode) and ifirst = 0; a
// second search that finds no root falls back to c(k).  The output is the
// real*4 group velocity of the two roots.  h = 0.005 (h0, surfdisp96.f:113).
// The two periods of a group-velocity period t (surfdisp96.f:226-233):
// t1a = t/(1.+h), t1b = t/(1.-h), real*8 quotients stored in real*4, h = 0.005.
__device__ __forceinline__ void group_periods(double t, float& t1a, float& t1b)
{
    t1a = __double2float_rn(__ddiv_rn(t, (double)__fadd_rn(1.0f, 0.005f)));
    t1b = __double2float_rn(__ddiv_rn(t, (double)__fsub_rn(1.0f, 0.005f)));
}

// An output object of the root search may also take the two roots behind a
// group velocity: out.group_roots(k, c0, c1), c0 the secant-refined root at
// t1a, c1 the one at t1b, or 0 where the second search found no root and
// surfdisp96 used c0 in its place.  Detected at compile time.
template <class O, class = void>
struct HasGroupRoots { static constexpr bool value = false; };
template <class O>
struct HasGroupRoots<O, decltype((void)std::declval<O&>().group_roots(0, 0.0, 0.0))> {
    static constexpr bool value = true;
};

// FAST (DAZI_FORM_FAST_ROOT, Rayleigh/Love phase velocity): the scan is
// getsol's, point for point, so the bracket and with it the mode are the
// reference's; the bracket is then refined by Brent's method (inverse
// quadratic interpolation / secant / bisection; R. P. Brent, Algorithms for
// Minimization without Derivatives, 1973, ch. 4) to kFastRootTol * c instead
// of nevill()'s hybrid to 1e-6 * c.  The root is the exact one to that
// tolerance (the reference's lies anywhere in its final 1e-6 * c bracket);
// the next period's scan starts 1.5 dc below it.  About 3.5 instead of 12
// refinement evaluations per period on uneven columns.
constexpr double kFastRootTol = 1.0e-10;

// Brent's state: the last step and the one before (FAST instantiations only)
struct BrentSteps { double bd, be; };
struct NoBrentSteps {};

template <bool GROUP = false, bool FAST = false>
struct RootSM : std::conditional_t<FAST, BrentSteps, NoBrentSteps> {
    static_assert(!(GROUP && FAST), "the Brent refinement serves phase velocity");
    enum Phase : int { START = 0, GS_FIRST, GS_SCAN, VER1, VER2, NEV_A, NEV_B, NEV_CD, DONE,
                       GR_START, BRENT_INIT, BRENT };
    // model constants
    double cc, cm, dc, cmax, tol;
    float betmx;
    int kmax;
    // period state
    int phase, k, idir, nev, nctrl, mm, evals, fail_k;
    bool ifirst;
    // FP32 coarse scan: sc32 enables it, p64 forces FP64 for the rest of the
    // current period (after a verification mismatch), want64 is the
    // precision of the pending request, d1x/d2x mark del1/del2 as FP64 values
    bool sc32, p64, want64, d1x, d2x;
    double c1, c2, c3, del1, del2, del3, clow, del1st, cprev, omega;
    double ceval;   // point to evaluate next
    double x[11], y[11];
    // group velocity: second search running, its period t1b, the first root
    // (and its secant refinement)
    bool second;
    float t1a, t1b;
    double cph, cph_t;

    __device__ void init(double cc_, float betmx_, int kmax_, double tol_, bool scan32 = false)
    {
        cc = cc_; cm = cc_; betmx = betmx_; kmax = kmax_; tol = tol_;
        sc32 = scan32; p64 = false; want64 = true; d1x = d2x = true;
        dc = fabs((double)0.005f);
        cmax = (double)betmx_ + dc;
        k = 0; phase = START; fail_k = -1; del1st = 0.0; cprev = 0.0; evals = 0;
        second = false; t1a = t1b = 0.0f; cph = 0.0; cph_t = 0.0;
    }

    // Runs the machine until it requests an evaluation (returns true, with
    // ceval/omega set) or finishes (returns false).  Results go through
    // out(k, c, ctight, evals): c is the reference's FP64 root (converged to
    // |c1 - c2| <= tol * c1, surfdisp96.f:608), ctight the secant root inside
    // that final bracket (error O(bracket^2)); both 0 without a root.
    template <class Out>
    __device__ bool next(double F, const double* periods, Out& out)
    {
        for (int guard = 0; guard < 64; ++guard) {
            switch (phase) {
            case START: {
                if (k >= kmax) { phase = DONE; return false; }
                if constexpr (GROUP) {
                    // the first search runs at dble(t1a)
                    group_periods(periods[k], t1a, t1b);
                    second = false;
                    omega = TWOPI / (double)t1a;
                } else {
                    omega = TWOPI / periods[k];
                }
                if (!p64) evals = 0;
                if (k == 0) { c1 = cc; clow = cc; ifirst = true; }
                else { c1 = cprev - 1.5 * dc; clow = cm; ifirst = false; }
                phase = GS_FIRST;
                return request(c1);
            }
            case GS_FIRST: {
                del1 = F;
                d1x = true;
                if (ifirst) del1st = del1;
                const double plmn = fsign1(del1st) * fsign1(del1);
                idir = (ifirst || plmn >= 0.0) ? +1 : -1;
                return scan_next();
            }
            case GS_SCAN: {
                // an FP32 value near zero is re-evaluated in FP64
                if (!want64 && fabs(F) < (double)kScanTrust32) return request(c2);
                del2 = F;
                d2x = want64;
                if (fsign1(del1) != fsign1(del2)) {
                    // bracketed: both end values in FP64 before nevill()
                    if (!d1x) { phase = VER1; return request(c1); }
                    if (!d2x) { phase = VER2; return request(c2); }
                    if constexpr (FAST) { phase = BRENT_INIT; continue; }
                    return begin_nevill();
                }
                c1 = c2;
                del1 = del2;
                d1x = d2x;
                if (c1 < cm || c1 >= cmax) {
                    if (GROUP && second) { group_out(cph, 0.0, out); continue; }
                    fail();
                    return false;
                }
                return scan_next();
            }
            case VER1: {
                if (fsign1(F) != fsign1(del1)) { restart_fp64(); continue; }
                del1 = F;
                d1x = true;
                if (!d2x) { phase = VER2; return request(c2); }
                if constexpr (FAST) { phase = BRENT_INIT; continue; }
                return begin_nevill();
            }
            case VER2: {
                if (fsign1(F) != fsign1(del2)) { restart_fp64(); continue; }
                del2 = F;
                d2x = true;
                if constexpr (FAST) { phase = BRENT_INIT; continue; }
                return begin_nevill();
            }
            case BRENT_INIT: {
                if constexpr (FAST) {
                    // a = c1 (del1), b = c2 (del2): getsol's bracket; c = a
                    c3 = c1; del3 = del1;
                    this->bd = c2 - c1; this->be = this->bd;
                    nctrl = 0;
                    if (brent_iter(out)) return true;
                    if (phase != DONE) continue;
                }
                return false;
            }
            case BRENT: {
                if constexpr (FAST) {
                    del2 = F;
                    if (brent_iter(out)) return true;
                    if (phase != DONE) continue;
                }
                return false;
            }
            case NEV_A:
            case NEV_CD: {
                del3 = F;
                // top of the nevill loop
                nctrl = nctrl + 1;
                if (nctrl >= 100) { if (finish(out)) continue; return false; }
                if (c3 < fmin(c1, c2) || c3 > fmax(c1, c2)) {
                    nev = 0;
                    c3 = 0.5 * (c1 + c2);
                    phase = NEV_B;
                    return request(c3);
                }
                if (update(out)) return true;
                if (phase != DONE) continue;
                return false;
            }
            case NEV_B: {
                del3 = F;
                if (update(out)) return true;
                if (phase != DONE) continue;
                return false;
            }
            case GR_START: {
                // second getsol of a group-velocity period
                omega = TWOPI / (double)t1b;
                ifirst = false;
                clow = 0.0 + 1.0e-2 * dc;
                c1 = cph - 1.5 * dc;
                phase = GS_FIRST;
                return request(c1);
            }
            default:
                return false;
            }
        }
        phase = DONE;   // unreachable for finite input; keeps the loop bounded
        return false;
    }

  private:
    // The secant root inside the final bracket [c1, c2] (c3 when the
    // bracket does not straddle a sign change): error O(bracket^2).  The
    // same step as finish()'s for phase velocity, written out there.
    __device__ double secant_root() const
    {
        const double dd = del2 - del1;
        if (dd != 0.0 && fsign1(del1) != fsign1(del2)) {
            const double s = c1 - del1 * (c2 - c1) / dd;
            if (s >= fmin(c1, c2) && s <= fmax(c1, c2)) return s;
        }
        return c3;
    }

    __device__ bool request(double c)
    {
        ceval = c;
        want64 = true;
        ++evals;
        return true;
    }

    // a scan point: FP32 unless disabled or the period was restarted
    __device__ bool request_scan(double c)
    {
        ceval = c;
        want64 = !(sc32 && !p64);
        ++evals;
        return true;
    }

    __device__ bool begin_nevill()
    {
        // nevill() starts with one halving
        nev = 1; nctrl = 1; mm = 1;
        c3 = 0.5 * (c1 + c2);
        phase = NEV_A;
        return request(c3);
    }

    // An FP32 sign disagreed with FP64 at a verified point: run the period
    // again from its start with every evaluation in FP64 (the reference's
    // sequence of points, hence its root).
    __device__ void restart_fp64()
    {
        p64 = true;
        phase = START;
    }

    __device__ bool scan_next()
    {
        for (int it = 0; it < 4; ++it) {
            c2 = (idir > 0) ? c1 + dc : c1 - dc;
            if (c2 <= clow) { idir = +1; c1 = clow; continue; }
            break;
        }
        phase = GS_SCAN;
        return request_scan(c2);
    }

    __device__ void fail()
    {
        fail_k = k;
        phase = DONE;
    }

    // Group velocity of period k from the roots at t1a (c0) and t1b (c1),
    // surfdisp96.f:293-299, in real*4 without fused operations:
    //   gvel = (1/t1a - 1/t1b) / (1/(t1a*cc0) - 1/(t1b*cc1))
    // then the next period.  cbt: the secant-refined second root, 0 when
    // the second search fell back to c0.
    template <class Out>
    __device__ void group_out(double cb, double cbt, Out& out)
    {
        const float cc0 = __double2float_rn(cph), cc1 = __double2float_rn(cb);
        const float num = __fsub_rn(__fdiv_rn(1.0f, t1a), __fdiv_rn(1.0f, t1b));
        const float den = __fsub_rn(__fdiv_rn(1.0f, __fmul_rn(t1a, cc0)),
                                    __fdiv_rn(1.0f, __fmul_rn(t1b, cc1)));
        const double g = (double)__fdiv_rn(num, den);
        out(k, g, g, evals);
        if constexpr (HasGroupRoots<Out>::value) out.group_roots(k, cph_t, cbt);
        ++k;
        p64 = false;
        second = false;
        phase = START;
    }

    // End of nevill() for this period: getsol's acceptance test, then the
    // next period (or, for group velocity, the second search).  Returns
    // true when the machine should keep running.
    template <class Out>
    __device__ bool finish(Out& out)
    {
        if constexpr (GROUP) {
            if (second) {
                // a root above betmx counts as none found: cb(k) = c(k)
                const bool none = c3 > (double)betmx;
                double cbt = 0.0;
                if constexpr (HasGroupRoots<Out>::value) cbt = none ? 0.0 : secant_root();
                group_out(none ? cph : c3, cbt, out);
                return true;
            }
        }
        if (c3 > (double)betmx) { out(k, 0.0, 0.0, evals); fail(); return false; }
        if constexpr (GROUP) {
            cph = c3;
            if constexpr (HasGroupRoots<Out>::value) cph_t = secant_root();
            cprev = c3;
            second = true;
            phase = GR_START;
            return true;
        }
        // secant root inside the final bracket [c1, c2] (opposite signs)
        double ct = c3;
        const double dd = del2 - del1;
        if (dd != 0.0 && fsign1(del1) != fsign1(del2)) {
            const double s = c1 - del1 * (c2 - c1) / dd;
            if (s >= fmin(c1, c2) && s <= fmax(c1, c2)) ct = s;
        }
        out(k, c3, ct, evals);
        cprev = c3;
        ++k;
        p64 = false;
        phase = START;
        return true;
    }

    // One step of Brent's method on the bracket [b, c] = [c2, c3] with the
    // previous iterate a = c1 (values del2, del3, del1).  Returns true when a
    // new evaluation was requested; otherwise the period finished (phase
    // START) or the model failed (phase DONE).
    template <class Out>
    __device__ bool brent_iter(Out& out)
    {
        double& bd = this->bd;
        double& be = this->be;
        if ((del2 > 0.0) == (del3 > 0.0)) { c3 = c1; del3 = del1; bd = c2 - c1; be = bd; }
        if (fabs(del3) < fabs(del2)) {
            c1 = c2; c2 = c3; c3 = c1;
            del1 = del2; del2 = del3; del3 = del1;
        }
        const double tol1 = 2.0 * 2.220446049250313e-16 * fabs(c2) + 0.5 * kFastRootTol * fabs(c2);
        const double xm = 0.5 * (c3 - c2);
        if (fabs(xm) <= tol1 || del2 == 0.0 || ++nctrl >= 100) {
            // getsol's acceptance test, then the next period
            if (c2 > (double)betmx) { out(k, 0.0, 0.0, evals); fail(); return false; }
            out(k, c2, c2, evals);
            cprev = c2;
            ++k;
            p64 = false;
            phase = START;
            return false;
        }
        if (fabs(be) >= tol1 && fabs(del1) > fabs(del2)) {
            const double sr = del2 / del1;
            double p, q;
            if (c1 == c3) {
                p = 2.0 * xm * sr;
                q = 1.0 - sr;
            } else {
                const double qa = del1 / del3, r = del2 / del3;
                p = sr * (2.0 * xm * qa * (qa - r) - (c2 - c1) * (r - 1.0));
                q = (qa - 1.0) * (r - 1.0) * (sr - 1.0);
            }
            if (p > 0.0) q = -q; else p = -p;
            if (2.0 * p < fmin(3.0 * xm * q - fabs(tol1 * q), fabs(be * q))) { be = bd; bd = p / q; }
            else { bd = xm; be = bd; }
        } else {
            bd = xm; be = bd;
        }
        c1 = c2; del1 = del2;
        c2 += fabs(bd) > tol1 ? bd : (xm > 0.0 ? tol1 : -tol1);
        phase = BRENT;
        return request(c2);
    }

    // Bracket update, convergence test and choice of the next point (the
    // body of the nevill loop after c3 is known).  Returns true when a new
    // evaluation was requested; otherwise the period finished (phase START)
    // or the model failed (phase DONE).
    template <class Out>
    __device__ bool update(Out& out)
    {
        const double s13 = del1 - del3;
        const double s32 = del3 - del2;
        if (fsign1(del3) * fsign1(del1) < 0.0) { c2 = c3; del2 = del3; }
        else { c1 = c3; del1 = del3; }
        if (fabs(c1 - c2) <= tol * c1) { finish(out); return false; }
        if (fsign1(s13) != fsign1(s32)) nev = 0;
        const double ss1 = fabs(del1), s1 = (double)0.01f * ss1;
        const double ss2 = fabs(del2), s2 = (double)0.01f * ss2;
        phase = NEV_CD;
        if (s1 > ss2 || s2 > ss1 || nev == 0) {
            c3 = 0.5 * (c1 + c2);
            nev = 1; mm = 1;
            return request(c3);
        }
        if (nev == 2) { x[mm] = c3; y[mm] = del3; }
        else { x[0] = c1; y[0] = del1; x[1] = c2; y[1] = del2; mm = 1; }
        for (int kk = 1; kk <= mm; ++kk) {
            const int j = mm - kk;
            const double denom = y[mm] - y[j];
            if (fabs(denom) < 1.0e-10 * fabs(y[mm])) {
                c3 = 0.5 * (c1 + c2);
                nev = 1; mm = 1;
                return request(c3);
            }
            x[j] = (-y[j] * x[j + 1] + y[mm] * x[j]) / denom;
        }
        c3 = x[0];
        nev = 2;
        mm = mm + 1;
        if (mm > 10) mm = 10;
        return request(c3);
    }
};

// Scan start of a model, surfdisp96.f:139-206: slowest layer -> gtsolh ->
// backed off by 0.95 * 0.90 in single precision.  Also returns betmx.
template <class LayerF>
__device__ void scan_start(LayerF layerf, int mmax, double& cc, float& betmx)
{
    float betmn = 1.e20f;
    betmx = -1.e20f;
    int jmn = 0;
    bool jsol = true;
    for (int i = 0; i < mmax; ++i) {
        float4 L = layerf(i);
        if (L.z > 0.01f && L.z < betmn) { betmn = L.z; jmn = i; jsol = true; }
        else if (L.z <= 0.01f && L.y < betmn) { betmn = L.y; jmn = i; jsol = false; }
        if (L.z > betmx) betmx = L.z;
    }
    float cc1;
    if (!jsol) cc1 = betmn;
    else { float4 L = layerf(jmn); cc1 = gtsolh(L.y, L.z); }
    cc1 = __fmul_rn(0.95f, cc1);
    cc1 = __fmul_rn(0.90f, cc1);
    cc = (double)cc1;
}

// Drive one model per lane through the whole period list with warp-uniform
// evaluation steps.  All 32 lanes of the warp must call this together;
// inactive lanes pass active = false.  IFUNC 2 is Rayleigh (dltar4), 1 Love
// (dltar1); GROUP selects group velocity.  The FP32 scan applies to
// Rayleigh phase velocity only.  Returns the 0-based first failing period
// or -1.
template <int IFUNC = 2, bool GROUP = false, bool FAST = false, class M, class Out>
__device__ int solve_model_warp(bool active, const M& mdl, int mmax, double cc, float betmx,
                                const double* periods, int kmax, double tol, Out& out,
                                int* total_evals = nullptr, bool scan32 = false)
{
    static_assert(IFUNC == 1 || IFUNC == 2, "ifunc is 1 (Love) or 2 (Rayleigh)");
    constexpr bool kScan32 = M::kF32 && IFUNC == 2 && !GROUP;
    RootSM<GROUP, FAST> sm;
    sm.init(cc, betmx, kmax, tol, kScan32 && scan32);
    bool want = active ? sm.next(0.0, periods, out) : false;
    int tot = want ? 1 : 0;
    while (__any_sync(0xffffffffu, want)) {
        double F = 0.0;
        // one precision per warp step: FP32 only when every waiting lane is
        // on an FP32 scan step; otherwise all evaluate in FP64 (a scan lane
        // then receives an exact value)
        bool step32 = false;
        if constexpr (kScan32) step32 = !__any_sync(0xffffffffu, want && sm.want64);
        if constexpr (kScan32) {
            if (want && step32)
                F = (double)dltar4_f32([&](int m) { return mdl.layerf(m); }, mmax,
                                       (float)(sm.omega / sm.ceval), (float)sm.omega);
        }
        if (want && !step32) {
            if constexpr (IFUNC == 1) F = dltar1(mdl, mmax, sm.omega / sm.ceval, sm.omega);
            else F = dltar4(mdl, mmax, sm.omega / sm.ceval, sm.omega);
            sm.want64 = true;
        }
        if (want) {
            want = sm.next(F, periods, out);
            tot += want ? 1 : 0;
        }
    }
    if (active && sm.fail_k >= 0)
        for (int kk = sm.fail_k; kk < kmax; ++kk) out(kk, 0.0, 0.0, kk == sm.fail_k ? sm.evals : 0);
    if (total_evals) *total_evals = tot;
    return active ? sm.fail_k : -1;
}

}  // namespace dk
