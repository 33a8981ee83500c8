// Device-side model preparation for the depth-kernel stage.
//
// Every single-precision step is written with round-to-nearest intrinsics so
// the compiler cannot fuse a multiply and an add: the layer values the secular
// function sees are then bit-identical to the reference Fortran, which does
// these steps in real*4 arithmetic without FMA.
//
//   brocher       DepthKernel1D.f90:187-200 (depthkernel_empirical_vp_rho)
//   layer split   CalSurfG.f90:2490-2549    (refineGrid2LayerMdl)
//   flattening    surfdisp96.f:480-547      (sphere; density factor
//                 btp**(-2.275) for Rayleigh, ifunc = 2, btp**(-5) for Love)
//
// The layer split and the flattening depend only on the node depths, so they
// form a "geometry" shared by every column with the same depth grid.  The
// velocity-dependent part (a, b, rho per layer) is rebuilt per column and per
// perturbed model.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dk {

constexpr int NL = 200;   // max refined layers (surfdisp96.f:57, NL = 200)
constexpr int NP = 160;   // max periods (surfdisp96.f:59, NP = 160)
constexpr int NZMAX = NL; // max depth nodes (DepthKernel1D.f90:14)

// Per-layer geometry of one depth grid.
struct Geometry {
    int rmax;                // refined layers including the half-space
    int nz;
    int8_t pad[8];
    // per layer (index m = 0 .. rmax-1)
    int16_t node[NL];        // interval i (0-based) the sublayer belongs to; nz-1 for the half-space
    int16_t sub[NL];         // 2*j-1 (odd multiplier of the midpoint interpolation)
    int16_t den[NL];         // 2*nsublay(i)
    int16_t nsub_of_node[NZMAX]; // nsublay per interval (splice bookkeeping)
    float dflat[NL];         // flattened thickness (0 for the half-space)
    float btp[NL];           // flattening velocity factor, stored real*4
    float rhofac[NL];        // btp**(-2.275) in single precision (Rayleigh)
    float rhofac_love[NL];   // btp**(-5) in single precision (Love)
    double tmp[NL];          // flattening velocity factor in double
    float rthk[NL];          // refined thickness before flattening
    // tregn96's own flattening of the TI model (R = 6371 km,
    // tregn96.f:774-841) and its sphericity factors (bldsph, :1301-1383)
    float tdflat[NL];        // flattened thickness (0 for the half-space)
    double f275[NL];         // tmp**(-0.275): moduli A, C, L, N
    double f2275[NL];        // tmp**(-2.275): density
    float vtp[NL];           // partial-derivative velocity factor
};

// ---------------------------------------------------------------- Brocher
__device__ __forceinline__ void brocher(float x, float& vp, float& rho)
{
    float x2 = __fmul_rn(x, x), x3 = __fmul_rn(x2, x), x4 = __fmul_rn(x2, x2);
    float t = __fadd_rn(0.9409f, __fmul_rn(2.0947f, x));
    t = __fsub_rn(t, __fmul_rn(0.8206f, x2));
    t = __fadd_rn(t, __fmul_rn(0.2683f, x3));
    t = __fsub_rn(t, __fmul_rn(0.0251f, x4));
    vp = t;
    float p2 = __fmul_rn(t, t), p3 = __fmul_rn(p2, t), p4 = __fmul_rn(p2, p2);
    float p5 = __fmul_rn(p3, p2);
    float r = __fsub_rn(__fmul_rn(1.6612f, t), __fmul_rn(0.4721f, p2));
    r = __fadd_rn(r, __fmul_rn(0.0671f, p3));
    r = __fsub_rn(r, __fmul_rn(0.0043f, p4));
    r = __fadd_rn(r, __fmul_rn(0.000106f, p5));
    rho = r;
}

// Love-wave density factor btp**(-5), surfdisp96.f:539: an integer power
// of a real*4 value, which gfortran -O3 expands as x^2 * (x^2 * x) and
// inverts with one real*4 division.
__device__ __forceinline__ float love_rhofac(float btp)
{
    const float x2 = __fmul_rn(btp, btp);
    return __fdiv_rn(1.0f, __fmul_rn(__fmul_rn(x2, btp), x2));
}

// Midpoint-interpolated sublayer value, CalSurfG.f90:2527-2529:
//   v(i) + (2j-1)*(v(i+1)-v(i))/(2*nsublay(i))      all real*4
__device__ __forceinline__ float sublayer_value(float vi, float vi1, int sub, int den)
{
    return __fadd_rn(vi, __fdiv_rn(__fmul_rn((float)sub, __fsub_rn(vi1, vi)), (float)den));
}

// Build the geometry of one depth grid (one thread).  Returns rmax, or -1 if
// the refined stack would exceed NL layers.
__device__ inline int build_geometry(Geometry& g, const float* depz, int nz, float minthk0)
{
    int k = 0;
    for (int i = 0; i < nz - 1; ++i) {
        float thk = __fsub_rn(depz[i + 1], depz[i]);
        float minthk = __fdiv_rn(thk, minthk0);
        int ns = (int)__fdiv_rn(__fadd_rn(thk, 1.0e-4f), minthk) + 1;
        g.nsub_of_node[i] = (int16_t)ns;
        if (ns < 1 || k + ns + 1 > NL) { g.rmax = -1; return -1; }
        float newthk = __fdiv_rn(thk, (float)ns);
        for (int j = 1; j <= ns; ++j) {
            g.node[k] = (int16_t)i;
            g.sub[k] = (int16_t)(2 * j - 1);
            g.den[k] = (int16_t)(2 * ns);
            g.rthk[k] = newthk;
            ++k;
        }
    }
    g.node[k] = (int16_t)(nz - 1);
    g.sub[k] = 0;
    g.den[k] = 1;
    g.rthk[k] = 0.0f;
    g.nsub_of_node[nz - 1] = 1;
    const int rmax = k + 1;
    g.rmax = rmax;
    g.nz = nz;
    // sphere(0, ...): flattening of thickness and the velocity factor
    const double ar = 6370.0;
    double dr = 0.0, r0 = ar;
    for (int m = 0; m < rmax; ++m) {
        float dm = (m == rmax - 1) ? 1.0f : g.rthk[m];
        dr = __dadd_rn(dr, (double)dm);
        double r1 = __dsub_rn(ar, dr);
        double z0 = __dmul_rn(ar, log(__ddiv_rn(ar, r0)));
        double z1 = __dmul_rn(ar, log(__ddiv_rn(ar, r1)));
        g.dflat[m] = (m == rmax - 1) ? 0.0f : (float)__dsub_rn(z1, z0);
        double tmp = __ddiv_rn(__dadd_rn(ar, ar), __dadd_rn(r0, r1));
        g.tmp[m] = tmp;
        float btp = (float)tmp;
        g.btp[m] = btp;
        // powf(btp, -2.275f), formed in double and rounded once
        g.rhofac[m] = (float)pow((double)btp, (double)(-2.275f));
        g.rhofac_love[m] = love_rhofac(btp);
        r0 = r1;
    }
    // sphere_tdisp96(): radius 6371 (a real*4 constant), the half-space
    // again entered with thickness 1
    {
        const double ar2 = (double)6371.0f;
        double q0 = ar2;
        for (int m = 0; m < rmax; ++m) {
            const float dm = (m == rmax - 1) ? 1.0f : g.rthk[m];
            const double q1 = __dsub_rn(q0, (double)dm);
            const double z0 = __dmul_rn(ar2, log(__ddiv_rn(ar2, q0)));
            const double z1 = __dmul_rn(ar2, log(__ddiv_rn(ar2, q1)));
            const float td = (float)__dsub_rn(z1, z0);
            g.tdflat[m] = (m == rmax - 1) ? 0.0f : td;
            const double t2 = __ddiv_rn(__dadd_rn(ar2, ar2), __dadd_rn(q0, q1));
            g.f2275[m] = pow(t2, (double)(-2.275f));
            g.f275[m] = pow(t2, (double)(-0.2750f));
            // bldsph() reads the flattened thickness, the half-space as 1
            g.vtp[m] = td;   // temporary: flattened thickness incl. half-space
            q0 = q1;
        }
        const double ar = 6370.0;
        double p0 = ar;
        for (int m = 0; m < rmax; ++m) {
            const double zd = (m == rmax - 1) ? 1.0 : (double)g.vtp[m];
            const double p1 = __dmul_rn(p0, exp(-__ddiv_rn(zd, ar)));
            g.vtp[m] = (float)__ddiv_rn(__dadd_rn(ar, ar), __dadd_rn(p0, p1));
            p0 = p1;
        }
    }
    return rmax;
}

// Flattened layer values (a, b, rho) of layer m given the node values;
// ifunc 1 (Love) or 2 (Rayleigh) selects sphere()'s density factor.
__device__ __forceinline__ float4 flat_layer(const Geometry& g, int m, const float* vp,
                                             const float* vs, const float* rho, int ifunc = 2)
{
    int i = g.node[m];
    float rvp, rvs, rrh;
    if (m == g.rmax - 1) {
        rvp = vp[i]; rvs = vs[i]; rrh = rho[i];
    } else {
        rvp = sublayer_value(vp[i], vp[i + 1], g.sub[m], g.den[m]);
        rvs = sublayer_value(vs[i], vs[i + 1], g.sub[m], g.den[m]);
        rrh = sublayer_value(rho[i], rho[i + 1], g.sub[m], g.den[m]);
    }
    double t = g.tmp[m];
    float4 L;
    L.x = g.dflat[m];
    L.y = (float)__dmul_rn((double)rvp, t);
    L.z = (float)__dmul_rn((double)rvs, t);
    L.w = __fmul_rn(rrh, ifunc == 1 ? g.rhofac_love[m] : g.rhofac[m]);
    return L;
}

// Per-layer constants the secular function needs, precomputed once per model
// so the layer loop has no division by model parameters.
struct LayerD {
    double d;      // flattened thickness
    double ia;     // 1 / Vp
    double ib;     // 1 / Vs
    double b2;     // Vs^2
    double rho;    // density
    double irho;   // 1 / density
};

__device__ __forceinline__ LayerD make_layerd(float4 L)
{
    LayerD o;
    o.d = (double)L.x;
    o.ia = 1.0 / (double)L.y;
    o.ib = 1.0 / (double)L.z;
    o.b2 = (double)L.z * (double)L.z;
    o.rho = (double)L.w;
    o.irho = 1.0 / (double)L.w;
    return o;
}

// gtsolh(), surfdisp96.f:361-382: Rayleigh half-space speed, real*4.
__device__ inline float gtsolh(float a, float b)
{
    float c = __fmul_rn(0.95f, b);
    for (int i = 0; i < 5; ++i) {
        float gamma = __fdiv_rn(b, a);
        float kappa = __fdiv_rn(c, b);
        float k2 = __fmul_rn(kappa, kappa);
        float gk = __fmul_rn(gamma, kappa);
        float gk2 = __fmul_rn(gk, gk);
        float fac1 = __fsqrt_rn(__fsub_rn(1.0f, gk2));
        float fac2 = __fsqrt_rn(__fsub_rn(1.0f, k2));
        float tk = __fsub_rn(2.0f, k2);
        float fr = __fsub_rn(__fmul_rn(tk, tk), __fmul_rn(__fmul_rn(4.0f, fac1), fac2));
        float frp = -__fmul_rn(__fmul_rn(4.0f, tk), kappa);
        frp = __fadd_rn(frp, __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(4.0f, fac2), gamma), gamma), kappa), fac1));
        frp = __fadd_rn(frp, __fdiv_rn(__fmul_rn(__fmul_rn(4.0f, fac1), kappa), fac2));
        frp = __fdiv_rn(frp, b);
        c = __fsub_rn(c, __fdiv_rn(fr, frp));
    }
    return c;
}

}  // namespace dk
