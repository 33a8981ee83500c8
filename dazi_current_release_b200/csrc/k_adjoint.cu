// Adjoint form of the isotropic depth kernel: implicit differentiation of
// the Rayleigh dispersion root.
//
// At a root c of the secular function F(c; m) (dltar4, surfdisp96.f:767-865)
//     dc/dm = -(dF/dm) / (dF/dc),   dF/dc = -(wvno/c) dF/dwvno,
// for every layer parameter m (flattened Vp, Vs, density).  The kernels the
// reference obtains by perturb-and-recompute (DepthKernel1D.f90:102-185,
// sen_X = (c(X+dX/2) - c(X-dX/2))/dX at each depth node) are these
// derivatives chained through the Earth flattening (surfdisp96.f:480-547:
// a_flat = a*tmp, b_flat = b*tmp, rho_flat = rho*btp**-2.275) and the
// sublayer interpolation (CalSurfG.f90:2527-2529: each sublayer value is
// (1-f) v(i) + f v(i+1), f = (2j-1)/(2 nsublay)).
//
// F is a chain of 5x5 compound-matrix products, e(m) = e(m+1) CA_m / n_m from
// the half-space up to the surface, F = e(0)[0].  With the top-down vectors
// g(0) = (1,0,0,0,0), g(m+1) = CA_m g(m) / n_m, F = e(m).g(m) at every m, so
//     dF/dtheta_m = e(m+1) . (dCA_m/dtheta) . g(m) / n_m.
// One thread owns one (column, period):
//   1. bottom-up sweep at the root, storing e(m+1) and 1/n_m per layer in a
//      global scratch block of the thread's warp (6 doubles per layer,
//      [layer][6][lane] so a warp's stores coalesce); the 5x5 matrices are
//      not stored;
//   2. top-down sweep that recomputes CA_m with forward-mode tangents in
//      (Vp_m, Vs_m, wvno) -- density enters each element as a power, so its
//      derivative is read off the values -- and accumulates the node kernels.
// The evanescent layer functions carry factored-out exponentials (var(),
// surfdisp96.f:868-985); the tangents treat those scale factors as constants,
// which differentiates the true secular function times one positive factor
// common to every derivative, so the ratio is exact even slightly off the
// root.  The root itself is the phase-1 root refined by a secant step inside
// the reference's final Neville bracket.
#include "dk_secular.cuh"
#include "dk_fastmath.cuh"
#include "dk_kernels.cuh"

namespace dk {

// ------------------------------------------------------------ tangent type
struct D3 {
    double v, d0, d1, d2;
};
__device__ __forceinline__ D3 mk(double v) { return {v, 0.0, 0.0, 0.0}; }
__device__ __forceinline__ D3 operator+(const D3& a, const D3& b) { return {a.v + b.v, a.d0 + b.d0, a.d1 + b.d1, a.d2 + b.d2}; }
__device__ __forceinline__ D3 operator-(const D3& a, const D3& b) { return {a.v - b.v, a.d0 - b.d0, a.d1 - b.d1, a.d2 - b.d2}; }
__device__ __forceinline__ D3 operator-(const D3& a) { return {-a.v, -a.d0, -a.d1, -a.d2}; }
__device__ __forceinline__ D3 operator*(const D3& a, const D3& b)
{
    return {a.v * b.v, fma(a.v, b.d0, a.d0 * b.v), fma(a.v, b.d1, a.d1 * b.v), fma(a.v, b.d2, a.d2 * b.v)};
}
__device__ __forceinline__ D3 operator*(double s, const D3& a) { return {s * a.v, s * a.d0, s * a.d1, s * a.d2}; }
__device__ __forceinline__ D3 operator*(const D3& a, double s) { return s * a; }
__device__ __forceinline__ D3 operator+(const D3& a, double s) { return {a.v + s, a.d0, a.d1, a.d2}; }
__device__ __forceinline__ D3 operator-(const D3& a, double s) { return {a.v - s, a.d0, a.d1, a.d2}; }
__device__ __forceinline__ D3 operator-(double s, const D3& a) { return {s - a.v, -a.d0, -a.d1, -a.d2}; }
// a / b given ib = 1/b.v
__device__ __forceinline__ D3 div_by(const D3& a, const D3& b, double ib)
{
    const double q = a.v * ib;
    return {q, (a.d0 - q * b.d0) * ib, (a.d1 - q * b.d1) * ib, (a.d2 - q * b.d2) * ib};
}

// Layer functions of var() with tangents.  P (or S) part for one wave type:
// vertical wavenumber r = sqrt(|wvno^2 - xk^2|), phase arg = r*d, and the
// (cos, sin/r, r*sin) triple in oscillatory or scaled-hyperbolic form.
struct WaveD3 {
    D3 r, cosf, sinr, rsin;   // cos, sin/r, r*sin  (x = -r sin in the oscillatory case)
    double scale_exp;         // factored-out exponent (0 when oscillatory)
    double escale;            // exp(-scale_exp) (1 when oscillatory)
    bool evan;
};

__device__ __forceinline__ void wave_d3(const D3& wvno, const D3& xk, double d, WaveD3& o)
{
    const D3 s = wvno + xk;
    const D3 t = wvno - xk;
    const double sg = t.v < 0.0 ? -1.0 : 1.0;
    const D3 prod = s * (sg * t);                 // (wvno + xk) |wvno - xk|
    const double r = fast_sqrt(prod.v);
    const double ir = r > 0.0 ? fast_rcp(r) : 0.0;
    const double h = 0.5 * ir;
    o.r = {r, prod.d0 * h, prod.d1 * h, prod.d2 * h};
    const D3 p = o.r * d;
    if (wvno.v < xk.v) {
        double sp, cp;
        sincos(p.v, &sp, &cp);
        o.evan = false;
        o.scale_exp = 0.0;
        o.escale = 1.0;
        o.cosf = {cp, -sp * p.d0, -sp * p.d1, -sp * p.d2};
        const D3 sn = {sp, cp * p.d0, cp * p.d1, cp * p.d2};
        o.sinr = div_by(sn, o.r, ir);
        o.rsin = -(o.r * sn);                      // x = -r sin(p), z = -r sin(q)
    } else if (wvno.v == xk.v) {
        o.evan = false;
        o.scale_exp = 0.0;
        o.escale = 1.0;
        o.cosf = mk(1.0);
        o.sinr = mk(d);
        o.rsin = mk(0.0);
    } else {
        const double ep = exp(-p.v);
        const double fac = (p.v < 16.0) ? ep * ep : 0.0;
        const double cs = (1.0 + fac) * 0.5, ss = (1.0 - fac) * 0.5;
        o.evan = true;
        o.scale_exp = p.v;
        o.escale = ep;
        // d(cosh) = sinh dp, d(sinh) = cosh dp, with the scale e^-p held
        o.cosf = {cs, ss * p.d0, ss * p.d1, ss * p.d2};
        const D3 sn = {ss, cs * p.d0, cs * p.d1, cs * p.d2};
        o.sinr = div_by(sn, o.r, ir);
        o.rsin = o.r * sn;
    }
}

// The 19 distinct compound-matrix entries (dnka(), surfdisp96.f:1018-1062).
template <class T>
struct CAset {
    T c11, c12, c13, c14, c15, c21, c22, c23, c24, c41, c42, c43, c51, c53, c31, c32, c33, c34, c35;
};

template <class T>
__device__ __forceinline__ void dnka_t(CAset<T>& C, const T& wvno2, const T& gam, const T& gammk,
                                       double rho, double irho, const T& a0, const T& cosp,
                                       const T& w, const T& x, const T& cosq, const T& y,
                                       const T& z)
{
    const T cpcq = cosp * cosq, cpy = cosp * y, cpz = cosp * z;
    const T cqw = cosq * w, cqx = cosq * x;
    const T xy = x * y, xz = x * z, wy = w * y, wz = w * z;
    const T gamm1 = gam - 1.0, twgm1 = gam + gamm1, gmgmk = gam * gammk;
    const T gmgm1 = gam * gamm1, gm1sq = gamm1 * gamm1;
    const double rho2 = rho * rho, r2inv = irho * irho;
    const T a0pq = a0 - cpcq;
    C.c11 = cpcq - 2.0 * gmgm1 * a0pq - gmgmk * xz - wvno2 * gm1sq * wy;
    C.c12 = (wvno2 * cpy - cqx) * irho;
    C.c13 = -(twgm1 * a0pq + gammk * xz + wvno2 * gamm1 * wy) * irho;
    C.c14 = (cpz - wvno2 * cqw) * irho;
    C.c15 = -(2.0 * wvno2 * a0pq + xz + wvno2 * wvno2 * wy) * r2inv;
    C.c21 = (gmgmk * cpz - gm1sq * cqw) * rho;
    C.c22 = cpcq;
    C.c23 = gammk * cpz - gamm1 * cqw;
    C.c24 = -wz;
    C.c41 = (gm1sq * cpy - gmgmk * cqx) * rho;
    C.c42 = -xy;
    C.c43 = gamm1 * cpy - gammk * cqx;
    C.c51 = -(2.0 * gmgmk * gm1sq * a0pq + gmgmk * gmgmk * xz + gm1sq * gm1sq * wy) * rho2;
    C.c53 = -(gammk * gamm1 * twgm1 * a0pq + gam * gammk * gammk * xz + gamm1 * gm1sq * wy) * rho;
    const T tt = -2.0 * wvno2;
    C.c31 = tt * C.c53;
    C.c32 = tt * C.c43;
    C.c33 = a0 + 2.0 * (cpcq - C.c11);
    C.c34 = tt * C.c23;
    C.c35 = tt * C.c13;
}

// Half-space starting vector (dltar4, surfdisp96.f:789-808) with tangents.
__device__ __forceinline__ void halfspace_d3(const D3& wvno, const D3& xka, const D3& xkb,
                                             const D3& gammk, double rho, D3 e[5])
{
    const D3 wvno2 = wvno * wvno;
    const D3 sa = wvno + xka, ta = wvno - xka;
    const D3 pa = sa * ((ta.v < 0.0 ? -1.0 : 1.0) * ta);
    const D3 sb = wvno + xkb, tb = wvno - xkb;
    const D3 pb = sb * ((tb.v < 0.0 ? -1.0 : 1.0) * tb);
    const double ra = fast_sqrt(pa.v), rb = fast_sqrt(pb.v);
    const double ha = ra > 0 ? 0.5 * fast_rcp(ra) : 0.0, hb = rb > 0 ? 0.5 * fast_rcp(rb) : 0.0;
    const D3 Ra = {ra, pa.d0 * ha, pa.d1 * ha, pa.d2 * ha};
    const D3 Rb = {rb, pb.d0 * hb, pb.d1 * hb, pb.d2 * hb};
    const D3 gam = gammk * wvno2;
    const D3 gamm1 = gam - 1.0;
    const D3 rab = Ra * Rb;
    e[0] = (rho * rho) * (gamm1 * gamm1 - gam * gammk * rab);
    e[1] = -rho * Ra;
    e[2] = rho * (gamm1 - gammk * rab);
    e[3] = rho * Rb;
    e[4] = wvno2 - rab;
}

// sum_ij u_i CA_ij v_j for the value and the three tangents, plus the
// density derivative (entries scale as rho^pow).
struct Contract {
    double v, d0, d1, d2, drho;
};

__device__ __forceinline__ void acc_entry(Contract& s, double uv, const D3& c, int pw)
{
    s.v = fma(uv, c.v, s.v);
    s.d0 = fma(uv, c.d0, s.d0);
    s.d1 = fma(uv, c.d1, s.d1);
    s.d2 = fma(uv, c.d2, s.d2);
    if (pw) s.drho = fma(uv * (double)pw, c.v, s.drho);
}

__device__ __forceinline__ Contract contract(const CAset<D3>& C, const double u[5], const double g[5])
{
    Contract s = {0, 0, 0, 0, 0};
    // row 1: c11 c12 c13 c14 c15
    acc_entry(s, u[0] * g[0], C.c11, 0); acc_entry(s, u[0] * g[1], C.c12, -1);
    acc_entry(s, u[0] * g[2], C.c13, -1); acc_entry(s, u[0] * g[3], C.c14, -1);
    acc_entry(s, u[0] * g[4], C.c15, -2);
    // row 2: c21 c22 c23 c24 c14
    acc_entry(s, u[1] * g[0], C.c21, 1); acc_entry(s, u[1] * g[1], C.c22, 0);
    acc_entry(s, u[1] * g[2], C.c23, 0); acc_entry(s, u[1] * g[3], C.c24, 0);
    acc_entry(s, u[1] * g[4], C.c14, -1);
    // row 3: c31 c32 c33 c34 c35
    acc_entry(s, u[2] * g[0], C.c31, 1); acc_entry(s, u[2] * g[1], C.c32, 0);
    acc_entry(s, u[2] * g[2], C.c33, 0); acc_entry(s, u[2] * g[3], C.c34, 0);
    acc_entry(s, u[2] * g[4], C.c35, -1);
    // row 4: c41 c42 c43 c22 c12
    acc_entry(s, u[3] * g[0], C.c41, 1); acc_entry(s, u[3] * g[1], C.c42, 0);
    acc_entry(s, u[3] * g[2], C.c43, 0); acc_entry(s, u[3] * g[3], C.c22, 0);
    acc_entry(s, u[3] * g[4], C.c12, -1);
    // row 5: c51 c41 c53 c21 c11
    acc_entry(s, u[4] * g[0], C.c51, 2); acc_entry(s, u[4] * g[1], C.c41, 1);
    acc_entry(s, u[4] * g[2], C.c53, 1); acc_entry(s, u[4] * g[3], C.c21, 1);
    acc_entry(s, u[4] * g[4], C.c11, 0);
    return s;
}

// g_new = CA g (values only)
__device__ __forceinline__ void matvec(const CAset<D3>& C, const double g[5], double o[5])
{
    o[0] = C.c11.v * g[0] + C.c12.v * g[1] + C.c13.v * g[2] + C.c14.v * g[3] + C.c15.v * g[4];
    o[1] = C.c21.v * g[0] + C.c22.v * g[1] + C.c23.v * g[2] + C.c24.v * g[3] + C.c14.v * g[4];
    o[2] = C.c31.v * g[0] + C.c32.v * g[1] + C.c33.v * g[2] + C.c34.v * g[3] + C.c35.v * g[4];
    o[3] = C.c41.v * g[0] + C.c42.v * g[1] + C.c43.v * g[2] + C.c22.v * g[3] + C.c12.v * g[4];
    o[4] = C.c51.v * g[0] + C.c41.v * g[1] + C.c53.v * g[2] + C.c21.v * g[3] + C.c11.v * g[4];
}

// Build the tangent CA of layer m.  Tangent directions: 0 = Vp_m, 1 = Vs_m,
// 2 = wvno.
__device__ __forceinline__ void layer_ca_d3(const float4& L, double wvno_v, double omega,
                                            CAset<D3>& C)
{
    const double a = (double)L.y, b = (double)L.z, rho = (double)L.w, d = (double)L.x;
    const double ia = fast_rcp(a), ib = fast_rcp(b), iom = fast_rcp(omega);
    const D3 wvno = {wvno_v, 0.0, 0.0, 1.0};
    const double xka_v = omega * ia, xkb_v = omega * ib;
    const D3 xka = {xka_v, -xka_v * ia, 0.0, 0.0};     // d(omega/a)/da
    const D3 xkb = {xkb_v, 0.0, -xkb_v * ib, 0.0};
    const double gk = 2.0 * b * b * (iom * iom);
    const D3 gammk = {gk, 0.0, 2.0 * gk * ib, 0.0};
    const D3 wvno2 = wvno * wvno;
    const D3 gam = gammk * wvno2;
    WaveD3 P, S;
    wave_d3(wvno, xka, d, P);
    wave_d3(wvno, xkb, d, S);
    const double exa = (P.evan ? P.scale_exp : 0.0) + (S.evan ? S.scale_exp : 0.0);
    // exp(-exa) from the waves' own exponentials
    const D3 a0 = mk(exa < 60.0 ? P.escale * S.escale : 0.0);   // the "1" of cosh^2 - sinh^2
    dnka_t(C, wvno2, gam, gammk, rho, fast_rcp(rho), a0, P.cosf, P.sinr, P.rsin, S.cosf, S.sinr, S.rsin);
}

// Value-only layer functions (same expressions as wave_d3 without tangents).
__device__ __forceinline__ void wave_val(double wvno, double xk, double d, double& cosf,
                                         double& sinr, double& rsin, bool& evan, double& sexp,
                                         double& escale)
{
    const double r = fast_sqrt((wvno + xk) * fabs(wvno - xk));
    const double p = r * d;
    if (wvno < xk) {
        double sp, cp;
        sincos(p, &sp, &cp);
        evan = false; sexp = 0.0; escale = 1.0;
        cosf = cp; sinr = sp * fast_rcp(r); rsin = -r * sp;
    } else if (wvno == xk) {
        evan = false; sexp = 0.0; escale = 1.0;
        cosf = 1.0; sinr = d; rsin = 0.0;
    } else {
        const double ep = exp(-p);
        const double fac = (p < 16.0) ? ep * ep : 0.0;
        evan = true; sexp = p; escale = ep;
        cosf = (1.0 + fac) * 0.5;
        const double ss = (1.0 - fac) * 0.5;
        sinr = ss * fast_rcp(r); rsin = r * ss;
    }
}

// One bottom-up step f = e CA_m (values); returns the max-norm of f.
__device__ __forceinline__ double layer_step_val(const float4& L, double wvno, double omega,
                                                 const double e[5], double f[5])
{
    const double a = (double)L.y, b = (double)L.z, rho = (double)L.w, d = (double)L.x;
    const double wvno2 = wvno * wvno;
    const double iom = fast_rcp(omega);
    const double gammk = 2.0 * b * b * (iom * iom);
    const double gam = gammk * wvno2;
    double cp, wp, xp, cq, yq, zq, ep_, eq_, sp_, sq_;
    bool evp, evq;
    wave_val(wvno, omega * fast_rcp(a), d, cp, wp, xp, evp, ep_, sp_);
    wave_val(wvno, omega * fast_rcp(b), d, cq, yq, zq, evq, eq_, sq_);
    const double exa = (evp ? ep_ : 0.0) + (evq ? eq_ : 0.0);
    const double a0 = (exa < 60.0) ? sp_ * sq_ : 0.0;   // exp(-exa)
    CAset<double> C;
    dnka_t(C, wvno2, gam, gammk, rho, fast_rcp(rho), a0, cp, wp, xp, cq, yq, zq);
    f[0] = e[0] * C.c11 + e[1] * C.c21 + e[2] * C.c31 + e[3] * C.c41 + e[4] * C.c51;
    f[1] = e[0] * C.c12 + e[1] * C.c22 + e[2] * C.c32 + e[3] * C.c42 + e[4] * C.c41;
    f[2] = e[0] * C.c13 + e[1] * C.c23 + e[2] * C.c33 + e[3] * C.c43 + e[4] * C.c53;
    f[3] = e[0] * C.c14 + e[1] * C.c24 + e[2] * C.c34 + e[3] * C.c22 + e[4] * C.c21;
    f[4] = e[0] * C.c15 + e[1] * C.c14 + e[2] * C.c35 + e[3] * C.c12 + e[4] * C.c11;
    double t1 = fmax(fmax(fmax(fabs(f[0]), fabs(f[1])), fmax(fabs(f[2]), fabs(f[3]))), fabs(f[4]));
    if (t1 < 1.0e-40) t1 = 1.0;
    return t1;
}

// ---------------------------------------------------------------- kernel
// Warp-level work queue over (tile, period) tasks: a warp takes one task and
// its 32 lanes are the tile's 32 columns at that period.
__device__ __forceinline__ long long next_task(unsigned* queue)
{
    unsigned t = 0;
    if ((threadIdx.x & 31) == 0) t = atomicAdd(queue, 1u);
    return (long long)__shfl_sync(0xffffffffu, t, 0);
}

// Group velocity (igr > 0).  surfdisp96 forms
//     U = (1/t1a - 1/t1b) / (1/(t1a c0) - 1/(t1b c1))
// from the phase roots c0 at t1a and c1 at t1b (surfdisp96.f:226-233,
// 293-299), so with D = 1/t1a - 1/t1b
//     dU/dm = wa dc0/dm + wb dc1/dm,  wa = U^2 / (D t1a c0^2),
//                                     wb = -U^2 / (D t1b c1^2),
// two phase adjoints ("passes") at (t1a, c0) and (t1b, c1).  Where the
// second search found no root (c1 = 0 here) the reference used c0 for c1:
// U = c0 and the derivative is dc0/dm, one pass.  U is differentiated in
// FP64; the reference rounds it to real*4.
struct GroupPasses {
    double per_a, per_b, wa, wb;
    int n;
};

__device__ __forceinline__ GroupPasses group_passes(double t, double c0, double c1)
{
    float t1a, t1b;
    group_periods(t, t1a, t1b);
    GroupPasses g;
    g.per_a = (double)t1a;
    g.per_b = (double)t1b;
    g.wa = 1.0; g.wb = 0.0; g.n = 1;
    if (c1 > 0.0) {
        const double ia = 1.0 / g.per_a, ib = 1.0 / g.per_b;
        const double D = ia - ib;
        const double U = D / (ia / c0 - ib / c1);
        const double u2d = U * U / D;
        g.wa = u2d * ia / (c0 * c0);
        g.wb = -u2d * ib / (c1 * c1);
        g.n = 2;
    }
    return g;
}

// Per-warp adjoint scratch row of layer (or node) m: [row][6][lane].
__device__ __forceinline__ double* scr_row(double* scr, int m)
{
    return scr + (long long)m * 6 * TILE;
}

// Depth cut of the phase-velocity sweep: below a depth where the shear
// waves have decayed by E = sum over the layers above of nu_b d, nu_b =
// sqrt(k^2 - (omega / b)^2) (layers with c < b), the stack's effect on the
// secular function and its partials is of relative order exp(-2 E); the
// first layer with E >= kAdjDepthCut above it is taken as the half-space
// and the ones below are not swept (their partials, of that relative
// order, are written as zero).
constexpr double kAdjDepthCut = 16.0;

// Layers the sweep of one (column, period) covers, the last one taken as
// the half-space: rmax, or m + 1 for the first solid layer m with E >=
// kAdjDepthCut above it.  lay: the column's flat layers (d, a, b, rho), layer
// m at lay[m * TILE].
__device__ __forceinline__ int adj_cut_layers(const float4* lay, int rmax, double omega, double wvno)
{
    const double k2 = wvno * wvno;
    double ex = 0.0;
    for (int m = 0; m < rmax - 1; ++m) {
        const float4 L = lay[(long long)m * TILE];
        if (ex >= kAdjDepthCut && L.z > 0.0f) return m + 1;
        if (L.z > 0.0f) {
            const double kb = omega / (double)L.z;
            const double nb2 = k2 - kb * kb;
            if (nb2 > 0.0) ex += sqrt(nb2) * (double)L.x;
        }
    }
    return rmax;
}

// Sort key of the pair (column lane `lane` of tile t, period k): 0 no such
// pair, 1 no root (the kernels are written as zero), else 1 + the layers
// its sweep covers (adj_cut_layers, at most NL).
__device__ __forceinline__ int adj_pair_key(const AdjArgs& a, long long t, int lane, int k)
{
    const Tables& T = a.T;
    const long long s = t * TILE + lane;
    if (s >= T.ncols) return 0;
    const ColMeta M = T.meta[s];
    if (k >= M.K) return 0;
    const double c0 = a.croot[M.cr_b + (long long)TILE * k];
    if (!(c0 > 0.0)) return 1;
    const double omega = TWOPI / a.periods[M.per_b + k];
    return 1 + adj_cut_layers(T.flat + T.tile_lbase[t] + lane, M.rmax, omega, omega / c0);
}

// The Rayleigh adjoint of one (column, period): lane `lane` of task `task`
// (tile, period), with scr the lane's column of its warp's scratch block;
// phase velocity or (GROUP) the group velocity's two passes.  With a.order
// set (phase velocity), the lane takes the pair a.order lists at its place
// and sweeps the layers its key gives (adj_cut_layers).  The second pass stages its node values in
// scratch rows the top-down sweep has already read (node i is complete only
// once the sweep is past layer i, since every interval holds a sublayer;
// i <= nz - 2 < rmax - 1 rows) and the half-space node in registers, then
// adds them to the first pass's outputs.
template <bool GROUP>
__device__ __forceinline__ void adjoint_rayleigh_task(const AdjArgs& a, long long task, int lane, double* scr)
{
    const Tables& T = a.T;
    constexpr long long nslots = TILE;
    const int2 tk = T.tasks[task];
    // the (column, period) pair: the task's period at column `lane`, or
    // (phase velocity, a.order set) the pair adj_order_kernel placed here
    int cl = lane, k = tk.y, key = 0;
    if (!GROUP && a.order) {
        const int e = a.order[task * TILE + lane];
        key = e >> 16;
        if (key == 0) return;
        cl = e & 31;
        k = (e >> 5) & 0x7ff;
    }
    const long long s = (long long)tk.x * TILE + cl;
    if (s >= T.ncols) return;
    const ColMeta M = T.meta[s];
    if (k >= M.K) return;
    const double c0 = a.croot[M.cr_b + (long long)TILE * k];
    const int nz = M.nz, rmax = M.rmax;
    // layers swept, the last taken as the half-space (adj_cut_layers)
    const int rm = key >= 2 ? key - 1 : rmax;
    double* dvs = a.sen_vs + M.sen_b + T.sen_sk * k;
    double* dvp = a.sen_vp + M.sen_b + T.sen_sk * k;
    double* drh = a.sen_rho + M.sen_b + T.sen_sk * k;
    const long long nstride = M.sen_is;   // node stride in the outputs
    if (!(c0 > 0.0)) {
        for (int i = 0; i < nz; ++i) { dvs[nstride * i] = 0.0; dvp[nstride * i] = 0.0; drh[nstride * i] = 0.0; }
        return;
    }
    double omega = TWOPI / a.periods[M.per_b + k];
    double wvno = omega / c0;
    GroupPasses gp{};
    int npass = 1;
    if constexpr (GROUP) {
        gp = group_passes(a.periods[M.per_b + k], c0, a.croot_b[M.cr_b + (long long)TILE * k]);
        npass = gp.n;
    }
    const long long lbase = T.tile_lbase[tk.x] + cl;
    const float4* lay = T.flat + lbase;            // layer m at lay[m * TILE]
    const ChainRec* chr = T.ch + lbase;
#pragma unroll 1
    for (int pass = 0; pass < npass; ++pass) {
        const bool staged = GROUP && pass > 0;   // second group pass
        double croot = c0;
        if constexpr (GROUP) {
            croot = pass ? a.croot_b[M.cr_b + (long long)TILE * k] : c0;
            omega = TWOPI / (pass ? gp.per_b : gp.per_a);
            wvno = omega / croot;
        }
        auto put = [&](int node, double vs, double vp, double rh) {
            if (staged) {
                double* row = scr_row(scr, node);
                row[0] = vs; row[TILE] = vp; row[2 * TILE] = rh;
            } else {
                dvs[nstride * node] = vs; dvp[nstride * node] = vp; drh[nstride * node] = rh;
            }
        };
        // ---- 1. bottom-up sweep: store e(m+1) and 1/n_m for m = rm-2 .. 0
        double e[5];
        {
            const float4 L = lay[(long long)(rm - 1) * TILE];
            const double aa = L.y, bb = L.z;
            const D3 w = mk(wvno);
            const D3 xka = mk(omega / aa), xkb = mk(omega / bb);
            const D3 gk = mk(2.0 * bb * bb / (omega * omega));
            D3 h[5];
            halfspace_d3(w, xka, xkb, gk, (double)L.w, h);
            for (int q = 0; q < 5; ++q) e[q] = h[q].v;
        }
        for (int m = rm - 2; m >= 0; --m) {
            const float4 L = lay[(long long)m * TILE];
            double f[5];
            const double nrm = layer_step_val(L, wvno, omega, e, f);
            double* sp = scr + (long long)m * 6 * nslots;
            for (int q = 0; q < 5; ++q) sp[q * nslots] = e[q];
            const double inv = fast_rcp(nrm);
            sp[5 * nslots] = inv;
            for (int q = 0; q < 5; ++q) e[q] = f[q] * inv;
        }
        // ---- 2. top-down sweep with tangents
        double gv[5] = {1.0, 0.0, 0.0, 0.0, 0.0};
        double dFdw = 0.0;
        double acc_vs = 0.0, acc_vp = 0.0, acc_rh = 0.0;   // current node (top of interval)
        double nxt_vs = 0.0, nxt_vp = 0.0, nxt_rh = 0.0;   // next node (bottom of interval)
        int cur_node = 0;
        int gexp = 0;   // g is kept as gv * 2^gexp
        for (int m = 0; m <= rm - 2; ++m) {
            const ChainRec ch = chr[(long long)m * TILE];
            const int node = ch.node;
            if (node != cur_node) {
                // interval cur_node finished: node cur_node is complete
                put(cur_node, acc_vs, acc_vp, acc_rh);
                acc_vs = nxt_vs; acc_vp = nxt_vp; acc_rh = nxt_rh;
                nxt_vs = nxt_vp = nxt_rh = 0.0;
                cur_node = node;
            }
            const float4 L = lay[(long long)m * TILE];
            CAset<D3> C;
            layer_ca_d3(L, wvno, omega, C);
            const double* sp = scr + (long long)m * 6 * nslots;
            double u[5];
            for (int q = 0; q < 5; ++q) u[q] = sp[q * nslots];
            const double inv = sp[5 * nslots];
            const Contract sc5 = contract(C, u, gv);
            const double sc = ldexp(inv, gexp);
            dFdw = fma(sc5.d2, sc, dFdw);
            const double dFda = sc5.d0 * sc, dFdb = sc5.d1 * sc, dFdr = sc5.drho * sc * fast_rcp((double)L.w);
            // chain to nodes: a_flat = tmp * ((1-f) vp_i + f vp_i+1), etc.
            const double tmpm = ch.tmp, rf = (double)ch.rhofac;
            const double fw = (double)ch.sub * fast_rcp((double)ch.den);
            acc_vp = fma(dFda * tmpm, 1.0 - fw, acc_vp); nxt_vp = fma(dFda * tmpm, fw, nxt_vp);
            acc_vs = fma(dFdb * tmpm, 1.0 - fw, acc_vs); nxt_vs = fma(dFdb * tmpm, fw, nxt_vs);
            acc_rh = fma(dFdr * rf, 1.0 - fw, acc_rh);   nxt_rh = fma(dFdr * rf, fw, nxt_rh);
            double gn[5];
            matvec(C, gv, gn);
            double mx = 0.0;
            for (int q = 0; q < 5; ++q) { gn[q] *= inv; mx = fmax(mx, fabs(gn[q])); }
            int ex = 0;
            if (mx > 0.0) frexp(mx, &ex);
            for (int q = 0; q < 5; ++q) gv[q] = ldexp(gn[q], -ex);
            gexp += ex;
        }
        // half-space (layer rm - 1).  Without a cut (rm = rmax) its
        // contributions go to node nz-1, together with the bottom sublayers
        // of interval nz-2 already in nxt_*.  With a cut, layer rm - 1 is a
        // sublayer of interval ch.node and is chained to that interval's two
        // nodes as the layers above it are; the nodes below get zero.
        {
            const int m = rm - 1;
            const float4 L = lay[(long long)m * TILE];
            const ChainRec ch = chr[(long long)m * TILE];
            const double aa = L.y, bb = L.z, rho = L.w;
            const D3 w = {wvno, 0.0, 0.0, 1.0};
            const D3 xka = {omega / aa, -omega / (aa * aa), 0.0, 0.0};
            const D3 xkb = {omega / bb, 0.0, -omega / (bb * bb), 0.0};
            const double gkv = 2.0 * bb * bb / (omega * omega);
            const D3 gk = {gkv, 0.0, 2.0 * gkv / bb, 0.0};
            D3 h[5];
            halfspace_d3(w, xka, xkb, gk, rho, h);
            const double sc = ldexp(1.0, gexp);
            double s0 = 0, s1 = 0, s2 = 0, sr = 0;
            const int pw[5] = {2, 1, 1, 1, 0};
            for (int q = 0; q < 5; ++q) {
                s0 = fma(h[q].d0, gv[q], s0);
                s1 = fma(h[q].d1, gv[q], s1);
                s2 = fma(h[q].d2, gv[q], s2);
                sr = fma((double)pw[q] * h[q].v, gv[q], sr);
            }
            dFdw = fma(s2, sc, dFdw);
            const double tmpm = ch.tmp, rf = (double)ch.rhofac;
            if (rm < rmax) {
                if (ch.node != cur_node) {
                    put(cur_node, acc_vs, acc_vp, acc_rh);
                    acc_vs = nxt_vs; acc_vp = nxt_vp; acc_rh = nxt_rh;
                    nxt_vs = nxt_vp = nxt_rh = 0.0;
                    cur_node = ch.node;
                }
                const double fw = (double)ch.sub * fast_rcp((double)ch.den);
                const double dFda = s0 * sc, dFdb = s1 * sc, dFdr = sr * sc / rho;
                acc_vp = fma(dFda * tmpm, 1.0 - fw, acc_vp); nxt_vp = fma(dFda * tmpm, fw, nxt_vp);
                acc_vs = fma(dFdb * tmpm, 1.0 - fw, acc_vs); nxt_vs = fma(dFdb * tmpm, fw, nxt_vs);
                acc_rh = fma(dFdr * rf, 1.0 - fw, acc_rh);   nxt_rh = fma(dFdr * rf, fw, nxt_rh);
                put(cur_node, acc_vs, acc_vp, acc_rh);
                put(cur_node + 1, nxt_vs, nxt_vp, nxt_rh);
                for (int i = cur_node + 2; i < nz; ++i) put(i, 0.0, 0.0, 0.0);
            } else {
                put(cur_node, acc_vs, acc_vp, acc_rh);
                nxt_vp = fma(s0 * sc, tmpm, nxt_vp);
                nxt_vs = fma(s1 * sc, tmpm, nxt_vs);
                nxt_rh = fma(sr * sc / rho, rf, nxt_rh);
                if (!staged) {
                    dvs[nstride * (nz - 1)] = nxt_vs;
                    dvp[nstride * (nz - 1)] = nxt_vp;
                    drh[nstride * (nz - 1)] = nxt_rh;
                }
            }
        }
        // ---- 3. dc/dm = -F_m / F_c = (c / (wvno F_wvno)) F_m
        double scale = croot / (wvno * dFdw);
        if constexpr (GROUP) scale *= pass ? gp.wb : gp.wa;
        if (!staged) {
            for (int i = 0; i < nz; ++i) {
                dvs[nstride * i] *= scale;
                dvp[nstride * i] *= scale;
                drh[nstride * i] *= scale;
            }
        } else {
            for (int i = 0; i < nz - 1; ++i) {
                const double* row = scr_row(scr, i);
                dvs[nstride * i] = fma(scale, row[0], dvs[nstride * i]);
                dvp[nstride * i] = fma(scale, row[TILE], dvp[nstride * i]);
                drh[nstride * i] = fma(scale, row[2 * TILE], drh[nstride * i]);
            }
            dvs[nstride * (nz - 1)] = fma(scale, nxt_vs, dvs[nstride * (nz - 1)]);
            dvp[nstride * (nz - 1)] = fma(scale, nxt_vp, dvp[nstride * (nz - 1)]);
            drh[nstride * (nz - 1)] = fma(scale, nxt_rh, drh[nstride * (nz - 1)]);
        }
    }   // pass
}

// The persistent loop: a warp takes (tile, period) tasks off the queue;
// scr is its lane's column of the warp's scratch block.
template <bool GROUP>
__device__ __forceinline__ void adjoint_rayleigh(const AdjArgs& a)
{
    const long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    double* scr = a.scratch + (slot / TILE) * a.scr_layers * 6 * TILE + lane;
    for (;;) {
        const long long task = next_task(a.queue);
        if (task >= a.T.ntasks) break;
        adjoint_rayleigh_task<GROUP>(a, task, lane, scr);
    }
}

// MINB: minimum resident blocks of 128 threads per SM the register
// allocation aims for (the autotuner picks one of the instantiations).
template <int MINB>
__global__ void __launch_bounds__(128, MINB)
adjoint_kernel(AdjArgs a)
{
    adjoint_rayleigh<false>(a);
}

template <int MINB>
__global__ void __launch_bounds__(128, MINB)
adjoint_group_kernel(AdjArgs a)
{
    adjoint_rayleigh<true>(a);
}

// ------------------------------------------------------------------ Love
// Adjoint form for Love waves (dltar1, surfdisp96.f:704-763).  F is the top
// component of a chain of 2x2 Haskell-Thomson steps from the half-space up:
//     e(m) = e(m+1) M_m / n_m,   M = [[cos q, y/mu], [mu z, cos q]],
// mu = rho b^2, e(rmax-1) = (rho rb, 1/b^2) for the half-space.  With
// g(0) = (1,0), g(m+1) = M_m g(m) / n_m, dF/dtheta_m = e(m+1) dM_m g(m) / n_m
// (and dF/dtheta = (dh/dtheta) . g for the half-space), for theta = the
// layer's flattened Vs and density and the wavenumber.  Vp does not enter:
// its kernel is zero.  Evanescent layers hold their factored-out e^-q as a
// constant, as in the Rayleigh kernel above, which leaves the ratio
// dF/dtheta / dF/dwvno exact.
struct Love3 {
    D3 cosq, m01, m10;   // M00 = M11 = cosq, M01 = y / mu, M10 = mu z
};

// One layer's M with tangents in (b, rho, wvno).
__device__ __forceinline__ void love_layer_d3(double b, double rho, double d, double wvno_v,
                                              double omega, Love3& o)
{
    const double ib = fast_rcp(b);
    const D3 wvno = {wvno_v, 0.0, 0.0, 1.0};
    const double xkb_v = omega * ib;
    const D3 xkb = {xkb_v, -xkb_v * ib, 0.0, 0.0};   // d(omega/b)/db
    const D3 s = wvno + xkb, t = wvno - xkb;
    const D3 prod = s * ((t.v < 0.0 ? -1.0 : 1.0) * t);
    const double r = fast_sqrt(prod.v);
    const double ir = r > 0.0 ? fast_rcp(r) : 0.0;
    const double h = 0.5 * ir;
    const D3 rb = {r, prod.d0 * h, prod.d1 * h, prod.d2 * h};
    const D3 q = rb * d;
    D3 cosq, y, z;
    if (wvno_v < xkb_v) {
        double sq, cq;
        sincos(q.v, &sq, &cq);
        cosq = {cq, -sq * q.d0, -sq * q.d1, -sq * q.d2};
        const D3 sn = {sq, cq * q.d0, cq * q.d1, cq * q.d2};
        y = div_by(sn, rb, ir);
        z = -(rb * sn);
    } else if (wvno_v == xkb_v) {
        cosq = mk(1.0);
        y = mk(d);
        z = mk(0.0);
    } else {
        const double fac = q.v < 16.0 ? exp(-2.0 * q.v) : 0.0;
        const double cs = (1.0 + fac) * 0.5, ss = (1.0 - fac) * 0.5;
        // d(cosh) = sinh dq, d(sinh) = cosh dq under the held scale e^-q
        cosq = {cs, ss * q.d0, ss * q.d1, ss * q.d2};
        const D3 sn = {ss, cs * q.d0, cs * q.d1, cs * q.d2};
        y = div_by(sn, rb, ir);
        z = rb * sn;
    }
    const D3 mu = {rho * b * b, 2.0 * rho * b, b * b, 0.0};
    o.cosq = cosq;
    o.m01 = div_by(y, mu, fast_rcp(mu.v));
    o.m10 = mu * z;
}

// One bottom-up step f = e M (values); returns the max-norm of f (1 below
// 1e-40), as dltar1 normalises.
__device__ __forceinline__ double love_step_val(double b, double rho, double d, double wvno,
                                                double omega, const double e[2], double f[2])
{
    Love3 M;
    love_layer_d3(b, rho, d, wvno, omega, M);
    f[0] = e[0] * M.cosq.v + e[1] * M.m10.v;
    f[1] = e[0] * M.m01.v + e[1] * M.cosq.v;
    double t1 = fmax(fabs(f[0]), fabs(f[1]));
    if (t1 < 1.0e-40) t1 = 1.0;
    return t1;
}

// Half-space vector (rho rb, 1/b^2) with tangents in (b, rho, wvno).
__device__ __forceinline__ void love_halfspace_d3(double b, double rho, double wvno_v, double omega,
                                                  D3 h[2])
{
    const double ib = fast_rcp(b);
    const D3 wvno = {wvno_v, 0.0, 0.0, 1.0};
    const double xkb_v = omega * ib;
    const D3 xkb = {xkb_v, -xkb_v * ib, 0.0, 0.0};
    const D3 s = wvno + xkb, t = wvno - xkb;
    const D3 prod = s * ((t.v < 0.0 ? -1.0 : 1.0) * t);
    const double r = fast_sqrt(prod.v);
    const double hh = r > 0.0 ? 0.5 * fast_rcp(r) : 0.0;
    const D3 rb = {r, prod.d0 * hh, prod.d1 * hh, prod.d2 * hh};
    h[0] = D3{rho, 0.0, 1.0, 0.0} * rb;
    h[1] = {ib * ib, -2.0 * ib * ib * ib, 0.0, 0.0};
}

// The Love adjoint of one (column, period), as adjoint_rayleigh_task: phase
// velocity or (GROUP) the group velocity's two passes, staged likewise.
template <bool GROUP>
__device__ __forceinline__ void adjoint_love_task(const AdjArgs& a, long long task, int lane, double* scr)
{
    const Tables& T = a.T;
    constexpr long long nslots = TILE;   // scratch per warp [layer][3 of 6][lane]
    const int2 tk = T.tasks[task];
    const long long s = (long long)tk.x * TILE + lane;
    const int k = tk.y;
    if (s >= T.ncols) return;
    const ColMeta M = T.meta[s];
    if (k >= M.K) return;
    const double c0 = a.croot[task * TILE + lane];
    const int nz = M.nz, rmax = M.rmax;
    double* dvs = a.sen_vs + M.sen_b + T.sen_sk * k;
    double* dvp = a.sen_vp + M.sen_b + T.sen_sk * k;
    double* drh = a.sen_rho + M.sen_b + T.sen_sk * k;
    const long long nstride = M.sen_is;
    for (int i = 0; i < nz; ++i) dvp[nstride * i] = 0.0;   // Love waves do not see Vp
    if (!(c0 > 0.0)) {
        for (int i = 0; i < nz; ++i) { dvs[nstride * i] = 0.0; drh[nstride * i] = 0.0; }
        return;
    }
    double omega = TWOPI / a.periods[M.per_b + k];
    double wvno = omega / c0;
    GroupPasses gp{};
    int npass = 1;
    if constexpr (GROUP) {
        gp = group_passes(a.periods[M.per_b + k], c0, a.croot_b[task * TILE + lane]);
        npass = gp.n;
    }
    const long long lbase = T.tile_lbase[tk.x] + lane;
    const float4* lay = T.flat + lbase;            // layer m at lay[m * TILE]: (d, a, b, rho)
    const ChainRec* chr = T.ch + lbase;
#pragma unroll 1
    for (int pass = 0; pass < npass; ++pass) {
        const bool staged = GROUP && pass > 0;   // second group pass
        double croot = c0;
        if constexpr (GROUP) {
            croot = pass ? a.croot_b[task * TILE + lane] : c0;
            omega = TWOPI / (pass ? gp.per_b : gp.per_a);
            wvno = omega / croot;
        }
        auto put = [&](int node, double vs, double rh) {
            if (staged) {
                double* row = scr_row(scr, node);
                row[3 * TILE] = vs; row[4 * TILE] = rh;
            } else {
                dvs[nstride * node] = vs; drh[nstride * node] = rh;
            }
        };
        // ---- 1. bottom-up sweep: store e(m+1) and 1/n_m for m = rmax-2 .. 0
        double e[2];
        {
            const float4 L = lay[(long long)(rmax - 1) * TILE];
            D3 h[2];
            love_halfspace_d3((double)L.z, (double)L.w, wvno, omega, h);
            e[0] = h[0].v; e[1] = h[1].v;
        }
        for (int m = rmax - 2; m >= 0; --m) {
            const float4 L = lay[(long long)m * TILE];
            double f[2];
            const double nrm = love_step_val((double)L.z, (double)L.w, (double)L.x, wvno, omega, e, f);
            double* sp = scr + (long long)m * 6 * nslots;
            sp[0] = e[0]; sp[nslots] = e[1];
            const double inv = fast_rcp(nrm);
            sp[2 * nslots] = inv;
            e[0] = f[0] * inv; e[1] = f[1] * inv;
        }
        // ---- 2. top-down sweep with tangents
        double gv[2] = {1.0, 0.0};
        int gexp = 0;                 // g is kept as gv * 2^gexp
        double dFdw = 0.0;
        double acc_vs = 0.0, acc_rh = 0.0, nxt_vs = 0.0, nxt_rh = 0.0;
        int cur_node = 0;
        for (int m = 0; m <= rmax - 2; ++m) {
            const ChainRec ch = chr[(long long)m * TILE];
            const int node = ch.node;
            if (node != cur_node) {
                put(cur_node, acc_vs, acc_rh);
                acc_vs = nxt_vs; acc_rh = nxt_rh;
                nxt_vs = nxt_rh = 0.0;
                cur_node = node;
            }
            const float4 L = lay[(long long)m * TILE];
            Love3 C;
            love_layer_d3((double)L.z, (double)L.w, (double)L.x, wvno, omega, C);
            const double* sp = scr + (long long)m * 6 * nslots;
            const double u0 = sp[0], u1 = sp[nslots], inv = sp[2 * nslots];
            const double sc = ldexp(inv, gexp);
            // u . dM . g,  M = [[c, m01], [m10, c]]
            auto contract = [&](double dc, double d01, double d10) {
                return u0 * (dc * gv[0] + d01 * gv[1]) + u1 * (d10 * gv[0] + dc * gv[1]);
            };
            const double dFdb = contract(C.cosq.d0, C.m01.d0, C.m10.d0) * sc;
            const double dFdr = contract(C.cosq.d1, C.m01.d1, C.m10.d1) * sc;
            dFdw = fma(contract(C.cosq.d2, C.m01.d2, C.m10.d2), sc, dFdw);
            // chain to nodes: b_flat = tmp ((1-f) vs_i + f vs_i+1), rho likewise
            const double tmpm = ch.tmp, rf = (double)ch.rhofac;
            const double fw = (double)ch.sub * fast_rcp((double)ch.den);
            acc_vs = fma(dFdb * tmpm, 1.0 - fw, acc_vs); nxt_vs = fma(dFdb * tmpm, fw, nxt_vs);
            acc_rh = fma(dFdr * rf, 1.0 - fw, acc_rh);   nxt_rh = fma(dFdr * rf, fw, nxt_rh);
            // g <- M g / n, rescaled by a power of two
            double g0 = (C.cosq.v * gv[0] + C.m01.v * gv[1]) * inv;
            double g1 = (C.m10.v * gv[0] + C.cosq.v * gv[1]) * inv;
            const double mx = fmax(fabs(g0), fabs(g1));
            int ex = 0;
            if (mx > 0.0) frexp(mx, &ex);
            gv[0] = ldexp(g0, -ex); gv[1] = ldexp(g1, -ex);
            gexp += ex;
        }
        // half-space: its contributions go to node nz-1
        {
            const int m = rmax - 1;
            const float4 L = lay[(long long)m * TILE];
            const ChainRec ch = chr[(long long)m * TILE];
            D3 h[2];
            love_halfspace_d3((double)L.z, (double)L.w, wvno, omega, h);
            const double sc = ldexp(1.0, gexp);
            const double s0 = (h[0].d0 * gv[0] + h[1].d0 * gv[1]) * sc;
            const double s1 = (h[0].d1 * gv[0] + h[1].d1 * gv[1]) * sc;
            dFdw = fma(h[0].d2 * gv[0] + h[1].d2 * gv[1], sc, dFdw);
            const double tmpm = ch.tmp, rf = (double)ch.rhofac;
            put(cur_node, acc_vs, acc_rh);
            nxt_vs = fma(s0, tmpm, nxt_vs);
            nxt_rh = fma(s1, rf, nxt_rh);
            if (!staged) {
                dvs[nstride * (nz - 1)] = nxt_vs;
                drh[nstride * (nz - 1)] = nxt_rh;
            }
        }
        // ---- 3. dc/dm = -F_m / F_c = (c / (wvno F_wvno)) F_m
        double scale = croot / (wvno * dFdw);
        if constexpr (GROUP) scale *= pass ? gp.wb : gp.wa;
        if (!staged) {
            for (int i = 0; i < nz; ++i) {
                dvs[nstride * i] *= scale;
                drh[nstride * i] *= scale;
            }
        } else {
            for (int i = 0; i < nz - 1; ++i) {
                const double* row = scr_row(scr, i);
                dvs[nstride * i] = fma(scale, row[3 * TILE], dvs[nstride * i]);
                drh[nstride * i] = fma(scale, row[4 * TILE], drh[nstride * i]);
            }
            dvs[nstride * (nz - 1)] = fma(scale, nxt_vs, dvs[nstride * (nz - 1)]);
            drh[nstride * (nz - 1)] = fma(scale, nxt_rh, drh[nstride * (nz - 1)]);
        }
    }   // pass
}

// The persistent loop of the Love adjoint (as adjoint_rayleigh).
template <bool GROUP>
__device__ __forceinline__ void adjoint_love(const AdjArgs& a)
{
    const long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    double* scr = a.scratch + (slot / TILE) * a.scr_layers * 6 * TILE + lane;
    for (;;) {
        const long long task = next_task(a.queue);
        if (task >= a.T.ntasks) break;
        adjoint_love_task<GROUP>(a, task, lane, scr);
    }
}

template <int MINB>
__global__ void __launch_bounds__(128, MINB)
adjoint_love_kernel(AdjArgs a)
{
    adjoint_love<false>(a);
}

template <int MINB>
__global__ void __launch_bounds__(128, MINB)
adjoint_love_group_kernel(AdjArgs a)
{
    adjoint_love<true>(a);
}

template __global__ void adjoint_love_kernel<3>(AdjArgs);
template __global__ void adjoint_love_group_kernel<3>(AdjArgs);
template __global__ void adjoint_group_kernel<3>(AdjArgs);

template __global__ void adjoint_kernel<2>(AdjArgs);
template __global__ void adjoint_kernel<3>(AdjArgs);
template __global__ void adjoint_kernel<4>(AdjArgs);

// One block per tile: every (column, period) pair's key (adj_pair_key),
// then a counting sort of the tile's pairs by key into order, so that the
// 32 lanes of a task sweep to nearly the same depth.  The results do not
// depend on the order: each pair is computed by one lane alone.
__global__ void __launch_bounds__(TI_ORDER_THREADS)
adj_order_kernel(AdjArgs a, int* order, const long long* tile_tbase, const long long* tile_tasks)
{
    __shared__ unsigned short key[NP * TILE];
    __shared__ int hist[NL + 2];
    const long long t = blockIdx.x;
    const int np = (int)tile_tasks[t] * TILE;     // tile_tasks <= NP (checked by the table build)
    for (int i = threadIdx.x; i < NL + 2; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        const int kk = adj_pair_key(a, t, p & 31, p >> 5);
        key[p] = (unsigned short)kk;
        atomicAdd(&hist[kk], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int i = 0; i < NL + 2; ++i) {
            const int h = hist[i];
            hist[i] = run;
            run += h;
        }
    }
    __syncthreads();
    int* out = order + tile_tbase[t] * TILE;
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        const int kk = key[p];
        out[atomicAdd(&hist[kk], 1)] = (kk << 16) | p;
    }
}

}  // namespace dk
