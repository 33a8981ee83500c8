// Gc/Gs (azimuthal anisotropy) depth kernel Lsen_Gsc on the GPU.
//
// Reference: depthkernelTI (code/src_inv_iso_joint/depthkernelTI.f90:86-169)
// turns each column into a transversely isotropic layer stack
// (TA = TC = rho Vp^2, TL = TN = rho Vs^2, TF = TA - 2 TL, Q = 150/50) and
// calls CPS tregn96 (tregn96.f:52-722) with the surfdisp96 phase velocities.
// tregn96 computes the Rayleigh eigenfunctions at that velocity -- a complex
// compound-matrix up-sweep (up, dnka_tregn) combined with a Haskell
// down-sweep (down, hska) -- then the variational partials from layer energy
// integrals (energy, intijr), the attenuation shift of c (gammap) and the
// sphericity factors (sprayl).  The splice then forms, per depth interval j,
//     Lsen_Gsc(j) = sum_{sublayers k of j} dc/dA_k TA_k + dc/dL_k TL_k.
//
// One thread owns one (column, period).  The eigenvalues of an isotropic
// input layer are real (their discriminant is (omega^2 (1/Vs^2 - 1/Vp^2))^2),
// so the up- and down-sweeps run in real arithmetic: an oscillatory layer
// (negative eigenvalue, imaginary vertical wavenumber) maps onto cos/sin
// forms exactly as tregn96's complex varsv evaluates them.  Only the energy
// integrals, where the eigenvector matrices carry imaginary wavenumbers,
// use complex arithmetic.  The up-sweep's compound vectors go to a global
// scratch slot per thread ([layer][slot], coalesced); the down-sweep builds
// eigenfunctions and energy integrals interface by interface and stores the
// raw partials in the same slots for the final normalised splice.
#include <utility>

#include "dk_secular.cuh"
#include "dk_fastmath.cuh"
#include "dk_kernels.cuh"

namespace dk {

// Divisions and square roots use dk_fastmath.cuh (the sweep is held to 1e-5
// of the oracle, not to bit parity).

// Depth cut of the Gc/Gs sweep: the accumulated vertical decay exponent
// (sum of nu d from the surface) at which a layer is taken as the
// half-space.  Against the full sweep, on 400 columns of the uneven
// workload (host build): per-column rel-L2 of Lsen_Gsc 5e-11 at 16
// (2.6e-19 at 25, 3.9e-8 at 12), i.e. far below the real*4 output's
// resolution, while 18 % of the layer items are left out.
constexpr double kTiDepthCut = 16.0;

// ------------------------------------------------------------ complex
struct zc { double re, im; };
__device__ __forceinline__ zc Z(double r, double i = 0.0) { return {r, i}; }
__device__ __forceinline__ zc operator+(zc a, zc b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ zc operator-(zc a, zc b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ zc operator-(zc a) { return {-a.re, -a.im}; }
__device__ __forceinline__ zc operator*(zc a, zc b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ zc operator*(double s, zc a) { return {s * a.re, s * a.im}; }
// |b|^2 of the layer quantities here (wavenumbers, eigenvalues, their
// products) stays far inside the double range, so a / b is formed as
// a conj(b) / |b|^2 without rescaling, and |z| is compared through |z|^2.
__device__ __forceinline__ double znorm2(zc a) { return a.re * a.re + a.im * a.im; }
__device__ __forceinline__ zc zdiv(zc a, zc b)
{
    const double in = fast_rcp(znorm2(b));
    return {(a.re * b.re + a.im * b.im) * in, (a.im * b.re - a.re * b.im) * in};
}
__device__ __forceinline__ zc zsqrt(zc a)
{
    // principal square root (branch cut on the negative real axis)
    const double m = fast_sqrt(znorm2(a));
    double re = fast_sqrt(0.5 * (m + fabs(a.re)));
    if (re == 0.0) return Z(0.0, 0.0);
    double im = a.im * fast_rcp(2.0 * re);
    if (a.re < 0.0) { const double t = fabs(im); im = copysign(re, a.im); re = t; }
    return {re, im};
}
__device__ __forceinline__ zc zexp(zc a)
{
    double s, c;
    sincos(a.im, &s, &c);
    const double e = exp(a.re);
    return {e * c, e * s};
}

// ------------------------------------------------------- TI layer model
// A layer as tregn96 holds it: TiRec (dk_table.cuh) with TC = TA, TN = TL
// (depthkernelTI.f90:124-131), plus the period-independent combinations,
// formed from the stored record where the layer is read (the compiler keeps
// only those a call site uses).
struct TiLayer {
    double TA, TL, rho, TF;
    double iTA, iTL;          // 1 / TC, 1 / TL           (TC = TA)
    double TFoTA, TAF;        // TF / TC, TA - TF^2 / TC
    double rhoTA, rhoTL;      // rho / TC, rho / TL
    double ah, bv;            // sqrt(TA / rho) (= av), sqrt(TL / rho) (= bh)
    double eta, ieta;         // TF / (TA - 2 TL), its reciprocal
    double td;                // flattened thickness (0 for the half-space)
};

__device__ __forceinline__ TiLayer ti_layer(const TiRec* p)
{
    const TiRec r = *p;
    TiLayer L;
    L.TA = r.TA; L.TL = r.TL; L.rho = r.rho; L.TF = r.TF; L.td = r.td;
    L.iTA = fast_rcp(r.TA);
    L.iTL = fast_rcp(r.TL);
    const double irho = fast_rcp(r.rho);
    L.TFoTA = r.TF * L.iTA;
    L.TAF = r.TA - r.TF * L.TFoTA;
    L.rhoTA = r.rho * L.iTA;
    L.rhoTL = r.rho * L.iTL;
    L.ah = fast_sqrt(r.TA * irho);
    L.bv = fast_sqrt(r.TL * irho);
    L.eta = r.TF * fast_rcp(r.TA - 2.0 * r.TL);
    L.ieta = fast_rcp(L.eta);
    return L;
}

// gettiegn() (tregn96.f:3166-3361) for real eigenvalues.  rp/rsv are the
// vertical wavenumbers: a non-negative real value, or (osc = true) the
// magnitude of an imaginary one.
struct TiEig {
    double x11, x21, x31, x41, x12, x22, x32, x42, np, nsv;
    double rp, rsv;
    bool oscp, oscs;
    bool ok;
};

// The same with complex eigenvectors and wavenumbers (general case).
struct TiEigZ {
    zc x11, x21, x31, x41, x12, x22, x32, x42, np, nsv, rp, rsv;
};

__device__ __forceinline__ void ti_eigen(const TiLayer& L, double omg, double wvn, double wvno2, TiEig& o)
{
    const double om2 = omg * omg;
    const double wvn2 = wvn * wvn;
    const double a = wvn * L.TFoTA, b = L.iTA;
    const double c = -L.rho * om2 + wvn2 * L.TAF;
    const double d = -wvn, e = L.iTL, f = -L.rho * om2;
    const double ddef = wvn2 - om2 * L.rhoTL;
    const double aabc = wvn2 - om2 * L.rhoTA;
    const double bb = 2.0 * a * d + e * c + f * b;
    const double cc = ddef * aabc;
    const double disc = bb * bb - 4.0 * cc;
    o.ok = disc >= 0.0;
    const double srt = fast_sqrt(fmax(disc, 0.0));
    double L1 = 0.5 * (bb + srt);
    double L2 = fabs(L1) > 0.0 ? cc * fast_rcp(L1) : 0.5 * (bb - srt);
    if (fabs(wvno2 - L2) < fabs(wvno2 - L1)) { const double t = L1; L1 = L2; L2 = t; }
    o.oscp = L1 < 0.0;
    o.oscs = L2 < 0.0;
    o.rp = fast_sqrt(fabs(L1));
    o.rsv = fast_sqrt(fabs(L2));
    const double bcaa = b * c + a * a, ddef2 = d * d + e * f;
    double x12 = b * d - a * e;
    double x22 = b * L2 - e * bcaa;
    double x32 = L2 - (a * d + c * e);
    double x42 = -a * L2 + d * bcaa;
    double x11 = -e * L1 + b * ddef2;
    double x21 = b * d - a * e;
    double x31 = d * L1 - a * ddef2;
    double x41 = -(L1 - a * d - b * f);
    if (wvn != 0.0) {
        const double z1 = wvn * fast_rcp(x11);
        x11 *= z1; x21 *= z1; x31 *= z1; x41 *= z1;
        const double z2 = wvn * fast_rcp(x22);
        x12 *= z2; x22 *= z2; x32 *= z2; x42 *= z2;
    }
    o.x11 = x11; o.x21 = x21; o.x31 = x31; o.x41 = x41;
    o.x12 = x12; o.x22 = x22; o.x32 = x32; o.x42 = x42;
    o.np = x11 * x41 - x21 * x31;
    o.nsv = x12 * x42 - x22 * x32;
}

// varsv() (tregn96.f:3363-3475) on the real representation.
struct TiVar {
    double cosp, rsinp, sinpr, cosq, rsinq, sinqr, pex, svex;
};

__device__ __forceinline__ void ti_var_one(double r, bool osc, double dm, double& cosf,
                                           double& rsin, double& sinr, double& ex)
{
    if (!osc) {
        const double pr = r * dm;
        ex = pr;
        const double fac = pr < 15.0 ? exp(-2.0 * pr) : 0.0;
        cosf = 0.5 * (1.0 + fac);
        const double sn = 0.5 * (1.0 - fac);
        rsin = r * sn;
        sinr = (fabs(pr) < 1.0e-5 && r < 1.0e-5) ? dm : sn * fast_rcp(r);
    } else {
        const double pi = r * dm;
        ex = 0.0;
        double sn, cs;
        sincos(pi, &sn, &cs);
        cosf = cs;
        rsin = -r * sn;                               // (i r)(i sin)
        sinr = (r < 1.0e-5) ? dm : sn * fast_rcp(r);    // (i sin)/(i r)
    }
}

// Compound-matrix element tables of dnka_tregn (tregn96.f:1992-2987): each
// needed element tca(I,J) is a signed sum of x(a,k)x(b,k) x(c,l)x(d,l) times
// trig factors of modes k and l (f: 0 = cos, 1 = sin/r, 2 = r sin,
// 3 = the exact same-mode value 4 a_k^2 exp(-ex)), in two groups subtracted.
struct TT { signed char sg, a, b, k, c, d, l, fk, fl, grp; };
// All terms, element after element: terms kTTo[q] .. kTTo[q+1]-1 form the
// q-th needed element, in the order t11 t12 t13 t15 t16 t21 t22 t23 t25 t31
// t32 t33 t51 t52 t61.
constexpr TT kTT[72] = {
    // tca(1,1)
    {-1,1,3,1,2,4,1,3,3,0}, {-1,1,4,1,2,3,2,0,0,0}, {-1,1,4,2,2,3,1,0,0,0}, {+1,1,3,1,2,4,2,1,1,0}, {+1,1,3,2,2,4,1,2,2,0}, {-1,1,3,2,2,4,2,3,3,0},
    // tca(1,2)
    {-1,1,4,1,2,2,2,0,1,0}, {-1,1,4,2,2,2,1,0,2,0}, {-1,1,2,1,2,4,2,0,1,1}, {-1,1,2,2,2,4,1,0,2,1},
    // tca(1,3)
    {+1,1,4,1,2,1,1,3,3,0}, {+1,1,4,1,1,2,2,0,0,0}, {+1,1,4,2,2,1,1,0,0,0}, {-1,1,1,1,2,4,2,1,1,0}, {-1,1,1,2,2,4,1,2,2,0}, {+1,1,4,2,1,2,2,3,3,0},
    // tca(1,5)
    {-1,1,3,1,1,2,2,1,0,0}, {-1,1,3,2,2,1,1,2,0,0}, {-1,1,1,1,2,3,2,1,0,1}, {-1,1,1,2,2,3,1,2,0,1},
    // tca(1,6)
    {-1,1,2,1,1,2,2,0,0,0}, {-1,1,2,2,2,1,1,0,0,0}, {+1,1,1,1,2,2,2,1,1,0}, {+1,1,1,2,2,2,1,2,2,0}, {-1,1,2,1,2,1,1,3,3,0}, {-1,1,2,2,1,2,2,3,3,0},
    // tca(2,1)
    {-1,1,4,1,3,3,2,0,2,0}, {-1,1,4,2,3,3,1,0,1,0}, {-1,1,3,1,3,4,2,1,0,1}, {-1,1,3,2,3,4,1,2,0,1},
    // tca(2,2)
    {-1,1,4,1,3,2,2,0,0,0}, {+1,1,2,1,3,4,2,0,0,0}, {-1,1,4,2,3,2,1,0,0,0}, {+1,1,2,2,3,4,1,0,0,0},
    // tca(2,3)
    {+1,1,4,1,3,1,2,0,2,0}, {+1,1,4,2,3,1,1,0,1,0}, {+1,1,1,1,3,4,2,1,0,1}, {+1,1,1,2,3,4,1,2,0,1},
    // tca(2,5)
    {-1,1,3,1,3,1,2,1,2,0}, {-1,1,3,2,3,1,1,2,1,0}, {-1,1,1,1,3,3,2,1,2,1}, {-1,1,1,2,3,3,1,2,1,1},
    // tca(3,1)
    {-1,1,4,1,4,3,2,0,0,0}, {-1,1,4,2,4,3,1,0,0,0}, {+1,1,3,2,4,4,1,2,2,0}, {+1,1,3,1,4,4,2,1,1,0}, {-1,1,4,1,4,3,1,3,3,0}, {-1,1,4,2,4,3,2,3,3,0},
    // tca(3,2)
    {-1,1,4,1,4,2,2,0,1,0}, {-1,1,4,2,4,2,1,0,2,0}, {-1,1,2,1,4,4,2,0,1,1}, {-1,1,2,2,4,4,1,0,2,1},
    // tca(3,3)
    {+1,1,4,1,4,1,2,0,0,0}, {+1,1,4,2,4,1,1,0,0,0}, {-1,1,1,1,4,4,2,1,1,0}, {-1,1,1,2,4,4,1,2,2,0}, {+1,1,4,1,4,1,1,3,3,0}, {+1,1,4,2,4,1,2,3,3,0},
    // tca(5,1)
    {-1,2,4,1,4,3,2,2,0,0}, {-1,2,4,2,4,3,1,1,0,0}, {-1,2,3,1,4,4,2,0,1,1}, {-1,2,3,2,4,4,1,0,2,1},
    // tca(5,2)
    {-1,2,4,1,4,2,2,2,1,0}, {-1,2,4,2,4,2,1,1,2,0}, {+1,2,2,1,4,4,2,2,1,0}, {+1,2,2,2,4,4,1,1,2,0},
    // tca(6,1)
    {-1,3,4,1,4,3,2,0,0,0}, {-1,3,4,2,4,3,1,0,0,0}, {+1,3,3,1,4,4,2,1,1,0}, {+1,3,3,2,4,4,1,2,2,0}, {-1,3,4,1,4,3,1,3,3,0}, {-1,3,4,2,4,3,2,3,3,0},
};
constexpr int kTTo[16] = {0, 6, 10, 16, 20, 26, 30, 34, 38, 42, 48, 52, 58, 62, 66, 72};

// One term with compile-time indices (registers only).
template <int I, class T, class F>
__device__ __forceinline__ T tca_term(const T (&xs)[5][3], const F (&fac)[3][4])
{
    constexpr TT t = kTT[I];
    T v = (xs[t.a][t.k] * xs[t.b][t.k]) * (xs[t.c][t.l] * xs[t.d][t.l]);
    if constexpr (t.sg < 0) v = -v;
    if constexpr (t.fk == 3) return v * fac[t.k][3];
    else return (v * fac[t.k][t.fk]) * fac[t.l][t.fl];
}

template <class T, class F, int... Is>
__device__ __forceinline__ T tca_expand(const T (&xs)[5][3], const F (&fac)[3][4],
                                        std::integer_sequence<int, Is...>)
{
    T g0{}, g1{};
    ((kTT[Is].grp ? (g1 = g1 + tca_term<Is>(xs, fac)) : (g0 = g0 + tca_term<Is>(xs, fac))), ...);
    return g0 - g1;
}

template <int LO, class S> struct Shift;
template <int LO, int... Is>
struct Shift<LO, std::integer_sequence<int, Is...>> {
    using type = std::integer_sequence<int, (LO + Is)...>;
};

template <int Q, class T, class F>
__device__ __forceinline__ T tca_elem(const T (&xs)[5][3], const F (&fac)[3][4])
{
    using S = typename Shift<kTTo[Q], std::make_integer_sequence<int, kTTo[Q + 1] - kTTo[Q]>>::type;
    return tca_expand(xs, fac, S{});
}

// The up-sweep step with the real compound matrix: ee = cdv * CA, each
// tca element folded into ee as soon as it is formed (CA is never held):
//   CA rows  (t11 t12 t13 t15 t16) (t21 t22 t23 t25 t15)
//            (2t31 2t32 2t33-dfac -2t23 -2t13) (t51 t52 -t32 t22 t12)
//            (t61 t51 -t31 t21 t11)
__device__ __forceinline__ void ti_compound_apply(const TiEig& E, const TiVar& v, const double c[5],
                                                  double ee[5])
{
    const double ex = v.pex + v.svex;
    const double dfac = ex > 35.0 ? 0.0 : exp(-ex);
    const double a1 = 0.5 * fast_rcp(E.np), a2 = 0.5 * fast_rcp(E.nsv);
    double fac[3][4];
    fac[1][0] = 2.0 * a1 * v.cosp; fac[1][1] = 2.0 * a1 * v.sinpr; fac[1][2] = 2.0 * a1 * v.rsinp;
    fac[1][3] = 4.0 * a1 * a1 * dfac;
    fac[2][0] = 2.0 * a2 * v.cosq; fac[2][1] = 2.0 * a2 * v.sinqr; fac[2][2] = 2.0 * a2 * v.rsinq;
    fac[2][3] = 4.0 * a2 * a2 * dfac;
    double xs[5][3];
    xs[1][1] = E.x11; xs[2][1] = E.x21; xs[3][1] = E.x31; xs[4][1] = E.x41;
    xs[1][2] = E.x12; xs[2][2] = E.x22; xs[3][2] = E.x32; xs[4][2] = E.x42;
    const double c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3], c4 = c[4];
    const double c2x2 = 2.0 * c2;
    double e0, e1, e2, e3, e4;
    {   const double t = tca_elem<0>(xs, fac);  e0 = c0 * t;  e4 = c4 * t; }           // t11
    {   const double t = tca_elem<1>(xs, fac);  e1 = c0 * t;  e4 += c3 * t; }          // t12
    {   const double t = tca_elem<2>(xs, fac);  e2 = c0 * t;  e4 -= c2x2 * t; }        // t13
    {   const double t = tca_elem<3>(xs, fac);  e3 = c0 * t;  e4 += c1 * t; }          // t15
    {   const double t = tca_elem<4>(xs, fac);  e4 += c0 * t; }                         // t16
    {   const double t = tca_elem<5>(xs, fac);  e0 += c1 * t; e3 += c4 * t; }          // t21
    {   const double t = tca_elem<6>(xs, fac);  e1 += c1 * t; e3 += c3 * t; }          // t22
    {   const double t = tca_elem<7>(xs, fac);  e2 += c1 * t; e3 -= c2x2 * t; }        // t23
    {   const double t = tca_elem<8>(xs, fac);  e3 += c1 * t; }                         // t25
    {   const double t = tca_elem<9>(xs, fac);  e0 += c2x2 * t; e2 -= c4 * t; }        // t31
    {   const double t = tca_elem<10>(xs, fac); e1 += c2x2 * t; e2 -= c3 * t; }        // t32
    {   const double t = tca_elem<11>(xs, fac); e2 += c2 * (2.0 * t - dfac); }          // t33
    {   const double t = tca_elem<12>(xs, fac); e0 += c3 * t; e1 += c4 * t; }          // t51
    {   const double t = tca_elem<13>(xs, fac); e1 += c3 * t; }                         // t52
    {   const double t = tca_elem<14>(xs, fac); e0 += c4 * t; }                         // t61
    ee[0] = e0; ee[1] = e1; ee[2] = e2; ee[3] = e3; ee[4] = e4;
}

// E and E^-1 of a layer (evalg, tregn96.f:3055-3105) as complex matrices.
__device__ __forceinline__ void ti_emat(const TiEigZ& E, zc e[4][4], zc ei[4][4])
{
    const zc rp = E.rp, rsv = E.rsv;
    const zc x11 = E.x11, x21 = E.x21, x31 = E.x31, x41 = E.x41;
    const zc x12 = E.x12, x22 = E.x22, x32 = E.x32, x42 = E.x42;
    const zc d1 = (2.0 * rp) * E.np, d2 = (2.0 * rsv) * E.nsv;
    const zc i1 = zdiv(Z(1.0), d1), i2 = zdiv(Z(1.0), d2);   // 1/(2 rp NP), 1/(2 rsv NSV)
    ei[0][0] = (x41 * rp) * i1;    ei[1][0] = x42 * i2;
    ei[2][0] = (x41 * rp) * i1;    ei[3][0] = -(x42 * i2);
    ei[0][1] = -(x31 * i1);        ei[1][1] = -((x32 * rsv) * i2);
    ei[2][1] = x31 * i1;           ei[3][1] = -((x32 * rsv) * i2);
    ei[0][2] = -((x21 * rp) * i1); ei[1][2] = -(x22 * i2);
    ei[2][2] = -((x21 * rp) * i1); ei[3][2] = x22 * i2;
    ei[0][3] = x11 * i1;           ei[1][3] = (x12 * rsv) * i2;
    ei[2][3] = -(x11 * i1);        ei[3][3] = (x12 * rsv) * i2;
    e[0][0] = x11; e[1][0] = x21 * rp; e[2][0] = x31; e[3][0] = x41 * rp;
    e[0][1] = x12 * rsv; e[1][1] = x22; e[2][1] = x32 * rsv; e[3][1] = x42;
    e[0][2] = x11; e[1][2] = -(x21 * rp); e[2][2] = x31; e[3][2] = -(x41 * rp);
    e[0][3] = -(x12 * rsv); e[1][3] = x22; e[2][3] = -(x32 * rsv); e[3][3] = x42;
}

// The six energy integrals of a layer (intijr, tregn96.f:4073-4245):
// (1,1) (1,3) (2,2) (2,4) (3,3) (4,4).  top/bot = (ur, uz, tz, tr) at the
// layer's top and bottom interface; half = the lower half-space.  fg holds
// the layer's ffunc/gfunc/h1func/h2func values (FA, GA, FB, GB, H1, H2).
__device__ __forceinline__ void ti_integrals_z(const TiEigZ& E, const zc fg[6], const double top[4],
                                               const double bot[4], bool half, double out[6])
{
    zc e[4][4], ei[4][4];
    ti_emat(E, e, ei);
    const zc ra = E.rp, rb = E.rsv;
    auto pot = [&](int r, const double u[4]) {
        return (u[0] * ei[r][0] + u[1] * ei[r][1]) + (u[2] * ei[r][2] + u[3] * ei[r][3]);
    };
    const zc km1pd = pot(2, top), km1sd = pot(3, top);
    constexpr int IJ[6][2] = {{0, 0}, {0, 2}, {1, 1}, {1, 3}, {2, 2}, {3, 3}};
    if (!half) {
        const zc kmpu = pot(0, bot), kmsu = pot(1, bot);
        const zc FA = fg[0], GA = fg[1], FB = fg[2], GB = fg[3], H1 = fg[4], H2 = fg[5];
        const zc pu2 = kmpu * kmpu, pd2 = km1pd * km1pd, su2 = kmsu * kmsu, sd2 = km1sd * km1sd;
        const zc pusu = kmpu * kmsu, pdsd = km1pd * km1sd, pusd = kmpu * km1sd, pdsu = km1pd * kmsu;
        const zc pupd = kmpu * km1pd, susd = kmsu * km1sd;
        // (potential product) x (ffunc/gfunc/h1func/h2func) once per layer;
        // each integral then needs only the real part of EE x W
        const zc W1 = pu2 * FA, W2 = pd2 * FA, W3 = su2 * FB, W4 = sd2 * FB;
        const zc W5 = pusu * H1, W6 = pdsd * H1, W7 = pusd * H2, W8 = pdsu * H2;
        const zc W9 = pupd * GA, W10 = susd * GB;
        auto re_mul = [](zc a, zc b) { return a.re * b.re - a.im * b.im; };
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const int i = IJ[q][0], j = IJ[q][1];
            auto EE = [&](int a, int b) { return e[i][a] * e[j][b]; };
            auto SY = [&](int a, int b) { return EE(a, b) + EE(b, a); };
            double r = re_mul(EE(0, 0), W1) + re_mul(EE(2, 2), W2);
            r += re_mul(EE(1, 1), W3) + re_mul(EE(3, 3), W4);
            r += re_mul(SY(0, 1), W5) + re_mul(SY(2, 3), W6);
            r += re_mul(SY(0, 3), W7) + re_mul(SY(1, 2), W8);
            r += re_mul(SY(0, 2), W9) + re_mul(SY(1, 3), W10);
            out[q] = r;
        }
    } else {
        const zc pd2 = km1pd * km1pd, sd2 = km1sd * km1sd, pdsd = km1pd * km1sd;
        const zc i2a = zdiv(Z(1.0), 2.0 * ra), iab = zdiv(Z(1.0), ra + rb), i2b = zdiv(Z(1.0), 2.0 * rb);
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const int i = IJ[q][0], j = IJ[q][1];
            auto EE = [&](int a, int b) { return e[i][a] * e[j][b]; };
            zc r = (EE(2, 2) * pd2) * i2a;
            r = r + ((EE(2, 3) + EE(3, 2)) * pdsd) * iab;
            r = r + (EE(3, 3) * sd2) * i2b;
            out[q] = r.re;
        }
    }
}

// One wave of a layer with a real eigenvalue: varsv's quantities
// (tregn96.f:3363-3475) and ea = exp(-nu d), the one transcendental that
// ffunc/gfunc/h1func/h2func also need (real nu = r: exp(-r d); imaginary
// nu = i r: cos(r d) - i sin(r d)).  exp(-2 nu d) is formed as ea^2 and
// exp(-(nu_a + nu_b) d) as ea eb, with the reference's cut-offs.
struct TiWave {
    double cosf, rsin, sinr, ex;
    double er, ei;
};

__device__ __forceinline__ TiWave ti_wave(double r, bool osc, double dm)
{
    TiWave w;
    if (!osc) {
        const double pr = r * dm;
        w.ex = pr;
        const double e1 = exp(-pr);
        const double fac = pr < 15.0 ? e1 * e1 : 0.0;
        w.cosf = 0.5 * (1.0 + fac);
        const double sn = 0.5 * (1.0 - fac);
        w.rsin = r * sn;
        w.sinr = (fabs(pr) < 1.0e-5 && r < 1.0e-5) ? dm : sn * fast_rcp(r);
        w.er = e1;
        w.ei = 0.0;
    } else {
        const double pi = r * dm;
        w.ex = 0.0;
        double sn, cs;
        sincos(pi, &sn, &cs);
        w.cosf = cs;
        w.rsin = -r * sn;                             // (i r)(i sin)
        w.sinr = (r < 1.0e-5) ? dm : sn * fast_rcp(r);  // (i sin)/(i r)
        w.er = cs;
        w.ei = -sn;
    }
    return w;
}

// ----------------------------------------------------- complex layer path
// A layer whose TI eigenvalues form a complex-conjugate pair (deep layers
// at short periods, where tregn96's flattening leaves F unmapped and eta
// departs from 1).  The layer's propagators are real by construction; as in
// tregn96 the compound and Haskell matrices are formed in complex arithmetic
// and their real parts carried on.
__device__ __noinline__ void ti_eigen_z(const TiLayer& L, double omg, double wvn, double wvno2, TiEigZ& o)
{
    const double om2 = omg * omg;
    const double wvn2 = wvn * wvn;
    const zc a = Z(wvn * L.TFoTA), b = Z(L.iTA);
    const zc c = Z(-L.rho * om2 + wvn2 * L.TAF);
    const zc d = Z(-wvn), e = Z(L.iTL), f = Z(-L.rho * om2);
    const zc ddef = Z(wvn2 - om2 * L.rhoTL);
    const zc aabc = Z(wvn2 - om2 * L.rhoTA);
    const zc bb = (2.0 * (a * d) + e * c) + f * b;
    const zc cc = ddef * aabc;
    zc srt = zsqrt(bb * bb - 4.0 * cc);
    if (srt.im < 0.0) srt = -srt;
    zc L1, L2;
    if (bb.re < 0.0 && srt.re < 0.0) {
        L2 = 0.5 * (bb - srt);
        L1 = znorm2(L2) > 0.0 ? zdiv(cc, L2) : 0.5 * (bb + srt);
    } else {
        L1 = 0.5 * (bb + srt);
        L2 = znorm2(L1) > 0.0 ? zdiv(cc, L1) : 0.5 * (bb - srt);
    }
    if (znorm2(Z(wvno2) - L2) < znorm2(Z(wvno2) - L1)) { const zc t = L1; L1 = L2; L2 = t; }
    zc rp = zsqrt(L1), rsv = zsqrt(L2);
    if (rp.re < 0.0) rp = -rp;
    if (rsv.re < 0.0) rsv = -rsv;
    const zc bcaa = b * c + a * a, ddef2 = d * d + e * f;
    zc x12 = b * d - a * e;
    zc x22 = b * L2 - e * bcaa;
    zc x32 = L2 - (a * d + c * e);
    zc x42 = -(a * L2) + d * bcaa;
    zc x11 = -(e * L1) + b * ddef2;
    zc x21 = b * d - a * e;
    zc x31 = d * L1 - a * ddef2;
    zc x41 = -((L1 - a * d) - b * f);
    if (wvn != 0.0) {
        const zc z1 = zdiv(Z(wvn), x11);
        x11 = x11 * z1; x21 = x21 * z1; x31 = x31 * z1; x41 = x41 * z1;
        const zc z2 = zdiv(Z(wvn), x22);
        x12 = x12 * z2; x22 = x22 * z2; x32 = x32 * z2; x42 = x42 * z2;
    }
    o.x11 = x11; o.x21 = x21; o.x31 = x31; o.x41 = x41;
    o.x12 = x12; o.x22 = x22; o.x32 = x32; o.x42 = x42;
    o.np = x11 * x41 - x21 * x31;
    o.nsv = x12 * x42 - x22 * x32;
    o.rp = rp;
    o.rsv = rsv;
}

struct TiVarZ {
    zc cosp, rsinp, sinpr, cosq, rsinq, sinqr;
    double pex, svex;
};

__device__ __noinline__ void ti_var_z_one(zc r, double dm, zc& cosf, zc& rsin, zc& sinr, double& ex)
{
    const zc p = dm * r;
    ex = p.re;
    double sn, cs;
    sincos(p.im, &sn, &cs);
    const zc ep = Z(cs / 2.0, sn / 2.0), em = Z(ep.re, -ep.im);
    const double fac = p.re < 15.0 ? exp(-2.0 * p.re) : 0.0;
    cosf = ep + fac * em;
    const zc s = ep - fac * em;
    rsin = r * s;
    sinr = (fabs(p.re) < 1.0e-5 && znorm2(r) < 1.0e-10) ? Z(dm) : zdiv(s, r);
}

__device__ void ti_compound_z(const TiEigZ& E, const TiVarZ& v, double ca[5][5])
{
    const double ex = v.pex + v.svex;
    const double dfac = ex > 35.0 ? 0.0 : exp(-ex);
    const zc a1 = zdiv(Z(0.5), E.np), a2 = zdiv(Z(0.5), E.nsv);
    zc fac[3][4];
    fac[1][0] = (2.0 * a1) * v.cosp; fac[1][1] = (2.0 * a1) * v.sinpr; fac[1][2] = (2.0 * a1) * v.rsinp;
    fac[1][3] = (4.0 * dfac) * (a1 * a1);
    fac[2][0] = (2.0 * a2) * v.cosq; fac[2][1] = (2.0 * a2) * v.sinqr; fac[2][2] = (2.0 * a2) * v.rsinq;
    fac[2][3] = (4.0 * dfac) * (a2 * a2);
    zc xs[5][3];
    xs[1][1] = E.x11; xs[2][1] = E.x21; xs[3][1] = E.x31; xs[4][1] = E.x41;
    xs[1][2] = E.x12; xs[2][2] = E.x22; xs[3][2] = E.x32; xs[4][2] = E.x42;
    // the term table expanded at compile time (as the real path does): the
    // factors stay in registers
    const double t11 = tca_elem<0>(xs, fac).re, t12 = tca_elem<1>(xs, fac).re;
    const double t13 = tca_elem<2>(xs, fac).re, t15 = tca_elem<3>(xs, fac).re;
    const double t16 = tca_elem<4>(xs, fac).re, t21 = tca_elem<5>(xs, fac).re;
    const double t22 = tca_elem<6>(xs, fac).re, t23 = tca_elem<7>(xs, fac).re;
    const double t25 = tca_elem<8>(xs, fac).re, t31 = tca_elem<9>(xs, fac).re;
    const double t32 = tca_elem<10>(xs, fac).re, t33 = tca_elem<11>(xs, fac).re;
    const double t51 = tca_elem<12>(xs, fac).re, t52 = tca_elem<13>(xs, fac).re;
    const double t61 = tca_elem<14>(xs, fac).re;
    ca[0][0] = t11; ca[0][1] = t12; ca[0][2] = t13; ca[0][3] = t15; ca[0][4] = t16;
    ca[1][0] = t21; ca[1][1] = t22; ca[1][2] = t23; ca[1][3] = t25; ca[1][4] = t15;
    ca[2][0] = 2.0 * t31; ca[2][1] = 2.0 * t32; ca[2][2] = 2.0 * t33 - dfac;
    ca[2][3] = -2.0 * t23; ca[2][4] = -2.0 * t13;
    ca[3][0] = t51; ca[3][1] = t52; ca[3][2] = -t32; ca[3][3] = t22; ca[3][4] = t12;
    ca[4][0] = t61; ca[4][1] = t51; ca[4][2] = -t31; ca[4][3] = t21; ca[4][4] = t11;
}

__device__ void ti_haskell_z(const TiEigZ& E, const TiVarZ& V, double v[4], double& cpex)
{
    const bool pbig = V.pex > V.svex;
    const double dd = fabs(V.pex - V.svex);
    const double f = dd > 40.0 ? 0.0 : exp(-dd);
    const double fp = pbig ? 1.0 : f, fs = pbig ? f : 1.0;
    cpex = pbig ? V.pex : V.svex;
    const zc cosp = zdiv(fp * V.cosp, E.np), sinpr = zdiv(fp * V.sinpr, E.np), rsinp = zdiv(fp * V.rsinp, E.np);
    const zc cossv = zdiv(fs * V.cosq, E.nsv), sinsvr = zdiv(fs * V.sinqr, E.nsv), rsinsv = zdiv(fs * V.rsinq, E.nsv);
    const zc x11 = E.x11, x21 = E.x21, x31 = E.x31, x41 = E.x41;
    const zc x12 = E.x12, x22 = E.x22, x32 = E.x32, x42 = E.x42;
    double A[4][4];
    A[0][0] = ((x11 * x41) * cosp + (x12 * x42) * cossv).re;
    A[0][1] = (-((x11 * x31) * sinpr) - (x12 * x32) * rsinsv).re;
    A[0][2] = (-((x11 * x21) * cosp) - (x12 * x22) * cossv).re;
    A[0][3] = ((x11 * x11) * sinpr + (x12 * x12) * rsinsv).re;
    A[1][0] = ((x21 * x41) * rsinp + (x22 * x42) * sinsvr).re;
    A[1][1] = (-((x21 * x31) * cosp) - (x22 * x32) * cossv).re;
    A[1][2] = (-((x21 * x21) * rsinp) - (x22 * x22) * sinsvr).re;
    A[2][0] = ((x31 * x41) * cosp + (x32 * x42) * cossv).re;
    A[2][1] = (-((x31 * x31) * sinpr) - (x32 * x32) * rsinsv).re;
    A[3][0] = ((x41 * x41) * rsinp + (x42 * x42) * sinsvr).re;
    A[1][3] = -A[0][2]; A[2][2] = A[1][1]; A[2][3] = -A[0][1];
    A[3][1] = -A[2][0]; A[3][2] = -A[1][0]; A[3][3] = A[0][0];
    double o[4];
    for (int i = 0; i < 4; ++i) o[i] = A[i][0] * v[0] + A[i][1] * v[1] + A[i][2] * v[2] + A[i][3] * v[3];
    for (int i = 0; i < 4; ++i) v[i] = o[i];
}

// Haskell matrix (hska, tregn96.f:3477-3559) applied to v: v <- AA v.
__device__ __forceinline__ void ti_haskell(const TiEig& E, const TiVar& V, double v[4], double& cpex)
{
    // the larger exponent is factored out; the other wave is scaled by
    // exp(-|pex - svex|) (0 beyond 40)
    const bool pbig = V.pex > V.svex;
    const double dd = fabs(V.pex - V.svex);
    const double f = dd > 40.0 ? 0.0 : exp(-dd);
    const double fp = pbig ? 1.0 : f, fs = pbig ? f : 1.0;
    cpex = pbig ? V.pex : V.svex;
    const double inp = fast_rcp(E.np), ins = fast_rcp(E.nsv);
    const double cosp = fp * V.cosp * inp, sinpr = fp * V.sinpr * inp, rsinp = fp * V.rsinp * inp;
    const double cossv = fs * V.cosq * ins, sinsvr = fs * V.sinqr * ins, rsinsv = fs * V.rsinq * ins;
    const double x11 = E.x11, x21 = E.x21, x31 = E.x31, x41 = E.x41;
    const double x12 = E.x12, x22 = E.x22, x32 = E.x32, x42 = E.x42;
    double A[4][4];
    A[0][0] = x11 * x41 * cosp + x12 * x42 * cossv;
    A[0][1] = -x11 * x31 * sinpr - x12 * x32 * rsinsv;
    A[0][2] = -x11 * x21 * cosp - x12 * x22 * cossv;
    A[0][3] = x11 * x11 * sinpr + x12 * x12 * rsinsv;
    A[1][0] = x21 * x41 * rsinp + x22 * x42 * sinsvr;
    A[1][1] = -x21 * x31 * cosp - x22 * x32 * cossv;
    A[1][2] = -x21 * x21 * rsinp - x22 * x22 * sinsvr;
    A[2][0] = x31 * x41 * cosp + x32 * x42 * cossv;
    A[2][1] = -x31 * x31 * sinpr - x32 * x32 * rsinsv;
    A[3][0] = x41 * x41 * rsinp + x42 * x42 * sinsvr;
    A[1][3] = -A[0][2]; A[2][2] = A[1][1]; A[2][3] = -A[0][1];
    A[3][1] = -A[2][0]; A[3][2] = -A[1][0]; A[3][3] = A[0][0];
    double o[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) o[i] = A[i][0] * v[0] + A[i][1] * v[1] + A[i][2] * v[2] + A[i][3] * v[3];
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = o[i];
}

// ffunc/gfunc/h1func/h2func values (tregn96.f:1385-1473: FA, GA, FB, GB,
// H1, H2) of a layer with complex eigenvalues: exp(-nu d) of the two waves
// once, exp(-2 nu d) and exp(-(nu_a + nu_b) d) as their products, with the
// reference's cut-offs on the real part of the exponent (40, and 75 for
// gfunc).  Re(nu) >= 0, so the products cannot overflow.
__device__ __forceinline__ void ti_fgh_z(zc ra, zc rb, double dm, zc fg[6])
{
    const zc aa = dm * ra, ab = dm * rb;
    const zc ea = aa.re < 75.0 ? zexp(-aa) : Z(0.0);
    const zc eb = ab.re < 75.0 ? zexp(-ab) : Z(0.0);
    fg[0] = znorm2(ra) < 1.0e-16 ? Z(dm) : zdiv(Z(1.0) - (aa.re < 40.0 ? ea * ea : Z(0.0)), 2.0 * ra);
    fg[1] = dm * ea;
    fg[2] = znorm2(rb) < 1.0e-16 ? Z(dm) : zdiv(Z(1.0) - (ab.re < 40.0 ? eb * eb : Z(0.0)), 2.0 * rb);
    fg[3] = dm * eb;
    const zc sab = rb + ra;
    fg[4] = znorm2(sab) < 1.0e-16 ? Z(dm)
            : zdiv(Z(1.0) - (dm * sab.re < 40.0 ? ea * eb : Z(0.0)), sab);
    fg[5] = znorm2(rb - ra) < 1.0e-16 ? Z(dm)
            : zdiv((ab.re < 40.0 ? eb : Z(0.0)) - (aa.re < 40.0 ? ea : Z(0.0)), ra - rb);
}

// Energy integrals of a layer with real eigenvalues, evanescent and
// oscillatory waves alike: the sums of ti_integrals_z, in mostly real
// arithmetic, with one code path for both kinds of layer (so the lanes of a
// warp do not split between them).
//   - Each entry of E is a real factor times 1, nu_a or nu_b (nu = r for an
//     evanescent wave, i r for an oscillatory one).  The six integrals pair
//     rows (i, j) of equal parity, so e[i][a] e[j][b] is real for two P or
//     two S columns (times nu^2 = +-r^2 where the rows carry nu), and real
//     times nu_b (even rows) or nu_a (odd rows) for a P and an S column.
//   - The potentials are A + B / nu with A, B real.
//   - With the ten products W = (potential product) x (ffunc, gfunc,
//     h1func, h2func value), each integral is a real combination of Re W
//     and Re(nu W).
__device__ __forceinline__ zc ti_over_nu(double A, double B, double ir, bool osc)
{
    // A + B / nu: 1 / nu = 1 / r, or -i / r
    return osc ? Z(A, -B * ir) : Z(A + B * ir, 0.0);
}
__device__ __forceinline__ double ti_re_nu(double r, bool osc, zc w)
{
    // Re(nu w)
    return osc ? -r * w.im : r * w.re;
}
__device__ __forceinline__ void ti_integrals_wave(const TiEig& E, const TiWave& P, const TiWave& S,
                                                  double dm, const double top[4], const double bot[4],
                                                  double out[6])
{
    const double ra = E.rp, rb = E.rsv;
    const bool oa = E.oscp, ob = E.oscs;
    const double ira = fast_rcp(ra), irb = fast_rcp(rb);
    const double x11 = E.x11, x21 = E.x21, x31 = E.x31, x41 = E.x41;
    const double x12 = E.x12, x22 = E.x22, x32 = E.x32, x42 = E.x42;
    // potentials: rows 0 / 2 of E^-1 (P up / down) and 1 / 3 (S up / down)
    const double hp = 0.5 * fast_rcp(E.np), hs = 0.5 * fast_rcp(E.nsv);
    const zc kmpu = ti_over_nu((bot[0] * x41 - bot[2] * x21) * hp, (bot[3] * x11 - bot[1] * x31) * hp, ira, oa);
    const zc km1pd = ti_over_nu((top[0] * x41 - top[2] * x21) * hp, (top[1] * x31 - top[3] * x11) * hp, ira, oa);
    const zc kmsu = ti_over_nu((bot[3] * x12 - bot[1] * x32) * hs, (bot[0] * x42 - bot[2] * x22) * hs, irb, ob);
    const zc km1sd = ti_over_nu((top[3] * x12 - top[1] * x32) * hs, (top[2] * x22 - top[0] * x42) * hs, irb, ob);
    // ffunc/gfunc/h1func/h2func from the waves' exp(-nu d), with the
    // reference's cut-offs on the real part of nu d (40; 75 for gfunc)
    const zc ea = Z(P.er, P.ei), eb = Z(S.er, S.ei);
    const double xa = oa ? 0.0 : dm * ra, xb = ob ? 0.0 : dm * rb;
    auto ffun = [&](double r, bool osc, double x, zc e) {
        if (r < 1.0e-08) return Z(dm);
        const zc n = Z(1.0) - (x < 40.0 ? e * e : Z(0.0));
        const double h = 0.5 * fast_rcp(r);           // n / (2 nu)
        return osc ? Z(n.im * h, -n.re * h) : Z(n.re * h, n.im * h);
    };
    const zc FA = ffun(ra, oa, xa, ea), FB = ffun(rb, ob, xb, eb);
    const zc GA = xa < 75.0 ? dm * ea : Z(0.0);
    const zc GB = xb < 75.0 ? dm * eb : Z(0.0);
    const zc nua = oa ? Z(0.0, ra) : Z(ra), nub = ob ? Z(0.0, rb) : Z(rb);
    const zc sab = nub + nua;
    const zc H1 = znorm2(sab) < 1.0e-16 ? Z(dm)
                  : zdiv(Z(1.0) - (dm * sab.re < 40.0 ? ea * eb : Z(0.0)), sab);
    const zc H2 = znorm2(nub - nua) < 1.0e-16 ? Z(dm)
                  : zdiv((xb < 40.0 ? eb : Z(0.0)) - (xa < 40.0 ? ea : Z(0.0)), nua - nub);
    // the ten products
    const zc W1 = (kmpu * kmpu) * FA, W2 = (km1pd * km1pd) * FA;
    const zc W3 = (kmsu * kmsu) * FB, W4 = (km1sd * km1sd) * FB;
    const zc W5 = (kmpu * kmsu) * H1, W6 = (km1pd * km1sd) * H1;
    const zc W7 = (kmpu * km1sd) * H2, W8 = (km1pd * kmsu) * H2;
    const zc W9 = (kmpu * km1pd) * GA, W10 = (kmsu * km1sd) * GB;
    const double U5a = ti_re_nu(ra, oa, W5), U6a = ti_re_nu(ra, oa, W6);
    const double U7a = ti_re_nu(ra, oa, W7), U8a = ti_re_nu(ra, oa, W8);
    const double U5b = ti_re_nu(rb, ob, W5), U6b = ti_re_nu(rb, ob, W6);
    const double U7b = ti_re_nu(rb, ob, W7), U8b = ti_re_nu(rb, ob, W8);
    const double kaa = oa ? -(ra * ra) : ra * ra, kbb = ob ? -(rb * rb) : rb * rb;   // nu^2
    // real factors of E (the nu factors taken out)
    const double ep[4][4] = {{x11, x12, x11, -x12}, {x21, x22, -x21, x22},
                             {x31, x32, x31, -x32}, {x41, x42, -x41, x42}};
    constexpr int IJ[6][2] = {{0, 0}, {0, 2}, {1, 1}, {1, 3}, {2, 2}, {3, 3}};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const int i = IJ[q][0], j = IJ[q][1];
        const bool odd = (i & 1) != 0;
        auto ee = [&](int a, int b) { return ep[i][a] * ep[j][b]; };
        auto sy = [&](int a, int b) { return ee(a, b) + ee(b, a); };
        const double pp = ee(0, 0) * W1.re + ee(2, 2) * W2.re + sy(0, 2) * W9.re;
        const double ss = ee(1, 1) * W3.re + ee(3, 3) * W4.re + sy(1, 3) * W10.re;
        const double mx = odd ? sy(0, 1) * U5a + sy(2, 3) * U6a + sy(0, 3) * U7a + sy(1, 2) * U8a
                              : sy(0, 1) * U5b + sy(2, 3) * U6b + sy(0, 3) * U7b + sy(1, 2) * U8b;
        out[q] = (odd ? kaa : 1.0) * pp + (odd ? 1.0 : kbb) * ss + mx;
    }
}

// Small fixed-size vectors passed by value to the out-of-line paths (so
// the hot loop keeps its vectors in registers).
struct D4 { double v[4]; };
struct D5 { double v[5]; };
struct D6 { double v[6]; };
struct UpOut { D5 ee; double pexsv; };
struct DownOut { D4 vv; double cpex; };

// Up-sweep step of a layer with complex eigenvalues: ee = cdv * CA.
__device__ __noinline__ UpOut ti_up_general(TiLayer L, double omega, double wvno, double wvno2, D5 cdv)
{
    TiEigZ EZ;
    ti_eigen_z(L, omega, wvno, wvno2, EZ);
    TiVarZ VZ;
    ti_var_z_one(EZ.rp, L.td, VZ.cosp, VZ.rsinp, VZ.sinpr, VZ.pex);
    ti_var_z_one(EZ.rsv, L.td, VZ.cosq, VZ.rsinq, VZ.sinqr, VZ.svex);
    double ca[5][5];
    ti_compound_z(EZ, VZ, ca);
    UpOut o;
    for (int i = 0; i < 5; ++i)
        o.ee.v[i] = cdv.v[0] * ca[0][i] + cdv.v[1] * ca[1][i] + cdv.v[2] * ca[2][i] +
                    cdv.v[3] * ca[3][i] + cdv.v[4] * ca[4][i];
    o.pexsv = VZ.pex + VZ.svex;
    return o;
}

// Down-sweep Haskell step of a layer with complex eigenvalues.
__device__ __noinline__ DownOut ti_down_general(TiLayer L, double omega, double wvno, double wvno2, D4 vv)
{
    TiEigZ EZ;
    ti_eigen_z(L, omega, wvno, wvno2, EZ);
    TiVarZ VZ;
    ti_var_z_one(EZ.rp, L.td, VZ.cosp, VZ.rsinp, VZ.sinpr, VZ.pex);
    ti_var_z_one(EZ.rsv, L.td, VZ.cosq, VZ.rsinq, VZ.sinqr, VZ.svex);
    DownOut o;
    o.vv = vv;
    ti_haskell_z(EZ, VZ, o.vv.v, o.cpex);
    return o;
}

// Energy integrals of the half-space or of a layer with complex
// eigenvalues (complex exponentials).
__device__ __noinline__ D6 ti_integrals_general(TiLayer L, double omega, double wvno, double wvno2,
                                                D4 top, D4 bot, bool half)
{
    // only layers whose eigenvalues are complex come here (the real ones
    // take ti_integrals_wave / ti_integrals_halfspace)
    TiEigZ EZ;
    ti_eigen_z(L, omega, wvno, wvno2, EZ);
    zc fg[6];
    if (!half) ti_fgh_z(EZ.rp, EZ.rsv, L.td, fg);
    D6 o;
    ti_integrals_z(EZ, fg, top.v, bot.v, half, o.v);
    return o;
}

// Energy integrals of the half-space (half = 1 in intijr): only its upper
// interface's potentials (km1pd, km1sd) contribute, and for exp(-nu z) on
// z > 0 ffunc -> 1/(2 nu), h1func -> 1/(nu_a + nu_b), gfunc = h2func = 0.
// With real eigenvalues this is ti_integrals_wave's real form (same E
// factors, same potentials); complex eigenvalues go through the general
// path.  Called once per (column, period), out of line, so the warps do not
// fetch the general path's code at the end of every task.
__device__ __noinline__ D6 ti_integrals_halfspace(TiLayer L, double omega, double wvno, double wvno2,
                                                  D4 top)
{
    TiEig E;
    ti_eigen(L, omega, wvno, wvno2, E);
    if (!E.ok) {
        const D4 zero = {{0.0, 0.0, 0.0, 0.0}};
        return ti_integrals_general(L, omega, wvno, wvno2, top, zero, true);
    }
    const double ra = E.rp, rb = E.rsv;
    const bool oa = E.oscp, ob = E.oscs;
    const double ira = fast_rcp(ra), irb = fast_rcp(rb);
    const double x11 = E.x11, x21 = E.x21, x31 = E.x31, x41 = E.x41;
    const double x12 = E.x12, x22 = E.x22, x32 = E.x32, x42 = E.x42;
    const double hp = 0.5 * fast_rcp(E.np), hs = 0.5 * fast_rcp(E.nsv);
    const double* t = top.v;
    const zc km1pd = ti_over_nu((t[0] * x41 - t[2] * x21) * hp, (t[1] * x31 - t[3] * x11) * hp, ira, oa);
    const zc km1sd = ti_over_nu((t[3] * x12 - t[1] * x32) * hs, (t[2] * x22 - t[0] * x42) * hs, irb, ob);
    // 1 / (2 nu): 1/(2r) or -i/(2r)
    const zc FA = oa ? Z(0.0, -0.5 * ira) : Z(0.5 * ira);
    const zc FB = ob ? Z(0.0, -0.5 * irb) : Z(0.5 * irb);
    const zc nua = oa ? Z(0.0, ra) : Z(ra), nub = ob ? Z(0.0, rb) : Z(rb);
    const zc H1 = zdiv(Z(1.0), nua + nub);
    const zc W2 = (km1pd * km1pd) * FA, W4 = (km1sd * km1sd) * FB, W6 = (km1pd * km1sd) * H1;
    const double U6a = ti_re_nu(ra, oa, W6), U6b = ti_re_nu(rb, ob, W6);
    const double kaa = oa ? -(ra * ra) : ra * ra, kbb = ob ? -(rb * rb) : rb * rb;
    const double ep[4][4] = {{x11, x12, x11, -x12}, {x21, x22, -x21, x22},
                             {x31, x32, x31, -x32}, {x41, x42, -x41, x42}};
    constexpr int IJ[6][2] = {{0, 0}, {0, 2}, {1, 1}, {1, 3}, {2, 2}, {3, 3}};
    D6 o;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const int i = IJ[q][0], j = IJ[q][1];
        const bool odd = (i & 1) != 0;
        const double pp = ep[i][2] * ep[j][2] * W2.re;
        const double ss = ep[i][3] * ep[j][3] * W4.re;
        const double mx = (ep[i][2] * ep[j][3] + ep[i][3] * ep[j][2]) * (odd ? U6a : U6b);
        o.v[q] = (odd ? kaa : 1.0) * pp + (odd ? 1.0 : kbb) * ss + mx;
    }
    return o;
}

// Haskell step (hska) of an evanescent or oscillatory layer with real
// eigenvalues, from its waves.
__device__ __forceinline__ void ti_haskell_w(const TiEig& E, const TiWave& P, const TiWave& S, double v[4],
                                             double& cpex)
{
    TiVar V;
    V.cosp = P.cosf; V.rsinp = P.rsin; V.sinpr = P.sinr; V.pex = P.ex;
    V.cosq = S.cosf; V.rsinq = S.rsin; V.sinqr = S.sinr; V.svex = S.ex;
    ti_haskell(E, V, v, cpex);
}

// Max-norm scaling by a power of two (exact; the exponent is carried in
// ex2 as a natural-log amount, like cnormc/rnormc's log(t1)).
__device__ __forceinline__ double pow2_normalise(double* v, int n)
{
    double mx = 0.0;
    for (int i = 0; i < n; ++i) mx = fmax(mx, fabs(v[i]));
    if (!(mx > 1.0e-40)) return 0.0;
    int ex;
    frexp(mx, &ex);
    for (int i = 0; i < n; ++i) v[i] = ldexp(v[i], -ex);
    return (double)ex * 0.6931471805599453;
}

// Compound vector of the half-space: the 2x2 minors of rows 1-2 of its
// E^-1 (evalg, up).
__device__ __noinline__ D5 ti_halfspace_cdv(TiLayer L, double omega, double wvno, double wvno2)
{
    TiEigZ E;
    ti_eigen_z(L, omega, wvno, wvno2, E);
    zc e[4][4], G[4][4];
    ti_emat(E, e, G);
    D5 c;
    c.v[0] = (G[0][0] * G[1][1] - G[0][1] * G[1][0]).re;
    c.v[1] = (G[0][0] * G[1][2] - G[0][2] * G[1][0]).re;
    c.v[2] = (G[0][0] * G[1][3] - G[0][3] * G[1][0]).re;
    c.v[3] = (G[0][1] * G[1][3] - G[0][3] * G[1][1]).re;
    c.v[4] = (G[0][2] * G[1][3] - G[0][3] * G[1][2]).re;
    return c;
}

__device__ __forceinline__ long long ti_next_task(unsigned* queue)
{
    unsigned t = 0;
    if ((threadIdx.x & 31) == 0) t = atomicAdd(queue, 1u);
    return (long long)__shfl_sync(0xffffffffu, t, 0);
}

// Number of layers the sweep of one (column, period) covers, the last taken
// as the half-space (the depth cut, kTiDepthCut): where the waves have
// decayed by exp(-E) with E = sum of nu d over the layers above and
// E >= kTiDepthCut, that layer is taken as the half-space and the ones
// below are not swept.  The compound vectors above it and the
// eigenfunction energy at and below it are exponentially small in E
// against the surface's, so the partials above move by far less than a
// real*4 ulp and the ones below the cut (of that size) are left out of the
// splice (written as zero).  nu is the isotropic vertical S wavenumber
// sqrt(k^2 - omega^2 rho / L) of the flattened layer (the smaller of the
// two; the TI ones differ by well under 1 %).  Only short periods over
// deep stacks are cut, which is where the complex-eigenvalue layers lie.
__device__ __forceinline__ int ti_cut_layers(const TiRec* tir, int rmax, double omega, double wvno2)
{
    double ex = 0.0;
    for (int m = 0; m < rmax - 1; ++m) {
        if (ex >= kTiDepthCut) return m + 1;
        const TiRec r = tir[(long long)m * TILE];
        const double nb2 = wvno2 - omega * omega * r.rho / r.TL;
        if (nb2 > 0.0) ex += sqrt(nb2) * r.td;
    }
    return rmax;
}

// tregn96.f:430-479: twopi real*4, t and cp real*4
__device__ __forceinline__ double ti_omega(const TiArgs& a, const ColMeta& M, int k)
{
    const float twopi = 6.2831855f;
    return (double)twopi / (double)(float)a.periods[M.per_b + k];
}

// Sort key of the pair (column lane `lane` of tile t, period k): 0 no such
// pair, 1 no root (the period's Lsen_Gsc row is written as zero), else
// 1 + the layers its sweep covers (ti_cut_layers, at most NL).
__device__ __forceinline__ int ti_pair_key(const TiArgs& a, long long t, int lane, int k)
{
    const Tables& T = a.T;
    const long long s = t * TILE + lane;
    if (s >= T.ncols) return 0;
    const ColMeta M = T.meta[s];
    if (k >= M.K) return 0;
    const float cpf = (float)a.pv[M.pv_b + T.pv_sk * k];
    if (!(cpf > 0.0f)) return 1;
    if (!a.cut) return 1 + M.rmax;
    const double omega = ti_omega(a, M, k);
    const double wvno = omega / (double)cpf;
    return 1 + ti_cut_layers(T.ti + T.tile_lbase[t] + lane, M.rmax, omega, wvno * wvno);
}

// One (column, period) of the Gc/Gs kernel: the pair at a.order[task * 32
// + tl] of task `task`, run by lane tl with the thread's scratch block at
// scr (layer m, entry q at scr[(m * TI_SCR_Q + q) * TILE]).
__device__ __forceinline__ void ti_task(const TiArgs& a, long long task, int tl, double* scr)
{
    const Tables& T = a.T;
    constexpr long long nslots = TILE;
    {
        const int e = a.order[task * TILE + tl];
        const int key = e >> 16;
        if (key == 0) return;
        const int lane = e & 31, k = (e >> 5) & 0x7ff;
        const int2 tk = T.tasks[task];
        const long long s = (long long)tk.x * TILE + lane;
        const ColMeta M = T.meta[s];
        const int rmax = M.rmax, nz = M.nz;
        float* lout = a.lsen + M.ls_b + T.ls_sk * k;
        const long long jstride = M.ls_is;
        if (key == 1) {
            for (int j = 0; j < nz - 1; ++j) lout[jstride * j] = 0.0f;
            return;
        }
        const int rm = key - 1;
        const float cpf = (float)a.pv[M.pv_b + T.pv_sk * k];
        const long long lbase = T.tile_lbase[tk.x] + lane;
        const TiRec* tir = T.ti + lbase;              // layer m at tir[m * TILE]
        const ChainRec* chr = T.ch + lbase;
        const double omega = ti_omega(a, M, k);
        const double wvno = omega / (double)cpf;
        const double wvno2 = wvno * wvno;
        const double iwvno = 1.0 / wvno, iwvno2 = 1.0 / wvno2;
        // ---- up() (compound vectors from the half-space upward), then
        // down() + svfunc() + energy() (interface by interface), as one loop
        // of 2 rm - 1 steps (rm: the layers ti_cut_layers gives, the last
        // as the half-space): steps 0 .. rm-2 are up-sweep layers
        // rm-2 .. 0, the rest down-sweep layers 0 .. rm-1.  A layer's
        // eigen-solution and waves are formed at the top of the step by the
        // one copy of that code, in both sweeps, so the down-sweep forms
        // them again instead of reading them back: the per-layer scratch is
        // the compound vector and its exponent sum only.

        constexpr int Q = TI_SCR_Q;
        double cdv[5];
        double exsum = 0.0;
        {
            const D5 c = ti_halfspace_cdv(ti_layer(tir + (long long)(rm - 1) * TILE), omega, wvno, wvno2);
            double* sp = scr + (long long)(rm - 1) * Q * nslots;
#pragma unroll
            for (int q = 0; q < 5; ++q) { cdv[q] = c.v[q]; sp[q * nslots] = cdv[q]; }
            sp[5 * nslots] = 0.0;
        }
        double exe0 = 0.0, if1213 = 0.0;
        double top[4] = {0.0, 0.0, 0.0, 0.0}, vv[4] = {1.0, 0.0, 0.0, 0.0};
        double exa = 0.0;
        double sumi0 = 0.0, sumi1 = 0.0, sumi2 = 0.0, gsum = 0.0;
        const double pi_ = 3.141592653589493;   // gammap's constant, as in the reference
        const double lw = log(omega / (2.0 * pi_ * 1.0)) / pi_;
        const int nsteps = 2 * rm - 1;
        for (int step = 0; step < nsteps; ++step) {
            const bool up = step < rm - 1;
            const int m = up ? rm - 2 - step : step - (rm - 1);
            const bool half = (m == rm - 1);
            const TiLayer L = ti_layer(tir + (long long)m * TILE);
            TiEig E;
            TiWave P, S;
            E.ok = false;
            if (!half) {
                ti_eigen(L, omega, wvno, wvno2, E);
                if (E.ok) {
                    // P and S waves through one copy of the wave code
#pragma unroll 1
                    for (int w = 0; w < 2; ++w) {
                        const TiWave t = ti_wave(w ? E.rsv : E.rp, w ? E.oscs : E.oscp, L.td);
                        if (w) S = t; else P = t;
                    }
                }
            }
            const bool fast = E.ok;
            if (up) {
                double* sp = scr + (long long)m * Q * nslots;
                double ee[5];
                double pexsv;
                if (fast) {
                    TiVar V;
                    V.cosp = P.cosf; V.rsinp = P.rsin; V.sinpr = P.sinr; V.pex = P.ex;
                    V.cosq = S.cosf; V.rsinq = S.rsin; V.sinqr = S.sinr; V.svex = S.ex;
                    ti_compound_apply(E, V, cdv, ee);
                    pexsv = P.ex + S.ex;
                } else {
                    D5 c5;
#pragma unroll
                    for (int i = 0; i < 5; ++i) c5.v[i] = cdv[i];
                    const UpOut u = ti_up_general(L, omega, wvno, wvno2, c5);
#pragma unroll
                    for (int i = 0; i < 5; ++i) ee[i] = u.ee.v[i];
                    pexsv = u.pexsv;
                }
                const double exn = pow2_normalise(ee, 5);
                exsum = exsum + pexsv + exn;
#pragma unroll
                for (int q = 0; q < 5; ++q) { cdv[q] = ee[q]; sp[q * nslots] = ee[q]; }
                sp[5 * nslots] = exsum;
                continue;
            }
            if (m == 0) {
                // the surface: exe(1), and ur, uz, tz, tr from the top
                // compound vector
                exe0 = exsum;
                const double f1213 = -cdv[1];
                if1213 = 1.0 / f1213;
                top[0] = cdv[2] / cdv[1]; top[1] = 1.0; top[2] = 0.0; top[3] = 0.0;
            }
            double bot[4] = {0.0, 0.0, 0.0, 0.0};
            if (!half) {
                double cpex;
                if (fast) {
                    ti_haskell_w(E, P, S, vv, cpex);
                } else {
                    D4 v4;
#pragma unroll
                    for (int i = 0; i < 4; ++i) v4.v[i] = vv[i];
                    const DownOut d = ti_down_general(L, omega, wvno, wvno2, v4);
#pragma unroll
                    for (int i = 0; i < 4; ++i) vv[i] = d.vv.v[i];
                    cpex = d.cpex;
                }
                const double ex2 = pow2_normalise(vv, 4);
                exa = exa + cpex + ex2;
                // eigenfunctions at interface m+1 (svfunc)
                const double* sp = scr + (long long)(m + 1) * Q * nslots;
                const double cd1 = sp[0], cd2 = sp[nslots], cd3 = sp[2 * nslots];
                const double cd4 = -cd3, cd5 = sp[3 * nslots], cd6 = sp[4 * nslots];
                const double exe = sp[5 * nslots];
                const double tz1 = -vv[3], tz2 = -vv[2], tz3 = vv[1], tz4 = vv[0];
                const double uu1 = tz2 * cd6 - tz3 * cd5 + tz4 * cd4;
                const double uu2 = -tz1 * cd6 + tz3 * cd3 - tz4 * cd2;
                const double uu3 = tz1 * cd5 - tz2 * cd3 + tz4 * cd1;
                const double uu4 = -tz1 * cd4 + tz2 * cd2 - tz3 * cd1;
                const double ext = exa + exe - exe0;
                if (ext > -80.0 && ext < 80.0) {
                    const double fact = exp(ext) * if1213;
                    bot[0] = uu1 * fact; bot[1] = uu2 * fact; bot[2] = uu3 * fact; bot[3] = uu4 * fact;
                }
            }
            // energy integrals of layer m (typelyr 0, or 1 for the half-space)
            double I[6];
            if (fast) {
                // real eigenvalues, evanescent or oscillatory waves: one path
                ti_integrals_wave(E, P, S, L.td, top, bot, I);
            } else {
                D4 t4, b4;
#pragma unroll
                for (int i = 0; i < 4; ++i) { t4.v[i] = top[i]; b4.v[i] = bot[i]; }
                const D6 r = half ? ti_integrals_halfspace(L, omega, wvno, wvno2, t4)
                                  : ti_integrals_general(L, omega, wvno, wvno2, t4, b4, false);
#pragma unroll
                for (int i = 0; i < 6; ++i) I[i] = r.v[i];
            }
            const double TA = L.TA, TF = L.TF, TL = L.TL, rho = L.rho;
            const double ah = L.ah, av = L.ah, bv = L.bv;
            const double eta = L.eta;
            const double a12 = -wvno, a14 = L.iTL, a21 = wvno * L.TFoTA, a23 = L.iTA;
            const double URUR = I[0], UZUZ = I[2];
            const double DURDUR = a12 * a12 * I[2] + 2.0 * a12 * a14 * I[3] + a14 * a14 * I[5];
            const double DUZDUZ = a21 * a21 * I[0] + 2.0 * a21 * a23 * I[1] + a23 * a23 * I[4];
            const double URDUZ = a21 * I[0] + a23 * I[1];
            const double UZDUR = a12 * I[2] + a14 * I[3];
            sumi0 += rho * (URUR + UZUZ);
            sumi1 += TL * UZUZ + TA * URUR;
            sumi2 += TL * UZDUR - TF * URDUZ;
            const double facah = rho * ah * (URUR - 2.0 * eta * URDUZ * iwvno);
            const double facav = rho * av * DUZDUZ * iwvno2;
            const double facbv = rho * bv * (UZUZ + 2.0 * UZDUR * iwvno + DURDUR * iwvno2 + 4.0 * eta * URDUZ * iwvno);
            const double facn = -TF * URDUZ * iwvno * L.ieta;
            // gammap() (facbh = 0; Q = 150 / 50, reference frequency 1 Hz)
            gsum += lw * (facbv * bv * (double)(1.0f / 50.0f));
            gsum += lw * ((facav * av + facah * ah) * (double)(1.0f / 150.0f));
            // raw partials for the splice (slot m is free: its compound
            // vector was consumed one step earlier)
            double* so = scr + (long long)m * Q * nslots;
            so[0] = facah; so[nslots] = facbv; so[2 * nslots] = facn;
#pragma unroll
            for (int i = 0; i < 4; ++i) top[i] = bot[i];
        }
        // ---- normalisation, attenuation shift, sphericity, splice
        const double ugr = (wvno * sumi1 + sumi2) / (omega * sumi0);
        const double un = ugr * sumi0;
        const double dcq = gsum / un;
        const double cq = omega / wvno + dcq;
        const double wq = omega / cq;
        const double c2 = omega / wq;
        const double tq = c2 / (2.0 * 6370.0 * omega);
        const double tm = sqrt(1.0 + tq * tq);
        const double tm3 = tm * tm * tm;
        const double iun = 1.0 / un, iuntm3 = iun / tm3;
        const SpRec* spr = T.sp + lbase;
        // the half-space (rmax - 1) and the layers below the depth cut add
        // nothing; their records are not read
        const int mlim = rm < rmax - 1 ? rm : rmax - 1;
        int m = 0;
        for (int j = 0; j < nz - 1; ++j) {
            float acc = 0.0f;
            for (; m < mlim && chr[(long long)m * TILE].node == j; ++m) {
                const SpRec R = spr[(long long)m * TILE];
                const double* so = scr + (long long)m * Q * nslots;
                const double vt = (double)R.vtp;
                const double vah = so[0] * vt * iuntm3;
                const double vbv = so[nslots] * vt * iuntm3;
                const double vn = so[2 * nslots] * iun;
                const float dah = fabs(vah) < 1.0e-36 ? 0.0f : (float)vah;
                const float dbv = fabs(vbv) < 1.0e-36 ? 0.0f : (float)vbv;
                const float dn = fabs(vn) < 1.0e-36 ? 0.0f : (float)vn;
                // depthkernelTI.f90:152-162 (real*4)
                const float dA = __fsub_rn(__fmul_rn(R.cA1, dah), __fmul_rn(R.cA2, dn));
                const float dL = __fadd_rn(__fmul_rn(R.cL1, dbv), __fmul_rn(R.cL2, dn));
                acc = __fadd_rn(__fadd_rn(acc, __fmul_rn(dA, R.TA)), __fmul_rn(dL, R.TL));
            }
            lout[jstride * j] = acc;
            if (!isfinite(acc) && a.errflag) atomicOr(a.errflag, 1);
        }
    }
}

// MINB: minimum resident blocks of 128 threads per SM the register
// allocation aims for (the autotuner picks one of the instantiations).
template <int MINB>
__global__ void __launch_bounds__(128, MINB)
ti_kernel(TiArgs a)
{
    // scratch: per warp [layer][q][lane] -- compile-time strides
    const long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    double* scr = a.scratch + (slot / TILE) * a.scr_layers * TI_SCR_Q * TILE + lane;
    for (;;) {
        const long long task = ti_next_task(a.queue);
        if (task >= a.T.ntasks) break;
        ti_task(a, task, lane, scr);
    }
}

// One block per tile: every (column, period) pair's key (ti_pair_key), then
// a counting sort of the tile's pairs by key into a.order, so that the 32
// lanes of a task sweep to nearly the same depth.  With lanes bound to the
// tile's columns, the lanes of a task at a short period would stop at
// depths differing by up to the whole stack, and the task would take the
// deepest.  The results do not depend on the order: each pair is computed
// by one lane alone, the same arithmetic on whichever lane.
__global__ void __launch_bounds__(TI_ORDER_THREADS)
ti_order_kernel(TiArgs a, const long long* tile_tbase, const long long* tile_tasks)
{
    __shared__ unsigned short key[NP * TILE];
    __shared__ int hist[NL + 2];
    const long long t = blockIdx.x;
    const int np = (int)tile_tasks[t] * TILE;     // tile_tasks <= NP (checked by the table build)
    for (int i = threadIdx.x; i < NL + 2; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        const int kk = ti_pair_key(a, t, p & 31, p >> 5);
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
    int* out = a.order + tile_tbase[t] * TILE;
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        const int kk = key[p];
        out[atomicAdd(&hist[kk], 1)] = (kk << 16) | p;
    }
}

template __global__ void ti_kernel<2>(TiArgs);
template __global__ void ti_kernel<3>(TiArgs);
template __global__ void ti_kernel<4>(TiArgs);
template __global__ void ti_kernel<6>(TiArgs);
template __global__ void ti_kernel<8>(TiArgs);

}  // namespace dk
