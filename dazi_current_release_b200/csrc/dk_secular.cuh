// Rayleigh secular function and the reference's root search, in FP64 on the
// CUDA cores.
//
//   dltar4 + var + dnka + normc   surfdisp96.f:767-865, 868-985, 1018-1062, 989-1014
//   getsol (bracket)              surfdisp96.f:384-476
//   nevill + half (refine)        surfdisp96.f:551-680
//   surfdisp96 period loop        surfdisp96.f:52-354 (Rayleigh, phase, mode 1)
//
// The layer chain is a sequential product of 5x5 Dunkin compound matrices,
// so it runs one model per thread; the tensor cores have no role here.  The
// model is reached through an accessor object (`M::layer(m)` returning the
// flattened thickness, Vp, Vs and density of layer m as a float4), so the
// same code serves the base model, a perturbed model of the finite-difference
// form and a model staged in shared memory.
#pragma once
#include "dk_model.cuh"

namespace dk {

constexpr double TWOPI = 2.0 * 3.141592653589793;

__device__ __forceinline__ double fsign1(double x) { return signbit(x) ? -1.0 : 1.0; }

// Secular-function value at wavenumber wvno, angular frequency omega.
// Normalisation factors of each layer product are discarded (they do not move
// the root), exactly as normc() does in the reference.
template <class M>
__device__ __noinline__ double dltar4(const M& mdl, int mmax, double wvno, double omega)
{
    if (omega < 1.0e-4) omega = 1.0e-4;
    const double wvno2 = wvno * wvno;
    float4 L = mdl.layer(mmax - 1);
    double a = (double)L.y, b = (double)L.z, rho1 = (double)L.w;
    double xka = omega / a, xkb = omega / b;
    double ra = sqrt((wvno + xka) * fabs(wvno - xka));
    double rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
    double t = b / omega;
    double gammk = 2.0 * t * t;
    double gam = gammk * wvno2;
    double gamm1 = gam - 1.0;
    double e0 = rho1 * rho1 * (gamm1 * gamm1 - gam * gammk * ra * rb);
    double e1 = -rho1 * ra;
    double e2 = rho1 * (gamm1 - gammk * ra * rb);
    double e3 = rho1 * rb;
    double e4 = wvno2 - ra * rb;
    for (int m = mmax - 2; m >= 0; --m) {
        L = mdl.layer(m);
        const double dpth = (double)L.x;
        a = (double)L.y; b = (double)L.z; rho1 = (double)L.w;
        xka = omega / a; xkb = omega / b;
        t = b / omega;
        gammk = 2.0 * t * t;
        gam = gammk * wvno2;
        ra = sqrt((wvno + xka) * fabs(wvno - xka));
        rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
        const double p = ra * dpth, q = rb * dpth;
        // var(): cos/sin (oscillatory) or scaled cosh/sinh (evanescent)
        double pex = 0.0, sex = 0.0, w, x, cosp, y, z, cosq;
        if (wvno < xka) {
            double sp, cp;
            sincos(p, &sp, &cp);
            w = sp / ra; x = -ra * sp; cosp = cp;
        } else if (wvno == xka) {
            cosp = 1.0; w = dpth; x = 0.0;
        } else {
            pex = p;
            double fac = (p < 16.0) ? exp(-2.0 * p) : 0.0;
            cosp = (1.0 + fac) * 0.5;
            double sinp = (1.0 - fac) * 0.5;
            w = sinp / ra; x = ra * sinp;
        }
        if (wvno < xkb) {
            double sq, cq;
            sincos(q, &sq, &cq);
            y = sq / rb; z = -rb * sq; cosq = cq;
        } else if (wvno == xkb) {
            cosq = 1.0; y = dpth; z = 0.0;
        } else {
            sex = q;
            double fac = (q < 16.0) ? exp(-2.0 * q) : 0.0;
            cosq = (1.0 + fac) * 0.5;
            double sinq = (1.0 - fac) * 0.5;
            y = sinq / rb; z = rb * sinq;
        }
        const double exa = pex + sex;
        const double a0 = (exa < 60.0) ? exp(-exa) : 0.0;
        const double cpcq = cosp * cosq, cpy = cosp * y, cpz = cosp * z;
        const double cqw = cosq * w, cqx = cosq * x;
        const double xy = x * y, xz = x * z, wy = w * y, wz = w * z;
        // dnka(): Dunkin compound matrix
        const double gamm1l = gam - 1.0, twgm1 = gam + gamm1l, gmgmk = gam * gammk;
        const double gmgm1 = gam * gamm1l, gm1sq = gamm1l * gamm1l;
        const double rinv = 1.0 / rho1, rho2 = rho1 * rho1, r2inv = rinv * rinv;
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
        // ee(i) = sum_j e(j) * ca(j,i), with ca's symmetries
        //   ca(2,5)=ca(1,4) ca(4,4)=ca(2,2) ca(4,5)=ca(1,2) ca(5,2)=ca(4,1)
        //   ca(5,4)=ca(2,1) ca(5,5)=ca(1,1)
        double f0 = e0 * c11 + e1 * c21 + e2 * c31 + e3 * c41 + e4 * c51;
        double f1 = e0 * c12 + e1 * c22 + e2 * c32 + e3 * c42 + e4 * c41;
        double f2 = e0 * c13 + e1 * c23 + e2 * c33 + e3 * c43 + e4 * c53;
        double f3 = e0 * c14 + e1 * c24 + e2 * c34 + e3 * c22 + e4 * c21;
        double f4 = e0 * c15 + e1 * c14 + e2 * c35 + e3 * c12 + e4 * c11;
        // normc()
        double t1 = fmax(fmax(fmax(fabs(f0), fabs(f1)), fmax(fabs(f2), fabs(f3))), fabs(f4));
        if (t1 < 1.0e-40) t1 = 1.0;
        const double tinv = 1.0 / t1;
        e0 = f0 * tinv; e1 = f1 * tinv; e2 = f2 * tinv; e3 = f3 * tinv; e4 = f4 * tinv;
    }
    return e0;
}

// Root-search state of one model: the reference keeps del1st in a SAVE
// variable of getsol; here it lives with the model.
struct RootState {
    double del1st;
    int evals;
};

template <class M>
__device__ __forceinline__ double secular(const M& mdl, int mmax, double c, double omega, RootState& st)
{
    st.evals++;
    return dltar4(mdl, mmax, omega / c, omega);
}

// nevill(), surfdisp96.f:551-668
template <class M>
__device__ double nevill(const M& mdl, int mmax, double t, double c1, double c2,
                         double del1, double del2, double tol, RootState& st)
{
    double x[11], y[11];
    const double omega = TWOPI / t;
    double c3 = 0.5 * (c1 + c2);
    double del3 = secular(mdl, mmax, c3, omega, st);
    int nev = 1, nctrl = 1, mm = 1;
    for (;;) {
        nctrl = nctrl + 1;
        if (nctrl >= 100) break;
        if (c3 < fmin(c1, c2) || c3 > fmax(c1, c2)) {
            nev = 0;
            c3 = 0.5 * (c1 + c2);
            del3 = secular(mdl, mmax, c3, omega, st);
        }
        const double s13 = del1 - del3;
        const double s32 = del3 - del2;
        if (fsign1(del3) * fsign1(del1) < 0.0) { c2 = c3; del2 = del3; }
        else { c1 = c3; del1 = del3; }
        if (fabs(c1 - c2) <= tol * c1) break;
        if (fsign1(s13) != fsign1(s32)) nev = 0;
        const double ss1 = fabs(del1), s1 = (double)0.01f * ss1;
        const double ss2 = fabs(del2), s2 = (double)0.01f * ss2;
        if (s1 > ss2 || s2 > ss1 || nev == 0) {
            c3 = 0.5 * (c1 + c2);
            del3 = secular(mdl, mmax, c3, omega, st);
            nev = 1; mm = 1;
        } else {
            if (nev == 2) { x[mm] = c3; y[mm] = del3; }
            else { x[0] = c1; y[0] = del1; x[1] = c2; y[1] = del2; mm = 1; }
            bool bad = false;
            for (int kk = 1; kk <= mm; ++kk) {
                const int j = mm - kk;        // 0-based
                const double denom = y[mm] - y[j];
                if (fabs(denom) < 1.0e-10 * fabs(y[mm])) { bad = true; break; }
                x[j] = (-y[j] * x[j + 1] + y[mm] * x[j]) / denom;
            }
            if (bad) {
                c3 = 0.5 * (c1 + c2);
                del3 = secular(mdl, mmax, c3, omega, st);
                nev = 1; mm = 1;
            } else {
                c3 = x[0];
                del3 = secular(mdl, mmax, c3, omega, st);
                nev = 2;
                mm = mm + 1;
                if (mm > 10) mm = 10;
            }
        }
    }
    return c3;
}

// getsol(), surfdisp96.f:384-476.  Returns true when a root was found.
template <class M>
__device__ bool getsol(const M& mdl, int mmax, double t1, double& c1io, double clow,
                       double dc, double cm, float betmx, bool ifirst, double tol,
                       RootState& st)
{
    double c1 = c1io, c2;
    const double omega = TWOPI / t1;
    double del1 = secular(mdl, mmax, c1, omega, st), del2;
    if (ifirst) st.del1st = del1;
    const double plmn = fsign1(st.del1st) * fsign1(del1);
    int idir = (ifirst || plmn >= 0.0) ? +1 : -1;
    const double cmax = (double)betmx + dc;
    // The scan is bounded by [cm, betmx + dc) as in the reference, but a
    // hard iteration cap keeps every thread finite even on degenerate input.
    for (int it = 0; it < 200000; ++it) {
        c2 = (idir > 0) ? c1 + dc : c1 - dc;
        if (c2 <= clow) { idir = +1; c1 = clow; continue; }
        del2 = secular(mdl, mmax, c2, omega, st);
        if (fsign1(del1) != fsign1(del2)) {
            c1 = nevill(mdl, mmax, t1, c1, c2, del1, del2, tol, st);
            c1io = c1;
            return !(c1 > (double)betmx);
        }
        c1 = c2;
        del1 = del2;
        if (c1 < cm || c1 >= cmax) { c1io = c1; return false; }
    }
    c1io = c1;
    return false;
}

// Scan start of a model, surfdisp96.f:139-206: slowest layer -> gtsolh ->
// backed off by 0.95 * 0.90 in single precision.  Also returns betmx.
template <class M>
__device__ void scan_start(const M& mdl, int mmax, double& cc, float& betmx)
{
    float betmn = 1.e20f;
    betmx = -1.e20f;
    int jmn = 0;
    bool jsol = true;
    for (int i = 0; i < mmax; ++i) {
        float4 L = mdl.layer(i);
        if (L.z > 0.01f && L.z < betmn) { betmn = L.z; jmn = i; jsol = true; }
        else if (L.z <= 0.01f && L.y < betmn) { betmn = L.y; jmn = i; jsol = false; }
        if (L.z > betmx) betmx = L.z;
    }
    float cc1;
    if (!jsol) cc1 = betmn;
    else { float4 L = mdl.layer(jmn); cc1 = gtsolh(L.y, L.z); }
    cc1 = __fmul_rn(0.95f, cc1);
    cc1 = __fmul_rn(0.90f, cc1);
    cc = (double)cc1;
}

// surfdisp96 period loop (Rayleigh fundamental-mode phase velocity).
// Writes c (unrounded FP64 root) for k = 0..kmax-1 through `out(k, c, evals)`
// and returns the 0-based index of the first period without a root, or -1.
// After a failure the reference sets that and all later periods to zero.
template <class M, class Out>
__device__ int surfdisp_column(const M& mdl, int mmax, const double* periods, int kmax,
                               double tol, Out out)
{
    double cc;
    float betmx;
    scan_start(mdl, mmax, cc, betmx);
    const double dc = fabs((double)0.005f);
    const double onea = 1.5;
    const double cm = cc;
    RootState st;
    st.del1st = 0.0;
    double cprev = 0.0;
    for (int k = 0; k < kmax; ++k) {
        st.evals = 0;
        double c1, clow;
        bool ifirst;
        if (k == 0) { c1 = cc; clow = cc; ifirst = true; }
        else { c1 = cprev - onea * dc; clow = cm; ifirst = false; }
        const bool ok = getsol(mdl, mmax, periods[k], c1, clow, dc, cm, betmx, ifirst, tol, st);
        if (!ok) {
            out(k, 0.0, st.evals);
            for (int kk = k + 1; kk < kmax; ++kk) out(kk, 0.0, 0);
            return k;
        }
        cprev = c1;
        out(k, c1, st.evals);
    }
    return -1;
}

}  // namespace dk
