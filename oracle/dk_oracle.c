/*
 * CPU ORACLE — test infrastructure only.
 *
 * A C restatement of DAzi's per-column dispersion and isotropic depth-kernel
 * stage, used as the checker for the CUDA library and as the timed CPU
 * baseline.  Nothing in the shipped library links, loads or calls this code.
 *
 * It follows the reference Fortran routine by routine (paths are within the
 * reference project):
 *   code/src_inv_iso_joint/surfdisp96.f   surfdisp96 :52-354, gtsolh :361-382,
 *       getsol :384-476, sphere :480-547, nevill :551-668, half :670-680,
 *       dltar4 :767-865, var :868-985, normc :989-1014, dnka :1018-1062,
 *       dltar1 (Love) :704-763
 *   code/src_inv_iso_joint/DepthKernel1D.f90  depthkernel_column_fd :102-185,
 *       depthkernel_empirical_vp_rho :187-200
 *   code/src_inv_iso_joint/CalSurfG.f90   depthkernel :1-113,
 *       refineGrid2LayerMdl :2490-2549
 *
 * Type rules kept from the Fortran: model arrays are real*4 (float) and every
 * store into them rounds to float; secular-function arithmetic is real*8;
 * implicitly-real scalars (cc0, cc1, betmn, betmx, t1a) are float; the
 * returned phase velocity is sngl(c) widened back to double.  The two SAVE
 * variables of the Fortran (del1st in getsol, dhalf in sphere) become explicit
 * per-call state, which makes the oracle re-entrant and safe under OpenMP.
 *
 * Parity status: pinned.  The phase velocities reproduce the reference's own
 * golden output examples/test4_Yunnan/voro/period_phaseVMOD.dat (tests under
 * tests/test_oracle_golden.py).
 *
 * Build: oracle/Makefile -> oracle/_build/liboracle_dk.so (gcc, -O2,
 * -ffp-contract=off so no fused multiply-add changes the rounding).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "dk_oracle.h"

#define NL 200
#define NP 160

/* Fortran DSIGN(1.0d0, x): +1 unless the sign bit of x is set. */
static inline double fsign1(double x) { return signbit(x) ? -1.0 : 1.0; }

/* ------------------------------------------------------------------------ */
/* Brocher empirical relations, DepthKernel1D.f90:187-200.  Integer powers are
 * expanded the way gfortran expands them (x^3 = x^2*x, x^4 = x^2*x^2,
 * x^5 = x^3*x^2), all in single precision.                                  */
void or_brocher(int nz, const float *vs, float *vp, float *rho)
{
    for (int k = 0; k < nz; ++k) {
        float x = vs[k];
        float x2 = x * x, x3 = x2 * x, x4 = x2 * x2;
        float t = 0.9409f + 2.0947f * x;
        t = t - 0.8206f * x2;
        t = t + 0.2683f * x3;
        t = t - 0.0251f * x4;
        vp[k] = t;
        float p = t, p2 = p * p, p3 = p2 * p, p4 = p2 * p2, p5 = p3 * p2;
        float r = 1.6612f * p - 0.4721f * p2;
        r = r + 0.0671f * p3;
        r = r - 0.0043f * p4;
        r = r + 0.000106f * p5;
        rho[k] = r;
    }
}

/* Node model -> layer stack, CalSurfG.f90:2490-2549 (refineLayerMdl in
 * CalSurfGAniso_Joint.f90:146-196 is the same plus the nsublay output).
 * Returns rmax, or -1 when the stack would exceed NL layers.               */
int or_refine(float minthk0, int nz, const float *dep, const float *vp,
              const float *vs, const float *rho, float *rthk, float *rvp,
              float *rvs, float *rrho, int *nsublay)
{
    int k = 0;
    float initdep = 0.0f;
    for (int i = 0; i < nz - 1; ++i) {
        float thk = dep[i + 1] - dep[i];
        float minthk = thk / minthk0;
        int ns = (int)((thk + 1.0e-4f) / minthk) + 1;
        if (nsublay) nsublay[i] = ns;
        if (k + ns + 1 > NL) return -1;
        float newthk = thk / (float)ns;
        float dvp = vp[i + 1] - vp[i], dvs = vs[i + 1] - vs[i];
        float drh = rho[i + 1] - rho[i];
        float den = (float)(2 * ns);
        for (int j = 1; j <= ns; ++j) {
            float odd = (float)(2 * j - 1);
            rthk[k] = newthk;
            initdep = initdep + newthk;
            rvp[k] = vp[i] + (odd * dvp) / den;
            rvs[k] = vs[i] + (odd * dvs) / den;
            rrho[k] = rho[i] + (odd * drh) / den;
            ++k;
        }
    }
    rthk[k] = 0.0f;
    rvp[k] = vp[nz - 1];
    rvs[k] = vs[nz - 1];
    rrho[k] = rho[nz - 1];
    return k + 1;
}

/* ------------------------------------------------------------------------ */
/* Layer model after Earth flattening (surfdisp96.f COMMON/modl).           */
typedef struct {
    int mmax, llw;
    int f32;              /* 1: store model values as real*4 (the reference) */
    double d[NL], a[NL], b[NL], rho[NL], rtp[NL], dtp[NL], btp[NL];
    double dhalf;         /* SAVE dhalf of sphere()                          */
    double del1st;        /* SAVE del1st of getsol()                         */
    double tol;           /* nevill relative tolerance (reference: 1e-6)     */
    long evals;           /* secular-function evaluations                    */
    long scan_evals;      /* of which getsol's bracket scan (checker counter) */
} sd_model;

/* A store into a real*4 model array; identity in exact-model mode. */
static inline double rf(const sd_model *m, double x) { return m->f32 ? (double)(float)x : x; }

/* sphere(), surfdisp96.f:480-547 */
static void sd_sphere(sd_model *m, int ifunc, int iflag)
{
    const double ar = 6370.0;
    double dr = 0.0, r0 = ar;
    int n = m->mmax;
    m->d[n - 1] = 1.0;
    if (iflag == 0) {
        for (int i = 0; i < n; ++i) {
            m->dtp[i] = m->d[i];
            m->rtp[i] = m->rho[i];
        }
        for (int i = 0; i < n; ++i) {
            dr = dr + m->d[i];
            double r1 = ar - dr;
            double z0 = ar * log(ar / r0);
            double z1 = ar * log(ar / r1);
            m->d[i] = rf(m, z1 - z0);
            double tmp = (ar + ar) / (r0 + r1);
            m->a[i] = rf(m, m->a[i] * tmp);
            m->b[i] = rf(m, m->b[i] * tmp);
            m->btp[i] = rf(m, tmp);
            r0 = r1;
        }
        m->dhalf = m->d[n - 1];
    } else {
        m->d[n - 1] = m->dhalf;
        for (int i = 0; i < n; ++i) {
            if (ifunc == 1) {
                if (m->f32) {
                    /* btp**(-5): integer power, expanded then inverted */
                    float x = (float)m->btp[i], x2 = x * x, x5 = (x2 * x) * x2;
                    m->rho[i] = (double)((float)m->rtp[i] * (1.0f / x5));
                } else {
                    m->rho[i] = m->rtp[i] * pow(m->btp[i], -5.0);
                }
            } else if (ifunc == 2) {
                if (m->f32)
                    m->rho[i] = (double)((float)m->rtp[i] * powf((float)m->btp[i], -2.275f));
                else
                    m->rho[i] = m->rtp[i] * pow(m->btp[i], (double)-2.275f);
            }
        }
    }
    m->d[n - 1] = 0.0;
}

/* gtsolh(), surfdisp96.f:361-382: Rayleigh speed of a half-space, float.   */
static float sd_gtsolh(float a, float b)
{
    float c = 0.95f * b;
    for (int i = 0; i < 5; ++i) {
        float gamma = b / a;
        float kappa = c / b;
        float k2 = kappa * kappa;
        float gk = gamma * kappa;
        float gk2 = gk * gk;
        float fac1 = sqrtf(1.0f - gk2);
        float fac2 = sqrtf(1.0f - k2);
        float tk = 2.0f - k2;
        float fr = tk * tk - (4.0f * fac1) * fac2;
        float frp = -((4.0f * tk) * kappa);
        frp = frp + (((4.0f * fac2) * gamma) * gamma) * kappa / fac1;
        frp = frp + ((4.0f * fac1) * kappa) / fac2;
        frp = frp / b;
        c = c - fr / frp;
    }
    return c;
}

/* var(), surfdisp96.f:868-985: the products the compound matrix needs.    */
typedef struct { double a0, cpcq, cpy, cpz, cqw, cqx, xy, xz, wy, wz; } sd_var;

static void sd_varf(double p, double q, double ra, double rb, double wvno,
                    double xka, double xkb, double dpth, sd_var *v,
                    double *w_out, double *cosp_out)
{
    double pex = 0.0, sex = 0.0, w = 0, x = 0, cosp = 0, sinp, y = 0, z = 0,
           cosq = 0, sinq, fac;
    if (wvno < xka) {
        sinp = sin(p); w = sinp / ra; x = -ra * sinp; cosp = cos(p);
    } else if (wvno == xka) {
        cosp = 1.0; w = dpth; x = 0.0;
    } else if (wvno > xka) {
        pex = p;
        fac = 0.0;
        if (p < 16) fac = exp(-2.0 * p);
        cosp = (1.0 + fac) * 0.5;
        sinp = (1.0 - fac) * 0.5;
        w = sinp / ra; x = ra * sinp;
    }
    if (wvno < xkb) {
        sinq = sin(q); y = sinq / rb; z = -rb * sinq; cosq = cos(q);
    } else if (wvno == xkb) {
        cosq = 1.0; y = dpth; z = 0.0;
    } else if (wvno > xkb) {
        sex = q;
        fac = 0.0;
        if (q < 16) fac = exp(-2.0 * q);
        cosq = (1.0 + fac) * 0.5;
        sinq = (1.0 - fac) * 0.5;
        y = sinq / rb; z = rb * sinq;
    }
    double exa = pex + sex;
    v->a0 = 0.0;
    if (exa < 60.0) v->a0 = exp(-exa);
    v->cpcq = cosp * cosq; v->cpy = cosp * y; v->cpz = cosp * z;
    v->cqw = cosq * w; v->cqx = cosq * x;
    v->xy = x * y; v->xz = x * z; v->wy = w * y; v->wz = w * z;
    if (w_out) *w_out = w;
    if (cosp_out) *cosp_out = cosp;
}

/* dnka(), surfdisp96.f:1018-1062: Dunkin's 5x5 compound layer matrix,
 * stored ca[row][col] with Fortran's ca(row,col).                          */
static void sd_dnka(double ca[5][5], double wvno2, double gam, double gammk,
                    double rho, const sd_var *v)
{
    const double one = 1.0, two = 2.0;
    double gamm1 = gam - one, twgm1 = gam + gamm1, gmgmk = gam * gammk;
    double gmgm1 = gam * gamm1, gm1sq = gamm1 * gamm1, rho2 = rho * rho;
    double a0pq = v->a0 - v->cpcq;
    ca[0][0] = ((v->cpcq - (two * gmgm1) * a0pq) - gmgmk * v->xz) - (wvno2 * gm1sq) * v->wy;
    ca[0][1] = (wvno2 * v->cpy - v->cqx) / rho;
    ca[0][2] = -(((twgm1 * a0pq + gammk * v->xz) + (wvno2 * gamm1) * v->wy) / rho);
    ca[0][3] = (v->cpz - wvno2 * v->cqw) / rho;
    ca[0][4] = -((((two * wvno2) * a0pq + v->xz) + (wvno2 * wvno2) * v->wy) / rho2);
    ca[1][0] = (gmgmk * v->cpz - gm1sq * v->cqw) * rho;
    ca[1][1] = v->cpcq;
    ca[1][2] = gammk * v->cpz - gamm1 * v->cqw;
    ca[1][3] = -v->wz;
    ca[1][4] = ca[0][3];
    ca[3][0] = (gm1sq * v->cpy - gmgmk * v->cqx) * rho;
    ca[3][1] = -v->xy;
    ca[3][2] = gamm1 * v->cpy - gammk * v->cqx;
    ca[3][3] = ca[1][1];
    ca[3][4] = ca[0][1];
    ca[4][0] = -((((two * gmgmk) * gm1sq) * a0pq + (gmgmk * gmgmk) * v->xz + (gm1sq * gm1sq) * v->wy) * rho2);
    ca[4][1] = ca[3][0];
    ca[4][2] = -((((gammk * gamm1) * twgm1) * a0pq + ((gam * gammk) * gammk) * v->xz + (gamm1 * gm1sq) * v->wy) * rho);
    ca[4][3] = ca[1][0];
    ca[4][4] = ca[0][0];
    double t = -two * wvno2;
    ca[2][0] = t * ca[4][2];
    ca[2][1] = t * ca[3][2];
    ca[2][2] = v->a0 + two * (v->cpcq - ca[0][0]);
    ca[2][3] = t * ca[1][2];
    ca[2][4] = t * ca[0][2];
}

/* normc(), surfdisp96.f:989-1014 (the log exponent is discarded there).   */
static void sd_normc(double ee[5])
{
    double t1 = 0.0;
    for (int i = 0; i < 5; ++i) if (fabs(ee[i]) > t1) t1 = fabs(ee[i]);
    if (t1 < 1.0e-40) t1 = 1.0;
    for (int i = 0; i < 5; ++i) ee[i] = ee[i] / t1;
}

/* dltar4(), surfdisp96.f:767-865: Rayleigh secular function F(c, T).      */
static double sd_dltar4(sd_model *m, double wvno, double omga)
{
    m->evals++;
    const int mmax = m->mmax;
    double omega = omga;
    if (omega < 1.0e-4) omega = 1.0e-4;
    double wvno2 = wvno * wvno;
    double xka = omega / (double)m->a[mmax - 1];
    double xkb = omega / (double)m->b[mmax - 1];
    double wvnop = wvno + xka, wvnom = fabs(wvno - xka);
    double ra = sqrt(wvnop * wvnom);
    wvnop = wvno + xkb; wvnom = fabs(wvno - xkb);
    double rb = sqrt(wvnop * wvnom);
    double t = (double)m->b[mmax - 1] / omega;
    double gammk = 2.0 * t * t;
    double gam = gammk * wvno2;
    double gamm1 = gam - 1.0;
    double rho1 = (double)m->rho[mmax - 1];
    double e[5], ee[5], ca[5][5];
    e[0] = (rho1 * rho1) * (gamm1 * gamm1 - ((gam * gammk) * ra) * rb);
    e[1] = -(rho1 * ra);
    e[2] = rho1 * (gamm1 - (gammk * ra) * rb);
    e[3] = rho1 * rb;
    e[4] = wvno2 - ra * rb;
    for (int mm = mmax - 2; mm >= m->llw - 1; --mm) {
        xka = omega / (double)m->a[mm];
        xkb = omega / (double)m->b[mm];
        t = (double)m->b[mm] / omega;
        gammk = 2.0 * t * t;
        gam = gammk * wvno2;
        wvnop = wvno + xka; wvnom = fabs(wvno - xka);
        ra = sqrt(wvnop * wvnom);
        wvnop = wvno + xkb; wvnom = fabs(wvno - xkb);
        rb = sqrt(wvnop * wvnom);
        double dpth = (double)m->d[mm];
        rho1 = (double)m->rho[mm];
        double p = ra * dpth, q = rb * dpth;
        sd_var v;
        sd_varf(p, q, ra, rb, wvno, xka, xkb, dpth, &v, NULL, NULL);
        sd_dnka(ca, wvno2, gam, gammk, rho1, &v);
        for (int i = 0; i < 5; ++i) {
            double cr = 0.0;
            for (int j = 0; j < 5; ++j) cr = cr + e[j] * ca[j][i];
            ee[i] = cr;
        }
        sd_normc(ee);
        for (int i = 0; i < 5; ++i) e[i] = ee[i];
    }
    if (m->llw != 1) {
        /* water layer on top, surfdisp96.f:844-861 */
        xka = omega / (double)m->a[0];
        wvnop = wvno + xka; wvnom = fabs(wvno - xka);
        ra = sqrt(wvnop * wvnom);
        double dpth = (double)m->d[0];
        rho1 = (double)m->rho[0];
        double p = ra * dpth, znul = 1.0e-5, w, cosp;
        sd_var v;
        sd_varf(p, znul, ra, znul, wvno, xka, znul, dpth, &v, &w, &cosp);
        double w0 = -rho1 * w;
        return cosp * e[0] + w0 * e[1];
    }
    return e[0];
}

/* dltar1(), surfdisp96.f:704-763: Love-wave secular function.              */
static double sd_dltar1(sd_model *m, double wvno, double omega)
{
    m->evals++;
    const int mmax = m->mmax;
    double beta1 = (double)m->b[mmax - 1], rho1 = (double)m->rho[mmax - 1];
    double xkb = omega / beta1;
    double wvnop = wvno + xkb, wvnom = fabs(wvno - xkb);
    double rb = sqrt(wvnop * wvnom);
    double e1 = rho1 * rb, e2 = 1.0 / (beta1 * beta1);
    for (int mm = mmax - 2; mm >= m->llw - 1; --mm) {
        beta1 = (double)m->b[mm];
        rho1 = (double)m->rho[mm];
        double xmu = rho1 * beta1 * beta1;
        xkb = omega / beta1;
        wvnop = wvno + xkb; wvnom = fabs(wvno - xkb);
        rb = sqrt(wvnop * wvnom);
        double q = (double)m->d[mm] * rb, sinq, y, z, cosq;
        if (wvno < xkb) {
            sinq = sin(q); y = sinq / rb; z = -rb * sinq; cosq = cos(q);
        } else if (wvno == xkb) {
            cosq = 1.0; y = (double)m->d[mm]; z = 0.0;
        } else {
            double fac = 0.0;
            if (q < 16) fac = exp(-2.0 * q);
            cosq = (1.0 + fac) * 0.5;
            sinq = (1.0 - fac) * 0.5;
            y = sinq / rb; z = rb * sinq;
        }
        double e10 = e1 * cosq + (e2 * xmu) * z;
        double e20 = (e1 * y) / xmu + e2 * cosq;
        double xnor = fabs(e10), ynor = fabs(e20);
        if (ynor > xnor) xnor = ynor;
        if (xnor < 1.0e-40) xnor = 1.0;
        e1 = e10 / xnor;
        e2 = e20 / xnor;
    }
    return e1;
}

static double sd_dltar(sd_model *m, double wvno, double omega, int ifunc)
{
    return ifunc == 1 ? sd_dltar1(m, wvno, omega) : sd_dltar4(m, wvno, omega);
}

static const double TWOPI = 2.0 * 3.141592653589793;

/* half(), surfdisp96.f:670-680 */
static void sd_half(sd_model *m, double c1, double c2, double *c3,
                    double *del3, double omega, int ifunc)
{
    *c3 = 0.5 * (c1 + c2);
    *del3 = sd_dltar(m, omega / *c3, omega, ifunc);
}

/* nevill(), surfdisp96.f:551-668: hybrid bisection / Neville refinement.  */
static double sd_nevill(sd_model *m, double t, double c1, double c2,
                        double del1, double del2, int ifunc)
{
    double x[20], y[20], c3, del3;
    double omega = TWOPI / t;
    int nev = 1, nctrl = 1, mm = 1;
    sd_half(m, c1, c2, &c3, &del3, omega, ifunc);
    for (;;) {
        nctrl = nctrl + 1;
        if (nctrl >= 100) break;
        if (c3 < fmin(c1, c2) || c3 > fmax(c1, c2)) {
            nev = 0;
            sd_half(m, c1, c2, &c3, &del3, omega, ifunc);
        }
        double s13 = del1 - del3;
        double s32 = del3 - del2;
        if (fsign1(del3) * fsign1(del1) < 0.0) {
            c2 = c3; del2 = del3;
        } else {
            c1 = c3; del1 = del3;
        }
        if (fabs(c1 - c2) <= m->tol * c1) break;
        if (fsign1(s13) != fsign1(s32)) nev = 0;
        double ss1 = fabs(del1), s1 = (double)0.01f * ss1;
        double ss2 = fabs(del2), s2 = (double)0.01f * ss2;
        if (s1 > ss2 || s2 > ss1 || nev == 0) {
            sd_half(m, c1, c2, &c3, &del3, omega, ifunc);
            nev = 1; mm = 1;
        } else {
            if (nev == 2) {
                x[mm] = c3; y[mm] = del3;
            } else {
                x[0] = c1; y[0] = del1; x[1] = c2; y[1] = del2; mm = 1;
            }
            int bad = 0;
            for (int kk = 1; kk <= mm; ++kk) {
                int j = mm - kk + 1;                 /* Fortran index */
                double denom = y[mm] - y[j - 1];
                if (fabs(denom) < 1.0e-10 * fabs(y[mm])) { bad = 1; break; }
                x[j - 1] = (-y[j - 1] * x[j] + y[mm] * x[j - 1]) / denom;
            }
            if (bad) {
                sd_half(m, c1, c2, &c3, &del3, omega, ifunc);
                nev = 1; mm = 1;
            } else {
                c3 = x[0];
                del3 = sd_dltar(m, omega / c3, omega, ifunc);
                nev = 2;
                mm = mm + 1;
                if (mm > 10) mm = 10;
            }
        }
    }
    return c3;
}

/* getsol(), surfdisp96.f:384-476.  Returns 1 on success, -1 on failure.   */
static int sd_getsol(sd_model *m, double t1, double *c1p, double clow,
                     double dc, double cm, float betmx, int ifunc, int ifirst)
{
    double c1 = *c1p, c2, del1, del2;
    double omega = TWOPI / t1;
    const long e_in = m->evals;
    del1 = sd_dltar(m, omega / c1, omega, ifunc);
    if (ifirst == 1) m->del1st = del1;
    double plmn = fsign1(m->del1st) * fsign1(del1);
    int idir;
    if (ifirst == 1) idir = +1;
    else if (plmn >= 0.0) idir = +1;
    else idir = -1;
    for (;;) {
        if (idir > 0) c2 = c1 + dc; else c2 = c1 - dc;
        if (c2 <= clow) {
            idir = +1;
            c1 = clow;
            continue;
        }
        del2 = sd_dltar(m, omega / c2, omega, ifunc);
        if (fsign1(del1) != fsign1(del2)) break;
        c1 = c2;
        del1 = del2;
        if (c1 < cm) { *c1p = c1; m->scan_evals += m->evals - e_in; return -1; }
        if (c1 >= ((double)betmx + dc)) { *c1p = c1; m->scan_evals += m->evals - e_in; return -1; }
    }
    m->scan_evals += m->evals - e_in;
    c1 = sd_nevill(m, t1, c1, c2, del1, del2, ifunc);
    *c1p = c1;
    if (c1 > (double)betmx) return -1;
    return 1;
}

/* surfdisp96(), surfdisp96.f:52-354.  Fundamental and higher modes of
 * Love (iwave=1) or Rayleigh (iwave=2) phase (igr=0) or group (igr>0)
 * velocity.  evals_per_period (may be NULL) receives the secular-function
 * evaluation count of each period.  round_f32 = 1 reproduces the reference
 * output cg(k) = sngl(c(k)); 0 returns the unrounded double root.
 * Returns 0, or the 1-based index of the first period with no root.       */
static int sd_run(const double *thkm, const double *vpm, const double *vsm,
                  const double *rhom, int nlayer, int iflsph, int iwave, int mode,
                  int igr, int kmax, const double *t, double *cg, double tol,
                  int model_f32, int round_f32, int *evals_per_period,
                  int *scan_per_period)
{
    if (nlayer < 1 || nlayer > NL || kmax < 1 || kmax > NP) return -1;
    sd_model mdl;
    sd_model *m = &mdl;
    m->mmax = nlayer;
    m->f32 = model_f32 ? 1 : 0;
    m->tol = tol;
    m->evals = 0;
    m->scan_evals = 0;
    m->del1st = 0.0;
    for (int i = 0; i < nlayer; ++i) {
        m->b[i] = vsm[i]; m->a[i] = vpm[i]; m->d[i] = thkm[i]; m->rho[i] = rhom[i];
    }
    int idispl = 0, idispr = 0;
    if (iwave == 1) idispl = kmax; else if (iwave == 2) idispr = kmax;
    const float ddc0 = 0.005f, sone0 = 1.500f, h0 = 0.005f;
    m->llw = 1;
    if (m->b[0] <= 0.0) m->llw = 2;
    const double one = 1.0e-2;
    if (iflsph == 1) sd_sphere(m, 0, 0);
    int jmn = 0, jsol = 1;
    float betmx = -1.e20f, betmn = 1.e20f;
    for (int i = 0; i < m->mmax; ++i) {
        float bi = (float)m->b[i], ai = (float)m->a[i];
        if (bi > 0.01f && bi < betmn) {
            betmn = bi; jmn = i; jsol = 1;
        } else if (bi <= 0.01f && ai < betmn) {
            betmn = ai; jmn = i; jsol = 0;
        }
        if (bi > betmx) betmx = bi;
    }
    int first_fail = 0;
    double c[NP], cb[NP];
    for (int ifunc = 1; ifunc <= 2; ++ifunc) {
        if (ifunc == 1 && idispl <= 0) continue;
        if (ifunc == 2 && idispr <= 0) continue;
        if (iflsph == 1) sd_sphere(m, ifunc, 1);
        float ddc = ddc0, sone = sone0, h = h0;
        if (sone < 0.01f) sone = 2.0f;
        double onea = (double)sone;
        float cc1;
        if (jsol == 0) cc1 = betmn;
        else cc1 = sd_gtsolh((float)m->a[jmn], (float)m->b[jmn]);
        cc1 = 0.95f * cc1;
        cc1 = 0.90f * cc1;
        double cc = (double)cc1;
        double dc = fabs((double)ddc);
        double c1 = cc, cm = cc, clow = cc;
        for (int i = 0; i < kmax; ++i) { cb[i] = 0.0; c[i] = 0.0; }
        int ift = 999;
        for (int iq = 1; iq <= mode; ++iq) {
            int is = 1, ie = kmax, k, failed = 0;
            for (k = is; k <= ie; ++k) {
                if (k >= ift) { failed = 1; break; }
                double t1 = t[k - 1];
                float t1a, t1b = 0.0f;
                if (igr > 0) {
                    t1a = (float)(t1 / (double)(1.0f + h));
                    t1b = (float)(t1 / (double)(1.0f - h));
                    t1 = (double)t1a;
                } else {
                    t1a = (float)t1;
                }
                int ifirst;
                if (k == is && iq == 1) {
                    c1 = cc; clow = cc; ifirst = 1;
                } else if (k == is && iq > 1) {
                    c1 = c[is - 1] + one * dc; clow = c1; ifirst = 1;
                } else if (k > is && iq > 1) {
                    ifirst = 0;
                    clow = c[k - 1] + one * dc;
                    c1 = c[k - 2];
                    if (c1 < clow) c1 = clow;
                } else {
                    ifirst = 0;
                    c1 = c[k - 2] - onea * dc;
                    clow = cm;
                }
                long e0 = m->evals, s0 = m->scan_evals;
                int iret = sd_getsol(m, t1, &c1, clow, dc, cm, betmx, ifunc, ifirst);
                if (scan_per_period) scan_per_period[k - 1] = (int)(m->scan_evals - s0);
                if (iret == -1) {
                    if (evals_per_period) evals_per_period[k - 1] = (int)(m->evals - e0);
                    failed = 1;
                    break;
                }
                c[k - 1] = c1;
                if (igr > 0) {
                    t1 = (double)t1b;
                    ifirst = 0;
                    clow = cb[k - 1] + one * dc;
                    c1 = c1 - onea * dc;
                    iret = sd_getsol(m, t1, &c1, clow, dc, cm, betmx, ifunc, ifirst);
                    if (iret == -1) c1 = c[k - 1];
                    cb[k - 1] = c1;
                } else {
                    c1 = 0.0;
                }
                if (evals_per_period) evals_per_period[k - 1] = (int)(m->evals - e0);
                if (scan_per_period) scan_per_period[k - 1] = (int)(m->scan_evals - s0);
                float cc0 = (float)c[k - 1];
                float ccb = (float)c1;
                if (igr == 0) {
                    cg[k - 1] = round_f32 ? (double)cc0 : c[k - 1];
                } else if (m->f32) {
                    float gvel = (1.0f / t1a - 1.0f / t1b) /
                                 (1.0f / (t1a * cc0) - 1.0f / (t1b * ccb));
                    cg[k - 1] = (double)gvel;
                } else {
                    /* exact-model checker: the same quotient of the FP64 roots
                     * in double, so that differences resolve its derivative */
                    const double ia = 1.0 / (double)t1a, ib = 1.0 / (double)t1b;
                    cg[k - 1] = (ia - ib) / (ia / c[k - 1] - ib / c1);
                }
            }
            if (failed) {
                /* surfdisp96.f:1700-1770: zero this and all later periods */
                if (iq > 1) { /* higher mode: mark and continue */ }
                if (!first_fail) first_fail = k;
                ift = k;
                for (int i = k; i <= ie; ++i) {
                    cg[i - 1] = 0.0;
                    if (evals_per_period && i > k) evals_per_period[i - 1] = 0;
                    if (scan_per_period && i > k) scan_per_period[i - 1] = 0;
                }
            }
        }
    }
    return first_fail;
}

int or_surfdisp96_ex(const float *thkm, const float *vpm, const float *vsm,
                     const float *rhom, int nlayer, int iflsph, int iwave,
                     int mode, int igr, int kmax, const double *t, double *cg,
                     double tol, int round_f32, int *evals_per_period)
{
    double d[NL], a[NL], b[NL], r[NL];
    if (nlayer < 1 || nlayer > NL) return -1;
    for (int i = 0; i < nlayer; ++i) { d[i] = thkm[i]; a[i] = vpm[i]; b[i] = vsm[i]; r[i] = rhom[i]; }
    /* the reference model is real*4 whatever the output rounding */
    return sd_run(d, a, b, r, nlayer, iflsph, iwave, mode, igr, kmax, t, cg, tol, 1,
                  round_f32, evals_per_period, NULL);
}

/* The same with the evaluation count of every period split: scan_per_period
 * receives getsol's bracket-scan evaluations (the rest of evals_per_period
 * are nevill's).  A checker counter; the arithmetic is or_surfdisp96_ex's. */
int or_surfdisp96_split(const float *thkm, const float *vpm, const float *vsm,
                        const float *rhom, int nlayer, int kmax, const double *t, double *cg,
                        int *evals_per_period, int *scan_per_period)
{
    double d[NL], a[NL], b[NL], r[NL];
    if (nlayer < 1 || nlayer > NL) return -1;
    for (int i = 0; i < nlayer; ++i) { d[i] = thkm[i]; a[i] = vpm[i]; b[i] = vsm[i]; r[i] = rhom[i]; }
    return sd_run(d, a, b, r, nlayer, 1, 2, 1, 0, kmax, t, cg, 1.0e-6, 1, 1, evals_per_period,
                  scan_per_period);
}

/* Exact-model variant (checker): double model arrays, no real*4 stores. */
int or_surfdisp96_d(const double *thkm, const double *vpm, const double *vsm,
                    const double *rhom, int nlayer, int iflsph, int kmax,
                    const double *t, double *cg, double tol)
{
    return sd_run(thkm, vpm, vsm, rhom, nlayer, iflsph, 2, 1, 0, kmax, t, cg, tol, 0, 0, NULL,
                  NULL);
}

int or_surfdisp96(const float *thkm, const float *vpm, const float *vsm,
                  const float *rhom, int nlayer, int iflsph, int iwave,
                  int mode, int igr, int kmax, const double *t, double *cg)
{
    return or_surfdisp96_ex(thkm, vpm, vsm, rhom, nlayer, iflsph, iwave,
                            mode, igr, kmax, t, cg, 1.0e-6, 1, NULL);
}

/* ------------------------------------------------------------------------ */
/* Double-precision layer split for the exact-model mode (same arithmetic as
 * or_refine without real*4 stores).                                         */
static int refine_d(double minthk0, int nz, const double *dep, const double *vp,
                    const double *vs, const double *rho, double *rthk, double *rvp,
                    double *rvs, double *rrho)
{
    int k = 0;
    for (int i = 0; i < nz - 1; ++i) {
        /* the sublayer count uses the real*4 rule so the layering is the
         * reference's */
        float thkf = (float)dep[i + 1] - (float)dep[i];
        int ns = (int)((thkf + 1.0e-4f) / (thkf / (float)minthk0)) + 1;
        if (k + ns + 1 > NL) return -1;
        double thk = dep[i + 1] - dep[i];
        for (int j = 1; j <= ns; ++j) {
            double f = (double)(2 * j - 1) / (double)(2 * ns);
            rthk[k] = thk / ns;
            rvp[k] = vp[i] + f * (vp[i + 1] - vp[i]);
            rvs[k] = vs[i] + f * (vs[i + 1] - vs[i]);
            rrho[k] = rho[i] + f * (rho[i + 1] - rho[i]);
            ++k;
        }
    }
    rthk[k] = 0.0; rvp[k] = vp[nz - 1]; rvs[k] = vs[nz - 1]; rrho[k] = rho[nz - 1];
    return k + 1;
}

/* One column: pv plus central finite-difference kernels,
 * DepthKernel1D.f90:102-185.  vp/rho given explicitly (the reference's
 * depthkernel derives them from vs by Brocher first).
 * precision 0 (the reference): real*4 model arithmetic, root to tol, output
 *   sngl(c), perturbation and divisor in single precision:
 *     vs_pert = vs -/+ 0.5*dln*vs  (float),  sen = (cg2 - cg1)/dble(dln*vs)
 * precision 1: as 0 but the roots are not rounded to FP32;
 * precision 2 (exact-model checker): the model pipeline in double, no FP32
 *   stores anywhere, divisor = the exact step.  With a tight tol and a small
 *   dln this resolves the derivative itself.                               */
int or_column_fd(int nz, const float *vs, const float *vp, const float *rho,
                 int kmax, const double *periods, int iwave, int igr,
                 const float *depz, float minthk, float dlnvs, float dlnvp,
                 float dlnrho, double tol, int precision, double *pv,
                 double *sen_vs, double *sen_vp, double *sen_rho,
                 long *evals)
{
    if (kmax > NP || nz > NL || nz < 2) return -1;
    double cg0[NP], cg1[NP], cg2[NP];
    int ev[NP];
    long tot = 0;
    const int model_f32 = precision < 2, out_f32 = precision == 0;
    double rthk[NL], rvp[NL], rvs[NL], rrho[NL];
    float fthk[NL], fvp[NL], fvs[NL], frho[NL];
    float depm[NL], vpm[NL], vsm[NL], rhom[NL];
    double ddep[NL], dvp[NL], dvs[NL], drho[NL];
    for (int i = 0; i < nz; ++i) {
        depm[i] = depz[i]; vsm[i] = vs[i]; vpm[i] = vp[i]; rhom[i] = rho[i];
        ddep[i] = depz[i]; dvs[i] = vs[i]; dvp[i] = vp[i]; drho[i] = rho[i];
    }
    /* model -> roots for the current node arrays */
#define RUN_MODEL(CG)                                                                 \
    do {                                                                              \
        int rm_;                                                                      \
        if (model_f32) {                                                              \
            rm_ = or_refine(minthk, nz, depm, vpm, vsm, rhom, fthk, fvp, fvs, frho, NULL); \
            if (rm_ < 0) return -2;                                                   \
            for (int q_ = 0; q_ < rm_; ++q_) {                                        \
                rthk[q_] = fthk[q_]; rvp[q_] = fvp[q_]; rvs[q_] = fvs[q_]; rrho[q_] = frho[q_]; \
            }                                                                         \
        } else {                                                                      \
            rm_ = refine_d(minthk, nz, ddep, dvp, dvs, drho, rthk, rvp, rvs, rrho);   \
            if (rm_ < 0) return -2;                                                   \
        }                                                                             \
        st_ = sd_run(rthk, rvp, rvs, rrho, rm_, 1, iwave, 1, igr, kmax, periods, CG,  \
                     tol, model_f32, out_f32, ev, NULL);                              \
        for (int k_ = 0; k_ < kmax; ++k_) tot += ev[k_];                              \
    } while (0)
    int st_ = 0;
    RUN_MODEL(cg0);
    const int status = st_;
    for (int k = 0; k < kmax; ++k) pv[k] = cg0[k];
    for (int i = 0; i < nz; ++i) {
        for (int par = 0; par < 3; ++par) {
            float *arr = par == 0 ? vsm : (par == 1 ? vpm : rhom);
            double *darr = par == 0 ? dvs : (par == 1 ? dvp : drho);
            const float *base = par == 0 ? vs : (par == 1 ? vp : rho);
            float dln = par == 0 ? dlnvs : (par == 1 ? dlnvp : dlnrho);
            double *sen = par == 0 ? sen_vs : (par == 1 ? sen_vp : sen_rho);
            double div;
            if (model_f32) {
                const float delta = (0.5f * dln) * base[i];
                arr[i] = base[i] - delta;
                RUN_MODEL(cg1);
                arr[i] = base[i] + delta;
                RUN_MODEL(cg2);
                arr[i] = base[i];
                div = (double)(dln * base[i]);
            } else {
                const double delta = 0.5 * (double)dln * (double)base[i];
                darr[i] = (double)base[i] - delta;
                RUN_MODEL(cg1);
                darr[i] = (double)base[i] + delta;
                RUN_MODEL(cg2);
                darr[i] = base[i];
                div = 2.0 * delta;
            }
            for (int k = 0; k < kmax; ++k)
                sen[(size_t)i * kmax + k] = (cg2[k] - cg1[k]) / div;
        }
    }
#undef RUN_MODEL
    if (evals) *evals = tot;
    return status;
}

/* depthkernel(), CalSurfG.f90:1-113 (default_fortran_fd backend), over a
 * 1-based column range [col_start, col_start+col_count) of the nx*ny grid.
 * vel is (nx,ny,nz) Fortran order; outputs are (nx*ny,kmax[,nz]) Fortran
 * order, written only for the selected columns.  vp_in/rho_in, when not
 * NULL, replace the Brocher relations (same layout as vel).
 * dln is the relative step (the reference uses 0.01, CalSurfG.f90:33-35);
 * precision as in or_column_fd (0 = the reference).
 * status_out (may be NULL, length nx*ny) receives the 1-based first failing
 * period per column, 0 when every period has a root.                       */
int or_depthkernel(int nx, int ny, int nz, const float *vel,
                   const float *vp_in, const float *rho_in, double *pvRc,
                   double *sen_vs, double *sen_vp, double *sen_rho, int iwave,
                   int igr, int kmax, const double *tRc, const float *depz,
                   float minthk, int col_start, int col_count, int nthreads,
                   double tol, int precision, float dln, int *status_out, long *evals_out)
{
    if (nx < 1 || ny < 1 || nz < 2 || nz > NL || kmax < 1 || kmax > NP) return -1;
    const long ncol = (long)nx * ny;
    if (col_start < 1 || col_count < 0 || col_start - 1 + (long)col_count > ncol) return -1;
    if (!(dln > 0.0f)) dln = 0.01f;   /* CalSurfG.f90:33-35 */
    long total_evals = 0;
    int bad = 0;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic) num_threads(nthreads) reduction(+:total_evals) reduction(|:bad)
#endif
    for (long cc = 0; cc < col_count; ++cc) {
        long post = col_start - 1 + cc;       /* 0-based column index */
        float vs[NL], vp[NL], rho[NL];
        double pv[NP];
        double *svs = malloc(sizeof(double) * 3 * (size_t)kmax * nz);
        if (!svs) { bad |= 1; continue; }
        double *svp = svs + (size_t)kmax * nz, *srh = svp + (size_t)kmax * nz;
        for (int k = 0; k < nz; ++k) vs[k] = vel[post + ncol * k];
        if (vp_in) {
            for (int k = 0; k < nz; ++k) { vp[k] = vp_in[post + ncol * k]; rho[k] = rho_in[post + ncol * k]; }
        } else {
            or_brocher(nz, vs, vp, rho);
        }
        long ev = 0;
        int st = or_column_fd(nz, vs, vp, rho, kmax, tRc, iwave, igr, depz,
                              minthk, dln, dln, dln, tol, precision, pv, svs,
                              svp, srh, &ev);
        if (st < 0) bad |= 1;
        total_evals += ev;
        if (status_out) status_out[post] = st < 0 ? -1 : st;
        for (int k = 0; k < kmax; ++k) pvRc[post + ncol * k] = pv[k];
        if (sen_vs) {
            for (int i = 0; i < nz; ++i)
                for (int k = 0; k < kmax; ++k) {
                    size_t o = (size_t)post + ncol * ((size_t)k + (size_t)kmax * i);
                    sen_vs[o] = svs[(size_t)i * kmax + k];
                    sen_vp[o] = svp[(size_t)i * kmax + k];
                    sen_rho[o] = srh[(size_t)i * kmax + k];
                }
        }
        free(svs);
    }
    if (evals_out) *evals_out = total_evals;
    return bad ? -1 : 0;
}

/* Phase velocity only, per column (depthkernel_column_phase_fd,
 * DepthKernel1D.f90:1-23), with per-(column, period) evaluation counts.    */
int or_phase(int nx, int ny, int nz, const float *vel, const float *vp_in,
             const float *rho_in, double *pvRc, int iwave, int igr, int kmax,
             const double *tRc, const float *depz, float minthk, int nthreads,
             double tol, int round_f32, int *evals_cp, int *status_out)
{
    if (nx < 1 || ny < 1 || nz < 2 || nz > NL || kmax < 1 || kmax > NP) return -1;
    const long ncol = (long)nx * ny;
    int bad = 0;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic) num_threads(nthreads) reduction(|:bad)
#endif
    for (long post = 0; post < ncol; ++post) {
        float vs[NL], vp[NL], rho[NL], rthk[NL], rvp[NL], rvs[NL], rrho[NL];
        double pv[NP];
        int ev[NP];
        for (int k = 0; k < nz; ++k) vs[k] = vel[post + ncol * k];
        if (vp_in) {
            for (int k = 0; k < nz; ++k) { vp[k] = vp_in[post + ncol * k]; rho[k] = rho_in[post + ncol * k]; }
        } else {
            or_brocher(nz, vs, vp, rho);
        }
        int rmax = or_refine(minthk, nz, depz, vp, vs, rho, rthk, rvp, rvs, rrho, NULL);
        if (rmax < 0) { bad |= 1; continue; }
        int st = or_surfdisp96_ex(rthk, rvp, rvs, rrho, rmax, 1, iwave, 1, igr,
                                  kmax, tRc, pv, tol, round_f32, ev);
        if (status_out) status_out[post] = st;
        for (int k = 0; k < kmax; ++k) {
            pvRc[post + ncol * k] = pv[k];
            if (evals_cp) evals_cp[post + ncol * k] = ev[k];
        }
    }
    return bad ? -1 : 0;
}
