/*
 * CPU ORACLE — test infrastructure only.
 *
 * C restatement of the parts of CPS tregn96 that DAzi's depthkernelTI
 * reaches, and of depthkernelTI's splice into Lsen_Gsc.  Used as the checker
 * of the CUDA TI kernel and as the CPU baseline; nothing shipped calls it.
 *
 * Reference (paths within the reference project):
 *   code/src_inv_iso_joint/tregn96.f
 *     tregn96 :52-722 (driver; hs = hr = 0, dogam, iflsph = 1)
 *     sphere_tdisp96 :774-841, bldsph :1301-1383, sprayl :1235-1299
 *     ffunc/gfunc/h1func/h2func :1385-1473, cnormc/rnormc :1475-1549
 *     svfunc :1559-1832, up :1834-1990, dnka_tregn :1992-2987
 *     evalg :2989-3164, gettiegn :3166-3361, varsv :3363-3475
 *     hska :3477-3559, down :3561-3709, gammap :3711-3775
 *     energy :3777-3994, getmat :3996-4071, intijr :4073-4245
 *   code/src_inv_iso_joint/depthkernelTI.f90:86-169 (column loop and splice)
 *   code/src_inv_iso_joint/CalSurfGAniso_Joint.f90:146-196 (refineLayerMdl)
 *
 * Scope: elastic layers only (DAzi's models have no water layer; a fluid
 * layer returns an error).  The source and receiver depths are 0, so no
 * layer is inserted (insert/srclyr/collap are identities; the reference
 * leaves hs/hr uninitialised and this is the value its defaults intend).
 * The SAVE/COMMON state of the Fortran becomes one explicit struct per call.
 * Complex arithmetic follows gfortran's rules: naive product, Smith-style
 * range-reduced quotient.
 *
 * Parity status: no golden vector of the reference pins Lsen_Gsc (its dump
 * files live outside the repository).  The restatement is checked by
 * physics against a second code path: the root of the TI secular function
 * (up()'s compound sweep) equals surfdisp96's golden-pinned root at
 * isotropic moduli, central differences of that root in A, C, F, L, N
 * equal the energy-integral partials converted to moduli, and sprayl,
 * gammap and the splice are checked in closed form (tests).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "dk_oracle.h"

#define NL 200
#define NP 160

/* ---------------------------------------------------------- complex ops */
typedef struct { double re, im; } cx;
static inline cx C(double r, double i) { cx z = {r, i}; return z; }
static inline cx cadd(cx a, cx b) { return C(a.re + b.re, a.im + b.im); }
static inline cx csub(cx a, cx b) { return C(a.re - b.re, a.im - b.im); }
static inline cx cneg(cx a) { return C(-a.re, -a.im); }
static inline cx cmul(cx a, cx b) { return C(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cx cscl(double s, cx a) { return C(s * a.re, s * a.im); }
static inline cx cdiv(cx a, cx b)
{
    /* range-reduced quotient (Smith) */
    if (fabs(b.re) >= fabs(b.im)) {
        double r = b.im / b.re, den = b.re + b.im * r;
        return C((a.re + a.im * r) / den, (a.im - a.re * r) / den);
    } else {
        double r = b.re / b.im, den = b.re * r + b.im;
        return C((a.re * r + a.im) / den, (a.im * r - a.re) / den);
    }
}
static inline double cabs_(cx a) { return hypot(a.re, a.im); }
static inline cx csqrt_(cx a) { double complex z = csqrt(a.re + I * a.im); return C(creal(z), cimag(z)); }
static inline cx cexp_(cx a) { double complex z = cexp(a.re + I * a.im); return C(creal(z), cimag(z)); }

/* -------------------------------------------------------- model state */
typedef struct {
    int mmax;
    int nsph, dogam;
    /* flattened model (COMMON/timod, double) */
    double zd[NL], zta[NL], ztc[NL], ztf[NL], ztl[NL], ztn[NL], zrho[NL];
    double zqai[NL], zqbi[NL], zfrefp[NL], zfrefs[NL];
    int iwat[NL];
    /* sphericity factors (COMMON/sphereL, real*4) */
    float vtp[NL], dtp[NL], rtp[NL];
    /* propagation results */
    cx cd[NL][5];
    double exe[NL], exa[NL];
    double vv[NL][4];
    double ur[NL], uz[NL], tz[NL], tr[NL];
    double dcdah[NL], dcdav[NL], dcdbh[NL], dcdbv[NL], dcdn[NL], dcdr[NL];
    double sumi0, sumi1, sumi2, sumi3, ugr;
    /* layer eigen-system from evalg (COMMON/emat) */
    cx e[4][4], einv[4][4], ra, rb;
} ti_state;

/* gettiegn(), tregn96.f:3166-3361 (elastic branch) */
typedef struct { cx rp, rsv, x11, x21, x31, x41, x12, x22, x32, x42, np, nsv; } tieig;

static void gettiegn(const ti_state *s, int m, double omg, double wvn, double wvno2, tieig *o)
{
    const double TA = s->zta[m], TC = s->ztc[m], TF = s->ztf[m], TL = s->ztl[m], TRho = s->zrho[m];
    cx a = C(wvn * TF / TC, 0), b = C(1.0 / TC, 0);
    cx c = C(-TRho * omg * omg + wvn * wvn * (TA - TF * TF / TC), 0);
    cx d = C(-wvn, 0), e = C(1.0 / TL, 0), f = C(-TRho * omg * omg, 0);
    cx ddef = C(wvn * wvn - TRho * omg * omg / TL, 0);
    cx aabc = C(wvn * wvn * TA / TC - TRho * omg * omg / TC, 0);
    cx bb = cadd(cadd(cscl(2.0, cmul(a, d)), cmul(e, c)), cmul(f, b));
    cx cc = cmul(ddef, aabc);
    cx srt = csqrt_(csub(cmul(bb, bb), cscl(4.0, cc)));
    if (srt.im < 0.0) srt = cneg(srt);
    cx L1, L2;
    if (bb.re < 0.0 && srt.re < 0.0) {
        L2 = cscl(0.5, csub(bb, srt));
        L1 = cabs_(L2) > 0.0 ? cdiv(cc, L2) : cscl(0.5, cadd(bb, srt));
    } else {
        L1 = cscl(0.5, cadd(bb, srt));
        L2 = cabs_(L1) > 0.0 ? cdiv(cc, L1) : cscl(0.5, csub(bb, srt));
    }
    cx xka2 = csub(C(wvno2, 0), L1), xkb2 = csub(C(wvno2, 0), L2);
    if (cabs_(xkb2) < cabs_(xka2)) { cx t = L1; L1 = L2; L2 = t; }
    cx rp = csqrt_(L1), rsv = csqrt_(L2);
    if (rp.re < 0.0) rp = cneg(rp);
    if (rsv.re < 0.0) rsv = cneg(rsv);
    cx bcaa = cadd(cmul(b, c), cmul(a, a));
    cx ddef2 = cadd(cmul(d, d), cmul(e, f));
    o->x12 = csub(cmul(b, d), cmul(a, e));
    o->x22 = csub(cmul(b, L2), cmul(e, bcaa));
    o->x32 = csub(L2, cadd(cmul(a, d), cmul(c, e)));
    o->x42 = cadd(cneg(cmul(a, L2)), cmul(d, bcaa));
    o->x11 = cadd(cneg(cmul(e, L1)), cmul(b, ddef2));
    o->x21 = csub(cmul(b, d), cmul(a, e));
    o->x31 = csub(cmul(d, L1), cmul(a, ddef2));
    o->x41 = cneg(csub(csub(L1, cmul(a, d)), cmul(b, f)));
    if (wvn != 0.0) {
        cx z = cdiv(C(wvn, 0), o->x11);
        o->x11 = cmul(o->x11, z); o->x21 = cmul(o->x21, z);
        o->x31 = cmul(o->x31, z); o->x41 = cmul(o->x41, z);
        z = cdiv(C(wvn, 0), o->x22);
        o->x12 = cmul(o->x12, z); o->x22 = cmul(o->x22, z);
        o->x32 = cmul(o->x32, z); o->x42 = cmul(o->x42, z);
    }
    o->np = csub(cmul(o->x11, o->x41), cmul(o->x21, o->x31));
    o->nsv = csub(cmul(o->x12, o->x42), cmul(o->x22, o->x32));
    o->rp = rp;
    o->rsv = rsv;
}

/* varsv(), tregn96.f:3363-3475 (elastic branch) */
typedef struct { cx cosp, cosq, rsinp, rsinq, sinpr, sinqr; double pex, svex; } tivar;

static void varsv(cx p, cx q, cx rp, cx rsv, double dm, tivar *v)
{
    double pr = p.re, pi = p.im, qr = q.re, qi = q.im;
    v->pex = pr;
    v->svex = qr;
    cx epp = C(cos(pi) / 2.0, sin(pi) / 2.0), epm = C(epp.re, -epp.im);
    cx eqp = C(cos(qi) / 2.0, sin(qi) / 2.0), eqm = C(eqp.re, -eqp.im);
    double pfac = pr < 15.0 ? exp(-2.0 * pr) : 0.0;
    v->cosp = cadd(epp, cscl(pfac, epm));
    cx sinp = csub(epp, cscl(pfac, epm));
    v->rsinp = cmul(rp, sinp);
    v->sinpr = (fabs(pr) < 1.0e-5 && cabs_(rp) < 1.0e-5) ? C(dm, 0) : cdiv(sinp, rp);
    double svfac = qr < 15.0 ? exp(-2.0 * qr) : 0.0;
    v->cosq = cadd(eqp, cscl(svfac, eqm));
    cx sinq = csub(eqp, cscl(svfac, eqm));
    v->rsinq = cmul(rsv, sinq);
    v->sinqr = (fabs(qr) < 1.0e-5 && cabs_(rsv) < 1.0e-5) ? C(dm, 0) : cdiv(sinq, rsv);
}

/* dnka_tregn(), tregn96.f:1992-2987 (elastic branch).
 * The 6x6 compound of the TI layer matrix, reduced to 5x5.  Each needed
 * element tca(I,J) is a signed sum of products x(a,k)x(b,k) x(c,l)x(d,l)
 * times a pair of trigonometric factors of modes k (P = 0) and l (SV = 1);
 * for k == l the cosh^2 - sinh^2 pair has been replaced by its exact value
 * 4 a_k^2 exp(-ex).  The terms are encoded below as
 *   {sign, a, b, k, c, d, l, fk, fl}   with f: 0 = c, 1 = s (sin/r),
 *   2 = ls (r sin), 3 = the exact same-mode factor 4 a^2 dfac,
 * and a group flag splitting "(first group) - (second group)".            */
typedef struct { signed char sg, a, b, k, c, d, l, fk, fl, grp; } tterm;

/* indices are 1-based rows of x, modes 1/2 as in the Fortran */
static const tterm T11[] = {
    {-1,1,3,1,2,4,1,3,3,0}, {-1,1,4,1,2,3,2,0,0,0}, {-1,1,4,2,2,3,1,0,0,0},
    {+1,1,3,1,2,4,2,1,1,0}, {+1,1,3,2,2,4,1,2,2,0}, {-1,1,3,2,2,4,2,3,3,0}};
static const tterm T12[] = {
    {-1,1,4,1,2,2,2,0,1,0}, {-1,1,4,2,2,2,1,0,2,0},
    {-1,1,2,1,2,4,2,0,1,1}, {-1,1,2,2,2,4,1,0,2,1}};
static const tterm T13[] = {
    {+1,1,4,1,2,1,1,3,3,0}, {+1,1,4,1,1,2,2,0,0,0}, {+1,1,4,2,2,1,1,0,0,0},
    {-1,1,1,1,2,4,2,1,1,0}, {-1,1,1,2,2,4,1,2,2,0}, {+1,1,4,2,1,2,2,3,3,0}};
static const tterm T15[] = {
    {-1,1,3,1,1,2,2,1,0,0}, {-1,1,3,2,2,1,1,2,0,0},
    {-1,1,1,1,2,3,2,1,0,1}, {-1,1,1,2,2,3,1,2,0,1}};
static const tterm T16[] = {
    {-1,1,2,1,1,2,2,0,0,0}, {-1,1,2,2,2,1,1,0,0,0}, {+1,1,1,1,2,2,2,1,1,0},
    {+1,1,1,2,2,2,1,2,2,0}, {-1,1,2,1,2,1,1,3,3,0}, {-1,1,2,2,1,2,2,3,3,0}};
static const tterm T21[] = {
    {-1,1,4,1,3,3,2,0,2,0}, {-1,1,4,2,3,3,1,0,1,0},
    {-1,1,3,1,3,4,2,1,0,1}, {-1,1,3,2,3,4,1,2,0,1}};
static const tterm T22[] = {
    {-1,1,4,1,3,2,2,0,0,0}, {+1,1,2,1,3,4,2,0,0,0}, {-1,1,4,2,3,2,1,0,0,0},
    {+1,1,2,2,3,4,1,0,0,0}};
static const tterm T23[] = {
    {+1,1,4,1,3,1,2,0,2,0}, {+1,1,4,2,3,1,1,0,1,0},
    {+1,1,1,1,3,4,2,1,0,1}, {+1,1,1,2,3,4,1,2,0,1}};
static const tterm T25[] = {
    {-1,1,3,1,3,1,2,1,2,0}, {-1,1,3,2,3,1,1,2,1,0},
    {-1,1,1,1,3,3,2,1,2,1}, {-1,1,1,2,3,3,1,2,1,1}};
static const tterm T31[] = {
    {-1,1,4,1,4,3,2,0,0,0}, {-1,1,4,2,4,3,1,0,0,0}, {+1,1,3,2,4,4,1,2,2,0},
    {+1,1,3,1,4,4,2,1,1,0}, {-1,1,4,1,4,3,1,3,3,0}, {-1,1,4,2,4,3,2,3,3,0}};
static const tterm T32[] = {
    {-1,1,4,1,4,2,2,0,1,0}, {-1,1,4,2,4,2,1,0,2,0},
    {-1,1,2,1,4,4,2,0,1,1}, {-1,1,2,2,4,4,1,0,2,1}};
static const tterm T33[] = {
    {+1,1,4,1,4,1,2,0,0,0}, {+1,1,4,2,4,1,1,0,0,0}, {-1,1,1,1,4,4,2,1,1,0},
    {-1,1,1,2,4,4,1,2,2,0}, {+1,1,4,1,4,1,1,3,3,0}, {+1,1,4,2,4,1,2,3,3,0}};
static const tterm T51[] = {
    {-1,2,4,1,4,3,2,2,0,0}, {-1,2,4,2,4,3,1,1,0,0},
    {-1,2,3,1,4,4,2,0,1,1}, {-1,2,3,2,4,4,1,0,2,1}};
static const tterm T52[] = {
    {-1,2,4,1,4,2,2,2,1,0}, {-1,2,4,2,4,2,1,1,2,0}, {+1,2,2,1,4,4,2,2,1,0},
    {+1,2,2,2,4,4,1,1,2,0}};
static const tterm T61[] = {
    {-1,3,4,1,4,3,2,0,0,0}, {-1,3,4,2,4,3,1,0,0,0}, {+1,3,3,1,4,4,2,1,1,0},
    {+1,3,3,2,4,4,1,2,2,0}, {-1,3,4,1,4,3,1,3,3,0}, {-1,3,4,2,4,3,2,3,3,0}};

static cx tca_eval(const tterm *t, int n, const cx x[5][3], const cx fac[3][4])
{
    cx g[2] = {C(0, 0), C(0, 0)};
    for (int i = 0; i < n; ++i) {
        cx v = cmul(cmul(x[t[i].a][t[i].k], x[t[i].b][t[i].k]),
                    cmul(x[t[i].c][t[i].l], x[t[i].d][t[i].l]));
        if (t[i].sg < 0) v = cneg(v);
        if (t[i].fk == 3) {
            v = cmul(v, fac[t[i].k][3]);           /* 4 a_k^2 dfac */
        } else {
            v = cmul(cmul(v, fac[t[i].k][t[i].fk]), fac[t[i].l][t[i].fl]);
        }
        g[t[i].grp] = cadd(g[t[i].grp], v);
    }
    return csub(g[0], g[1]);
}

static void dnka_tregn(cx CA[5][5], const tivar *v, const tieig *E, double ex)
{
    double dfac = ex > 35.0 ? 0.0 : exp(-ex);
    cx a1 = cdiv(C(0.5, 0), E->np), a2 = cdiv(C(0.5, 0), E->nsv);
    cx fac[3][4];
    /* mode 1 (P): c1, s1l, ls1; mode 2 (SV): c2, s2l, ls2 */
    fac[1][0] = cmul(cscl(2.0, a1), v->cosp);
    fac[1][1] = cmul(cscl(2.0, a1), v->sinpr);
    fac[1][2] = cmul(cscl(2.0, a1), v->rsinp);
    fac[1][3] = cscl(4.0 * dfac, cmul(a1, a1));
    fac[2][0] = cmul(cscl(2.0, a2), v->cosq);
    fac[2][1] = cmul(cscl(2.0, a2), v->sinqr);
    fac[2][2] = cmul(cscl(2.0, a2), v->rsinq);
    fac[2][3] = cscl(4.0 * dfac, cmul(a2, a2));
    cx x[5][3];
    x[1][1] = E->x11; x[2][1] = E->x21; x[3][1] = E->x31; x[4][1] = E->x41;
    x[1][2] = E->x12; x[2][2] = E->x22; x[3][2] = E->x32; x[4][2] = E->x42;
#define EV(T) tca_eval(T, (int)(sizeof(T) / sizeof(T[0])), x, fac)
    cx t11 = EV(T11), t12 = EV(T12), t13 = EV(T13), t15 = EV(T15), t16 = EV(T16);
    cx t21 = EV(T21), t22 = EV(T22), t23 = EV(T23), t25 = EV(T25);
    cx t31 = EV(T31), t32 = EV(T32), t33 = EV(T33), t51 = EV(T51), t52 = EV(T52), t61 = EV(T61);
#undef EV
    CA[0][0] = t11; CA[0][1] = t12; CA[0][2] = t13; CA[0][3] = t15; CA[0][4] = t16;
    CA[1][0] = t21; CA[1][1] = t22; CA[1][2] = t23; CA[1][3] = t25; CA[1][4] = t15;
    CA[2][0] = cscl(2.0, t31); CA[2][1] = cscl(2.0, t32);
    CA[2][2] = csub(cscl(2.0, t33), C(dfac, 0));
    CA[2][3] = cscl(-2.0, t23); CA[2][4] = cscl(-2.0, t13);
    CA[3][0] = t51; CA[3][1] = t52; CA[3][2] = cneg(t32); CA[3][3] = t22; CA[3][4] = t12;
    CA[4][0] = t61; CA[4][1] = t51; CA[4][2] = cneg(t31); CA[4][3] = t21; CA[4][4] = t11;
}

/* evalg(), tregn96.f:2989-3164: E, E^-1 of layer m (COMMON/emat) and the
 * half-space compound vector gbr (elastic). */
static void evalg(ti_state *s, int m, double wvno, double om, double om2, double wvno2, cx gbr[5])
{
    tieig E;
    gettiegn(s, m, om, wvno, wvno2, &E);
    s->ra = E.rp;
    s->rb = E.rsv;
    cx rp = E.rp, rsv = E.rsv;
    cx d1 = cmul(cscl(2.0, rp), E.np), d2 = cmul(cscl(2.0, rsv), E.nsv);
    cx d3 = cmul(cscl(-2.0, rp), E.np), d4 = cmul(cscl(-2.0, rsv), E.nsv);
    cx G[4][4];
    G[0][0] = cdiv(cmul(E.x41, rp), d1);  G[1][0] = cdiv(E.x42, d2);
    G[2][0] = cdiv(cneg(cmul(E.x41, rp)), d3); G[3][0] = cdiv(E.x42, d4);
    G[0][1] = cdiv(cneg(E.x31), d1);      G[1][1] = cdiv(cneg(cmul(E.x32, rsv)), d2);
    G[2][1] = cdiv(cneg(E.x31), d3);      G[3][1] = cdiv(cmul(E.x32, rsv), d4);
    G[0][2] = cdiv(cneg(cmul(E.x21, rp)), d1); G[1][2] = cdiv(cneg(E.x22), d2);
    G[2][2] = cdiv(cmul(E.x21, rp), d3);  G[3][2] = cdiv(cneg(E.x22), d4);
    G[0][3] = cdiv(E.x11, d1);            G[1][3] = cdiv(cmul(E.x12, rsv), d2);
    G[2][3] = cdiv(E.x11, d3);            G[3][3] = cdiv(cneg(cmul(E.x12, rsv)), d4);
    s->e[0][0] = E.x11; s->e[1][0] = cmul(E.x21, rp); s->e[2][0] = E.x31; s->e[3][0] = cmul(E.x41, rp);
    s->e[0][1] = cmul(E.x12, rsv); s->e[1][1] = E.x22; s->e[2][1] = cmul(E.x32, rsv); s->e[3][1] = E.x42;
    s->e[0][2] = E.x11; s->e[1][2] = cneg(cmul(E.x21, rp)); s->e[2][2] = E.x31; s->e[3][2] = cneg(cmul(E.x41, rp));
    s->e[0][3] = cneg(cmul(E.x12, rsv)); s->e[1][3] = E.x22; s->e[2][3] = cneg(cmul(E.x32, rsv)); s->e[3][3] = E.x42;
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) s->einv[i][j] = G[i][j];
    if (gbr) {
        gbr[0] = csub(cmul(G[0][0], G[1][1]), cmul(G[0][1], G[1][0]));
        gbr[1] = csub(cmul(G[0][0], G[1][2]), cmul(G[0][2], G[1][0]));
        gbr[2] = csub(cmul(G[0][0], G[1][3]), cmul(G[0][3], G[1][0]));
        /* CG(4) = G12 G23 - G13 G22 is not used */
        gbr[3] = csub(cmul(G[0][1], G[1][3]), cmul(G[0][3], G[1][1]));
        gbr[4] = csub(cmul(G[0][2], G[1][3]), cmul(G[0][3], G[1][2]));
    }
}

/* cnormc()/rnormc(), tregn96.f:1475-1549 */
static double cnormc(cx *ee, int n)
{
    double t1 = 0.0;
    for (int i = 0; i < n; ++i) if (cabs_(ee[i]) > t1) t1 = cabs_(ee[i]);
    if (t1 < 1.0e-40) t1 = 1.0;
    for (int i = 0; i < n; ++i) ee[i] = C(ee[i].re / t1, ee[i].im / t1);
    return log(t1);
}
static double rnormc(double *ee, int n)
{
    double t1 = 0.0;
    for (int i = 0; i < n; ++i) if (fabs(ee[i]) > t1) t1 = fabs(ee[i]);
    if (t1 < 1.0e-40) t1 = 1.0;
    for (int i = 0; i < n; ++i) ee[i] = ee[i] / t1;
    return log(t1);
}

/* up(), tregn96.f:1834-1990: compound vectors from the half-space up. */
static double up(ti_state *s, double omega, double wvno)
{
    const int mmax = s->mmax;
    double wvno2 = wvno * wvno, om2 = omega * omega;
    cx gbr[5];
    evalg(s, mmax - 1, wvno, omega, om2, wvno2, gbr);
    for (int i = 0; i < 5; ++i) s->cd[mmax - 1][i] = C(gbr[i].re, 0);
    s->exe[mmax - 1] = 0.0;
    double exsum = 0.0;
    for (int m = mmax - 2; m >= 0; --m) {
        tieig E;
        gettiegn(s, m, omega, wvno, wvno2, &E);
        cx p = cscl(s->zd[m], E.rp), q = cscl(s->zd[m], E.rsv);
        tivar v;
        varsv(p, q, E.rp, E.rsv, s->zd[m], &v);
        cx CA[5][5];
        dnka_tregn(CA, &v, &E, v.pex + v.svex);
        cx ee[5];
        for (int i = 0; i < 5; ++i) {
            cx cr = C(0, 0);
            for (int j = 0; j < 5; ++j) cr = cadd(cr, cmul(s->cd[m + 1][j], CA[j][i]));
            ee[i] = cr;
        }
        double exn = cnormc(ee, 5);
        exsum = exsum + v.pex + v.svex + exn;
        s->exe[m] = exsum;
        for (int i = 0; i < 5; ++i) s->cd[m][i] = ee[i];
    }
    return s->cd[0][0].re;
}

/* hska(), tregn96.f:3477-3559 (elastic): real 4x4 Haskell matrix. */
static void hska(double AA[4][4], cx tcosp, cx trsinp, cx tsinpr, cx tcossv, cx trsinsv,
                 cx tsinsvr, const tieig *E)
{
    cx cosp = cdiv(tcosp, E->np), sinpr = cdiv(tsinpr, E->np), rsinp = cdiv(trsinp, E->np);
    cx cossv = cdiv(tcossv, E->nsv), sinsvr = cdiv(tsinsvr, E->nsv), rsinsv = cdiv(trsinsv, E->nsv);
    const cx x11 = E->x11, x21 = E->x21, x31 = E->x31, x41 = E->x41;
    const cx x12 = E->x12, x22 = E->x22, x32 = E->x32, x42 = E->x42;
    AA[0][0] = cadd(cmul(cmul(x11, x41), cosp), cmul(cmul(x12, x42), cossv)).re;
    AA[0][1] = csub(cneg(cmul(cmul(x11, x31), sinpr)), cmul(cmul(x12, x32), rsinsv)).re;
    AA[0][2] = csub(cneg(cmul(cmul(x11, x21), cosp)), cmul(cmul(x12, x22), cossv)).re;
    AA[0][3] = cadd(cmul(cmul(x11, x11), sinpr), cmul(cmul(x12, x12), rsinsv)).re;
    AA[1][0] = cadd(cmul(cmul(x21, x41), rsinp), cmul(cmul(x22, x42), sinsvr)).re;
    AA[1][1] = csub(cneg(cmul(cmul(x21, x31), cosp)), cmul(cmul(x22, x32), cossv)).re;
    AA[1][2] = csub(cneg(cmul(cmul(x21, x21), rsinp)), cmul(cmul(x22, x22), sinsvr)).re;
    AA[2][0] = cadd(cmul(cmul(x31, x41), cosp), cmul(cmul(x32, x42), cossv)).re;
    AA[2][1] = csub(cneg(cmul(cmul(x31, x31), sinpr)), cmul(cmul(x32, x32), rsinsv)).re;
    AA[3][0] = cadd(cmul(cmul(x41, x41), rsinp), cmul(cmul(x42, x42), sinsvr)).re;
    AA[1][3] = -AA[0][2];
    AA[2][2] = AA[1][1];
    AA[2][3] = -AA[0][1];
    AA[3][1] = -AA[2][0];
    AA[3][2] = -AA[1][0];
    AA[3][3] = AA[0][0];
}

/* down(), tregn96.f:3561-3709: first column of the Haskell product. */
static void down(ti_state *s, double omega, double wvno)
{
    const int mmax = s->mmax;
    double om2 = omega * omega, wvno2 = wvno * wvno;
    s->vv[0][0] = 1.0; s->vv[0][1] = 0.0; s->vv[0][2] = 0.0; s->vv[0][3] = 0.0;
    s->exa[0] = 0.0;
    double exsum = 0.0;
    for (int m = 0; m < mmax - 1; ++m) {
        tieig E;
        gettiegn(s, m, omega, wvno, wvno2, &E);
        cx p = cscl(s->zd[m], E.rp), q = cscl(s->zd[m], E.rsv);
        tivar v;
        varsv(p, q, E.rp, E.rsv, s->zd[m], &v);
        double AA[4][4], cpex;
        if (v.pex > v.svex) {
            double dfac = (v.pex - v.svex) > 40.0 ? 0.0 : exp(-(v.pex - v.svex));
            cpex = v.pex;
            hska(AA, v.cosp, v.rsinp, v.sinpr, cscl(dfac, v.cosq), cscl(dfac, v.rsinq),
                 cscl(dfac, v.sinqr), &E);
        } else {
            double dfac = (v.svex - v.pex) > 40.0 ? 0.0 : exp(-(v.svex - v.pex));
            cpex = v.svex;
            hska(AA, cscl(dfac, v.cosp), cscl(dfac, v.rsinp), cscl(dfac, v.sinpr), v.cosq,
                 v.rsinq, v.sinqr, &E);
        }
        double aa0[4];
        for (int i = 0; i < 4; ++i) {
            double cc = 0.0;
            for (int j = 0; j < 4; ++j) cc = cc + AA[i][j] * s->vv[m][j];
            aa0[i] = cc;
        }
        double ex2 = rnormc(aa0, 4);
        exsum = exsum + cpex + ex2;
        s->exa[m + 1] = exsum;
        for (int i = 0; i < 4; ++i) s->vv[m + 1][i] = aa0[i];
    }
}

/* svfunc(), tregn96.f:1559-1832: eigenfunctions at every interface. */
static void svfunc(ti_state *s, double omega, double wvno)
{
    up(s, omega, wvno);
    down(s, omega, wvno);
    const int mmax = s->mmax;
    double f1213 = -s->cd[0][1].re;
    s->ur[0] = cdiv(s->cd[0][2], s->cd[0][1]).re;
    s->uz[0] = 1.0; s->tz[0] = 0.0; s->tr[0] = 0.0;
    for (int i = 1; i < mmax; ++i) {
        double cd1 = s->cd[i][0].re, cd2 = s->cd[i][1].re, cd3 = s->cd[i][2].re;
        double cd4 = -s->cd[i][2].re, cd5 = s->cd[i][3].re, cd6 = s->cd[i][4].re;
        double tz1 = -s->vv[i][3], tz2 = -s->vv[i][2], tz3 = s->vv[i][1], tz4 = s->vv[i][0];
        double uu1 = tz2 * cd6 - tz3 * cd5 + tz4 * cd4;
        double uu2 = -tz1 * cd6 + tz3 * cd3 - tz4 * cd2;
        double uu3 = tz1 * cd5 - tz2 * cd3 + tz4 * cd1;
        double uu4 = -tz1 * cd4 + tz2 * cd2 - tz3 * cd1;
        double ext = s->exa[i] + s->exe[i] - s->exe[0];
        if (ext > -80.0 && ext < 80.0) {
            double fact = exp(ext);
            s->ur[i] = uu1 * fact / f1213;
            s->uz[i] = uu2 * fact / f1213;
            s->tz[i] = uu3 * fact / f1213;
            s->tr[i] = uu4 * fact / f1213;
        } else {
            s->ur[i] = s->uz[i] = s->tz[i] = s->tr[i] = 0.0;
        }
    }
}

/* ffunc/gfunc/h1func/h2func, tregn96.f:1385-1473 */
static cx ffunc(cx nub, double dm)
{
    if (cabs_(nub) < 1.0e-08) return C(dm, 0);
    cx arg = cscl(dm, nub);
    cx exqq = arg.re < 40.0 ? cexp_(cscl(-2.0, arg)) : C(0, 0);
    return cdiv(csub(C(1, 0), exqq), cscl(2.0, nub));
}
static cx gfunc(cx nub, double dm)
{
    cx arg = cscl(dm, nub);
    if (arg.re < 75.0) return cscl(dm, cexp_(cneg(arg)));
    return C(0, 0);
}
static cx h1func(cx nua, cx nub, double dm)
{
    cx s = cadd(nub, nua);
    if (cabs_(s) < 1.0e-08) return C(dm, 0);
    cx arg = cscl(dm, cadd(nua, nub));
    cx exqq = arg.re < 40.0 ? cexp_(cneg(arg)) : C(0, 0);
    return cdiv(csub(C(1, 0), exqq), s);
}
static cx h2func(cx nua, cx nub, double dm)
{
    if (cabs_(csub(nub, nua)) < 1.0e-08) return C(dm, 0);
    cx arg = cscl(dm, nua);
    cx exqp = arg.re < 40.0 ? cexp_(cneg(arg)) : C(0, 0);
    arg = cscl(dm, nub);
    cx exqq = arg.re < 40.0 ? cexp_(cneg(arg)) : C(0, 0);
    return cdiv(csub(exqq, exqp), csub(nua, nub));
}

/* intijr(), tregn96.f:4073-4245 (elastic).  The six integrals a layer
 * needs, sharing one evalg call. */
static void intijr6(ti_state *s, int m, int typelyr, double om, double om2, double wvno,
                    double wvno2, double out[6])
{
    static const int IJ[6][2] = {{1, 1}, {1, 3}, {2, 2}, {2, 4}, {3, 3}, {4, 4}};
    evalg(s, m, wvno, om, om2, wvno2, NULL);
    cx (*e)[4] = s->e;
    cx (*ei)[4] = s->einv;
    cx ra = s->ra, rb = s->rb;
    for (int q = 0; q < 6; ++q) {
        const int i = IJ[q][0] - 1, j = IJ[q][1] - 1;
        cx r;
        if (typelyr == 0) {
            cx km1pd = cadd(cadd(cscl(s->ur[m], ei[2][0]), cscl(s->uz[m], ei[2][1])),
                            cadd(cscl(s->tz[m], ei[2][2]), cscl(s->tr[m], ei[2][3])));
            cx km1sd = cadd(cadd(cscl(s->ur[m], ei[3][0]), cscl(s->uz[m], ei[3][1])),
                            cadd(cscl(s->tz[m], ei[3][2]), cscl(s->tr[m], ei[3][3])));
            cx kmpu = cadd(cadd(cscl(s->ur[m + 1], ei[0][0]), cscl(s->uz[m + 1], ei[0][1])),
                           cadd(cscl(s->tz[m + 1], ei[0][2]), cscl(s->tr[m + 1], ei[0][3])));
            cx kmsu = cadd(cadd(cscl(s->ur[m + 1], ei[1][0]), cscl(s->uz[m + 1], ei[1][1])),
                           cadd(cscl(s->tz[m + 1], ei[1][2]), cscl(s->tr[m + 1], ei[1][3])));
            cx FA = ffunc(ra, s->zd[m]), GA = gfunc(ra, s->zd[m]);
            cx FB = ffunc(rb, s->zd[m]), GB = gfunc(rb, s->zd[m]);
            cx H1 = h1func(ra, rb, s->zd[m]), H2 = h2func(ra, rb, s->zd[m]);
#define EE(a, b) cmul(e[i][a], e[j][b])
#define SYM(a, b) cadd(EE(a, b), EE(b, a))
            r = cmul(cmul(EE(0, 0), cmul(kmpu, kmpu)), FA);
            r = cadd(r, cmul(cmul(EE(2, 2), cmul(km1pd, km1pd)), FA));
            r = cadd(r, cmul(cmul(EE(1, 1), cmul(kmsu, kmsu)), FB));
            r = cadd(r, cmul(cmul(EE(3, 3), cmul(km1sd, km1sd)), FB));
            r = cadd(r, cmul(H1, cadd(cmul(SYM(0, 1), cmul(kmpu, kmsu)),
                                      cmul(SYM(2, 3), cmul(km1pd, km1sd)))));
            r = cadd(r, cmul(H2, cadd(cmul(SYM(0, 3), cmul(kmpu, km1sd)),
                                      cmul(SYM(1, 2), cmul(km1pd, kmsu)))));
            r = cadd(r, cmul(GA, cmul(SYM(0, 2), cmul(kmpu, km1pd))));
            r = cadd(r, cmul(GB, cmul(SYM(1, 3), cmul(kmsu, km1sd))));
        } else {
            cx km1pd = cadd(cadd(cscl(s->ur[m], ei[2][0]), cscl(s->uz[m], ei[2][1])),
                            cadd(cscl(s->tz[m], ei[2][2]), cscl(s->tr[m], ei[2][3])));
            cx km1sd = cadd(cadd(cscl(s->ur[m], ei[3][0]), cscl(s->uz[m], ei[3][1])),
                            cadd(cscl(s->tz[m], ei[3][2]), cscl(s->tr[m], ei[3][3])));
            r = cdiv(cmul(EE(2, 2), cmul(km1pd, km1pd)), cscl(2.0, ra));
            r = cadd(r, cdiv(cmul(SYM(2, 3), cmul(km1pd, km1sd)), cadd(ra, rb)));
            r = cadd(r, cdiv(cmul(EE(3, 3), cmul(km1sd, km1sd)), cscl(2.0, rb)));
#undef EE
#undef SYM
        }
        out[q] = r.re;
    }
}

/* energy(), tregn96.f:3777-3994 (elastic) with getmat() :3996-4071 */
static void energy(ti_state *s, double om, double wvno)
{
    const int mmax = s->mmax;
    double sumi0 = 0, sumi1 = 0, sumi2 = 0, sumi3 = 0;
    double c = om / wvno, om2 = om * om, wvno2 = wvno * wvno;
    for (int m = 0; m < mmax; ++m) {
        double TA = s->zta[m], TC = s->ztc[m], TF = s->ztf[m], TL = s->ztl[m], TN = s->ztn[m];
        double rho = s->zrho[m];
        double ah = sqrt(TA / rho), av = sqrt(TC / rho), bh = sqrt(TN / rho), bv = sqrt(TL / rho);
        double eta = TF / (TA - 2.0 * TL);
        double a12 = -wvno, a14 = 1.0 / TL, a21 = wvno * TF / TC, a23 = 1.0 / TC;
        int typelyr = (m == mmax - 1) ? 1 : 0;
        double ints[6];
        intijr6(s, m, typelyr, om, om2, wvno, wvno2, ints);
        double INT11 = ints[0], INT13 = ints[1], INT22 = ints[2], INT24 = ints[3], INT33 = ints[4], INT44 = ints[5];
        double URUR = INT11, UZUZ = INT22;
        double DURDUR = a12 * a12 * INT22 + 2.0 * a12 * a14 * INT24 + a14 * a14 * INT44;
        double DUZDUZ = a21 * a21 * INT11 + 2.0 * a21 * a23 * INT13 + a23 * a23 * INT33;
        double URDUZ = a21 * INT11 + a23 * INT13;
        double UZDUR = a12 * INT22 + a14 * INT24;
        sumi0 = sumi0 + rho * (URUR + UZUZ);
        sumi1 = sumi1 + TL * UZUZ + TA * URUR;
        sumi2 = sumi2 + TL * UZDUR - TF * URDUZ;
        sumi3 = sumi3 + TL * DURDUR + TC * DUZDUZ;
        double facah = rho * ah * (URUR - 2.0 * eta * URDUZ / wvno);
        double facav = rho * av * DUZDUZ / wvno2;
        double facbh = 0.0;
        double facbv = rho * bv * (UZUZ + 2.0 * UZDUR / wvno + DURDUR / wvno2 + 4.0 * eta * URDUZ / wvno);
        double facn = -TF * URDUZ / (wvno * eta);
        s->dcdah[m] = facah; s->dcdav[m] = facav; s->dcdbh[m] = facbh;
        s->dcdbv[m] = facbv; s->dcdn[m] = facn;
        double facr = -0.5 * c * c * (URUR + UZUZ);
        s->dcdr[m] = 0.5 * (av * facav + ah * facah + bv * facbv) / rho + facr;
    }
    s->ugr = (wvno * sumi1 + sumi2) / (om * sumi0);
    for (int m = 0; m < mmax; ++m) {
        double u = s->ugr * sumi0;
        s->dcdah[m] /= u; s->dcdav[m] /= u; s->dcdbh[m] /= u;
        s->dcdbv[m] /= u; s->dcdr[m] /= u; s->dcdn[m] /= u;
    }
    s->sumi0 = sumi0; s->sumi1 = sumi1; s->sumi2 = sumi2; s->sumi3 = sumi3;
}

/* gammap(), tregn96.f:3711-3775: Q-dispersion shift of c (changes wvno). */
static double gammap(ti_state *s, double omega, double *wvno)
{
    double dc = 0.0;
    const double pi = 3.141592653589493;   /* sic, as in the reference */
    for (int m = 0; m < s->mmax; ++m) {
        double TA = s->zta[m], TC = s->ztc[m], TL = s->ztl[m], TN = s->ztn[m], rho = s->zrho[m];
        double ah = sqrt(TA / rho), av = sqrt(TC / rho), bh = sqrt(TN / rho), bv = sqrt(TL / rho);
        if (s->iwat[m] == 0) {
            double x = s->dcdbh[m] * bh * s->zqbi[m] + s->dcdbv[m] * bv * s->zqbi[m];
            double omgref = 2.0 * pi * s->zfrefs[m];
            dc = dc + log(omega / omgref) * x / pi;
        }
        double x = s->dcdav[m] * av * s->zqai[m] + s->dcdah[m] * ah * s->zqai[m];
        double omgref = 2.0 * pi * s->zfrefp[m];
        dc = dc + log(omega / omgref) * x / pi;
    }
    double c = omega / *wvno;
    c = c + dc;
    *wvno = omega / c;
    return dc;
}

/* tregn96 driver for one column, tregn96.f:52-722 (see the file header for
 * the scope).  Outputs dcdah/dcdbv/dcdn as real*4 (np x nl, period-major:
 * out[k*nl + layer]).  nsph / dogam switch sphericity and Q (the reference
 * uses 1 / 1).  Returns 0, or -1 on a fluid layer or bad sizes.           */
static int tregn96_run(int nl, const float *d_in, const float *TA_in, const float *TC_in,
                       const float *TF_in, const float *TL_in, const float *TN_in,
                       const float *TRho_in, const float *qai_in, const float *qbi_in,
                       const float *etapi_in, const float *etasi_in, const float *frefpi_in,
                       const float *frefsi_in, int nt, const float *t_in, const float *cp_in,
                       const double *cp_d, float *dcdah_out, float *dcdbv_out,
                       float *dcdn_out, int nsph, int dogam, double *full)
{
    if (nl < 2 || nl > NL || nt < 1 || nt > NP) return -1;
    ti_state *s = calloc(1, sizeof(ti_state));
    if (!s) return -1;
    s->mmax = nl;
    s->nsph = nsph;
    s->dogam = dogam;
    float d[NL], TA[NL], TC[NL], TF[NL], TN[NL], TL[NL], TRho[NL], qai[NL], qbi[NL];
    float frefpi[NL], frefsi[NL];
    for (int i = 0; i < nl; ++i) {
        d[i] = d_in[i]; TA[i] = TA_in[i]; TC[i] = TC_in[i]; TF[i] = TF_in[i];
        TN[i] = TN_in[i]; TL[i] = TL_in[i]; TRho[i] = TRho_in[i];
        qai[i] = qai_in[i]; qbi[i] = qbi_in[i];
        frefpi[i] = frefpi_in[i]; frefsi[i] = frefsi_in[i];
        if (TN[i] <= 1.0e-4f * TA[i]) { free(s); return -1; }   /* fluid: out of scope */
    }
    (void)etapi_in; (void)etasi_in;
    for (int i = 0; i < nl; ++i) {
        if (!dogam) { qai[i] = 0.0f; qbi[i] = 0.0f; }
        if (qai[i] > 1.0f) qai[i] = 1.0f / qai[i];
        if (qbi[i] > 1.0f) qbi[i] = 1.0f / qbi[i];
        s->zqai[i] = qai[i];
        s->zqbi[i] = qbi[i];
        if (frefpi[i] <= 0.0f) frefpi[i] = 1.0f;
        if (frefsi[i] <= 0.0f) frefsi[i] = 1.0f;
        s->zfrefp[i] = frefpi[i];
        s->zfrefs[i] = frefsi[i];
    }
    if (nsph > 0) {
        /* sphere_tdisp96(), tregn96.f:774-841, Rayleigh (ifunc = 2) */
        const float radius = 6371.0f;
        const double ar = radius;
        double r0 = ar + 0.0;
        d[nl - 1] = 1.0f;
        for (int i = 0; i < nl; ++i) {
            double r1 = r0 - (double)d[i];
            double z0 = ar * log(ar / r0);
            double z1 = ar * log(ar / r1);
            d[i] = (float)(z1 - z0);
            double tmp = (ar + ar) / (r0 + r1);
            float rhosph = TRho[i];
            TRho[i] = (float)((double)rhosph * pow(tmp, (double)(-2.275f)));
            const double f275 = pow(tmp, (double)(-0.2750f));
            TA[i] = (float)((double)TA[i] * f275);
            TC[i] = (float)((double)TC[i] * f275);
            float elsph = TL[i];
            TL[i] = (float)((double)elsph * f275);
            float ensph = TN[i];
            TN[i] = (float)((double)ensph * f275);
            r0 = r1;
        }
        d[nl - 1] = 0.0f;
    }
    for (int i = 0; i < nl; ++i) {
        s->zd[i] = d[i]; s->zta[i] = TA[i]; s->ztc[i] = TC[i]; s->ztl[i] = TL[i];
        s->ztn[i] = TN[i]; s->ztf[i] = TF[i]; s->zrho[i] = TRho[i];
        s->iwat[i] = (TN[i] < 0.0001f * TA[i]) ? 1 : 0;
    }
    if (nsph > 0) {
        /* bldsph(), tregn96.f:1301-1383 */
        const double ar = 6370.0;
        double r0 = ar;
        s->zd[nl - 1] = 1.0;
        for (int i = 0; i < nl; ++i) {
            double r1 = r0 * exp(-s->zd[i] / ar);
            double tmp = (ar + ar) / (r0 + r1);
            s->vtp[i] = (float)tmp;
            s->rtp[i] = (float)pow(tmp, (double)(-2.275f));
            s->dtp[i] = (float)(ar / r0);
            r0 = r1;
        }
        /* bldsph leaves zd(mmax) = 1.0: the half-space thickness is then only
         * read by intijr's half-space branch, which does not use it */
    }
    const float twopi = 2.0f * 3.141592654f;
    for (int k = 0; k < nt; ++k) {
        double t = (double)t_in[k];
        double omega = (double)twopi / t;
        double c = cp_d ? cp_d[k] : (double)cp_in[k];
        double wvno = omega / c;
        svfunc(s, omega, wvno);
        energy(s, omega, wvno);
        if (dogam) {
            gammap(s, omega, &wvno);
            c = omega / wvno;
        }
        if (nsph > 0) {
            /* sprayl(), tregn96.f:1235-1299 */
            const double ar = 6370.0;
            double tm = sqrt(1. + pow(c / (2. * ar * omega), 2));
            double tm3 = tm * tm * tm;
            for (int i = 0; i < nl; ++i) {
                s->dcdah[i] = s->dcdah[i] * (double)s->vtp[i] / tm3;
                s->dcdav[i] = s->dcdav[i] * (double)s->vtp[i] / tm3;
                s->dcdbh[i] = s->dcdbh[i] * (double)s->vtp[i] / tm3;
                s->dcdbv[i] = s->dcdbv[i] * (double)s->vtp[i] / tm3;
                s->dcdr[i] = s->dcdr[i] * (double)s->rtp[i] / tm3;
            }
        }
        if (full) {
            /* raw FP64 partials after sprayl, [k][ah,av,bh,bv,n,r][layer],
             * plus c after the Q shift in slot [k][6][0] (checker output) */
            double *fk = full + (size_t)k * 7 * nl;
            for (int i = 0; i < nl; ++i) {
                fk[0 * nl + i] = s->dcdah[i]; fk[1 * nl + i] = s->dcdav[i];
                fk[2 * nl + i] = s->dcdbh[i]; fk[3 * nl + i] = s->dcdbv[i];
                fk[4 * nl + i] = s->dcdn[i];  fk[5 * nl + i] = s->dcdr[i];
                fk[6 * nl + i] = 0.0;
            }
            fk[6 * nl] = c;
        }
        /* chksiz(), tregn96.f:1219-1233 */
        for (int i = 0; i < nl; ++i) {
            double v;
            v = s->dcdah[i]; dcdah_out[(size_t)k * nl + i] = fabs(v) < 1.0e-36 ? 0.0f : (float)v;
            v = s->dcdbv[i]; dcdbv_out[(size_t)k * nl + i] = fabs(v) < 1.0e-36 ? 0.0f : (float)v;
            v = s->dcdn[i];  dcdn_out[(size_t)k * nl + i] = fabs(v) < 1.0e-36 ? 0.0f : (float)v;
        }
    }
    free(s);
    return 0;
}

int or_tregn96_ex(int nl, const float *d_in, const float *TA_in, const float *TC_in,
                  const float *TF_in, const float *TL_in, const float *TN_in,
                  const float *TRho_in, const float *qai_in, const float *qbi_in,
                  const float *etapi_in, const float *etasi_in, const float *frefpi_in,
                  const float *frefsi_in, int nt, const float *t_in, const float *cp_in,
                  float *dcdah_out, float *dcdbv_out, float *dcdn_out, int nsph, int dogam,
                  double *full)
{
    return tregn96_run(nl, d_in, TA_in, TC_in, TF_in, TL_in, TN_in, TRho_in, qai_in, qbi_in,
                       etapi_in, etasi_in, frefpi_in, frefsi_in, nt, t_in, cp_in, NULL,
                       dcdah_out, dcdbv_out, dcdn_out, nsph, dogam, full);
}

/* The same with the phase velocities given in double (cp_d): a checker
 * entry that evaluates the partials at an exact root instead of at the
 * real*4 value depthkernelTI passes. */
int or_tregn96_cd(int nl, const float *d_in, const float *TA_in, const float *TC_in,
                  const float *TF_in, const float *TL_in, const float *TN_in,
                  const float *TRho_in, const float *qai_in, const float *qbi_in,
                  const float *etapi_in, const float *etasi_in, const float *frefpi_in,
                  const float *frefsi_in, int nt, const float *t_in, const double *cp_d,
                  float *dcdah_out, float *dcdbv_out, float *dcdn_out, int nsph, int dogam,
                  double *full)
{
    float cpf[NP];
    if (nt < 1 || nt > NP) return -1;
    for (int k = 0; k < nt; ++k) cpf[k] = (float)cp_d[k];
    return tregn96_run(nl, d_in, TA_in, TC_in, TF_in, TL_in, TN_in, TRho_in, qai_in, qbi_in,
                       etapi_in, etasi_in, frefpi_in, frefsi_in, nt, t_in, cpf, cp_d,
                       dcdah_out, dcdbv_out, dcdn_out, nsph, dogam, full);
}

/* ------------------------------------------------------------------------
 * Checker functions with no reference counterpart.  The TI Rayleigh secular
 * function of a flat double-precision model (no sphericity, no Q) is the
 * top entry of up()'s compound vector: the chain gettiegn -> varsv ->
 * dnka_tregn -> cnormc from the half-space (evalg) up.  Its fundamental
 * root, found by bracketing and Brent's method, and central differences of
 * that root with respect to the moduli of chosen layers give dc/dA, dc/dC,
 * dc/dF, dc/dL, dc/dN without svfunc/down/energy/intijr, the path that
 * forms tregn96's partials; the tests compare the two.                   */
static void ti_flat_model(ti_state *s, int nl, const double *d, const double *TA,
                          const double *TC, const double *TF, const double *TL,
                          const double *TN, const double *rho)
{
    s->mmax = nl;
    s->nsph = 0;
    s->dogam = 0;
    for (int i = 0; i < nl; ++i) {
        s->zd[i] = d[i]; s->zta[i] = TA[i]; s->ztc[i] = TC[i]; s->ztf[i] = TF[i];
        s->ztl[i] = TL[i]; s->ztn[i] = TN[i]; s->zrho[i] = rho[i];
        s->iwat[i] = 0;
    }
}

double or_ti_secular_d(int nl, const double *d, const double *TA, const double *TC,
                       const double *TF, const double *TL, const double *TN, const double *rho,
                       double omega, double c)
{
    if (nl < 2 || nl > NL) return NAN;
    ti_state *s = calloc(1, sizeof(ti_state));
    if (!s) return NAN;
    ti_flat_model(s, nl, d, TA, TC, TF, TL, TN, rho);
    double f = up(s, omega, omega / c);
    free(s);
    return f;
}

/* Root of F(c) = up() near c0: the bracket grows geometrically around c0
 * (first sign change on either side, nearest first), then Brent's method
 * (inverse quadratic interpolation / secant / bisection, R. P. Brent,
 * Algorithms for Minimization without Derivatives, 1973, ch. 4) until the
 * bracket is below xtol.  Returns 0, or -1 when no sign change lies within
 * 5 % of c0. */
static int ti_root(ti_state *s, double omega, double c0, double xtol, double *root)
{
#define TIF(c) up(s, omega, omega / (c))
    double f0 = TIF(c0);
    if (f0 == 0.0) { *root = c0; return 0; }
    double a = 0, b = 0, fa = 0, fb = 0;
    int found = 0;
    for (double del = 1e-9 * c0; del < 0.05 * c0 && !found; del *= 2.0) {
        double cl = c0 - del, cu = c0 + del;
        double fl = TIF(cl), fu = TIF(cu);
        if ((fu < 0) != (f0 < 0)) { a = c0; fa = f0; b = cu; fb = fu; found = 1; }
        else if ((fl < 0) != (f0 < 0)) { a = cl; fa = fl; b = c0; fb = f0; found = 1; }
    }
    if (!found) return -1;
    double c = a, fc = fa, dd = b - a, e = dd;
    for (int it = 0; it < 200; ++it) {
        if ((fb > 0) == (fc > 0)) { c = a; fc = fa; dd = b - a; e = dd; }
        if (fabs(fc) < fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
        double tol1 = 2.0 * 2.220446049250313e-16 * fabs(b) + 0.5 * xtol;
        double xm = 0.5 * (c - b);
        if (fabs(xm) <= tol1 || fb == 0.0) { *root = b; return 0; }
        if (fabs(e) >= tol1 && fabs(fa) > fabs(fb)) {
            double sr = fb / fa, p, q;
            if (a == c) { p = 2.0 * xm * sr; q = 1.0 - sr; }
            else {
                double qa = fa / fc, r = fb / fc;
                p = sr * (2.0 * xm * qa * (qa - r) - (b - a) * (r - 1.0));
                q = (qa - 1.0) * (r - 1.0) * (sr - 1.0);
            }
            if (p > 0) q = -q; else p = -p;
            double m1 = 3.0 * xm * q - fabs(tol1 * q), m2 = fabs(e * q);
            if (2.0 * p < (m1 < m2 ? m1 : m2)) { e = dd; dd = p / q; }
            else { dd = xm; e = dd; }
        } else { dd = xm; e = dd; }
        a = b; fa = fb;
        b += fabs(dd) > tol1 ? dd : (xm > 0 ? tol1 : -tol1);
        fb = TIF(b);
    }
#undef TIF
    *root = b;
    return 0;
}

int or_ti_root_d(int nl, const double *d, const double *TA, const double *TC, const double *TF,
                 const double *TL, const double *TN, const double *rho, double omega, double c0,
                 double xtol, double *root)
{
    if (nl < 2 || nl > NL) return -1;
    ti_state *s = calloc(1, sizeof(ti_state));
    if (!s) return -1;
    ti_flat_model(s, nl, d, TA, TC, TF, TL, TN, rho);
    int r = ti_root(s, omega, c0, xtol, root);
    free(s);
    return r;
}

/* Central differences of the root.  Perturbation p scales, in layers
 * lo[p]..hi[p] (0-based), the modulus kind[p] (0 A, 1 C, 2 F, 3 L, 4 N) by
 * (1 +- h), or with kind 5 both A and L (F, C, N and rho held).  For kinds
 * 0-4 on one layer dcdp[p] is dc/d(modulus); for kind 5 it is
 * dc/dh = sum over the layers of A dc/dA + L dc/dL.  OpenMP over the
 * perturbations.  Returns 0, or the number of failed roots. */
int or_ti_root_fd(int nl, const double *d, const double *TA, const double *TC, const double *TF,
                  const double *TL, const double *TN, const double *rho, double omega,
                  double c0, double h, double xtol, int npert, const int *lo, const int *hi,
                  const int *kind, double *dcdp, int nthreads)
{
    if (nl < 2 || nl > NL) return -1;
    int bad = 0;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic) num_threads(nthreads) reduction(+:bad)
#endif
    for (int p = 0; p < npert; ++p) {
        ti_state *s = calloc(1, sizeof(ti_state));
        if (!s) { ++bad; continue; }
        double cr[2];
        for (int sg = 0; sg < 2; ++sg) {
            const double f = sg == 0 ? 1.0 + h : 1.0 - h;
            ti_flat_model(s, nl, d, TA, TC, TF, TL, TN, rho);
            for (int m = lo[p]; m <= hi[p]; ++m) {
                switch (kind[p]) {
                case 0: s->zta[m] *= f; break;
                case 1: s->ztc[m] *= f; break;
                case 2: s->ztf[m] *= f; break;
                case 3: s->ztl[m] *= f; break;
                case 4: s->ztn[m] *= f; break;
                default: s->zta[m] *= f; s->ztl[m] *= f; break;
                }
            }
            if (ti_root(s, omega, c0, xtol, &cr[sg]) != 0) { ++bad; cr[sg] = NAN; }
        }
        double q = (cr[0] - cr[1]) / (2.0 * h);
        if (kind[p] <= 4) {
            const double *th = kind[p] == 0 ? TA : kind[p] == 1 ? TC : kind[p] == 2 ? TF
                             : kind[p] == 3 ? TL : TN;
            q /= th[lo[p]];
        }
        dcdp[p] = q;
        free(s);
    }
    return bad;
}

int or_tregn96(int nl, const float *d_in, const float *TA_in, const float *TC_in,
               const float *TF_in, const float *TL_in, const float *TN_in,
               const float *TRho_in, const float *qai_in, const float *qbi_in,
               const float *etapi_in, const float *etasi_in, const float *frefpi_in,
               const float *frefsi_in, int nt, const float *t_in, const float *cp_in,
               float *dcdah_out, float *dcdbv_out, float *dcdn_out)
{
    return or_tregn96_ex(nl, d_in, TA_in, TC_in, TF_in, TL_in, TN_in, TRho_in, qai_in, qbi_in,
                         etapi_in, etasi_in, frefpi_in, frefsi_in, nt, t_in, cp_in, dcdah_out,
                         dcdbv_out, dcdn_out, 1, 1, NULL);
}

/* depthkernelTI() column loop, depthkernelTI.f90:86-169, for the 1-based
 * column range [col_start, col_start+col_count).  pvRc (ncol,K) real*8 and
 * Lsen_Gsc (ncol,K,nz-1) real*4, Fortran order; vp_in/rho_in replace the
 * Brocher relations when not NULL.  status_out as or_depthkernel. */
int or_depthkernelTI(int nx, int ny, int nz, const float *vel, const float *vp_in,
                     const float *rho_in, double *pvRc, int iwave, int igr, int kmax,
                     const double *tRc, const float *depz, float minthk, float *Lsen,
                     int col_start, int col_count, int nthreads, int *status_out)
{
    if (nx < 1 || ny < 1 || nz < 2 || nz > NL || kmax < 1 || kmax > NP) return -1;
    const long ncol = (long)nx * ny;
    if (col_start < 1 || col_count < 0 || col_start - 1 + (long)col_count > ncol) return -1;
    int bad = 0;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic) num_threads(nthreads) reduction(|:bad)
#endif
    for (long cc = 0; cc < col_count; ++cc) {
        const long post = col_start - 1 + cc;
        float vs[NL], vp[NL], rho[NL], rthk[NL], rvp[NL], rvs[NL], rrho[NL];
        int nsub[NL];
        double cg[NP];
        for (int k = 0; k < nz; ++k) vs[k] = vel[post + ncol * k];
        if (vp_in) {
            for (int k = 0; k < nz; ++k) { vp[k] = vp_in[post + ncol * k]; rho[k] = rho_in[post + ncol * k]; }
        } else {
            or_brocher(nz, vs, vp, rho);
        }
        int rmax = or_refine(minthk, nz, depz, vp, vs, rho, rthk, rvp, rvs, rrho, nsub);
        if (rmax < 0) { bad |= 1; continue; }
        int st = or_surfdisp96_ex(rthk, rvp, rvs, rrho, rmax, 1, iwave, 1, igr, kmax, tRc, cg,
                                  1.0e-6, 1, NULL);
        if (status_out) status_out[post] = st;
        for (int k = 0; k < kmax; ++k) pvRc[post + ncol * k] = cg[k];
        float TA[NL], TC[NL], TF[NL], TL[NL], TN[NL], TR[NL], qp[NL], qs[NL], z0[NL], one[NL];
        for (int i = 0; i < rmax; ++i) {
            TA[i] = rrho[i] * (rvp[i] * rvp[i]);
            TC[i] = TA[i];
            TL[i] = rrho[i] * (rvs[i] * rvs[i]);
            TN[i] = TL[i];
            TF[i] = 1.0f * (TA[i] - 2.0f * TL[i]);
            TR[i] = rrho[i];
            qp[i] = 150.0f; qs[i] = 50.0f; z0[i] = 0.0f; one[i] = 1.0f;
        }
        float cp[NP], tt[NP];
        for (int k = 0; k < kmax; ++k) { cp[k] = (float)cg[k]; tt[k] = (float)tRc[k]; }
        float *dah = malloc(sizeof(float) * 3 * (size_t)kmax * rmax);
        if (!dah) { bad |= 1; continue; }
        float *dbv = dah + (size_t)kmax * rmax, *dn = dbv + (size_t)kmax * rmax;
        /* periods after a failed root keep cp = 0: tregn96 is not called for
         * them in effect (their kernels are left at zero below) */
        int kgood = kmax;
        for (int k = 0; k < kmax; ++k) if (!(cp[k] > 0.0f)) { kgood = k; break; }
        if (kgood > 0 &&
            or_tregn96(rmax, rthk, TA, TC, TF, TL, TN, TR, qp, qs, z0, z0, one, one, kgood, tt,
                       cp, dah, dbv, dn) != 0) {
            bad |= 1; free(dah); continue;
        }
        for (int i = 0; i < kmax; ++i) {
            for (int j = 0; j < nz - 1; ++j) Lsen[post + ncol * ((long)i + (long)kmax * j)] = 0.0f;
            if (i >= kgood) continue;
            int k = 0;
            for (int j = 0; j < nz - 1; ++j) {
                float acc = 0.0f;
                for (int jj = 0; jj < nsub[j]; ++jj, ++k) {
                    float tfd = TA[k] - 2.0f * TL[k];
                    float dA = 0.5f / (rrho[k] * rvp[k]) * dah[(size_t)i * rmax + k]
                               - TF[k] / (tfd * tfd) * dn[(size_t)i * rmax + k];
                    float dL = 0.5f / (rrho[k] * rvs[k]) * dbv[(size_t)i * rmax + k]
                               + 2.0f * TF[k] / (tfd * tfd) * dn[(size_t)i * rmax + k];
                    acc = acc + dA * TA[k] + dL * TL[k];
                }
                Lsen[post + ncol * ((long)i + (long)kmax * j)] = acc;
            }
        }
        free(dah);
    }
    return bad ? -1 : 0;
}

/* Ragged batch (CPU baseline of the batch interface): per column its own
 * depth grid (node_off) and periods (per_off); the reference's two stages,
 * depthkernel (FD, DepthKernel1D.f90:102-185) and depthkernelTI's tregn96
 * path (depthkernelTI.f90:93-162), with OpenMP over columns.  Outputs use the
 * batch layout: pv[per_off[c]+k], sen[sen_off[c] + k + K_c i],
 * lsen[ls_off[c] + k + K_c j].  Brocher Vp/rho.  Returns 0 or -1. */
static int ti_splice_column(int nz, int K, const double *per, int rmax, const float *rthk,
                            const float *rvp, const float *rvs, const float *rrho,
                            const int *nsub, const double *cg, float *L);

int or_batch(long ncols, const long *node_off, const float *depz, const float *vs_all,
             const long *per_off, const double *periods, float minthk, double *pv,
             const long *sen_off, double *svs, double *svp, double *srh, const long *ls_off,
             float *lsen, int nthreads)
{
    int bad = 0;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic) num_threads(nthreads) reduction(|:bad)
#endif
    for (long c = 0; c < ncols; ++c) {
        const int nz = (int)(node_off[c + 1] - node_off[c]);
        const int K = (int)(per_off[c + 1] - per_off[c]);
        if (nz < 2 || nz > NL || K < 1 || K > NP) { bad |= 1; continue; }
        const float *dep = depz + node_off[c];
        const float *vs = vs_all + node_off[c];
        const double *per = periods + per_off[c];
        float vp[NL], rho[NL];
        or_brocher(nz, vs, vp, rho);
        double *cpv = pv + per_off[c];
        double *a = svs ? svs + sen_off[c] : NULL, *b = svs ? svp + sen_off[c] : NULL;
        double *d = svs ? srh + sen_off[c] : NULL;
        double tmp1[NP * 4];
        if (svs) {
            if (or_column_fd(nz, vs, vp, rho, K, per, 2, 0, dep, minthk, 0.01f, 0.01f, 0.01f,
                             1.0e-6, 0, cpv, a, b, d, NULL) < 0) { bad |= 1; continue; }
        } else {
            (void)tmp1;
        }
        float rthk[NL], rvp[NL], rvs[NL], rrho[NL];
        int nsub[NL];
        int rmax = or_refine(minthk, nz, dep, vp, vs, rho, rthk, rvp, rvs, rrho, nsub);
        if (rmax < 0) { bad |= 1; continue; }
        double cg[NP];
        if (svs) { for (int k = 0; k < K; ++k) cg[k] = cpv[k]; }
        else {
            /* phase velocities alone when no kernel is asked for */
            or_surfdisp96_ex(rthk, rvp, rvs, rrho, rmax, 1, 2, 1, 0, K, per, cg, 1.0e-6, 1, NULL);
            for (int k = 0; k < K; ++k) cpv[k] = cg[k];
        }
        if (!lsen) continue;
        if (ti_splice_column(nz, K, per, rmax, rthk, rvp, rvs, rrho, nsub, cg,
                             lsen + ls_off[c]) != 0) bad |= 1;
    }
    return bad ? -1 : 0;
}

/* depthkernelTI's tregn96 call and splice for one refined column
 * (depthkernelTI.f90:124-162): the real*4 moduli, tregn96 with Q 150/50
 * and sphericity at the phase velocities cg (real*4 cp_in = sngl(cg); a
 * period without a root and all after it give 0), Lsen_Gsc (K x nz-1,
 * column-major) in real*4.  Returns 0 or -1. */
static int ti_splice_column(int nz, int K, const double *per, int rmax, const float *rthk,
                            const float *rvp, const float *rvs, const float *rrho,
                            const int *nsub, const double *cg, float *L)
{
    float TA[NL], TC[NL], TF[NL], TL[NL], TN[NL], TR[NL], qp[NL], qs[NL], z0[NL], one[NL];
    for (int i = 0; i < rmax; ++i) {
        TA[i] = rrho[i] * (rvp[i] * rvp[i]);
        TC[i] = TA[i];
        TL[i] = rrho[i] * (rvs[i] * rvs[i]);
        TN[i] = TL[i];
        TF[i] = 1.0f * (TA[i] - 2.0f * TL[i]);
        TR[i] = rrho[i];
        qp[i] = 150.0f; qs[i] = 50.0f; z0[i] = 0.0f; one[i] = 1.0f;
    }
    float cp[NP], tt[NP];
    int kgood = K;
    for (int k = 0; k < K; ++k) {
        cp[k] = (float)cg[k]; tt[k] = (float)per[k];
        if (!(cp[k] > 0.0f) && kgood == K) kgood = k;
    }
    float *dah = malloc(sizeof(float) * 3 * (size_t)K * rmax);
    if (!dah) return -1;
    float *dbv = dah + (size_t)K * rmax, *dn = dbv + (size_t)K * rmax;
    if (kgood > 0 && or_tregn96(rmax, rthk, TA, TC, TF, TL, TN, TR, qp, qs, z0, z0, one, one,
                                kgood, tt, cp, dah, dbv, dn) != 0) {
        free(dah);
        return -1;
    }
    for (int i = 0; i < K; ++i) {
        for (int j = 0; j < nz - 1; ++j) L[i + (long)K * j] = 0.0f;
        if (i >= kgood) continue;
        int k = 0;
        for (int j = 0; j < nz - 1; ++j) {
            float acc = 0.0f;
            for (int jj = 0; jj < nsub[j]; ++jj, ++k) {
                float tfd = TA[k] - 2.0f * TL[k];
                float dA = 0.5f / (rrho[k] * rvp[k]) * dah[(size_t)i * rmax + k]
                           - TF[k] / (tfd * tfd) * dn[(size_t)i * rmax + k];
                float dL = 0.5f / (rrho[k] * rvs[k]) * dbv[(size_t)i * rmax + k]
                           + 2.0f * TF[k] / (tfd * tfd) * dn[(size_t)i * rmax + k];
                acc = acc + dA * TA[k] + dL * TL[k];
            }
            L[i + (long)K * j] = acc;
        }
    }
    free(dah);
    return 0;
}

/* Lsen_Gsc of a ragged batch at given phase velocities (pv_in, batch
 * layout: tregn96 is called at sngl(pv_in), as depthkernelTI passes its
 * real*4 roots) or, with pv_in NULL, at surfdisp96's roots converged to
 * root_tol (1e-6: the reference's; smaller: a checker of the partials at
 * the exact root), which are written to pv_out.  OpenMP over columns. */
int or_batch_ti(long ncols, const long *node_off, const float *depz, const float *vs_all,
                const long *per_off, const double *periods, float minthk, const double *pv_in,
                double root_tol, double *pv_out, const long *ls_off, float *lsen, int nthreads)
{
    int bad = 0;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic) num_threads(nthreads) reduction(|:bad)
#endif
    for (long c = 0; c < ncols; ++c) {
        const int nz = (int)(node_off[c + 1] - node_off[c]);
        const int K = (int)(per_off[c + 1] - per_off[c]);
        if (nz < 2 || nz > NL || K < 1 || K > NP) { bad |= 1; continue; }
        const float *dep = depz + node_off[c];
        const float *vs = vs_all + node_off[c];
        const double *per = periods + per_off[c];
        float vp[NL], rho[NL], rthk[NL], rvp[NL], rvs[NL], rrho[NL];
        int nsub[NL];
        or_brocher(nz, vs, vp, rho);
        int rmax = or_refine(minthk, nz, dep, vp, vs, rho, rthk, rvp, rvs, rrho, nsub);
        if (rmax < 0) { bad |= 1; continue; }
        double cg[NP];
        if (pv_in) { for (int k = 0; k < K; ++k) cg[k] = pv_in[per_off[c] + k]; }
        else or_surfdisp96_ex(rthk, rvp, rvs, rrho, rmax, 1, 2, 1, 0, K, per, cg, root_tol, 1, NULL);
        if (pv_out) for (int k = 0; k < K; ++k) pv_out[per_off[c] + k] = cg[k];
        if (ti_splice_column(nz, K, per, rmax, rthk, rvp, rvs, rrho, nsub, cg,
                             lsen + ls_off[c]) != 0) bad |= 1;
    }
    return bad ? -1 : 0;
}

/* Vs-type kernels of a ragged batch with a chosen arithmetic: precision 0
 * is the reference's (real*4 model stores, sngl(c) roots, or_column_fd as
 * or_batch uses it), 2 the checker's exact-model pipeline (double model,
 * unrounded roots) with its own tol and dln.  status[c] as or_phase (first
 * failing period, 1-based, or 0).  OpenMP over columns.                    */
int or_batch_fd(long ncols, const long *node_off, const float *depz, const float *vs_all,
                const long *per_off, const double *periods, float minthk, double *pv,
                const long *sen_off, double *svs, double *svp, double *srh, int precision,
                double tol, float dln, int *status, int nthreads)
{
    int bad = 0;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic) num_threads(nthreads) reduction(|:bad)
#endif
    for (long c = 0; c < ncols; ++c) {
        const int nz = (int)(node_off[c + 1] - node_off[c]);
        const int K = (int)(per_off[c + 1] - per_off[c]);
        if (nz < 2 || nz > NL || K < 1 || K > NP) { bad |= 1; continue; }
        const float *vs = vs_all + node_off[c];
        float vp[NL], rho[NL];
        or_brocher(nz, vs, vp, rho);
        int st = or_column_fd(nz, vs, vp, rho, K, periods + per_off[c], 2, 0, depz + node_off[c],
                              minthk, dln, dln, dln, tol, precision, pv + per_off[c],
                              svs + sen_off[c], svp + sen_off[c], srh + sen_off[c], NULL);
        if (st < 0) bad |= 1;
        if (status) status[c] = st < 0 ? -1 : st;
    }
    return bad ? -1 : 0;
}

/* G rows of the LSMR system from the depth kernels, CalSurfG_parallel.f90
 * :2363-2400 (iso_phase_only, use_aniso_active): for each ray (a data row,
 * id ray_id[r], period index ray_period[r]) and each of its model cells
 * with |fdm| >= ftol (cell = (jj-1)*nvx + kk-1 of the nvx x nvz inner grid,
 * ascending within the ray), the dense parameter row
 *   row(i, cell)            = (sen_vp*coe_a + sen_rho*coe_rho + sen_vs)*fdm
 *   row(nparpi + i, cell)   = Lsen*fdmc,  row(2 nparpi + i, cell) = Lsen*fdms
 * (i = 1..nz-1, real*4 row; coe_a, coe_rho the Brocher derivatives at the
 * node velocity in real*4), then the entries |row| > ftol in parameter
 * order as (rw real*4, iw = ray id, col 1-based).  Kernel column of cell
 * (kk, jj): post = jj*(nvx+2)+kk (0-based), arrays in the reference's
 * layouts.  lsen == NULL: isotropic rows only.  Returns the number of
 * entries, or -1 when cap is exceeded / a cell index is invalid. */
static inline float or_coe_a(float v)
{
    const float v2 = v * v, v3 = v2 * v;
    return ((2.0947f - (float)(0.8206f * 2.0f) * v) + (float)(0.2683f * 3.0f) * v2) - (float)(0.0251f * 4.0f) * v3;
}

static inline float or_coe_rho(float v, float ca)
{
    const float v2 = v * v, v3 = v2 * v, v4 = v2 * v2;
    const float vp = (((0.9409f + 2.0947f * v) - 0.8206f * v2) + 0.2683f * v3) - 0.0251f * v4;
    const float p2 = vp * vp, p3 = p2 * vp, p4 = p2 * p2;
    const float poly = (((1.6612f - (float)(0.4721f * 2.0f) * vp) + (float)(0.0671f * 3.0f) * p2)
                        - (float)(0.0043f * 4.0f) * p3) + (float)(0.000106f * 5.0f) * p4;
    return ca * poly;
}

long or_grows(int nvx, int nvz, int nz, int K, const float *vels, const double *svs,
              const double *svp, const double *srh, const float *lsen, long nrays,
              const int *ray_period, const int *ray_id, const long *cell_off, const int *cell,
              const float *fdm, const float *fdmc, const float *fdms, float ftol, long cap,
              float *rw, int *iw, int *col, long *nnz_ray)
{
    const int nx = nvx + 2, ny = nvz + 2;
    const long nxy = (long)nx * ny, ncell = (long)nvx * nvz;
    const long nparpi = ncell * (nz - 1);
    const int nblk = lsen ? 3 : 1;
    float *row = malloc(sizeof(float) * nparpi * nblk);
    if (!row) return -1;
    long out = 0;
    for (long r = 0; r < nrays; ++r) {
        memset(row, 0, sizeof(float) * nparpi * nblk);
        const int k = ray_period[r];
        for (long e = cell_off[r]; e < cell_off[r + 1]; ++e) {
            const int c = cell[e];
            if (c < 0 || c >= ncell) { free(row); return -1; }
            if (!(fabsf(fdm[e]) >= ftol)) continue;
            const int kk = c % nvx + 1, jj = c / nvx + 1;
            const long post = (long)jj * nx + kk;
            for (int i = 0; i < nz - 1; ++i) {
                const float v = vels[post + nxy * i];
                const float ca = or_coe_a(v), cr = or_coe_rho(v, ca);
                const long ks = post + nxy * (k + (long)K * i);
                const double s = (svp[ks] * (double)ca + srh[ks] * (double)cr) + svs[ks];
                row[(long)i * ncell + c] = (float)(s * (double)fdm[e]);
                if (lsen) {
                    const float L = lsen[post + nxy * (k + (long)K * i)];
                    row[nparpi + (long)i * ncell + c] = L * fdmc[e];
                    row[2 * nparpi + (long)i * ncell + c] = L * fdms[e];
                }
            }
        }
        long n = 0;
        for (long q = 0; q < nparpi * nblk; ++q)
            if (fabsf(row[q]) > ftol) {
                if (out >= cap) { free(row); return -1; }
                rw[out] = row[q]; iw[out] = ray_id[r]; col[out] = (int)(q + 1);
                ++out; ++n;
            }
        if (nnz_ray) nnz_ray[r] = n;
    }
    free(row);
    return out;
}

/* FwdAzimuthalAniMap.f90:43-86: per inner column and period the real*4
 * sums cos = sum Lsen gc, sin = sum Lsen gs (intervals ascending), the
 * amplitude 0.5 sqrt(cos^2 + sin^2), its ratio to the isotropic phase
 * velocity (real*4) and the fast-axis angle 0.5 (atan2(sin, cos)/pi*180
 * [+360]) with pi real*8.  Outputs ((nx-2)*(ny-2), K) real*4. */
void or_azimap(int nx, int ny, int nz, int K, const float *lsen, const float *gc, const float *gs,
               const double *ciso, float *cosr, float *sinr, float *amp, float *rela, float *ang)
{
    const int nvx = nx - 2, nvz = ny - 2;
    const long nxy = (long)nx * ny, ncell = (long)nvx * nvz;
    const double pi = 3.1415926535898;
    for (int tt = 0; tt < K; ++tt)
        for (int jj = 1; jj <= nvz; ++jj)
            for (int ii = 1; ii <= nvx; ++ii) {
                const long post = (long)jj * nx + ii;
                float cs = 0.0f, sn = 0.0f;
                for (int k = 0; k < nz - 1; ++k) {
                    const float L = lsen[post + nxy * (tt + (long)K * k)];
                    const long g = (ii - 1) + (long)nvx * ((jj - 1) + (long)nvz * k);
                    cs = cs + L * gc[g];
                    sn = sn + L * gs[g];
                }
                const long o = (long)(jj - 1) * nvx + (ii - 1) + ncell * tt;
                const float a = 0.5f * sqrtf(cs * cs + sn * sn);
                float an = (float)((double)atan2f(sn, cs) / pi * 180.0);
                if (an < 0.0f) an = an + 360.0f;
                an = 0.5f * an;
                cosr[o] = cs; sinr[o] = sn; amp[o] = a;
                rela[o] = a / (float)ciso[o];
                ang[o] = an;
            }
}
