// TEST INFRASTRUCTURE ONLY: C restatement of the reference's first-arrival
// traveltime solver on the refined spherical grid (fast marching with a
// binary-heap narrow band), its source-grid refinement and the B-spline
// gridding of a phase-velocity map, and the source-receiver interpolation:
//   travel_parallel            CalSurfG_parallel.f90:125-336
//   fouds1_parallel            CalSurfG_parallel.f90:346-432
//   fouds2_parallel            CalSurfG_parallel.f90:443-622
//   addtree/downtree/updtree   CalSurfG_parallel.f90:631-803
//   gridder_parallel           CalSurfG_parallel.f90:811-909
//   bsplrefine_parallel        CalSurfG_parallel.f90:918-989
//   srtimes_parallel           CalSurfG_parallel.f90:997-1125
//   bilinear_parallel          CalSurfG_parallel.f90:2543-2566
//   per-(period, source) driver with source-grid refinement
//                              CalSurfG_parallel.f90:2085-2340
// Every quantity is REAL(KIND=i10) = real*4 in the reference, and every
// operation here is a float operation in the Fortran's order (built with
// -ffp-contract=off, as gfortran's x86-64 code has no FMA); SIN is sinf.
// Arrays keep the reference's (z, x) column-major layout: node (iz, ix),
// 1-based, at a[(ix - 1) * ld + (iz - 1)].
// Only tests/, the smoke check and bench.py's CPU legs use this file.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "dk_oracle.h"

#define AT(a, iz, ix) (a)[(size_t)((ix) - 1) * (size_t)ld + (size_t)((iz) - 1)]

typedef struct { int px, pz; } Bt;

typedef struct {
    int nnx, nnz, ld;
    float gox, goz, dnx, dnz, earth;
    int fom;
} Grid;

static const float kPi = 3.1415926535898f;   // globalp_local: REAL(i10) pi

// ------------------------------------------------------------ heap
// addtree_parallel (CalSurfG_parallel.f90:631-675)
static int addtree(int iz, int ix, int* ntr, int maxbt, int* nsts, const float* ttn, Bt* btg, int ld)
{
    if (*ntr >= maxbt) return -2;
    *ntr += 1;
    AT(nsts, iz, ix) = *ntr;
    btg[*ntr].px = ix;
    btg[*ntr].pz = iz;
    int tpc = *ntr, tpp = tpc / 2;
    while (tpp > 0) {
        if (AT(ttn, iz, ix) < AT(ttn, btg[tpp].pz, btg[tpp].px)) {
            AT(nsts, iz, ix) = tpp;
            AT(nsts, btg[tpp].pz, btg[tpp].px) = tpc;
            const Bt e = btg[tpc];
            btg[tpc] = btg[tpp];
            btg[tpp] = e;
            tpc = tpp;
            tpp = tpc / 2;
        } else {
            tpp = 0;
        }
    }
    return 0;
}

// downtree_parallel (CalSurfG_parallel.f90:686-761)
static void downtree(int* ntr, int* nsts, const float* ttn, Bt* btg, int ld)
{
    if (*ntr == 1) { *ntr -= 1; return; }
    AT(nsts, btg[*ntr].pz, btg[*ntr].px) = 1;
    btg[1] = btg[*ntr];
    *ntr -= 1;
    int tpp = 1, tpc = 2 * tpp;
    while (tpc < *ntr) {
        float rd1 = AT(ttn, btg[tpc].pz, btg[tpc].px);
        float rd2 = AT(ttn, btg[tpc + 1].pz, btg[tpc + 1].px);
        if (rd1 > rd2) tpc += 1;
        rd1 = AT(ttn, btg[tpc].pz, btg[tpc].px);
        rd2 = AT(ttn, btg[tpp].pz, btg[tpp].px);
        if (rd1 < rd2) {
            AT(nsts, btg[tpp].pz, btg[tpp].px) = tpc;
            AT(nsts, btg[tpc].pz, btg[tpc].px) = tpp;
            const Bt e = btg[tpc];
            btg[tpc] = btg[tpp];
            btg[tpp] = e;
            tpp = tpc;
            tpc = 2 * tpp;
        } else {
            tpc = *ntr + 1;
        }
    }
    if (tpc == *ntr) {
        const float rd1 = AT(ttn, btg[tpc].pz, btg[tpc].px);
        const float rd2 = AT(ttn, btg[tpp].pz, btg[tpp].px);
        if (rd1 < rd2) {
            AT(nsts, btg[tpp].pz, btg[tpp].px) = tpc;
            AT(nsts, btg[tpc].pz, btg[tpc].px) = tpp;
            const Bt e = btg[tpc];
            btg[tpc] = btg[tpp];
            btg[tpp] = e;
        }
    }
}

// updtree_parallel (CalSurfG_parallel.f90:770-803)
static void updtree(int iz, int ix, int* nsts, const float* ttn, Bt* btg, int ld)
{
    int tpc = AT(nsts, iz, ix), tpp = tpc / 2;
    while (tpp > 0) {
        if (AT(ttn, iz, ix) < AT(ttn, btg[tpp].pz, btg[tpp].px)) {
            AT(nsts, iz, ix) = tpp;
            AT(nsts, btg[tpp].pz, btg[tpp].px) = tpc;
            const Bt e = btg[tpc];
            btg[tpc] = btg[tpp];
            btg[tpp] = e;
            tpc = tpp;
            tpp = tpc / 2;
        } else {
            tpp = 0;
        }
    }
}

// ------------------------------------------------------------ local solvers
// the positive root of a t^2 + b t + c = 0, as the reference forms it
static float quad_root(float a, float b, float c)
{
    float rd1 = b * b - 4.0f * a * c;
    if (rd1 < 0.0f) rd1 = 0.0f;
    return (-b + sqrtf(rd1)) / (2.0f * a);
}

// fouds1_parallel (CalSurfG_parallel.f90:346-432): first-order upwind
static int fouds1(int iz, int ix, const Grid* g, const int* nsts, const float* veln, float* ttn)
{
    const int ld = g->ld;
    int tsw1 = 0;
    float travm = 0.0f;
    const float slown = 1.0f / AT(veln, iz, ix);
    const float ri = g->earth;
    const float risti = ri * sinf(g->gox + (float)(ix - 1) * g->dnx);
    for (int j = ix - 1; j <= ix + 1; j += 2) {
        for (int k = iz - 1; k <= iz + 1; k += 2) {
            if (j < 1 || j > g->nnx || k < 1 || k > g->nnz) continue;
            int swsol = 0;
            float a = 0, b = 0, c = 0, tref = 0;
            if (AT(nsts, iz, j) == 0) {
                swsol = 1;
                if (AT(nsts, k, ix) == 0) {
                    const float u = ri * g->dnx, v = risti * g->dnz;
                    const float em = AT(ttn, k, ix) - AT(ttn, iz, j);
                    a = u * u + v * v;
                    b = -2.0f * (u * u) * em;
                    c = (u * u) * (em * em - (v * v) * (slown * slown));
                    tref = AT(ttn, iz, j);
                } else {
                    a = 1.0f;
                    b = 0.0f;
                    c = -(slown * slown) * (ri * ri) * (g->dnx * g->dnx);
                    tref = AT(ttn, iz, j);
                }
            } else if (AT(nsts, k, ix) == 0) {
                swsol = 1;
                a = 1.0f;
                b = 0.0f;
                const float t = slown * risti * g->dnz;
                c = -(t * t);
                tref = AT(ttn, k, ix);
            }
            if (swsol) {
                const float trav = tref + quad_root(a, b, c);
                if (tsw1) travm = fminf(trav, travm);   // MIN of two non-NaN values
                else { travm = trav; tsw1 = 1; }
            }
        }
    }
    if (!tsw1) return -3;
    AT(ttn, iz, ix) = travm;
    return 0;
}

// fouds2_parallel (CalSurfG_parallel.f90:443-622): mixed-order upwind
static int fouds2(int iz, int ix, const Grid* g, const int* nsts, const float* veln, float* ttn)
{
    const int ld = g->ld;
    int tsw1 = 0;
    float travm = 0.0f;
    const float slown = 1.0f / AT(veln, iz, ix);
    const float ri = g->earth;
    const float risti = ri * sinf(g->gox + (float)(ix - 1) * g->dnx);
    for (int j = ix - 1; j <= ix + 1; j += 2) {
        if (j < 1 || j > g->nnx) continue;
        int swj = -1, j2;
        if (j == ix - 1) {
            j2 = j - 1;
            if (j2 >= 1 && AT(nsts, iz, j2) == 0) swj = 0;
        } else {
            j2 = j + 1;
            if (j2 <= g->nnx && AT(nsts, iz, j2) == 0) swj = 0;
        }
        if (AT(nsts, iz, j) == 0 && swj == 0) {
            swj = -1;
            if (AT(ttn, iz, j) > AT(ttn, iz, j2)) swj = 0;
        } else {
            swj = -1;
        }
        for (int k = iz - 1; k <= iz + 1; k += 2) {
            if (k < 1 || k > g->nnz) continue;
            int swk = -1, k2;
            if (k == iz - 1) {
                k2 = k - 1;
                if (k2 >= 1 && AT(nsts, k2, ix) == 0) swk = 0;
            } else {
                k2 = k + 1;
                if (k2 <= g->nnz && AT(nsts, k2, ix) == 0) swk = 0;
            }
            if (AT(nsts, k, ix) == 0 && swk == 0) {
                swk = -1;
                if (AT(ttn, k, ix) > AT(ttn, k2, ix)) swk = 0;
            } else {
                swk = -1;
            }
            int swsol = 0;
            float a = 0, b = 0, c = 0, tref = 0, tdiv = 1.0f, u, v, em;
            if (swj == 0) {
                swsol = 1;
                if (swk == 0) {
                    u = 2.0f * ri * g->dnx;
                    v = 2.0f * risti * g->dnz;
                    em = 4.0f * AT(ttn, iz, j) - AT(ttn, iz, j2) - 4.0f * AT(ttn, k, ix);
                    em = em + AT(ttn, k2, ix);
                    a = v * v + u * u;
                    b = 2.0f * em * (u * u);
                    c = (u * u) * (em * em - (slown * slown) * (v * v));
                    tref = 4.0f * AT(ttn, iz, j) - AT(ttn, iz, j2);
                    tdiv = 3.0f;
                } else if (AT(nsts, k, ix) == 0) {
                    u = risti * g->dnz;
                    v = 2.0f * ri * g->dnx;
                    em = 3.0f * AT(ttn, k, ix) - 4.0f * AT(ttn, iz, j) + AT(ttn, iz, j2);
                    a = v * v + 9.0f * (u * u);
                    b = 6.0f * em * (u * u);
                    c = (u * u) * (em * em - (slown * slown) * (v * v));
                    tref = AT(ttn, k, ix);
                    tdiv = 1.0f;
                } else {
                    u = 2.0f * ri * g->dnx;
                    a = 1.0f;
                    b = 0.0f;
                    c = -(u * u) * (slown * slown);
                    tref = 4.0f * AT(ttn, iz, j) - AT(ttn, iz, j2);
                    tdiv = 3.0f;
                }
            } else if (AT(nsts, iz, j) == 0) {
                swsol = 1;
                if (swk == 0) {
                    u = ri * g->dnx;
                    v = 2.0f * risti * g->dnz;
                    em = 3.0f * AT(ttn, iz, j) - 4.0f * AT(ttn, k, ix) + AT(ttn, k2, ix);
                    a = v * v + 9.0f * (u * u);
                    b = 6.0f * em * (u * u);
                    c = (u * u) * (em * em - (v * v) * (slown * slown));
                    tref = AT(ttn, iz, j);
                    tdiv = 1.0f;
                } else if (AT(nsts, k, ix) == 0) {
                    u = ri * g->dnx;
                    v = risti * g->dnz;
                    em = AT(ttn, k, ix) - AT(ttn, iz, j);
                    a = u * u + v * v;
                    b = -2.0f * (u * u) * em;
                    c = (u * u) * (em * em - (v * v) * (slown * slown));
                    tref = AT(ttn, iz, j);
                    tdiv = 1.0f;
                } else {
                    a = 1.0f;
                    b = 0.0f;
                    c = -(slown * slown) * (ri * ri) * (g->dnx * g->dnx);
                    tref = AT(ttn, iz, j);
                    tdiv = 1.0f;
                }
            } else {
                if (swk == 0) {
                    swsol = 1;
                    u = 2.0f * risti * g->dnz;
                    a = 1.0f;
                    b = 0.0f;
                    c = -(u * u) * (slown * slown);
                    tref = 4.0f * AT(ttn, k, ix) - AT(ttn, k2, ix);
                    tdiv = 3.0f;
                } else if (AT(nsts, k, ix) == 0) {
                    swsol = 1;
                    a = 1.0f;
                    b = 0.0f;
                    c = -(slown * slown) * (risti * risti) * (g->dnz * g->dnz);
                    tref = AT(ttn, k, ix);
                    tdiv = 1.0f;
                }
            }
            if (swsol) {
                const float trav = (tref + quad_root(a, b, c)) / tdiv;
                if (tsw1) travm = fminf(trav, travm);
                else { travm = trav; tsw1 = 1; }
            }
        }
    }
    if (!tsw1) return -3;
    AT(ttn, iz, ix) = travm;
    return 0;
}

// bilinear_parallel (CalSurfG_parallel.f90:2543-2566); nv[i][j] = nv(i+1, j+1)
static float bilinear(const float nv[2][2], float dsx, float dsz, float dnx, float dnz)
{
    float biv = 0.0f;
    for (int i = 1; i <= 2; ++i)
        for (int j = 1; j <= 2; ++j) {
            const float produ = (1.0f - fabsf(((float)(i - 1) * dnx - dsx) / dnx)) *
                                (1.0f - fabsf(((float)(j - 1) * dnz - dsz) / dnz));
            biv = biv + nv[i - 1][j - 1] * produ;
        }
    return biv;
}

// ------------------------------------------------------------ travel
// travel_parallel (CalSurfG_parallel.f90:125-336).  urg 0: from the source
// point; 1: on the refined source grid (the box vnl..vnr x vnt..vnb of
// coarse nodes), stopping once the popped node lies on a side of the
// refined grid, unless that side is the model's; 2: from the narrow band
// nsts holds (close nodes > 0).  As in the reference, the right and bottom
// sides are compared with this grid's own node counts (:249-254), so those
// two always stop the refined run.  Returns 0, -1 (source outside the
// grid), -2 (narrow band larger than maxbt), -3 (a node without an upwind
// solution), -5 (urg 2 without a close node: the field is undefined).
static int travel(float scx, float scz, int urg, const Grid* g, int vnl, int vnr, int vnt, int vnb,
                  int* nsts, const float* veln, float* ttn, Bt* btg, int maxbt)
{
    const int ld = g->ld, nnx = g->nnx, nnz = g->nnz;
    int isx = (int)((scx - g->gox) / g->dnx) + 1;
    int isz = (int)((scz - g->goz) / g->dnz) + 1;
    if (isx < 1 || isx > nnx || isz < 1 || isz > nnz) return -1;
    if (isx == nnx) isx -= 1;
    if (isz == nnz) isz -= 1;
    int ntr = 0, r;
    if (urg == 2) {
        for (int i = 1; i <= nnx; ++i)
            for (int j = 1; j <= nnz; ++j)
                if (AT(nsts, j, i) > 0 && (r = addtree(j, i, &ntr, maxbt, nsts, ttn, btg, ld))) return r;
        // the refined sweep stopped before it reached a coarse node (a source
        // in the last cell before the right or bottom side, which always
        // stops it): the reference's field is whatever its array held
        if (ntr == 0) return -5;
    } else {
        for (int i = 1; i <= nnx; ++i)
            for (int j = 1; j <= nnz; ++j) AT(nsts, j, i) = -1;
        float vss[2][2];
        for (int i = 1; i <= 2; ++i)
            for (int j = 1; j <= 2; ++j) vss[i - 1][j - 1] = AT(veln, isz - 1 + j, isx - 1 + i);
        const float dsx = (scx - g->gox) - (float)(isx - 1) * g->dnx;
        const float dsz = (scz - g->goz) - (float)(isz - 1) * g->dnz;
        const float vsrc = bilinear(vss, dsx, dsz, g->dnx, g->dnz);
        for (int i = 1; i <= 2; ++i)
            for (int j = 1; j <= 2; ++j) {
                const float ex = dsx - (float)(i - 1) * g->dnx, ez = dsz - (float)(j - 1) * g->dnz;
                const float ds = sqrtf(ex * ex + ez * ez);
                AT(ttn, isz - 1 + j, isx - 1 + i) = 2.0f * ds / (vss[i - 1][j - 1] + vsrc);
                if ((r = addtree(isz - 1 + j, isx - 1 + i, &ntr, maxbt, nsts, ttn, btg, ld))) return r;
            }
    }
    while (ntr > 0) {
        int ix = btg[1].px, iz = btg[1].pz;
        if (urg == 1) {
            int swrg = 0;
            if (ix == 1 && vnl != 1) swrg = 1;
            if (ix == nnx && vnr != nnx) swrg = 1;
            if (iz == 1 && vnt != 1) swrg = 1;
            if (iz == nnz && vnb != nnz) swrg = 1;
            if (swrg) { AT(nsts, iz, ix) = 0; break; }
        }
        AT(nsts, iz, ix) = 0;
        downtree(&ntr, nsts, ttn, btg, ld);
        for (int pass = 0; pass < 2; ++pass) {
            const int lo = pass == 0 ? ix - 1 : iz - 1;
            for (int i = lo; i <= lo + 2; i += 2) {
                const int niz = pass == 0 ? iz : i, nix = pass == 0 ? i : ix;
                if (pass == 0 ? (i < 1 || i > nnx) : (i < 1 || i > nnz)) continue;
                const int st = AT(nsts, niz, nix);
                if (st == -1 || st > 0) {
                    r = g->fom == 0 ? fouds1(niz, nix, g, nsts, veln, ttn) : fouds2(niz, nix, g, nsts, veln, ttn);
                    if (r) return r;
                    if (st == -1) {
                        if ((r = addtree(niz, nix, &ntr, maxbt, nsts, ttn, btg, ld))) return r;
                    } else {
                        updtree(niz, nix, nsts, ttn, btg, ld);
                    }
                }
            }
        }
    }
    return 0;
}

// ------------------------------------------------------------ gridding
// Cubic B-spline basis values at u (gridder_parallel :857-876): (1-u)^3/6,
// (4 - 6u^2 + 3u^3)/6, (1 + 3u + 3u^2 - 3u^3)/6, u^3/6.
static void bspline_basis(float u, float w[4])
{
    const float om = 1.0f - u, u2 = u * u, u3 = u2 * u;
    w[0] = om * om * om / 6.0f;
    w[1] = (4.0f - 6.0f * u2 + 3.0f * u3) / 6.0f;
    w[2] = (1.0f + 3.0f * u + 3.0f * u2 - 3.0f * u3) / 6.0f;
    w[3] = u3 / 6.0f;
}

// velv(i, j), i = 0..nvz+1, j = 0..nvx+1, from a phase-velocity map of the
// nx * ny grid (gridder_parallel :842-849: real(pv(i*(nvx+2)+j+1)))
static void fill_velv(int nvx, int nvz, const double* pv, float* velv)
{
    for (int i = 0; i <= nvz + 1; ++i)
        for (int j = 0; j <= nvx + 1; ++j)
            velv[(size_t)j * (nvz + 2) + i] = (float)pv[(size_t)i * (nvx + 2) + j];
}
#define VELV(i, j) velv[(size_t)(j) * (nvz + 2) + (i)]

// gridder_parallel (CalSurfG_parallel.f90:811-909): the propagation grid's
// velocities veln (nnz x nnx, ld = nnz) from the vertex values velv.
static void gridder(int nvx, int nvz, int gdx, int gdz, const float* velv, float* veln)
{
    const int nnz = (nvz - 1) * gdz + 1, ld = nnz;
    float ui[64][4], vi[64][4];
    for (int i = 1; i <= gdx + 1; ++i) bspline_basis((float)(i - 1) / (float)gdx, ui[i]);
    for (int i = 1; i <= gdz + 1; ++i) bspline_basis((float)(i - 1) / (float)gdz, vi[i]);
    for (int i = 1; i <= nvz - 1; ++i) {
        const int conz = i == nvz - 1 ? gdz + 1 : gdz;
        for (int j = 1; j <= nvx - 1; ++j) {
            const int conx = j == nvx - 1 ? gdx + 1 : gdx;
            for (int l = 1; l <= conz; ++l) {
                const int stz = gdz * (i - 1) + l;
                for (int m = 1; m <= conx; ++m) {
                    const int stx = gdx * (j - 1) + m;
                    float sumi = 0.0f;
                    for (int i1 = 1; i1 <= 4; ++i1) {
                        float sumj = 0.0f;
                        for (int j1 = 1; j1 <= 4; ++j1) sumj = sumj + ui[m][j1 - 1] * VELV(i - 2 + i1, j - 2 + j1);
                        sumi = sumi + vi[l][i1 - 1] * sumj;
                    }
                    AT(veln, stz, stx) = sumi;
                }
            }
        }
    }
}

// bsplrefine_parallel (CalSurfG_parallel.f90:918-989): the refined source
// grid's velocities (nnz x nnx nodes, ld = nnz) over the coarse box
// vnl..vnr x vnt..vnb, at sgdl times the coarse density.
static void bsplrefine(int vnl, int vnr, int vnt, int vnb, int nnx, int nnz, int nvx, int nvz, int gdx,
                       int gdz, int sgdl, const float* velv, float* veln)
{
    const int ld = nnz, nrxr = gdx * sgdl, nrzr = gdz * sgdl;
    float (*ui)[4] = malloc(sizeof(float[4]) * (size_t)(nrxr + 2));
    float (*vi)[4] = malloc(sizeof(float[4]) * (size_t)(nrzr + 2));
    for (int j = 1; j <= nrxr + 1; ++j) bspline_basis((float)(j - 1) / (float)nrxr, ui[j]);
    for (int i = 1; i <= nrzr + 1; ++i) bspline_basis((float)(i - 1) / (float)nrzr, vi[i]);
    const int origx = (vnl - 1) * sgdl + 1, origz = (vnt - 1) * sgdl + 1;
    for (int i = 1; i <= nvz - 1; ++i) {
        const int conz = i == nvz - 1 ? nrzr + 1 : nrzr;
        for (int j = 1; j <= nvx - 1; ++j) {
            const int conx = j == nvx - 1 ? nrxr + 1 : nrxr;
            for (int k = 1; k <= conz; ++k) {
                int st1 = gdz * (i - 1) + (k - 1) / sgdl + 1;
                if (st1 < vnt || st1 > vnb) continue;
                st1 = nrzr * (i - 1) + k;
                for (int l = 1; l <= conx; ++l) {
                    int st2 = gdx * (j - 1) + (l - 1) / sgdl + 1;
                    if (st2 < vnl || st2 > vnr) continue;
                    st2 = nrxr * (j - 1) + l;
                    float sum[4];
                    for (int i1 = 1; i1 <= 4; ++i1) {
                        float s = 0.0f;
                        for (int j1 = 1; j1 <= 4; ++j1) s = s + ui[l][j1 - 1] * VELV(i - 2 + i1, j - 2 + j1);
                        sum[i1 - 1] = vi[k][i1 - 1] * s;
                    }
                    const int idm1 = st1 - origz + 1, idm2 = st2 - origx + 1;
                    if (idm1 < 1 || idm1 > nnz || idm2 < 1 || idm2 > nnx) continue;
                    AT(veln, idm1, idm2) = sum[0] + sum[1] + sum[2] + sum[3];
                }
            }
        }
    }
    free(ui);
    free(vi);
}

// ------------------------------------------------------------ receivers
// srtimes_parallel (CalSurfG_parallel.f90:997-1125): the traveltime at a
// receiver, bilinear from its cell's four nodes, or, when source and
// receiver share a cell or lie closer than the smallest node spacing, the
// distance over the mean of the two interpolated velocities.  Returns 0 or
// -1 (receiver outside the grid).
static int srtimes(float scx, float scz, float rcx1, float rcz1, const Grid* g, const float* veln,
                   const float* ttn, float* out)
{
    const int ld = g->ld, nnx = g->nnx, nnz = g->nnz;
    const float earth = g->earth;
    int irx = (int)((rcx1 - g->gox) / g->dnx) + 1;
    int irz = (int)((rcz1 - g->goz) / g->dnz) + 1;
    int sw = 0;
    if (irx < 1 || irx > nnx || irz < 1 || irz > nnz) return -1;
    if (irx == nnx) irx -= 1;
    if (irz == nnz) irz -= 1;
    const int isx = (int)((scx - g->gox) / g->dnx) + 1;
    const int isz = (int)((scz - g->goz) / g->dnz) + 1;
    float dpl = g->dnx * earth;
    float rd1 = g->dnz * earth * sinf(g->gox);
    if (rd1 < dpl) dpl = rd1;
    rd1 = g->dnz * earth * sinf(g->gox + (float)(nnx - 1) * g->dnx);
    if (rd1 < dpl) dpl = rd1;
    float t = (scx - rcx1) * earth;
    float sred = t * t;
    t = (scz - rcz1) * earth * sinf(rcx1);
    sred = sred + t * t;
    sred = sqrtf(sred);
    if (sred < dpl) sw = 1;
    if (isx == irx && isz == irz) sw = 1;
    float trr;
    if (sw) {
        // the source's cell (not clamped here, :1062-1063): a source on the
        // last node would read past the grid, which the reference's
        // bounds-checked build stops on
        if (isx < 1 || isx >= nnx || isz < 1 || isz >= nnz) return -1;
        float vss[2][2];
        for (int k = 1; k <= 2; ++k)
            for (int l = 1; l <= 2; ++l) vss[k - 1][l - 1] = AT(veln, isz - 1 + l, isx - 1 + k);
        float drx = (scx - g->gox) - (float)(isx - 1) * g->dnx;
        float drz = (scz - g->goz) - (float)(isz - 1) * g->dnz;
        const float vels = bilinear(vss, drx, drz, g->dnx, g->dnz);
        for (int k = 1; k <= 2; ++k)
            for (int l = 1; l <= 2; ++l) vss[k - 1][l - 1] = AT(veln, irz - 1 + l, irx - 1 + k);
        drx = (rcx1 - g->gox) - (float)(irx - 1) * g->dnx;
        drz = (rcz1 - g->goz) - (float)(irz - 1) * g->dnz;
        const float velr = bilinear(vss, drx, drz, g->dnx, g->dnz);
        trr = 2.0f * sred / (vels + velr);
    } else {
        const float drx = (rcx1 - g->gox) - (float)(irx - 1) * g->dnx;
        const float drz = (rcz1 - g->goz) - (float)(irz - 1) * g->dnz;
        trr = 0.0f;
        for (int k = 1; k <= 2; ++k)
            for (int l = 1; l <= 2; ++l) {
                const float produ = (1.0f - fabsf(((float)(l - 1) * g->dnz - drz) / g->dnz)) *
                                    (1.0f - fabsf(((float)(k - 1) * g->dnx - drx) / g->dnx));
                trr = trr + AT(ttn, irz - 1 + l, irx - 1 + k) * produ;
            }
    }
    *out = trr;
    return 0;
}

// ------------------------------------------------------------ one source
// The traveltime field of one source on the coarse grid (nnz x nnx, ld =
// nnz) as the per-(period, source) loop of CalSurfG_parallel.f90:2148-2325
// forms it with source-grid refinement (asgr = 1): the refined grid over
// the coarse nodes within sgs of the source's cell, sgdl times denser,
// swept until its narrow band reaches the box's side (urg = 1); its nodes
// that coincide with coarse nodes carry their status and times over, alive
// nodes next to far ones are made close again, and the sweep finishes on
// the coarse grid (urg = 2).  asgr = 0 runs the coarse sweep from the
// source point.  ttn and nsts hold the coarse field and status on return.
static int one_source(const OrFmmParams* P, const float* velv, const float* veln, float x, float z,
                      float* ttn, int* nsts)
{
    const int nvx = P->nx - 2, nvz = P->ny - 2;
    const int nnx = (nvx - 1) * P->gdx + 1, nnz = (nvz - 1) * P->gdz + 1;
    const float dvx = P->dvxd * kPi / 180.0f, dvz = P->dvzd * kPi / 180.0f;
    Grid cg;
    cg.nnx = nnx; cg.nnz = nnz; cg.ld = nnz;
    cg.dnx = dvx / (float)P->gdx; cg.dnz = dvz / (float)P->gdz;
    cg.gox = (90.0f - P->goxd) * kPi / 180.0f;
    cg.goz = P->gozd * kPi / 180.0f;
    cg.earth = P->earth; cg.fom = P->fom;
    const int maxbt = (int)llround((double)P->snb * (double)nnx * (double)nnz);
    int r = 0;
    Bt* btg = NULL;
    if (!P->asgr) {
        btg = malloc(sizeof(Bt) * (size_t)(maxbt + 1));
        r = travel(x, z, 0, &cg, 0, 0, 0, 0, nsts, veln, ttn, btg, maxbt);
        free(btg);
        return r;
    }
    int isx = (int)((x - cg.gox) / cg.dnx) + 1;
    int isz = (int)((z - cg.goz) / cg.dnz) + 1;
    if (isx < 1 || isx > nnx || isz < 1 || isz > nnz) return -1;
    if (isx == nnx) isx -= 1;
    if (isz == nnz) isz -= 1;
    int vnl = isx - P->sgs; if (vnl < 1) vnl = 1;
    int vnr = isx + P->sgs; if (vnr > nnx) vnr = nnx;
    int vnt = isz - P->sgs; if (vnt < 1) vnt = 1;
    int vnb = isz + P->sgs; if (vnb > nnz) vnb = nnz;
    Grid rg;
    rg.nnx = (vnr - vnl) * P->sgdl + 1;
    rg.nnz = (vnb - vnt) * P->sgdl + 1;
    rg.ld = rg.nnz;
    rg.dnx = dvx / (float)(P->gdx * P->sgdl);
    rg.dnz = dvz / (float)(P->gdz * P->sgdl);
    // gorx = gox + dnx*(vnl-1) (:2189-2190) rounded once: the reference's
    // example run (examples/test4_Yunnan/smooth) was built with fused
    // multiply-adds, and this origin decides the source's refined cell for
    // sources on coarse nodes (two of its 46 sources land one refined cell
    // apart, 0.08 s, with two roundings)
    rg.gox = fmaf(cg.dnx, (float)(vnl - 1), cg.gox);
    rg.goz = fmaf(cg.dnz, (float)(vnt - 1), cg.goz);
    rg.earth = P->earth; rg.fom = P->fom;
    // the heap is sized from the larger of the two grids' dimensions, as the
    // reference reallocates it (:2208-2224)
    int maxbt_r = maxbt;
    if (rg.nnx > nnx || rg.nnz > nnz) {
        const int d1 = rg.nnx > nnx ? rg.nnx : nnx, d2 = rg.nnz > nnz ? rg.nnz : nnz;
        maxbt_r = (int)llround((double)P->snb * (double)d1 * (double)d2);
    }
    const size_t nr = (size_t)rg.nnx * rg.nnz;
    float* velr = malloc(sizeof(float) * nr);
    float* ttr = malloc(sizeof(float) * nr);
    int* nsr = malloc(sizeof(int) * nr);
    btg = malloc(sizeof(Bt) * (size_t)(maxbt_r + 1));
    for (size_t q = 0; q < nr; ++q) velr[q] = 0.0f;
    bsplrefine(vnl, vnr, vnt, vnb, rg.nnx, rg.nnz, nvx, nvz, P->gdx, P->gdz, P->sgdl, velv, velr);
    r = travel(x, z, 1, &rg, vnl, vnr, vnt, vnb, nsr, velr, ttr, btg, maxbt_r);
    if (!r) {
        // refined nodes on coarse nodes -> coarse status and times (:2245-2262)
        int ld = nnz;
        for (size_t q = 0; q < (size_t)nnx * nnz; ++q) nsts[q] = -1;
        for (int k = 1; k <= rg.nnz; k += P->sgdl) {
            const int idm1 = vnt + (k - 1) / P->sgdl;
            for (int l = 1; l <= rg.nnx; l += P->sgdl) {
                const int idm2 = vnl + (l - 1) / P->sgdl;
                const int st = nsr[(size_t)(l - 1) * rg.ld + (k - 1)];
                AT(nsts, idm1, idm2) = st;
                if (st >= 0) AT(ttn, idm1, idm2) = ttr[(size_t)(l - 1) * rg.ld + (k - 1)];
            }
        }
        // alive nodes next to far ones become close (:2290-2309)
        for (int k = 1; k <= nnx; ++k)
            for (int l = 1; l <= nnz; ++l) {
                if (AT(nsts, l, k) != 0) continue;
                if (l - 1 >= 1 && AT(nsts, l - 1, k) == -1) AT(nsts, l, k) = 1;
                if (l + 1 <= nnz && AT(nsts, l + 1, k) == -1) AT(nsts, l, k) = 1;
                if (k - 1 >= 1 && AT(nsts, l, k - 1) == -1) AT(nsts, l, k) = 1;
                if (k + 1 <= nnx && AT(nsts, l, k + 1) == -1) AT(nsts, l, k) = 1;
            }
        r = travel(x, z, 2, &cg, vnl, vnr, vnt, vnb, nsts, veln, ttn, btg, maxbt_r);
    }
    free(velr);
    free(ttr);
    free(nsr);
    free(btg);
    return r;
}

// ------------------------------------------------------------ batch
// The forward traveltimes of a data set: for every (period, source)
// instance, gridder on the period's phase-velocity map (pv column per
// period, nx * ny values, the x (latitude) index fastest), the source's
// field, then srtimes at each of its receivers (CSR rc_off).  times[r] in
// the order of the receivers.  ttn_out, when not NULL, receives each
// instance's coarse field (nnz * nnx floats per instance).  Returns 0 or
// the first instance's error (as above).
int or_fmm_batch(const OrFmmParams* P, const double* pv, int ninst, const int* inst_period,
                 const float* scx, const float* scz, const long* rc_off, const float* rcx,
                 const float* rcz, float* times, float* ttn_out, int nthreads)
{
    const int nvx = P->nx - 2, nvz = P->ny - 2;
    const int nnx = (nvx - 1) * P->gdx + 1, nnz = (nvz - 1) * P->gdz + 1;
    const size_t ncoarse = (size_t)nnx * nnz;
    int err = 0;
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int s = 0; s < ninst; ++s) {
        float* velv = malloc(sizeof(float) * (size_t)(nvx + 2) * (nvz + 2));
        float* veln = malloc(sizeof(float) * ncoarse);
        float* ttn = malloc(sizeof(float) * ncoarse);
        int* nsts = malloc(sizeof(int) * ncoarse);
        fill_velv(nvx, nvz, pv + (size_t)inst_period[s] * (size_t)P->nx * P->ny, velv);
        gridder(nvx, nvz, P->gdx, P->gdz, velv, veln);
        for (size_t q = 0; q < ncoarse; ++q) ttn[q] = 0.0f;
        int r = one_source(P, velv, veln, scx[s], scz[s], ttn, nsts);
        if (!r) {
            Grid cg;
            const float dvx = P->dvxd * kPi / 180.0f, dvz = P->dvzd * kPi / 180.0f;
            cg.nnx = nnx; cg.nnz = nnz; cg.ld = nnz;
            cg.dnx = dvx / (float)P->gdx; cg.dnz = dvz / (float)P->gdz;
            cg.gox = (90.0f - P->goxd) * kPi / 180.0f;
            cg.goz = P->gozd * kPi / 180.0f;
            cg.earth = P->earth; cg.fom = P->fom;
            for (long q = rc_off[s]; q < rc_off[s + 1] && !r; ++q)
                r = srtimes(scx[s], scz[s], rcx[q], rcz[q], &cg, veln, ttn, &times[q]);
        }
        if (ttn_out) memcpy(ttn_out + (size_t)s * ncoarse, ttn, sizeof(float) * ncoarse);
        if (r) {
#pragma omp critical(or_fmm_err)
            if (!err) err = r;
        }
        free(velv);
        free(veln);
        free(ttn);
        free(nsts);
    }
    return err;
}

// One coarse-grid field from a given velocity grid (nnz x nnx) and source,
// for tests that build their own grids: travel with urg = 0 (no source
// refinement).  nsts_out, when not NULL, receives the final status.
int or_fmm_travel(int nnx, int nnz, float gox, float goz, float dnx, float dnz, float earth, int fom,
                  float snb, const float* veln, float scx, float scz, float* ttn, int* nsts_out)
{
    Grid g;
    g.nnx = nnx; g.nnz = nnz; g.ld = nnz;
    g.gox = gox; g.goz = goz; g.dnx = dnx; g.dnz = dnz; g.earth = earth; g.fom = fom;
    const int maxbt = (int)llround((double)snb * (double)nnx * (double)nnz);
    int* nsts = malloc(sizeof(int) * (size_t)nnx * nnz);
    Bt* btg = malloc(sizeof(Bt) * (size_t)(maxbt + 1));
    const int r = travel(scx, scz, 0, &g, 0, 0, 0, 0, nsts, veln, ttn, btg, maxbt);
    if (nsts_out) memcpy(nsts_out, nsts, sizeof(int) * (size_t)nnx * nnz);
    free(nsts);
    free(btg);
    return r;
}
