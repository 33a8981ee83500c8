// First-arrival traveltimes on the refined spherical grid for many
// (period, source) instances at once: the reference's fast-marching solver
// (code/src_inv_iso_joint/CalSurfG_parallel.f90:125-336, travel_parallel,
// with fouds1/fouds2 :346-622 and the binary-heap narrow band :631-803),
// its source-grid refinement (:2148-2325, bsplrefine_parallel :918-989),
// the B-spline gridding of a phase-velocity map (gridder_parallel
// :811-909) and the receiver interpolation (srtimes_parallel :997-1125).
//
// Fast marching pops the narrow band's minimum one node at a time, and the
// value a node keeps depends on which neighbours were alive when it was
// last updated, ties included; a parallel front (several nodes accepted at
// once) changes those sets and so the times.  So each instance runs the
// reference's sequence exactly, on one warp: lane 0 marches (heap, upwind
// updates), the 32 lanes share the data-parallel steps (the refined grid's
// B-spline values, status resets, the transfer from the refined to the
// coarse grid, the receivers).  The instances (up to several thousand per
// data set) fill the GPU: a persistent grid of warps takes them from a
// queue, each with its own slice of the workspace.  The marching is a chain
// of dependent loads, so its speed is set by memory latency, not by
// bandwidth or FP32 throughput.
//
// Arithmetic: every value is real*4 as in the reference, every operation
// rounds on its own in the Fortran's order (k_fmm.cu, which includes this
// file, is compiled with -fmad=false; the one fused multiply-add, the refined grid's origin, is
// formed on the host as the reference's example build forms it), division
// and sqrtf are IEEE, and the ri*sin(colatitude) factors are tables the
// host fills with the C library's sinf.  The results equal the CPU
// restatement bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <cmath>
#include <vector>

#include "../../include/dazi_dk.h"

namespace dk {
namespace fmm {

constexpr int kWarpsPerBlock = 4;
// narrow-band heap positions each warp keeps in shared memory (1 .. 1535);
// bands larger than that (rare: the front of a 176 x 196 grid is at most
// ~750 nodes) continue in the warp's global workspace
constexpr int kHeapShared = 1536;

// A node of a field: its time and status, the reference's ttn and nsts
// (-1 far, 0 alive, > 0 its position in the narrow band's heap), side by
// side so that one load brings both.
struct Node {
    float t;
    int s;
};

// heap entry: the node's time (kept equal to its t while it is in the band)
// and its offset in the field's arrays ((ix - 1) * nnz + (iz - 1))
struct HeapE {
    float key;
    int idx;
};

// The band's heap: positions below kHeapShared in shared memory, the rest in
// the global workspace.  ShHeap is the fast path for a band that fits in
// shared memory (the usual case), MixHeap the general one.
struct ShHeap {
    HeapE* sh;
    __device__ __forceinline__ HeapE get(int i) const { return sh[i]; }
    __device__ __forceinline__ void put(int i, HeapE e) const { sh[i] = e; }
};

struct MixHeap {
    HeapE* sh;
    HeapE* gl;
    __device__ __forceinline__ HeapE get(int i) const { return i < kHeapShared ? sh[i] : gl[i]; }
    __device__ __forceinline__ void put(int i, HeapE e) const
    {
        if (i < kHeapShared) sh[i] = e;
        else gl[i] = e;
    }
};

struct Heap {
    HeapE* sh;   // positions < kHeapShared (shared memory on the GPU)
    HeapE* gl;   // all positions (global workspace; the low ones unused)
};

// One propagation grid of one instance: node (iz, ix), 1-based, at
// [(ix - 1) * nnz + (iz - 1)] as the reference's ttn(nnz, nnx).
struct FField {
    int nnx, nnz;
    float gox, goz, dnx, dnz, earth;
    int fom;
    const float* veln;
    const float* slow;    // 1 / veln, formed once per node (the reference's slown)
    const float* risti;   // [ix - 1]: earth * sin(gox + (ix - 1) * dnx)
    Node* node;
};

// (a field has at most 32767 x 32767 nodes: 32-bit offsets)
#define FN(iz, ix) F.node[((ix) - 1) * F.nnz + ((iz) - 1)]
#define FIDX(iz, ix) (((ix) - 1) * F.nnz + ((iz) - 1))
#define FV(iz, ix) F.veln[((ix) - 1) * F.nnz + ((iz) - 1)]
#define FS(iz, ix) F.slow[((ix) - 1) * F.nnz + ((iz) - 1)]

// error codes of one instance
constexpr int kErrOutside = 1;   // source or receiver outside the grid
constexpr int kErrBand = 2;      // narrow band beyond its capacity
constexpr int kErrNoSol = 3;     // a node without an upwind solution
constexpr int kErrSteps = 4;     // more pops than nodes (cannot happen)
constexpr int kErrNoBand = 5;    // no close node after the refined sweep

// ------------------------------------------------------------ heap
// addtree_parallel (CalSurfG_parallel.f90:631-675): the new node enters at
// the bottom and moves up while smaller than its parent (parents move down
// into the hole, as the reference's swaps leave them)
template <class H>
__device__ __forceinline__ void heap_add_in(const FField& F, int idx, float key, int ntr, const H& h)
{
    int tpc = ntr, tpp = tpc / 2;
    while (tpp > 0) {
        const HeapE p = h.get(tpp);
        if (!(key < p.key)) break;
        h.put(tpc, p);
        F.node[p.idx].s = tpc;
        tpc = tpp;
        tpp = tpc / 2;
    }
    h.put(tpc, HeapE{key, idx});
    F.node[idx].s = tpc;
}

__device__ int heap_add(const FField& F, int iz, int ix, float key, int& ntr, int cap, const Heap& h)
{
    if (ntr >= cap) return kErrBand;
    ntr += 1;
    if (ntr < kHeapShared) heap_add_in(F, FIDX(iz, ix), key, ntr, ShHeap{h.sh});
    else heap_add_in(F, FIDX(iz, ix), key, ntr, MixHeap{h.sh, h.gl});
    return 0;
}

// downtree_parallel (CalSurfG_parallel.f90:686-761): the root has been
// taken; the last entry moves to the root and down while a child is
// smaller (the smaller child; the right one only if strictly smaller, as
// the reference's rd1 > rd2 selects it)
template <class H>
__device__ __forceinline__ void heap_pop_in(const FField& F, int& ntr, const H& h)
{
    if (ntr == 1) { ntr = 0; return; }
    const HeapE last = h.get(ntr);
    ntr -= 1;
    int tpp = 1, tpc = 2;
    while (tpc <= ntr) {
        HeapE c = h.get(tpc);
        if (tpc < ntr) {
            const HeapE c2 = h.get(tpc + 1);
            if (c.key > c2.key) { c = c2; tpc += 1; }
        }
        if (!(c.key < last.key)) break;
        h.put(tpp, c);
        F.node[c.idx].s = tpp;
        tpp = tpc;
        tpc = 2 * tpp;
    }
    h.put(tpp, last);
    F.node[last.idx].s = tpp;
}

__device__ void heap_pop(const FField& F, int& ntr, const Heap& h)
{
    if (ntr < kHeapShared) heap_pop_in(F, ntr, ShHeap{h.sh});
    else heap_pop_in(F, ntr, MixHeap{h.sh, h.gl});
}

// ------------------------------------------------------------ upwind updates
// One quadrant of the upwind update of node (iz, ix): fouds1_parallel
// (CalSurfG_parallel.f90:346-432) for fom 0, fouds2_parallel (:443-622) for
// fom 1.  Quadrant (a, b) uses the x-neighbour j = ix - 1 + 2a, the
// z-neighbour k = iz - 1 + 2b and, for the second-order stencils, the nodes
// j2, k2 beyond them; it exists where j and k lie in the grid (the
// reference skips the others).  has: it gives a time (the reference's
// swsol); trav: that time.  The node's time is the minimum over its
// quadrants with a time (the reference's travm), which the GPU forms on
// four lanes at once.
__device__ void quadrant(const FField& F, int iz, int ix, int a, int b, int& has, float& trav)
{
    has = 0;
    trav = 0.0f;
    const int j = ix - 1 + 2 * a, j2 = ix - 2 + 4 * a;
    const int k = iz - 1 + 2 * b, k2 = iz - 2 + 4 * b;
    if (j < 1 || j > F.nnx || k < 1 || k > F.nnz) return;
    const bool inj2 = j2 >= 1 && j2 <= F.nnx, ink2 = k2 >= 1 && k2 <= F.nnz;
    const Node nj = FN(iz, j), nk = FN(k, ix);
    const Node nj2 = FN(iz, inj2 ? j2 : j), nk2 = FN(ink2 ? k2 : k, ix);
    const float slown = FS(iz, ix), ri = F.earth, risti = F.risti[ix - 1];
    const bool aj = nj.s == 0, ak = nk.s == 0;
    const float tj = nj.t, tk = nk.t, tj2 = nj2.t, tk2 = nk2.t;
    float qa = 1.0f, qb = 0.0f, qc = 0.0f, tref = 0.0f;
    bool third = false;    // tdiv = 3 (second-order operator); else 1
    if (F.fom == 0) {
        if (aj) {
            has = 1;
            if (ak) {
                const float u = ri * F.dnx, v = risti * F.dnz;
                const float em = tk - tj;
                qa = u * u + v * v;
                qb = -2.0f * (u * u) * em;
                qc = (u * u) * (em * em - (v * v) * (slown * slown));
            } else {
                qc = -(slown * slown) * (ri * ri) * (F.dnx * F.dnx);
            }
            tref = tj;
        } else if (ak) {
            has = 1;
            const float t = slown * risti * F.dnz;
            qc = -(t * t);
            tref = tk;
        }
    } else {
        // fouds2_parallel's eight cases in one form (the lanes of a warp sit
        // in different cases), with the reference's operation order:
        //   two neighbours:  qa = P + Q, qb = (c em) R, qc = R (em em - S (s s)),
        //                    em = ((x1 - x2) - x3) + x4;
        //   one neighbour:   qa = 1, qb = 0, qc = ((-(s s)) G) H;
        //   tref = g tA - tB.
        // Scaling by a power of two and swapping the factors of one product
        // are exact, so e.g. (-2 u^2) em = (-2 em) u^2 and (-u^2) s^2 =
        // ((-(s s)) u^2) 1 bit for bit; subtracting or adding 0 is exact.
        const bool swj = aj && inj2 && nj2.s == 0 && tj > tj2;
        const bool swk = ak && ink2 && nk2.s == 0 && tk > tk2;
        const float u1 = ri * F.dnx, u2 = 2.0f * ri * F.dnx;
        const float v1 = risti * F.dnz, v2 = 2.0f * risti * F.dnz;
        const float u1s = u1 * u1, u2s = u2 * u2, v1s = v1 * v1, v2s = v2 * v2;
        const float ss = slown * slown;
        const bool two = (swj || aj) && (swk || ak);
        has = (swj || aj || swk || ak) ? 1 : 0;
        // two neighbours: (swj, swk) (swj, ak) (aj, swk) (aj, ak)
        const float P = swj ? (swk ? v2s : u2s) : (swk ? v2s : u1s);
        const float Q = swj ? (swk ? u2s : 9.0f * v1s) : (swk ? 9.0f * u1s : v1s);
        const float cc = swj ? (swk ? 2.0f : 6.0f) : (swk ? 6.0f : -2.0f);
        const float R = swj ? (swk ? u2s : v1s) : u1s;
        const float S2 = swj ? (swk ? v2s : u2s) : (swk ? v2s : v1s);
        const float x1 = swj ? (swk ? 4.0f * tj : 3.0f * tk) : (swk ? 3.0f * tj : tk);
        const float x2 = (swj && swk) ? tj2 : 0.0f;
        const float x3 = swj ? 4.0f * (swk ? tk : tj) : (swk ? 4.0f * tk : tj);
        const float x4 = swj ? (swk ? tk2 : tj2) : (swk ? tk2 : 0.0f);
        // one neighbour: swj, aj, swk, ak alone
        const float G = swj ? u2s : aj ? ri * ri : swk ? v2s : risti * risti;
        const float H = swj ? 1.0f : aj ? F.dnx * F.dnx : swk ? 1.0f : F.dnz * F.dnz;
        if (two) {
            const float em = ((x1 - x2) - x3) + x4;
            qa = P + Q;
            qb = (cc * em) * R;
            qc = R * (em * em - S2 * ss);
        } else {
            qc = (-ss * G) * H;
        }
        // tref: 4 tj - tj2 (swj), tj (aj), 4 tk - tk2 (swk), tk (ak); with two
        // neighbours the x side's, but tk for (swj, ak)
        const bool xside = two ? !(swj && !swk) : (swj || aj);
        const bool second = two ? (swj && swk) : (swj || (!aj && swk));
        const float tA = xside ? tj : tk, tB = second ? (xside ? tj2 : tk2) : 0.0f;
        tref = (second ? 4.0f : 1.0f) * tA - tB;
        third = second;
    }
    if (!has) return;
    // the positive root of qa t^2 + qb t + qc (the reference's rd1, tdsh);
    // trav = (tref + tdsh) / tdiv, and x / 1 = x exactly
    float rd1 = qb * qb - 4.0f * qa * qc;
    if (rd1 < 0.0f) rd1 = 0.0f;
    const float tdsh = (-qb + sqrtf(rd1)) / (2.0f * qa);
    trav = third ? (tref + tdsh) / 3.0f : tref + tdsh;
}

// bilinear_parallel (CalSurfG_parallel.f90:2543-2566); nv[i][j] = nv(i+1, j+1)
__device__ float bilinear(const float nv[2][2], float dsx, float dsz, float dnx, float dnz)
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
// travel_parallel (CalSurfG_parallel.f90:125-336), as phases:
//   travel_start   the first band: urg 0 / 1 the four corners of the
//                  source's cell (statuses already -1); urg 2 the close
//                  nodes (status > 0) of the box vnl..vnr x vnt..vnb, the
//                  only place they can be, in the reference's order;
//   travel_pop     the band's minimum becomes alive; for urg 1 the sweep
//                  stops instead when that node lies on a side of the
//                  refined grid that is not the model's (compared, as in
//                  the reference, with this grid's own node counts on the
//                  right and bottom sides);
//   travel_nbr     the new time of neighbour q (x-1, x+1, z-1, z+1) of the
//                  popped node, if it is far or close;
//   commit_one     its band entry (added, or moved up: addtree_parallel
//                  :631-675, updtree_parallel :770-803).
// The reference runs travel_nbr and commit_one neighbour by neighbour;
// the new times depend only on alive nodes, which the commits do not
// change, so the four travel_nbr may also run first (travel_warp), with
// the commits tracking the heap positions they move (commit_one).
struct Box {
    int vnl, vnr, vnt, vnb;
};

__device__ int travel_start(const FField& F, int urg, float scx, float scz, const Box& B, const Heap& h,
                            int cap, int& ntr)
{
    int isx = (int)((scx - F.gox) / F.dnx) + 1;
    int isz = (int)((scz - F.goz) / F.dnz) + 1;
    if (isx < 1 || isx > F.nnx || isz < 1 || isz > F.nnz) return kErrOutside;
    if (isx == F.nnx) isx -= 1;
    if (isz == F.nnz) isz -= 1;
    ntr = 0;
    int r;
    if (urg == 2) {
        for (int i = B.vnl; i <= B.vnr; ++i)
            for (int j = B.vnt; j <= B.vnb; ++j) {
                const Node n = FN(j, i);
                if (n.s > 0 && (r = heap_add(F, j, i, n.t, ntr, cap, h))) return r;
            }
        // the refined sweep stopped before it reached a coarse node (a
        // source in the last cell before the right or bottom side, whose
        // refined sweep always stops there): the reference leaves the
        // field as its array held it, so this is reported, not computed
        return ntr == 0 ? kErrNoBand : 0;
    }
    float vss[2][2];
    for (int i = 1; i <= 2; ++i)
        for (int j = 1; j <= 2; ++j) vss[i - 1][j - 1] = FV(isz - 1 + j, isx - 1 + i);
    const float dsx = (scx - F.gox) - (float)(isx - 1) * F.dnx;
    const float dsz = (scz - F.goz) - (float)(isz - 1) * F.dnz;
    const float vsrc = bilinear(vss, dsx, dsz, F.dnx, F.dnz);
    for (int i = 1; i <= 2; ++i)
        for (int j = 1; j <= 2; ++j) {
            const float ex = dsx - (float)(i - 1) * F.dnx, ez = dsz - (float)(j - 1) * F.dnz;
            const float ds = sqrtf(ex * ex + ez * ez);
            const float t = 2.0f * ds / (vss[i - 1][j - 1] + vsrc);
            FN(isz - 1 + j, isx - 1 + i).t = t;
            if ((r = heap_add(F, isz - 1 + j, isx - 1 + i, t, ntr, cap, h))) return r;
        }
    return 0;
}

// returns true when the refined sweep stops (the node is made alive too)
__device__ bool travel_pop(const FField& F, int urg, const Box& B, const Heap& h, int& ntr, int& ix, int& iz)
{
    const HeapE root = h.sh[1];
    ix = root.idx / F.nnz + 1;
    iz = root.idx - (ix - 1) * F.nnz + 1;
    F.node[root.idx].s = 0;
    if (urg == 1 && ((ix == 1 && B.vnl != 1) || (ix == F.nnx && B.vnr != F.nnx) || (iz == 1 && B.vnt != 1) ||
                     (iz == F.nnz && B.vnb != F.nnz)))
        return true;
    heap_pop(F, ntr, h);
    return false;
}

// Neighbour q (x-1, x+1, z-1, z+1) of the popped (iz, ix), as explicit
// cases: written as one select per coordinate (q < 2 ? ix - 1 + 2 q : ix),
// lanes 0 and 1 of the warp got ix + 3 on the GPU (sm_100a, CUDA 12.9),
// seen with a self-recording build.
__device__ __forceinline__ bool nbr_of(const FField& F, int iz, int ix, int q, int& niz, int& nix)
{
    niz = iz;
    nix = ix;
    if (q == 0) nix = ix - 1;
    else if (q == 1) nix = ix + 1;
    else if (q == 2) niz = iz - 1;
    else niz = iz + 1;
    return nix >= 1 && nix <= F.nnx && niz >= 1 && niz <= F.nnz;
}

// Neighbour q's status st (0: alive or outside the grid, nothing to do)
// and, otherwise, its new time: the minimum over its quadrants.
__device__ int travel_nbr(const FField& F, int iz, int ix, int q, int& niz, int& nix, int& st, float& t)
{
    st = 0;
    if (!nbr_of(F, iz, ix, q, niz, nix)) return 0;
    st = FN(niz, nix).s;
    if (st == 0) return 0;
    int any = 0;
    float m = 0.0f;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            int has;
            float tr;
            quadrant(F, niz, nix, a, b, has, tr);
            if (has) {
                m = any ? fminf(tr, m) : tr;
                any = 1;
            }
        }
    if (!any) return kErrNoSol;
    t = m;
    return 0;
}

// The commits of one pop's four neighbours, in order.  A close node's
// status is its heap position, and an earlier commit's sift-up may move a
// later neighbour (a parent moving down): the positions st[] are updated
// as entries move, so no status is read back from memory (far stays far:
// the four neighbours are distinct nodes).
struct Pending {
    int z[4], x[4], st[4], idx[4];
    float t[4];
};

template <class H>
__device__ __forceinline__ void commit_in(const FField& F, Pending& P, int q, int tpc, const H& h)
{
    const int idx = P.idx[q];
    const float key = P.t[q];
    int tpp = tpc / 2;
    while (tpp > 0) {
        const HeapE p = h.get(tpp);
        if (!(key < p.key)) break;
        h.put(tpc, p);
        F.node[p.idx].s = tpc;
        // a later neighbour moved down: its position follows
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (r > q && P.st[r] > 0 && P.idx[r] == p.idx) P.st[r] = tpc;
        tpc = tpp;
        tpp = tpc / 2;
    }
    h.put(tpc, HeapE{key, idx});
    F.node[idx].s = tpc;
}

__device__ int commit_one(const FField& F, Pending& P, int q, const Heap& h, int& ntr, int cap)
{
    F.node[P.idx[q]].t = P.t[q];
    int tpc;
    if (P.st[q] < 0) {          // addtree_parallel: enters at the bottom
        if (ntr >= cap) return kErrBand;
        ntr += 1;
        tpc = ntr;
    } else {                    // updtree_parallel: from its position
        tpc = P.st[q];
    }
    if (ntr < kHeapShared) commit_in(F, P, q, tpc, ShHeap{h.sh});
    else commit_in(F, P, q, tpc, MixHeap{h.sh, h.gl});
    return 0;
}

// travel_warp's order on one thread (the host build's driver): after each
// pop the four neighbours' times first, then their commits.
__device__ int travel_four(const FField& F, int urg, float scx, float scz, const Box& B, const Heap& h, int cap)
{
    int ntr = 0, r;
    if ((r = travel_start(F, urg, scx, scz, B, h, cap, ntr))) return r;
    const long long maxpops = (long long)F.nnx * F.nnz + 4;
    for (long long pops = 0; ntr > 0; ++pops) {
        if (pops > maxpops) return kErrSteps;
        int ix, iz;
        if (travel_pop(F, urg, B, h, ntr, ix, iz)) break;
        Pending P;
        int e[4];
        for (int q = 0; q < 4; ++q) {
            P.t[q] = 0.0f;
            e[q] = travel_nbr(F, iz, ix, q, P.z[q], P.x[q], P.st[q], P.t[q]);
            P.idx[q] = FIDX(P.z[q], P.x[q]);
        }
        for (int q = 0; q < 4; ++q) {
            if (e[q]) return e[q];
            if (P.st[q] != 0 && (r = commit_one(F, P, q, h, ntr, cap))) return r;
        }
    }
    return 0;
}

// On a warp: lane 0 keeps the band; after each pop lanes 0..15 form the
// four neighbours' quadrant times at once (lane 4q + 2a + b: quadrant (a, b)
// of neighbour q) and each group of four takes its minimum.
__device__ int travel_warp(const FField& F, int urg, float scx, float scz, const Box& B, const Heap& h, int cap,
                           int lane)
{
    const unsigned all = 0xffffffffu;
    int ntr = 0, r = 0;
    if (lane == 0) r = travel_start(F, urg, scx, scz, B, h, cap, ntr);
    r = __shfl_sync(all, r, 0);
    if (r) return r;
    const long long maxpops = (long long)F.nnx * F.nnz + 4;
    for (long long pops = 0;; ++pops) {
        int code = 0;   // 1 done, 2 refined sweep stopped, 3 too many pops; else (ix << 16) | iz, +4
        if (lane == 0) {
            int ix, iz;
            if (ntr == 0) code = 1;
            else if (pops > maxpops) code = 3;
            else if (travel_pop(F, urg, B, h, ntr, ix, iz)) code = 2;
            else code = 4 + ((ix << 16) | iz);
        }
        code = __shfl_sync(all, code, 0);
        if (code < 4) return code == 3 ? kErrSteps : 0;
        const int ix = (code - 4) >> 16, iz = (code - 4) & 0xffff;
        __syncwarp();
        // lane 4q + 2a + b: quadrant (a, b) of neighbour q
        int niz = 0, nix = 0, st = 0, has = 0;
        float tr = 0.0f;
        if (lane < 16 && nbr_of(F, iz, ix, lane >> 2, niz, nix)) {
            // the status and the quadrant's nodes in one round of loads; the
            // quadrant's time is dropped for an alive neighbour
            st = FN(niz, nix).s;
            quadrant(F, niz, nix, (lane >> 1) & 1, lane & 1, has, tr);
            if (st == 0) has = 0;
        }
        // minimum over the quadrants with a time, within each group of four
        float m = has ? tr : __int_as_float(0x7f800000);
#pragma unroll
        for (int o = 1; o <= 2; o <<= 1) {
            m = fminf(m, __shfl_xor_sync(all, m, o));
            has |= __shfl_xor_sync(all, has, o);
        }
        const int e = (st != 0 && !has) ? kErrNoSol : 0;
        __syncwarp();
        Pending P;
        int eq[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            eq[q] = __shfl_sync(all, e, 4 * q);
            P.st[q] = __shfl_sync(all, st, 4 * q);
            P.z[q] = __shfl_sync(all, niz, 4 * q);
            P.x[q] = __shfl_sync(all, nix, 4 * q);
            P.t[q] = __shfl_sync(all, m, 4 * q);
            P.idx[q] = FIDX(P.z[q], P.x[q]);
        }
        if (lane == 0) {
            for (int q = 0; q < 4 && !r; ++q) {
                if (eq[q]) r = eq[q];
                else if (P.st[q] != 0) r = commit_one(F, P, q, h, ntr, cap);
            }
        }
        r = __shfl_sync(all, r, 0);
        if (r) return r;
        __syncwarp();
    }
}

// ------------------------------------------------------------ gridding
// cubic B-spline basis at u (gridder_parallel :857-876)
__device__ __forceinline__ void bspline_basis(float u, float w[4])
{
    const float om = 1.0f - u, u2 = u * u, u3 = u2 * u;
    w[0] = om * om * om / 6.0f;
    w[1] = (4.0f - 6.0f * u2 + 3.0f * u3) / 6.0f;
    w[2] = (1.0f + 3.0f * u + 3.0f * u2 - 3.0f * u3) / 6.0f;
    w[3] = u3 / 6.0f;
}

// The B-spline value at global node (stz, stx) (1-based) of a grid diced
// ncz x ncx per vertex cell, as gridder_parallel (ncz = gdz) and
// bsplrefine_parallel (ncz = gdz * sgdl) form it: cell i, offset l within
// it (the last cell holds one more node), velv(i, j) at velv[j * (nvz + 2) + i].
__device__ float bspline_node(const float* velv, int nvx, int nvz, int ncz, int ncx, int stz, int stx)
{
    int i = (stz - 1) / ncz + 1, j = (stx - 1) / ncx + 1;
    if (i > nvz - 1) i = nvz - 1;
    if (j > nvx - 1) j = nvx - 1;
    const int l = stz - ncz * (i - 1), m = stx - ncx * (j - 1);
    float ui[4], vi[4];
    bspline_basis((float)(m - 1) / (float)ncx, ui);
    bspline_basis((float)(l - 1) / (float)ncz, vi);
    const int ld = nvz + 2;
    float sum = 0.0f;
    for (int i1 = 1; i1 <= 4; ++i1) {
        float s = 0.0f;
        for (int j1 = 1; j1 <= 4; ++j1) s = s + ui[j1 - 1] * velv[(j - 2 + j1) * ld + (i - 2 + i1)];
        sum = sum + vi[i1 - 1] * s;
    }
    return sum;
}

// velv of every period map (real(pv), gridder_parallel :842-849) and the
// coarse grid's velocities veln and slownesses 1 / veln, one thread per
// value
__global__ void fmm_velv_kernel(const double* pv, int nx, int ny, int nper, float* velv)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long per = (long long)nx * ny;
    if (t >= per * nper) return;
    const long long p = t / per, r = t % per;
    const int i = (int)(r / nx), j = (int)(r % nx);   // i: z (longitude) vertex, j: x vertex
    velv[p * per + (long long)j * ny + i] = (float)pv[p * per + (long long)i * nx + j];
}

__global__ void fmm_gridder_kernel(const float* velv, int nvx, int nvz, int gdx, int gdz, int nper,
                                   float* veln, float* slow)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nnx = (nvx - 1) * gdx + 1, nnz = (nvz - 1) * gdz + 1;
    const long long nn = (long long)nnx * nnz;
    if (t >= nn * nper) return;
    const long long p = t / nn, r = t % nn;
    const int stx = (int)(r / nnz) + 1, stz = (int)(r % nnz) + 1;
    const float v = bspline_node(velv + p * (long long)(nvx + 2) * (nvz + 2), nvx, nvz, gdz, gdx, stz, stx);
    veln[t] = v;
    slow[t] = 1.0f / v;
}

// ------------------------------------------------------------ instances
// One (period, source) instance, laid out by the host.
struct FInst {
    int period;                 // map (and coarse velocity grid) index
    float scx, scz;             // source, colatitude / longitude (rad)
    int vnl, vnr, vnt, vnb;     // refined box in coarse nodes (asgr)
    int nrnx, nrnz;             // refined grid nodes
    float gorx, gorz;           // refined grid origin
    int cap;                    // narrow-band capacity (the reference's maxbt)
    long long rc_b, rc_e;       // receivers
    long long risti_r;          // offset of the refined grid's ri*sin table
};

struct FArgs {
    int ninst;
    const FInst* inst;
    int nnx, nnz, nvx, nvz, gdx, gdz, sgdl, fom, asgr;
    float gox, goz, dnx, dnz, drnx, drnz, earth, dpl;
    const float* velv;          // [period][(nvx + 2) * (nvz + 2)]
    const float* veln;          // [period][nnx * nnz]
    const float* slow;          // [period][nnx * nnz]: 1 / veln
    const float* risti_c;       // [nnx]
    const float* risti_r;
    const float* rcx;
    const float* rcz;
    const float* sin_rcx;       // [receiver]: sinf(rcx)
    float* times;
    float* ttn_out;             // [instance][nnx * nnz] or nullptr
    // per-warp workspace slots
    Node* w_node;               // coarse field
    Node* w_rnode;              // refined field
    float* w_vr;                // refined velocities
    float* w_sr;                // refined slownesses
    HeapE* w_heap;              // heap positions >= kHeapShared
    long long wc, wr, wh;       // slot sizes: coarse nodes, refined nodes, heap positions
    unsigned* queue;
    int* err;                   // first error code (0: none)
    int* err_inst;              // its instance
};

__device__ void record_error(const FArgs& a, int code, int s)
{
    if (atomicCAS(a.err, 0, code) == 0) *a.err_inst = s;
}

// srtimes_parallel (CalSurfG_parallel.f90:997-1125) for receiver q on the
// coarse field F (dpl, the smallest node spacing, and sin(rcx) come from the
// host)
__device__ int srtimes(const FArgs& a, const FField& F, float scx, float scz, long long q, float& out)
{
    const float rcx1 = a.rcx[q], rcz1 = a.rcz[q];
    int irx = (int)((rcx1 - F.gox) / F.dnx) + 1;
    int irz = (int)((rcz1 - F.goz) / F.dnz) + 1;
    if (irx < 1 || irx > F.nnx || irz < 1 || irz > F.nnz) return kErrOutside;
    if (irx == F.nnx) irx -= 1;
    if (irz == F.nnz) irz -= 1;
    const int isx = (int)((scx - F.gox) / F.dnx) + 1;
    const int isz = (int)((scz - F.goz) / F.dnz) + 1;
    float t = (scx - rcx1) * F.earth;
    float sred = t * t;
    t = (scz - rcz1) * F.earth * a.sin_rcx[q];
    sred = sred + t * t;
    sred = sqrtf(sred);
    const bool sw = sred < a.dpl || (isx == irx && isz == irz);
    float trr;
    if (sw) {
        // the source's cell is not clamped here (:1062-1063): a source on
        // the last node would read past the grid, which the reference's
        // bounds-checked build stops on
        if (isx < 1 || isx >= F.nnx || isz < 1 || isz >= F.nnz) return kErrOutside;
        float vss[2][2];
        for (int k = 1; k <= 2; ++k)
            for (int l = 1; l <= 2; ++l) vss[k - 1][l - 1] = FV(isz - 1 + l, isx - 1 + k);
        float drx = (scx - F.gox) - (float)(isx - 1) * F.dnx;
        float drz = (scz - F.goz) - (float)(isz - 1) * F.dnz;
        const float vels = bilinear(vss, drx, drz, F.dnx, F.dnz);
        for (int k = 1; k <= 2; ++k)
            for (int l = 1; l <= 2; ++l) vss[k - 1][l - 1] = FV(irz - 1 + l, irx - 1 + k);
        drx = (rcx1 - F.gox) - (float)(irx - 1) * F.dnx;
        drz = (rcz1 - F.goz) - (float)(irz - 1) * F.dnz;
        const float velr = bilinear(vss, drx, drz, F.dnx, F.dnz);
        trr = 2.0f * sred / (vels + velr);
    } else {
        const float drx = (rcx1 - F.gox) - (float)(irx - 1) * F.dnx;
        const float drz = (rcz1 - F.goz) - (float)(irz - 1) * F.dnz;
        trr = 0.0f;
        for (int k = 1; k <= 2; ++k)
            for (int l = 1; l <= 2; ++l) {
                const float produ = (1.0f - fabsf(((float)(l - 1) * F.dnz - drz) / F.dnz)) *
                                    (1.0f - fabsf(((float)(k - 1) * F.dnx - drx) / F.dnx));
                trr = trr + FN(irz - 1 + l, irx - 1 + k).t * produ;
            }
    }
    out = trr;
    return 0;
}

// The fields of an instance in workspace slot `slot`: C the coarse grid, R
// the refined source grid.
__device__ void inst_fields(const FArgs& a, const FInst& I, long long slot, FField& C, FField& R)
{
    C.nnx = a.nnx; C.nnz = a.nnz;
    C.gox = a.gox; C.goz = a.goz; C.dnx = a.dnx; C.dnz = a.dnz; C.earth = a.earth; C.fom = a.fom;
    C.veln = a.veln + (long long)I.period * a.nnx * a.nnz;
    C.slow = a.slow + (long long)I.period * a.nnx * a.nnz;
    C.risti = a.risti_c;
    C.node = a.w_node + slot * a.wc;
    R.nnx = I.nrnx; R.nnz = I.nrnz;
    R.gox = I.gorx; R.goz = I.gorz; R.dnx = a.drnx; R.dnz = a.drnz; R.earth = a.earth; R.fom = a.fom;
    R.risti = a.risti_r + I.risti_r;
    R.veln = a.w_vr + slot * a.wr;
    R.slow = a.w_sr + slot * a.wr;
    R.node = a.w_rnode + slot * a.wr;
}

__device__ __forceinline__ Box inst_box(const FInst& I) { return Box{I.vnl, I.vnr, I.vnt, I.vnb}; }

// The steps of one instance that the lanes share: lane `lane` of `nl`.
// The refined grid's velocities (bsplrefine_parallel), every status -1.
__device__ void step_init(const FArgs& a, const FInst& I, const FField& C, const FField& R, int lane, int nl)
{
    const long long nc = (long long)a.nnx * a.nnz;
    if (a.asgr) {
        const long long nr = (long long)I.nrnx * I.nrnz;
        const int origx = (I.vnl - 1) * a.sgdl + 1, origz = (I.vnt - 1) * a.sgdl + 1;
        const float* velv = a.velv + (long long)I.period * (a.nvx + 2) * (a.nvz + 2);
        float* vr = const_cast<float*>(R.veln);
        float* sr = const_cast<float*>(R.slow);
        for (long long q = lane; q < nr; q += nl) {
            const int idm2 = (int)(q / I.nrnz) + 1, idm1 = (int)(q % I.nrnz) + 1;
            const float v = bspline_node(velv, a.nvx, a.nvz, a.gdz * a.sgdl, a.gdx * a.sgdl,
                                         origz + idm1 - 1, origx + idm2 - 1);
            vr[q] = v;
            sr[q] = 1.0f / v;
            R.node[q].s = -1;
        }
    }
    for (long long q = lane; q < nc; q += nl) C.node[q].s = -1;
}

// Refined nodes on coarse nodes carry status and time over
// (CalSurfG_parallel.f90:2245-2262).
__device__ void step_map(const FArgs& a, const FInst& I, const FField& C, const FField& R, int lane, int nl)
{
    const int bz = I.vnb - I.vnt + 1, nbox = (I.vnr - I.vnl + 1) * bz;
    for (int q = lane; q < nbox; q += nl) {
        const int idm2 = I.vnl + q / bz, idm1 = I.vnt + q % bz;
        const int l = (idm2 - I.vnl) * a.sgdl + 1, k = (idm1 - I.vnt) * a.sgdl + 1;
        const Node rn = R.node[(long long)(l - 1) * I.nrnz + (k - 1)];
        Node& cn = C.node[(long long)(idm2 - 1) * a.nnz + (idm1 - 1)];
        cn.s = rn.s;
        if (rn.s >= 0) cn.t = rn.t;
    }
}

// Alive nodes next to far ones become close (:2290-2309), decided for 32
// box nodes per lane (chunk `base`) before any is written.
__device__ unsigned step_band_decide(const FArgs& a, const FInst& I, const FField& F, int base, int lane, int nl)
{
    const int bz = I.vnb - I.vnt + 1, nbox = (I.vnr - I.vnl + 1) * bz;
    unsigned mask = 0;
    for (int t = 0; t < 32; ++t) {
        const int q = base + t * nl + lane;
        if (q >= nbox) break;
        const int ix = I.vnl + q / bz, iz = I.vnt + q % bz;
        if (FN(iz, ix).s != 0) continue;
        if ((iz > 1 && FN(iz - 1, ix).s == -1) || (iz < F.nnz && FN(iz + 1, ix).s == -1) ||
            (ix > 1 && FN(iz, ix - 1).s == -1) || (ix < F.nnx && FN(iz, ix + 1).s == -1))
            mask |= 1u << t;
    }
    return mask;
}

__device__ void step_band_write(const FArgs& a, const FInst& I, const FField& F, int base, int lane, int nl,
                                unsigned mask)
{
    const int bz = I.vnb - I.vnt + 1;
    for (int t = 0; t < 32; ++t)
        if (mask >> t & 1u) {
            const int q = base + t * nl + lane;
            FN(I.vnt + q % bz, I.vnl + q / bz).s = 1;
        }
}

__device__ int box_nodes(const FInst& I) { return (I.vnr - I.vnl + 1) * (I.vnb - I.vnt + 1); }

// The receivers and the optional copy of the field.
__device__ void step_receivers(const FArgs& a, const FInst& I, const FField& C, int s, int lane, int nl)
{
    for (long long q = I.rc_b + lane; q < I.rc_e; q += nl) {
        float t = 0.0f;
        const int e = srtimes(a, C, I.scx, I.scz, q, t);
        if (e) record_error(a, e, s);
        else a.times[q] = t;
    }
    if (a.ttn_out) {
        const long long nc = (long long)a.nnx * a.nnz;
        float* o = a.ttn_out + (long long)s * nc;
        for (long long q = lane; q < nc; q += nl) o[q] = C.node[q].t;
    }
}

// One instance on one warp, its heap's first positions in `sh`.
__device__ void fmm_instance(const FArgs& a, int s, int lane, long long slot, HeapE* sh)
{
    const FInst I = a.inst[s];
    FField C, R;
    inst_fields(a, I, slot, C, R);
    const Heap heap{sh, a.w_heap + slot * a.wh};
    const Box B = inst_box(I);
    step_init(a, I, C, R, lane, 32);
    __syncwarp();
    int r = 0;
    if (a.asgr) {
        r = travel_warp(R, 1, I.scx, I.scz, B, heap, I.cap, lane);
        if (r) { if (lane == 0) record_error(a, r, s); return; }
        __syncwarp();
        step_map(a, I, C, R, lane, 32);
        __syncwarp();
        for (int base = 0; base < box_nodes(I); base += 32 * 32) {
            const unsigned mask = step_band_decide(a, I, C, base, lane, 32);
            __syncwarp();
            step_band_write(a, I, C, base, lane, 32, mask);
            __syncwarp();
        }
        r = travel_warp(C, 2, I.scx, I.scz, B, heap, I.cap, lane);
    } else {
        r = travel_warp(C, 0, I.scx, I.scz, B, heap, I.cap, lane);
    }
    if (r) { if (lane == 0) record_error(a, r, s); return; }
    __syncwarp();
    step_receivers(a, I, C, s, lane, 32);
}

__global__ void __launch_bounds__(32 * kWarpsPerBlock) fmm_kernel(FArgs a)
{
    __shared__ HeapE sheap[kWarpsPerBlock][kHeapShared];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long slot = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    for (;;) {
        unsigned s = 0;
        if (lane == 0) s = atomicAdd(a.queue, 1u);
        s = __shfl_sync(0xffffffffu, s, 0);
        if (s >= (unsigned)a.ninst) break;
        fmm_instance(a, (int)s, lane, slot, sheap[w]);
        __syncwarp();
    }
}

// ------------------------------------------------------------ host layout
constexpr float kPi = 3.1415926535898f;   // the reference's REAL(i10) pi

// The propagation grid of the model grid (CalSurfG_parallel.f90:1920-1930,
// 2068-2075), in the reference's real*4 operations.
struct FGrid {
    int nvx, nvz, nnx, nnz;
    float gox, goz, dvx, dvz, dnx, dnz, drnx, drnz, dpl;
    int maxbt;
};

inline int nint_cap(float snb, int a, int b)
{
    return (int)llround((double)snb * (double)a * (double)b);
}

inline FGrid grid_of(const dazi_fmm_params& p)
{
    FGrid g;
    g.nvx = p.nx - 2; g.nvz = p.ny - 2;
    g.nnx = (g.nvx - 1) * p.gdx + 1; g.nnz = (g.nvz - 1) * p.gdz + 1;
    g.dvx = p.dvxd * kPi / 180.0f; g.dvz = p.dvzd * kPi / 180.0f;
    g.gox = (90.0f - p.goxd) * kPi / 180.0f;
    g.goz = p.gozd * kPi / 180.0f;
    g.dnx = g.dvx / (float)p.gdx; g.dnz = g.dvz / (float)p.gdz;
    g.drnx = g.dvx / (float)(p.gdx * p.sgdl); g.drnz = g.dvz / (float)(p.gdz * p.sgdl);
    // srtimes_parallel's smallest node spacing (:1068-1072)
    g.dpl = g.dnx * p.earth;
    float rd1 = g.dnz * p.earth * sinf(g.gox);
    if (rd1 < g.dpl) g.dpl = rd1;
    rd1 = g.dnz * p.earth * sinf(g.gox + (float)(g.nnx - 1) * g.dnx);
    if (rd1 < g.dpl) g.dpl = rd1;
    g.maxbt = nint_cap(p.snb, g.nnx, g.nnz);
    return g;
}

inline int check_params(const dazi_fmm_params* p, const char** msg)
{
    if (!p) return *msg = "FMM: params is NULL", DAZI_ERR_BADARG;
    if (p->nx < 4 || p->ny < 4 || p->gdx < 1 || p->gdz < 1 || p->sgdl < 1 || p->sgs < 1 ||
        (p->fom != 0 && p->fom != 1) || (p->asgr != 0 && p->asgr != 1) || !(p->snb > 0.0f) ||
        !(p->earth > 0.0f) || !(p->dvxd > 0.0f) || !(p->dvzd > 0.0f))
        return *msg = "FMM: invalid grid or solver settings", DAZI_ERR_BADARG;
    const long long nnx = (long long)(p->nx - 3) * p->gdx + 1, nnz = (long long)(p->ny - 3) * p->gdz + 1;
    const long long nr = 2LL * p->sgs * p->sgdl + 1;
    if (nnx > 32767 || nnz > 32767 || nr > 32767)
        return *msg = "FMM: propagation grid beyond 32767 nodes per side", DAZI_ERR_LIMITS;
    return 0;
}

// Lay out the instances on the host: the refined box and origin of each
// source (CalSurfG_parallel.f90:2163-2200), its narrow-band capacity, and
// the ri*sin(colatitude) tables of its refined grid.
inline int layout(const dazi_fmm_params& p, const FGrid& g, int nper, int ninst, const int* per,
                  const float* scx, const float* scz, const long long* rc_off, std::vector<FInst>& inst,
                  std::vector<float>& risti_r, long long& wr, int& wh, const char** msg)
{
    inst.resize(ninst);
    risti_r.clear();
    wr = 1; wh = g.maxbt + 1;
    for (int s = 0; s < ninst; ++s) {
        FInst I{};
        if (per[s] < 0 || per[s] >= nper) return *msg = "FMM: period index outside the maps", DAZI_ERR_BADARG;
        if (rc_off[s + 1] < rc_off[s]) return *msg = "FMM: receiver offsets decrease", DAZI_ERR_BADARG;
        I.period = per[s];
        I.scx = scx[s]; I.scz = scz[s];
        I.rc_b = rc_off[s]; I.rc_e = rc_off[s + 1];
        I.cap = g.maxbt;
        int isx = (int)((scx[s] - g.gox) / g.dnx) + 1;
        int isz = (int)((scz[s] - g.goz) / g.dnz) + 1;
        if (!(isx >= 1 && isx <= g.nnx && isz >= 1 && isz <= g.nnz))
            return *msg = "FMM: source outside the model", DAZI_ERR_BADARG;
        if (p.asgr) {
            if (isx == g.nnx) isx -= 1;
            if (isz == g.nnz) isz -= 1;
            I.vnl = isx - p.sgs < 1 ? 1 : isx - p.sgs;
            I.vnr = isx + p.sgs > g.nnx ? g.nnx : isx + p.sgs;
            I.vnt = isz - p.sgs < 1 ? 1 : isz - p.sgs;
            I.vnb = isz + p.sgs > g.nnz ? g.nnz : isz + p.sgs;
            I.nrnx = (I.vnr - I.vnl) * p.sgdl + 1;
            I.nrnz = (I.vnb - I.vnt) * p.sgdl + 1;
            // the example build's fused multiply-add (one rounding)
            I.gorx = fmaf(g.dnx, (float)(I.vnl - 1), g.gox);
            I.gorz = fmaf(g.dnz, (float)(I.vnt - 1), g.goz);
            if (I.nrnx > g.nnx || I.nrnz > g.nnz)
                I.cap = nint_cap(p.snb, I.nrnx > g.nnx ? I.nrnx : g.nnx, I.nrnz > g.nnz ? I.nrnz : g.nnz);
            I.risti_r = (long long)risti_r.size();
            for (int ix = 1; ix <= I.nrnx; ++ix)
                risti_r.push_back(p.earth * sinf(I.gorx + (float)(ix - 1) * g.drnx));
            const long long n = (long long)I.nrnx * I.nrnz;
            if (n > wr) wr = n;
        }
        if (I.cap + 1 > wh) wh = I.cap + 1;
        inst[s] = I;
    }
    if (risti_r.empty()) risti_r.push_back(0.0f);
    return 0;
}

}  // namespace fmm
}  // namespace dk
