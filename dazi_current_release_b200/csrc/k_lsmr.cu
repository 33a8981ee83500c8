// LSMR on the GPU: the least-squares solve of the system the G rows fill.
//
// Reference: LSMR(m, n, leniw, lenrw, iw, rw, b, damp, atol, btol, conlim,
// itnlim, localSize, nout, x, istop, itn, normA, condA, normr, normAr,
// normx) of code/src_inv_iso_joint/lsmrModule.f90:36, with the sparse
// matrix as aprod.f90 reads it (rows iw(1:lenrw), columns
// iw(lenrw+1:2 lenrw), 1-based; values rw(1:lenrw), real*4), and the
// reference's SciPy backend of the same call
// (code/depthkernel_lab/scipy_lsmr_triplet_solver.py:60-90,
// scipy.sparse.linalg.lsmr, which has no local reorthogonalization).
//
// The algorithm is LSMR as published by D. C.-L. Fong and M. A. Saunders,
// "LSMR: An iterative algorithm for sparse least-squares problems", SIAM J.
// Sci. Comput. 33 (2011): Golub-Kahan bidiagonalisation of A, plane
// rotations turning it into the upper-bidiagonal R and R-bar, the updates of
// h, h-bar and x, the estimates of ||r||, ||A^T r||, ||A||, cond(A) and ||x||
// and the stopping rules istop = 1..7.  Here:
//   - the triplets are sorted on the device (stable radix sort) into CSR
//     copies of A and of A^T, so both products are gathers, one warp per
//     row, with no atomics: the results are reproducible;
//   - u and v are kept unnormalised with their scale factors (u = su u_raw,
//     v = sv v_raw), so each product also forms its new vector's sum of
//     squares and no separate scaling pass runs;
//   - every reduction is a fixed grid of per-block partial sums added in a
//     fixed order by the one-thread scalar kernel (the bidiagonalisation
//     scalars, the rotations, the estimates and the stopping tests all live
//     in device memory);
//   - an iteration is six launches (A v, scalars, A^T u, scalars and
//     rotations, h / h-bar / x update, tests); kChunk iterations are
//     captured once in a CUDA graph and the host reads the stop flag after
//     each graph launch.  Launches after the stop return at once.
// FP64 arithmetic throughout; the matrix values stay real*4 as the
// reference stores them.  Local reorthogonalization (localSize > 0 in the
// Fortran) is not done, as in the reference's SciPy backend.
#include <cuda_runtime.h>
#include <cub/cub.cuh>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <vector>

#include "../../include/dazi_dk.h"

namespace dk {
void set_last_error(const char* msg);

// Device memory of the LSMR entries comes from a private stream-ordered
// pool per device that keeps what it has been given between calls, so
// repeated solves of similar sizes take nothing from the driver after the
// first; dazi_dk_finalize gives it back (lsmr_release).
static std::mutex g_pool_mu;
static cudaMemPool_t g_pools[64] = {};

cudaMemPool_t lsmr_pool(int dev)
{
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        g_pools[dev] = p;
    }
    return g_pools[dev];
}

void lsmr_release()
{
    std::lock_guard<std::mutex> lk(g_pool_mu);
    for (cudaMemPool_t& p : g_pools)
        if (p) {
            cudaMemPoolDestroy(p);   // released once its outstanding allocations are freed
            p = nullptr;
        }
}
}

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kRedBlocks = 1184;     // fixed grid of the reducing kernels (148 SMs x 8)
constexpr int kChunk = 16;           // iterations per graph launch

// Solver state in device memory (one instance per solve).
struct State {
    // Golub-Kahan scalars; u = su u_raw, v = sv v_raw
    double alpha, beta, su, sv;
    int beta_pos;
    // rotations and estimates (the paper's notation)
    double normb, zetabar, alphabar, rho, rhobar, cbar, sbar;
    double betadd, betad, rhodold, tautildeold, thetatilde, zeta, d;
    double normA2, maxrbar, minrbar;
    double normA, condA, normr, normar, normx;
    // coefficients of the vector update of this iteration
    double c_hbar, c_x, c_h;
    // parameters
    double damp, atol, btol, ctol;
    int itnlim;
    // progress
    int itn, istop, done;
};

struct Mat {
    const long long* ptr;   // nrows + 1
    const int* idx;
    const float* val;
    int nrows;
};

__device__ __forceinline__ double block_sum(double v, double* sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < kWarps; ++i) s += sh[i];   // fixed order
    return s;
}

// y_raw = xs * (M x_raw) - ys * y_raw, row by row (one warp per row, a
// grid-stride loop over the rows on a fixed grid); part[block] = the
// block's sum of y_raw^2.  MODE 0: M = A (u step: xs = sv, ys = alpha su);
// MODE 1: M = A^T (v step: xs = su, ys = beta sv, skipped when beta = 0);
// MODE 2: the first v = A^T u (ys = 0).
// Each warp writes its own partial sum of squares (part[warp]), so a warp
// with fewer or shorter rows does not wait at a block barrier.
template <int MODE>
__global__ void __launch_bounds__(kThreads) spmv_kernel(Mat M, const double* __restrict__ x,
                                                        double* __restrict__ y,
                                                        double* __restrict__ part, State* S)
{
    if (S->done) return;
    if (MODE == 1 && !S->beta_pos) return;
    double xs, ys;
    if (MODE == 0) { xs = S->sv; ys = S->alpha * S->su; }
    else if (MODE == 1) { xs = S->su; ys = S->beta * S->sv; }
    else { xs = S->su; ys = 0.0; }
    const int lane = threadIdx.x & 31;
    const long long gw = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5);
    const long long nw = (long long)gridDim.x * kWarps;
    double sq = 0.0;
    for (long long r = gw; r < M.nrows; r += nw) {
        const long long a = M.ptr[r], b = M.ptr[r + 1];
        // the lane's products in the order k = a + lane, + 32, + 64, ...;
        // four of them in flight at once (the column and value loads, then
        // the gathers), added in that order
        double acc = 0.0;
        for (long long k0 = a + lane; k0 < b; k0 += 4 * 32) {
            int ix[4];
            float vv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const long long k = k0 + 32 * j;
                ix[j] = k < b ? M.idx[k] : -1;
                vv[j] = k < b ? M.val[k] : 0.0f;
            }
            double xv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) xv[j] = ix[j] >= 0 ? x[ix[j]] : 0.0;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (ix[j] >= 0) acc += (double)vv[j] * xv[j];
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            const double yr = xs * acc - (ys != 0.0 ? ys * y[r] : 0.0);
            y[r] = yr;
            sq += yr * yr;
        }
    }
    if (lane == 0) part[gw] = sq;
}

// The sum of n partials by one block of kThreads threads, in a fixed order
// (thread t adds part[t], part[t + kThreads], ...; then block_sum), so that
// the result does not depend on the run; valid in thread 0.  Every thread
// of the block must call it.  n: kRedBlocks (per-block partials of the
// vector kernels) or kRedWarps (per-warp partials of the products).
constexpr int kRedWarps = kRedBlocks * kWarps;

__device__ __forceinline__ double sum_parts(const double* part, int n, double* sh)
{
    double s = 0.0;
#pragma unroll 8
    for (int i = threadIdx.x; i < n; i += kThreads) s += part[i];   // loads in flight, adds in order
    return block_sum(s, sh);
}

__device__ __forceinline__ double sgn(double a) { return a > 0.0 ? 1.0 : (a < 0.0 ? -1.0 : 0.0); }

// A stable plane rotation: (c, s, r) with c a + s b = r, -s a + c b = 0
// (the paper's SymOrtho).
__device__ void sym_ortho(double a, double b, double& c, double& s, double& r)
{
    if (b == 0.0) { c = sgn(a); s = 0.0; r = fabs(a); }
    else if (a == 0.0) { c = 0.0; s = sgn(b); r = fabs(b); }
    else if (fabs(b) > fabs(a)) {
        const double tau = a / b;
        s = sgn(b) / sqrt(1.0 + tau * tau);
        c = s * tau;
        r = b / s;
    } else {
        const double tau = b / a;
        c = sgn(a) / sqrt(1.0 + tau * tau);
        s = c * tau;
        r = a / c;
    }
}

// b -> u_raw with its sum of squares
__global__ void __launch_bounds__(kThreads) copy_b_kernel(const double* __restrict__ b,
                                                          double* __restrict__ u, long long m,
                                                          double* __restrict__ part)
{
    __shared__ double sh[kWarps];
    double sq = 0.0;
    for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < m;
         i += (long long)gridDim.x * kThreads) {
        const double v = b[i];
        u[i] = v;
        sq += v * v;
    }
    const double s = block_sum(sq, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// beta = ||b||, u = b / beta
__global__ void __launch_bounds__(kThreads) init_beta_kernel(State* S, const double* part)
{
    __shared__ double sh[kWarps];
    const double ss = sum_parts(part, kRedBlocks, sh);
    if (threadIdx.x != 0) return;
    const double beta = sqrt(ss);
    S->beta = beta;
    S->normb = beta;
    S->beta_pos = beta > 0.0;
    S->su = beta > 0.0 ? 1.0 / beta : 1.0;
    S->itn = 0;
    S->istop = 0;
    S->done = 0;
    S->alpha = 0.0;
    S->sv = 1.0;
}

// alpha = ||A^T u||, v = A^T u / alpha; the starting values of the
// recurrences; stop at once when ||A^T b|| = 0 (x = 0 solves the problem)
__global__ void __launch_bounds__(kThreads) init_alpha_kernel(State* S, const double* part)
{
    __shared__ double sh[kWarps];
    const double ss = sum_parts(part, kRedWarps, sh);   // stale partials when beta = 0: not used
    if (threadIdx.x != 0) return;
    const double alpha = S->beta_pos ? sqrt(ss) : 0.0;
    S->alpha = alpha;
    S->sv = alpha > 0.0 ? 1.0 / alpha : 1.0;
    S->zetabar = alpha * S->beta;
    S->alphabar = alpha;
    S->rho = 1.0; S->rhobar = 1.0; S->cbar = 1.0; S->sbar = 0.0;
    S->betadd = S->beta; S->betad = 0.0; S->rhodold = 1.0; S->tautildeold = 0.0;
    S->thetatilde = 0.0; S->zeta = 0.0; S->d = 0.0;
    S->normA2 = alpha * alpha; S->maxrbar = 0.0; S->minrbar = 1.0e100;
    S->normA = sqrt(S->normA2); S->condA = 1.0; S->normx = 0.0; S->normr = S->beta;
    S->normar = alpha * S->beta;
    if (S->normar == 0.0 || S->itnlim <= 0) S->done = 1;
}

// h = v, h-bar = 0, x = 0
__global__ void __launch_bounds__(kThreads) init_vectors_kernel(const double* __restrict__ vraw,
                                                                double* __restrict__ h,
                                                                double* __restrict__ hbar,
                                                                double* __restrict__ x, long long n,
                                                                const State* S)
{
    const double sv = S->sv;
    for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
         i += (long long)gridDim.x * kThreads) {
        h[i] = sv * vraw[i];
        hbar[i] = 0.0;
        x[i] = 0.0;
    }
}

// after u = A v - alpha u: the iteration count, beta
__global__ void __launch_bounds__(kThreads) beta_kernel(State* S, const double* part)
{
    __shared__ double sh[kWarps];
    if (S->done) return;   // read by every thread before thread 0 writes anything
    const double ss = sum_parts(part, kRedWarps, sh);
    if (threadIdx.x != 0) return;
    S->itn += 1;
    const double beta = sqrt(ss);
    S->beta = beta;
    S->beta_pos = beta > 0.0;
    if (beta > 0.0) S->su = 1.0 / beta;
}

// after v = A^T u - beta v: alpha, the rotations, the coefficients of the
// vector update and the estimates of ||r||, ||A||, cond(A) and ||A^T r||
__global__ void __launch_bounds__(kThreads) rotate_kernel(State* S, const double* part)
{
    __shared__ double sh[kWarps];
    if (S->done) return;
    const double ss = sum_parts(part, kRedWarps, sh);   // stale partials when beta = 0: not used
    if (threadIdx.x != 0) return;
    State& T = *S;
    if (T.beta_pos) {
        const double alpha = sqrt(ss);
        T.alpha = alpha;
        if (alpha > 0.0) T.sv = 1.0 / alpha;
    }
    const double alpha = T.alpha, beta = T.beta;
    // Qhat_{k,2k+1}: the damping row
    double chat, shat, alphahat;
    sym_ortho(T.alphabar, T.damp, chat, shat, alphahat);
    // Q_k: B_k -> R_k
    const double rhoold = T.rho;
    double c, s, rho;
    sym_ortho(alphahat, beta, c, s, rho);
    T.rho = rho;
    const double thetanew = s * alpha;
    T.alphabar = c * alpha;
    // Qbar_k: R_k^T -> Rbar_k
    const double rhobarold = T.rhobar;
    const double zetaold = T.zeta;
    const double thetabar = T.sbar * rho;
    const double rhotemp = T.cbar * rho;
    double cbar, sbar, rhobar;
    sym_ortho(T.cbar * rho, thetanew, cbar, sbar, rhobar);
    T.cbar = cbar; T.sbar = sbar; T.rhobar = rhobar;
    T.zeta = cbar * T.zetabar;
    T.zetabar = -sbar * T.zetabar;
    // h-bar, x, h
    T.c_hbar = thetabar * rho / (rhoold * rhobarold);
    T.c_x = T.zeta / (rho * rhobar);
    T.c_h = thetanew / rho;
    // ||r||
    const double betaacute = chat * T.betadd;
    const double betacheck = -shat * T.betadd;
    const double betahat = c * betaacute;
    T.betadd = -s * betaacute;
    const double thetatildeold = T.thetatilde;
    double ctildeold, stildeold, rhotildeold;
    sym_ortho(T.rhodold, thetabar, ctildeold, stildeold, rhotildeold);
    T.thetatilde = stildeold * rhobar;
    T.rhodold = ctildeold * rhobar;
    T.betad = -stildeold * T.betad + ctildeold * betahat;
    T.tautildeold = (zetaold - thetatildeold * T.tautildeold) / rhotildeold;
    const double taud = (T.zeta - T.thetatilde * T.tautildeold) / T.rhodold;
    T.d = T.d + betacheck * betacheck;
    T.normr = sqrt(T.d + (T.betad - taud) * (T.betad - taud) + T.betadd * T.betadd);
    // ||A||
    T.normA2 = T.normA2 + beta * beta;
    T.normA = sqrt(T.normA2);
    T.normA2 = T.normA2 + alpha * alpha;
    // cond(A)
    T.maxrbar = fmax(T.maxrbar, rhobarold);
    if (T.itn > 1) T.minrbar = fmin(T.minrbar, rhobarold);
    T.condA = fmax(T.maxrbar, rhotemp) / fmin(T.minrbar, rhotemp);
    T.normar = fabs(T.zetabar);
}

// h-bar = h - c_hbar h-bar; x = x + c_x h-bar; h = v - c_h h (v = sv v_raw);
// part[block] = the block's sum of x^2
__global__ void __launch_bounds__(kThreads) update_kernel(const double* __restrict__ vraw,
                                                          double* __restrict__ h,
                                                          double* __restrict__ hbar,
                                                          double* __restrict__ x, long long n,
                                                          double* __restrict__ part, const State* S)
{
    __shared__ double sh[kWarps];
    if (S->done) return;
    const double c1 = S->c_hbar, c2 = S->c_x, c3 = S->c_h, sv = S->sv;
    double sq = 0.0;
    for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
         i += (long long)gridDim.x * kThreads) {
        const double hi = h[i];
        const double hb = hi - c1 * hbar[i];
        const double xi = x[i] + c2 * hb;
        hbar[i] = hb;
        x[i] = xi;
        h[i] = sv * vraw[i] - c3 * hi;
        sq += xi * xi;
    }
    const double s = block_sum(sq, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// ||x|| and the stopping rules (istop 1..7, the paper's order of precedence)
__global__ void __launch_bounds__(kThreads) test_kernel(State* S, const double* part)
{
    __shared__ double sh[kWarps];
    if (S->done) return;
    const double ss = sum_parts(part, kRedBlocks, sh);
    if (threadIdx.x != 0) return;
    State& T = *S;
    T.normx = sqrt(ss);
    const double test1 = T.normr / T.normb;
    const double test2 = (T.normA * T.normr) != 0.0 ? T.normar / (T.normA * T.normr) : INFINITY;
    const double test3 = 1.0 / T.condA;
    const double t1 = test1 / (1.0 + T.normA * T.normx / T.normb);
    const double rtol = T.btol + T.atol * T.normA * T.normx / T.normb;
    int istop = 0;
    if (T.itn >= T.itnlim) istop = 7;
    if (1.0 + test3 <= 1.0) istop = 6;
    if (1.0 + test2 <= 1.0) istop = 5;
    if (1.0 + t1 <= 1.0) istop = 4;
    if (test3 <= T.ctol) istop = 3;
    if (test2 <= T.atol) istop = 2;
    if (test1 <= rtol) istop = 1;
    T.istop = istop;
    if (istop > 0) T.done = 1;
}

// ---------------------------------------------------------------- CSR build
__global__ void keys_kernel(const int* __restrict__ a, int base, long long nnz, int lim,
                            int* __restrict__ keys, int* __restrict__ ord, int* __restrict__ bad)
{
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
         k += (long long)gridDim.x * blockDim.x) {
        const int v = a[k] - base;
        if (v < 0 || v >= lim) { atomicOr(bad, 1); keys[k] = 0; }
        else keys[k] = v;
        ord[k] = (int)k;
    }
}

__global__ void gather_kernel(const int* __restrict__ ord, const int* __restrict__ other, int base,
                              const float* __restrict__ val, long long nnz, int* __restrict__ idx,
                              float* __restrict__ vout)
{
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
         k += (long long)gridDim.x * blockDim.x) {
        const int o = ord[k];
        idx[k] = other[o] - base;
        vout[k] = val[o];
    }
}

// row pointers from the sorted keys: ptr[r] = first k with key >= r
__global__ void ptr_kernel(const int* __restrict__ skeys, long long nnz, int nrows,
                           long long* __restrict__ ptr)
{
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k <= nnz;
         k += (long long)gridDim.x * blockDim.x) {
        const int lo = k == 0 ? -1 : skeys[k - 1];
        const int hi = k == nnz ? nrows : skeys[k];
        for (int r = lo + 1; r <= hi; ++r) ptr[r] = k;
    }
}

// A pool allocation, freed in stream order on the stream it was made on
// (after every kernel queued there that uses it).
struct Buf {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~Buf() { if (p) cudaFreeAsync(p, s); }
    template <class T> T* as() { return (T*)p; }
};

int alloc(Buf& b, size_t bytes, cudaStream_t st)
{
    int dev = 0;
    cudaMemPool_t pool = cudaGetDevice(&dev) == cudaSuccess ? dk::lsmr_pool(dev) : nullptr;
    if (!pool || cudaMallocFromPoolAsync(&b.p, bytes ? bytes : 16, pool, st) != cudaSuccess) {
        b.p = nullptr;
        cudaGetLastError();
        dk::set_last_error("LSMR: device allocation failed");
        return DAZI_ERR_NOMEM;
    }
    b.s = st;
    return 0;
}

#define LK(call)                                                                  \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) {                                                  \
            char m_[200];                                                         \
            snprintf(m_, sizeof m_, "LSMR: CUDA error %s (%s)",                   \
                     cudaGetErrorString(e_), #call);                              \
            dk::set_last_error(m_);                                               \
            return DAZI_ERR_CUDA;                                                 \
        }                                                                         \
    } while (0)

// CSR of the triplets keyed by `key` (rows of A, or of A^T with the column
// indices as keys): a stable radix sort of the keys keeps equal keys in
// input order, so the layout (and with it every sum) is reproducible.
int build_csr(const int* key, const int* other, const float* val, int base, long long nnz,
              int nrows, int ncols_other, Buf& ptr, Buf& idx, Buf& v, cudaStream_t st)
{
    int r;
    Buf keys, skeys, ord, sord, bad, tmp;
    if ((r = alloc(keys, sizeof(int) * nnz, st)) || (r = alloc(skeys, sizeof(int) * nnz, st)) ||
        (r = alloc(ord, sizeof(int) * nnz, st)) || (r = alloc(sord, sizeof(int) * nnz, st)) ||
        (r = alloc(bad, sizeof(int), st)) || (r = alloc(ptr, sizeof(long long) * (nrows + 1), st)) ||
        (r = alloc(idx, sizeof(int) * nnz, st)) || (r = alloc(v, sizeof(float) * nnz, st)))
        return r;
    LK(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
    const int nb = 148 * 8;
    keys_kernel<<<nb, 256, 0, st>>>(key, base, nnz, nrows, keys.as<int>(), ord.as<int>(), bad.as<int>());
    LK(cudaGetLastError());
    // the other index must lie in range too
    keys_kernel<<<nb, 256, 0, st>>>(other, base, nnz, ncols_other, skeys.as<int>(), sord.as<int>(),
                                    bad.as<int>());
    LK(cudaGetLastError());
    int hbad = 0;
    LK(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    LK(cudaStreamSynchronize(st));
    if (hbad) {
        dk::set_last_error("LSMR: a row or column index lies outside the matrix");
        return DAZI_ERR_BADARG;
    }
    int bits = 1;
    while ((1ll << bits) < nrows) ++bits;
    size_t tb = 0;
    LK(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.as<int>(), skeys.as<int>(), ord.as<int>(),
                                       sord.as<int>(), (int)nnz, 0, bits, st));
    if ((r = alloc(tmp, tb, st))) return r;
    LK(cub::DeviceRadixSort::SortPairs(tmp.p, tb, keys.as<int>(), skeys.as<int>(), ord.as<int>(),
                                       sord.as<int>(), (int)nnz, 0, bits, st));
    gather_kernel<<<nb, 256, 0, st>>>(sord.as<int>(), other, base, val, nnz, idx.as<int>(),
                                      v.as<float>());
    LK(cudaGetLastError());
    ptr_kernel<<<nb, 256, 0, st>>>(skeys.as<int>(), nnz, nrows, ptr.as<long long>());
    LK(cudaGetLastError());
    return 0;
}

int check_args(int m, int n, long long nnz, double damp, double atol, double btol, double conlim,
               int itnlim)
{
    if (m < 1 || n < 1 || nnz < 0 || nnz > 2147483647ll) {
        dk::set_last_error("LSMR: m, n >= 1 and 0 <= nnz < 2^31 required");
        return DAZI_ERR_BADARG;
    }
    if (!(damp >= 0.0) || !(atol >= 0.0) || !(btol >= 0.0) || !(conlim >= 0.0) || itnlim < 0 ||
        !std::isfinite(damp) || !std::isfinite(atol) || !std::isfinite(btol)) {
        dk::set_last_error("LSMR: damp, atol, btol, conlim must be finite and >= 0, itnlim >= 0");
        return DAZI_ERR_BADARG;
    }
    return 0;
}

}  // namespace

extern "C" int dazi_lsmr_dev(int m, int n, long long nnz, const int* row, const int* col,
                             const float* val, int index_base, const double* b, double damp,
                             double atol, double btol, double conlim, int itnlim, double* x,
                             int* istop, int* itn, double* norms, void* stream)
{
    int r;
    if ((r = check_args(m, n, nnz, damp, atol, btol, conlim, itnlim))) return r;
    if ((nnz > 0 && (!row || !col || !val)) || !b || !x || !istop || !itn) {
        dk::set_last_error("LSMR: null argument");
        return DAZI_ERR_BADARG;
    }
    if (index_base != 0 && index_base != 1) {
        dk::set_last_error("LSMR: index_base is 0 or 1");
        return DAZI_ERR_BADARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        dk::set_last_error("no CUDA device");
        return DAZI_ERR_NODEVICE;
    }
    cudaStream_t st = (cudaStream_t)stream;
    Buf aptr, aidx, aval, tptr, tidx, tval;
    if ((r = build_csr(row, col, val, index_base, nnz, m, n, aptr, aidx, aval, st))) return r;
    if ((r = build_csr(col, row, val, index_base, nnz, n, m, tptr, tidx, tval, st))) return r;
    const Mat A{aptr.as<long long>(), aidx.as<int>(), aval.as<float>(), m};
    const Mat At{tptr.as<long long>(), tidx.as<int>(), tval.as<float>(), n};
    Buf u, v, h, hbar, part, sbuf;
    if ((r = alloc(u, sizeof(double) * m, st)) || (r = alloc(v, sizeof(double) * n, st)) ||
        (r = alloc(h, sizeof(double) * n, st)) || (r = alloc(hbar, sizeof(double) * n, st)) ||
        (r = alloc(part, sizeof(double) * kRedWarps * 3, st)) || (r = alloc(sbuf, sizeof(State), st)))
        return r;
    double* p0 = part.as<double>();
    double* p1 = p0 + kRedWarps;
    double* p2 = p1 + kRedWarps;
    State hs{};
    hs.damp = damp; hs.atol = atol; hs.btol = btol; hs.itnlim = itnlim;
    hs.ctol = conlim > 0.0 ? 1.0 / conlim : 0.0;
    State* S = sbuf.as<State>();
    LK(cudaMemcpyAsync(S, &hs, sizeof(State), cudaMemcpyHostToDevice, st));
    // u = b / ||b||, v = A^T u / ||A^T u||, h = v, h-bar = x = 0
    copy_b_kernel<<<kRedBlocks, kThreads, 0, st>>>(b, u.as<double>(), m, p0);
    init_beta_kernel<<<1, kThreads, 0, st>>>(S, p0);
    spmv_kernel<2><<<kRedBlocks, kThreads, 0, st>>>(At, u.as<double>(), v.as<double>(), p1, S);
    init_alpha_kernel<<<1, kThreads, 0, st>>>(S, p1);
    init_vectors_kernel<<<kRedBlocks, kThreads, 0, st>>>(v.as<double>(), h.as<double>(),
                                                        hbar.as<double>(), x, n, S);
    LK(cudaGetLastError());
    // kChunk iterations in one graph
    cudaStream_t cs;
    LK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    int* hdone = nullptr;                  // pinned: the stop flag after two chunks in turn
    cudaEvent_t ev[2] = {nullptr, nullptr};
    auto cleanup = [&]() {
        if (ge) cudaGraphExecDestroy(ge);
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cs);
        if (hdone) cudaFreeHost(hdone);
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
    };
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        dk::set_last_error("LSMR: stream capture failed");
        return DAZI_ERR_CUDA;
    }
    for (int it = 0; it < kChunk; ++it) {
        spmv_kernel<0><<<kRedBlocks, kThreads, 0, cs>>>(A, v.as<double>(), u.as<double>(), p0, S);
        beta_kernel<<<1, kThreads, 0, cs>>>(S, p0);
        spmv_kernel<1><<<kRedBlocks, kThreads, 0, cs>>>(At, u.as<double>(), v.as<double>(), p1, S);
        rotate_kernel<<<1, kThreads, 0, cs>>>(S, p1);
        update_kernel<<<kRedBlocks, kThreads, 0, cs>>>(v.as<double>(), h.as<double>(),
                                                       hbar.as<double>(), x, n, p2, S);
        test_kernel<<<1, kThreads, 0, cs>>>(S, p2);
    }
    if (cudaStreamEndCapture(cs, &g) != cudaSuccess ||
        cudaGraphInstantiate(&ge, g, 0) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        dk::set_last_error("LSMR: graph capture failed");
        return DAZI_ERR_CUDA;
    }
    if (cudaHostAlloc((void**)&hdone, 2 * sizeof(int), cudaHostAllocDefault) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        dk::set_last_error("LSMR: host flag allocation failed");
        return DAZI_ERR_CUDA;
    }
    // The graph runs on the caller's stream, in order with the set-up.  One
    // chunk runs ahead of the host's check of the stop flag: chunk c + 1 is
    // queued before the host waits for chunk c's flag, so the device does
    // not idle while the host reads it (a chunk queued after the stop does
    // nothing: every kernel returns once the solve is done).
    const int chunks = itnlim / kChunk + 2;
    int rc = 0;
    auto issue = [&](int c) {
        return cudaGraphLaunch(ge, st) == cudaSuccess &&
               cudaMemcpyAsync(&hdone[c & 1], &S->done, sizeof(int), cudaMemcpyDeviceToHost, st) ==
                   cudaSuccess &&
               cudaEventRecord(ev[c & 1], st) == cudaSuccess;
    };
    if (!issue(0)) rc = DAZI_ERR_CUDA;
    for (int c = 0; c < chunks && !rc; ++c) {
        if (c + 1 < chunks && !issue(c + 1)) { rc = DAZI_ERR_CUDA; break; }
        if (cudaEventSynchronize(ev[c & 1]) != cudaSuccess) { rc = DAZI_ERR_CUDA; break; }
        if (hdone[c & 1]) break;
    }
    // every queued chunk finishes before the graph, the flags and the
    // buffers go
    const cudaError_t se = cudaStreamSynchronize(st);
    if (rc || se != cudaSuccess) {
        cudaGetLastError();
        dk::set_last_error("LSMR: iteration launch failed");
        rc = DAZI_ERR_CUDA;
    }
    cleanup();
    if (rc) return rc;
    LK(cudaMemcpyAsync(&hs, S, sizeof(State), cudaMemcpyDeviceToHost, st));
    LK(cudaStreamSynchronize(st));
    *istop = hs.istop;
    *itn = hs.itn;
    if (norms) {
        norms[0] = hs.normA; norms[1] = hs.condA; norms[2] = hs.normr;
        norms[3] = hs.normar; norms[4] = hs.normx;
    }
    return DAZI_OK;
}

extern "C" int dazi_lsmr(const int* m, const int* n, const long long* leniw, const long long* lenrw,
                         const int* iw, const float* rw, const double* b, const double* damp,
                         const double* atol, const double* btol, const double* conlim,
                         const int* itnlim, const int* localSize, const int* nout, double* x,
                         int* istop, int* itn, double* normA, double* condA, double* normr,
                         double* normAr, double* normx)
{
    (void)localSize; (void)nout;
    if (!m || !n || !leniw || !lenrw || !b || !damp || !atol || !btol || !conlim || !itnlim ||
        !x || !istop || !itn || !normA || !condA || !normr || !normAr || !normx) {
        dk::set_last_error("LSMR: null argument");
        return DAZI_ERR_BADARG;
    }
    const long long nnz = *lenrw;
    if (nnz < 0 || *leniw < 2 * nnz || (nnz > 0 && (!iw || !rw))) {
        dk::set_last_error("LSMR: iw must hold lenrw row and lenrw column indices");
        return DAZI_ERR_BADARG;
    }
    int r;
    if ((r = check_args(*m, *n, nnz, *damp, *atol, *btol, *conlim, *itnlim))) return r;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        dk::set_last_error("no CUDA device");
        return DAZI_ERR_NODEVICE;
    }
    cudaStream_t st = nullptr;
    Buf dr, dc, dv, db, dx;
    if ((r = alloc(dr, sizeof(int) * nnz, st)) || (r = alloc(dc, sizeof(int) * nnz, st)) ||
        (r = alloc(dv, sizeof(float) * nnz, st)) || (r = alloc(db, sizeof(double) * *m, st)) ||
        (r = alloc(dx, sizeof(double) * *n, st)))
        return r;
    LK(cudaMemcpyAsync(dr.p, iw, sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
    LK(cudaMemcpyAsync(dc.p, iw + nnz, sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
    LK(cudaMemcpyAsync(dv.p, rw, sizeof(float) * nnz, cudaMemcpyHostToDevice, st));
    LK(cudaMemcpyAsync(db.p, b, sizeof(double) * *m, cudaMemcpyHostToDevice, st));
    double nrm[5];
    r = dazi_lsmr_dev(*m, *n, nnz, dr.as<int>(), dc.as<int>(), dv.as<float>(), 1, db.as<double>(),
                      *damp, *atol, *btol, *conlim, *itnlim, dx.as<double>(), istop, itn, nrm, st);
    if (r) return r;
    LK(cudaMemcpyAsync(x, dx.p, sizeof(double) * *n, cudaMemcpyDeviceToHost, st));
    LK(cudaStreamSynchronize(st));
    *normA = nrm[0]; *condA = nrm[1]; *normr = nrm[2]; *normAr = nrm[3]; *normx = nrm[4];
    return DAZI_OK;
}
