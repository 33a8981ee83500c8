// Plain (perturb-and-recompute) form of the isotropic depth kernel, and the
// per-column phase-velocity root search shared with the adjoint form.
//
// Reference: DepthKernel1D.f90:102-185 (depthkernel_column_fd) driven by
// CalSurfG.f90:86-107.  For each column the reference runs surfdisp96 on
// 1 + 6*nz models: the base model and, for every depth node, Vs, Vp and rho
// perturbed by -/+ dln/2 (dln = 0.01), then forms
//     sen_X(k, i) = (c_plus(k) - c_minus(k)) / (dln * X_i).
// iwave and igr pass through to surfdisp96 there, so the kernels are
// instantiated for Rayleigh and Love (IFUNC 2 / 1), phase and group
// velocity (GROUP); c is then the group velocity and sen_X its derivative.
//
// Layout on the GPU: one CTA per column, one thread per model.  The CTA
// stages the column's node values and its flattened base layer stack (as
// floats and as the FP64 per-layer constants of the secular function) in
// shared memory; a perturbed model differs from the base only in the
// sublayers of the two depth intervals that touch the perturbed node, so its
// thread reads the shared base stack and recomputes just those layers.
// Threads of one warp are perturbations of the same column and step through
// their root searches one secular evaluation at a time, in lock-step.  The
// FP32 phase velocities of the models go to a global scratch buffer and the
// CTA forms the quotients at the end.
#include "dk_secular.cuh"
#include "dk_kernels.cuh"

namespace dk {

// Base model staged in shared memory.
struct SharedModel {
    static constexpr bool kF32 = false;
    const LayerD* ld;
    __device__ __forceinline__ LayerD layer(int m) const { return ld[m]; }
};

// Perturbed model: shared base stack plus the recomputed affected layers.
struct PerturbedModel {
    static constexpr bool kF32 = false;
    const float4* lay;
    const LayerD* ld;
    const Geometry* g;
    const float* node_val;   // node values of the perturbed parameter
    const float* rhof;       // sphere()'s density factor per layer
    int pnode, par, lo, hi;
    float pval;              // perturbed node value
    __device__ __forceinline__ float4 layerf(int m) const {
        float4 L = lay[m];
        if (m >= lo && m <= hi) {
            const int i = g->node[m];
            float v;
            if (m == g->rmax - 1) {
                v = pval;   // half-space takes the deepest node value
            } else {
                const float vi = (i == pnode) ? pval : node_val[i];
                const float vi1 = (i + 1 == pnode) ? pval : node_val[i + 1];
                v = sublayer_value(vi, vi1, g->sub[m], g->den[m]);
            }
            if (par == 0)      L.z = (float)__dmul_rn((double)v, g->tmp[m]);
            else if (par == 1) L.y = (float)__dmul_rn((double)v, g->tmp[m]);
            else               L.w = __fmul_rn(v, rhof[m]);
        }
        return L;
    }
    __device__ __forceinline__ LayerD layer(int m) const {
        if (m >= lo && m <= hi) return make_layerd(layerf(m));
        return ld[m];
    }
};

__global__ void geometry_kernel(const float* __restrict__ depz, int nz, float minthk,
                                Geometry* __restrict__ g)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) build_geometry(*g, depz, nz, minthk);
}

// Load the node values of column `post` (Fortran (nx,ny,nz) layout, column
// stride ncol) into shared memory, deriving Vp and rho by Brocher when no
// explicit arrays are given.
__device__ __forceinline__ void load_column(int tid, int nthr, int nz, long long post,
                                            long long ncol, const float* __restrict__ vel,
                                            const float* __restrict__ vp_in,
                                            const float* __restrict__ rho_in,
                                            float* s_vs, float* s_vp, float* s_rho)
{
    for (int i = tid; i < nz; i += nthr) {
        const float vs = vel[post + ncol * i];
        float vp, rho;
        if (vp_in) { vp = vp_in[post + ncol * i]; rho = rho_in[post + ncol * i]; }
        else brocher(vs, vp, rho);
        s_vs[i] = vs; s_vp[i] = vp; s_rho[i] = rho;
    }
}

struct FdSmem {
    LayerD ld[NL];
    float4 lay[NL];
    float vs[NZMAX], vp[NZMAX], rho[NZMAX];
    int first[NZMAX + 2];
    double per[NP];
};

size_t fd_smem_bytes() { return sizeof(FdSmem); }
size_t fd_batch_smem_bytes() { return sizeof(FdSmem) + sizeof(Geometry); }

// One column of the finite-difference form: what the shared body needs.
struct FdColumn {
    const Geometry* g;
    int nz, K;
    long long pv_b, pv_sk;            // pv index = pv_b + pv_sk * k
    long long sen_b, sen_sk, sen_is;  // kernel index = sen_b + sen_sk * k + sen_is * i
    long long status_i;
    float* cbuf;                      // [fd_model_count][K] FP32 phase velocities
};

// Body shared by the grid and ragged kernels.  Node values and periods are
// already in S.vs/S.vp/S.rho and S.per; the whole block participates.
template <int IFUNC, bool GROUP>
__device__ void fd_column_body(const FdColumn& C, FdSmem& S, const FdArgs& a)
{
    const Geometry* g = C.g;
    const int nz = C.nz, K = C.K, rmax = g->rmax;
    const int nmod = fd_model_count(nz, a.sen_vs != nullptr);
    const int tid = threadIdx.x, nthr = blockDim.x;
    float* cbuf = C.cbuf;
    if (tid == 0) {
        int acc = 0;
        for (int i = 0; i < nz - 1; ++i) { S.first[i] = acc; acc += g->nsub_of_node[i]; }
        S.first[nz - 1] = acc;   // the half-space layer
        S.first[nz] = acc + 1;
    }
    __syncthreads();
    for (int m = tid; m < rmax; m += nthr) {
        const float4 L = flat_layer(*g, m, S.vp, S.vs, S.rho, IFUNC);
        S.lay[m] = L;
        S.ld[m] = make_layerd(L);
    }
    __syncthreads();

    const int rounds = (nmod + nthr - 1) / nthr;
    for (int r = 0; r < rounds; ++r) {
        const int q = r * nthr + tid;
        const bool active = q < nmod;
        float* myc = cbuf + (size_t)(active ? q : 0) * K;
        auto out = [&](int k, double c, double ct, int ev) { myc[k] = (float)c; };
        PerturbedModel mdl;
        mdl.lay = S.lay; mdl.ld = S.ld; mdl.g = g;
        mdl.rhof = IFUNC == 1 ? g->rhofac_love : g->rhofac;
        mdl.node_val = S.vs; mdl.pnode = 0; mdl.par = 0; mdl.pval = 0.f;
        mdl.lo = 1; mdl.hi = 0;   // empty range: the base model
        if (active && q > 0) {
            const int rr = q - 1;
            const int node = rr / 6, par = (rr % 6) / 2, sgn = rr & 1;
            const float* nv = par == 0 ? S.vs : (par == 1 ? S.vp : S.rho);
            const float x = nv[node];
            const float delta = __fmul_rn(__fmul_rn(0.5f, a.dln), x);
            mdl.node_val = nv; mdl.pnode = node; mdl.par = par;
            mdl.pval = sgn ? __fadd_rn(x, delta) : __fsub_rn(x, delta);
            mdl.lo = node >= 1 ? S.first[node - 1] : 0;
            mdl.hi = node <= nz - 2 ? S.first[node + 1] - 1 : rmax - 1;
        }
        double cc = 0.0;
        float betmx = 0.f;
        if (active) scan_start([&](int m) { return mdl.layerf(m); }, rmax, cc, betmx);
        int nev = 0;
        const int fk = solve_model_warp<IFUNC, GROUP>(active, mdl, rmax, cc, betmx, S.per, K, a.tol,
                                                      out, &nev);
        if (active && q == 0 && a.status) a.status[C.status_i] = fk < 0 ? 0 : fk + 1;
        if (a.nevals) {
            const unsigned long long w = __reduce_add_sync(0xffffffffu, (unsigned)nev);
            const unsigned long long wl = __reduce_add_sync(0xffffffffu, (unsigned)(nev * rmax));
            if ((tid & 31) == 0 && w) { atomicAdd(a.nevals, w); atomicAdd(a.nevals + 3, wl); }
        }
    }
    __syncthreads();
    // pv and the finite-difference quotients
    for (int k = tid; k < K; k += nthr) a.pv[C.pv_b + C.pv_sk * k] = (double)cbuf[k];
    if (a.sen_vs) {
        const int nent = 3 * nz * K;
        for (int e = tid; e < nent; e += nthr) {
            const int k = e % K, rest = e / K, par = rest % 3, i = rest / 3;
            const int base = 1 + 6 * i + 2 * par;
            const float* nv = par == 0 ? S.vs : (par == 1 ? S.vp : S.rho);
            const double cm = (double)cbuf[(size_t)base * K + k];
            const double cp = (double)cbuf[(size_t)(base + 1) * K + k];
            const double div = (double)__fmul_rn(a.dln, nv[i]);
            double* dst = par == 0 ? a.sen_vs : (par == 1 ? a.sen_vp : a.sen_rho);
            dst[C.sen_b + C.sen_sk * k + C.sen_is * i] = (cp - cm) / div;
        }
    }
}

template <int IFUNC, bool GROUP>
__global__ void __launch_bounds__(256)
fd_column_kernel(FdArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FdSmem& S = *reinterpret_cast<FdSmem*>(smem_raw);
    const int nz = a.nz, K = a.kmax;
    const long long post = (long long)a.col0 + blockIdx.x;   // 0-based column
    const long long ncol = a.ncol;
    const int tid = threadIdx.x, nthr = blockDim.x;
    load_column(tid, nthr, nz, post, ncol, a.vel, a.vp, a.rho, S.vs, S.vp, S.rho);
    for (int k = tid; k < K; k += nthr) S.per[k] = a.periods[k];
    FdColumn C;
    C.g = a.geo; C.nz = nz; C.K = K;
    C.pv_b = post; C.pv_sk = ncol;
    C.sen_b = post; C.sen_sk = ncol; C.sen_is = ncol * (long long)K;
    C.status_i = post;
    C.cbuf = a.cscratch + (size_t)blockIdx.x * fd_model_count(nz, a.sen_vs != nullptr) * K;
    fd_column_body<IFUNC, GROUP>(C, S, a);
}

// Ragged batch: column c = col0 + blockIdx.x has its own depth grid and
// periods (CSR offsets); its geometry is built in shared memory.
template <int IFUNC, bool GROUP>
__global__ void __launch_bounds__(256)
fd_batch_kernel(FdArgs a, FdBatch b)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FdSmem& S = *reinterpret_cast<FdSmem*>(smem_raw);
    Geometry& G = *reinterpret_cast<Geometry*>(smem_raw + sizeof(FdSmem));
    const long long c = (long long)a.col0 + blockIdx.x;
    const long long n0 = b.node_off[c], p0 = b.per_off[c];
    const int nz = (int)(b.node_off[c + 1] - n0), K = (int)(b.per_off[c + 1] - p0);
    const int tid = threadIdx.x, nthr = blockDim.x;
    for (int i = tid; i < nz; i += nthr) {
        const float vs = a.vel[n0 + i];
        float vp, rho;
        if (a.vp) { vp = a.vp[n0 + i]; rho = a.rho[n0 + i]; }
        else brocher(vs, vp, rho);
        S.vs[i] = vs; S.vp[i] = vp; S.rho[i] = rho;
    }
    for (int k = tid; k < K; k += nthr) S.per[k] = a.periods[p0 + k];
    if (tid == 0) build_geometry(G, b.depz + n0, nz, b.minthk);
    __syncthreads();
    FdColumn C;
    C.g = &G; C.nz = nz; C.K = K;
    C.pv_b = p0; C.pv_sk = 1;
    C.sen_b = b.sen_off ? b.sen_off[c] : 0; C.sen_sk = 1; C.sen_is = K;
    C.status_i = c;
    C.cbuf = a.cscratch + b.cbuf_off[c] - b.cbuf_off[a.col0];
    fd_column_body<IFUNC, GROUP>(C, S, a);
}

template __global__ void fd_column_kernel<2, false>(FdArgs);
template __global__ void fd_column_kernel<2, true>(FdArgs);
template __global__ void fd_column_kernel<1, false>(FdArgs);
template __global__ void fd_column_kernel<1, true>(FdArgs);
template __global__ void fd_batch_kernel<2, false>(FdArgs, FdBatch);
template __global__ void fd_batch_kernel<2, true>(FdArgs, FdBatch);
template __global__ void fd_batch_kernel<1, false>(FdArgs, FdBatch);
template __global__ void fd_batch_kernel<1, true>(FdArgs, FdBatch);

// ------------------------------------------------------------------------
// One thread per column (sorted position): the base-model root search (pv,
// and the FP64 roots the adjoint form differentiates).  A warp is one tile of
// the layer tables, so its 32 columns read each layer with coalesced loads.
struct TableModel {
    static constexpr bool kF32 = true;
    const LayerD* ld;
    const float4* flat;
    long long base;
    __device__ __forceinline__ LayerD layer(int m) const { return ld[base + (long long)m * TILE]; }
    __device__ __forceinline__ float4 layerf(int m) const { return flat[base + (long long)m * TILE]; }
};

// Root-search output of one column: pv (FP32-valued), and for the adjoint
// form the secant-refined FP64 roots, task-major.  For group velocity croot
// holds the root at t1a and croot_b the one at t1b (0: none, c0 used).
struct RootOut {
    const RootArgs& a;
    const ColMeta& M;
    __device__ __forceinline__ void operator()(int k, double cval, double ctight, int) const
    {
        a.pv[M.pv_b + a.T.pv_sk * k] = (double)(float)cval;
        if (a.croot) a.croot[M.cr_b + (long long)TILE * k] = ctight;
    }
    __device__ __forceinline__ void group_roots(int k, double c0, double c1) const
    {
        if (a.croot_b) {
            a.croot[M.cr_b + (long long)TILE * k] = c0;
            a.croot_b[M.cr_b + (long long)TILE * k] = c1;
        }
    }
};

// BT: threads per block (one thread per column); MINB: minimum resident
// blocks per SM the register allocation aims for (0: no constraint).  The
// autotuner picks one of the instantiations.  IFUNC / GROUP: Love or
// Rayleigh, group or phase velocity (the tables then hold the matching
// density flattening).
template <int BT, int MINB, int IFUNC, bool GROUP, bool FAST>
__global__ void __launch_bounds__(BT, MINB)
root_kernel(RootArgs a)
{
    const Tables& T = a.T;
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = s < T.ncols;
    const long long ss = active ? s : 0;
    const ColMeta M = T.meta[ss];
    const long long base = T.tile_lbase[ss / TILE] + (ss % TILE);
    const double* per = a.periods + M.per_b;
    TableModel mdl{T.ld, T.flat, base};
    RootOut out{a, M};
    double cc = 0.0;
    float betmx = 0.f;
    if (active) {
        const float4* lf = T.flat + base;
        scan_start([&](int m) { return lf[(long long)m * TILE]; }, M.rmax, cc, betmx);
    }
    int nev = 0;
    const int fk = solve_model_warp<IFUNC, GROUP, FAST>(active, mdl, M.rmax, cc, betmx, per, M.K,
                                                        a.tol, out, &nev, a.scan32 != 0);
    if (active && a.status) a.status[M.status_i] = fk < 0 ? 0 : fk + 1;
    if (a.nevals) {
        const unsigned long long w = __reduce_add_sync(0xffffffffu, (unsigned)nev);
        const unsigned long long wl = __reduce_add_sync(0xffffffffu, (unsigned)(nev * (active ? M.rmax : 0)));
        if ((threadIdx.x & 31) == 0 && w) { atomicAdd(a.nevals, w); atomicAdd(a.nevals + 3, wl); }
    }
}

template __global__ void root_kernel<64, 0, 2, false, false>(RootArgs);
template __global__ void root_kernel<128, 0, 2, false, false>(RootArgs);
template __global__ void root_kernel<256, 0, 2, false, false>(RootArgs);
template __global__ void root_kernel<128, 5, 2, false, false>(RootArgs);
template __global__ void root_kernel<64, 10, 2, false, false>(RootArgs);
template __global__ void root_kernel<128, 0, 2, true, false>(RootArgs);
template __global__ void root_kernel<128, 0, 1, false, false>(RootArgs);
template __global__ void root_kernel<128, 0, 1, true, false>(RootArgs);
// the Brent refinement of the bracket (DAZI_FORM_FAST_ROOT), Rayleigh phase
template __global__ void root_kernel<64, 0, 2, false, true>(RootArgs);
template __global__ void root_kernel<128, 0, 2, false, true>(RootArgs);
template __global__ void root_kernel<256, 0, 2, false, true>(RootArgs);
template __global__ void root_kernel<128, 5, 2, false, true>(RootArgs);
template __global__ void root_kernel<64, 10, 2, false, true>(RootArgs);

}  // namespace dk
