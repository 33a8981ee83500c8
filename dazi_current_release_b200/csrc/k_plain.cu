// Plain (perturb-and-recompute) form of the isotropic depth kernel, and the
// per-column phase-velocity root search shared with the adjoint form.
//
// Reference: DepthKernel1D.f90:102-185 (depthkernel_column_fd) driven by
// CalSurfG.f90:86-107.  For each column the reference runs surfdisp96 on
// 1 + 6*nz models: the base model and, for every depth node, Vs, Vp and rho
// perturbed by -/+ dln/2 (dln = 0.01), then forms
//     sen_X(k, i) = (c_plus(k) - c_minus(k)) / (dln * X_i).
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
    const LayerD* ld;
    __device__ __forceinline__ LayerD layer(int m) const { return ld[m]; }
};

// Perturbed model: shared base stack plus the recomputed affected layers.
struct PerturbedModel {
    const float4* lay;
    const LayerD* ld;
    const Geometry* g;
    const float* node_val;   // node values of the perturbed parameter
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
            else               L.w = __fmul_rn(v, g->rhofac[m]);
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

__global__ void __launch_bounds__(256)
fd_column_kernel(FdArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FdSmem& S = *reinterpret_cast<FdSmem*>(smem_raw);
    const Geometry* g = a.geo;
    const int nz = a.nz, K = a.kmax, rmax = g->rmax;
    const int nmod = 1 + 6 * nz;
    const long long post = (long long)a.col0 + blockIdx.x;   // 0-based column
    const long long ncol = a.ncol;
    const int tid = threadIdx.x, nthr = blockDim.x;
    // FP32 phase velocities of the column's 1 + 6 nz models, [model][K]
    float* cbuf = a.cscratch + (size_t)blockIdx.x * nmod * K;

    load_column(tid, nthr, nz, post, ncol, a.vel, a.vp, a.rho, S.vs, S.vp, S.rho);
    for (int k = tid; k < K; k += nthr) S.per[k] = a.periods[k];
    if (tid == 0) {
        int acc = 0;
        for (int i = 0; i < nz - 1; ++i) { S.first[i] = acc; acc += g->nsub_of_node[i]; }
        S.first[nz - 1] = acc;   // the half-space layer
        S.first[nz] = acc + 1;
    }
    __syncthreads();
    for (int m = tid; m < rmax; m += nthr) {
        const float4 L = flat_layer(*g, m, S.vp, S.vs, S.rho);
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
        const int fk = solve_model_warp(active, mdl, rmax, cc, betmx, S.per, K, a.tol, out, &nev);
        if (active && q == 0 && a.status) a.status[post] = fk < 0 ? 0 : fk + 1;
        if (a.nevals) {
            const unsigned long long w = __reduce_add_sync(0xffffffffu, (unsigned)nev);
            if ((tid & 31) == 0 && w) atomicAdd(a.nevals, w);
        }
    }
    __syncthreads();
    // pv and the finite-difference quotients, Fortran (ncol, K[, nz]) layout
    for (int k = tid; k < K; k += nthr) a.pv[post + ncol * k] = (double)cbuf[k];
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
            dst[post + ncol * ((long long)k + (long long)K * i)] = (cp - cm) / div;
        }
    }
}

// ------------------------------------------------------------------------
// One thread per column: the base-model root search (pv, and the FP64 roots
// the adjoint form differentiates).  Layer tables are [layer][column] so a
// warp's 32 columns read one layer with coalesced loads.
struct ColumnModel {
    const LayerD* ld;
    long long stride;
    __device__ __forceinline__ LayerD layer(int m) const { return ld[(long long)m * stride]; }
};

__global__ void build_layers_kernel(BuildArgs a)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncols) return;
    const long long post = a.col0 + c;
    const Geometry* g = a.geo;
    float vs[NZMAX], vp[NZMAX], rho[NZMAX];
    const int nz = a.nz;
    for (int i = 0; i < nz; ++i) {
        vs[i] = a.vel[post + a.ncol * i];
        if (a.vp) { vp[i] = a.vp[post + a.ncol * i]; rho[i] = a.rho[post + a.ncol * i]; }
        else brocher(vs[i], vp[i], rho[i]);
    }
    for (int m = 0; m < g->rmax; ++m) {
        const float4 L = flat_layer(*g, m, vp, vs, rho);
        a.layers[(long long)m * a.ncols + c] = L;
        a.layersd[(long long)m * a.ncols + c] = make_layerd(L);
        if (a.tilayers) {
            const int i = g->node[m];
            float4 t;
            if (m == g->rmax - 1) { t.x = vp[i]; t.y = vs[i]; t.z = rho[i]; }
            else {
                t.x = sublayer_value(vp[i], vp[i + 1], g->sub[m], g->den[m]);
                t.y = sublayer_value(vs[i], vs[i + 1], g->sub[m], g->den[m]);
                t.z = sublayer_value(rho[i], rho[i + 1], g->sub[m], g->den[m]);
            }
            t.w = 0.0f;
            a.tilayers[(long long)m * a.ncols + c] = t;
        }
    }
}

__global__ void __launch_bounds__(128)
root_kernel(RootArgs a)
{
    __shared__ double s_per[NP];
    for (int k = threadIdx.x; k < a.kmax; k += blockDim.x) s_per[k] = a.periods[k];
    __syncthreads();
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = c < a.ncols;
    const long long cc_ = active ? c : 0;
    const long long post = a.col0 + cc_;
    const int K = a.kmax;
    const int rmax = a.geo->rmax;
    ColumnModel mdl{a.layersd + cc_, a.ncols};
    auto out = [&](int k, double cval, double ctight, int ev) {
        a.pv[post + a.ncol * k] = (double)(float)cval;
        if (a.croot) a.croot[cc_ + a.ncols * k] = ctight;
        if (a.evals) a.evals[post + a.ncol * k] = ev;
    };
    double cc = 0.0;
    float betmx = 0.f;
    if (active) {
        const float4* lf = a.layers + cc_;
        scan_start([&](int m) { return lf[(long long)m * a.ncols]; }, rmax, cc, betmx);
    }
    int nev = 0;
    const int fk = solve_model_warp(active, mdl, rmax, cc, betmx, s_per, K, a.tol, out, &nev);
    if (active && a.status) a.status[post] = fk < 0 ? 0 : fk + 1;
    if (a.nevals) {
        const unsigned long long w = __reduce_add_sync(0xffffffffu, (unsigned)nev);
        if ((threadIdx.x & 31) == 0 && w) atomicAdd(a.nevals, w);
    }
}

}  // namespace dk
