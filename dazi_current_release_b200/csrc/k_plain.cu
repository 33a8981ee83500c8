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
// stages the column's node values and its flattened base layer stack in
// shared memory; a perturbed model differs from the base only in the
// sublayers of the two depth intervals that touch the perturbed node, so its
// thread reads the shared base stack and recomputes just those layers.
// Threads of one warp are perturbations of the same column, which keeps their
// root searches close to lock-step.  The FP32 phase velocities of all models
// land in shared memory and the CTA forms the quotients at the end.
#include "dk_secular.cuh"
#include "dk_kernels.cuh"

namespace dk {

// Base model staged in shared memory.
struct SharedModel {
    const float4* lay;
    __device__ __forceinline__ float4 layer(int m) const { return lay[m]; }
};

// Perturbed model: shared base stack plus the recomputed affected layers.
struct PerturbedModel {
    const float4* lay;
    const Geometry* g;
    const float* node_val;   // node values of the perturbed parameter
    int pnode, par, lo, hi;
    float pval;              // perturbed node value
    __device__ __forceinline__ float4 layer(int m) const {
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

__global__ void __launch_bounds__(256)
fd_column_kernel(FdArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const Geometry* g = a.geo;
    const int nz = a.nz, K = a.kmax, rmax = g->rmax;
    const int nmod = 1 + 6 * nz;
    float4* s_lay = reinterpret_cast<float4*>(smem);                 // NL
    float* s_vs = reinterpret_cast<float*>(s_lay + NL);              // NZMAX each
    float* s_vp = s_vs + NZMAX;
    float* s_rho = s_vp + NZMAX;
    int* s_first = reinterpret_cast<int*>(s_rho + NZMAX);            // NZMAX + 2
    double* s_per = reinterpret_cast<double*>(s_first + NZMAX + 2);  // NP

    const long long post = (long long)a.col0 + blockIdx.x;   // 0-based column
    const long long ncol = a.ncol;
    const int tid = threadIdx.x, nthr = blockDim.x;
    // FP32 phase velocities of the column's 1 + 6 nz models, [model][K]
    float* cbuf = a.cscratch + (size_t)blockIdx.x * nmod * K;

    load_column(tid, nthr, nz, post, ncol, a.vel, a.vp, a.rho, s_vs, s_vp, s_rho);
    for (int k = tid; k < K; k += nthr) s_per[k] = a.periods[k];
    if (tid == 0) {
        int acc = 0;
        for (int i = 0; i < nz - 1; ++i) { s_first[i] = acc; acc += g->nsub_of_node[i]; }
        s_first[nz - 1] = acc;   // the half-space layer
        s_first[nz] = acc + 1;
    }
    __syncthreads();
    for (int m = tid; m < rmax; m += nthr) s_lay[m] = flat_layer(*g, m, s_vp, s_vs, s_rho);
    __syncthreads();

    for (int q = tid; q < nmod; q += nthr) {
        float* myc = cbuf + (size_t)q * K;
        auto out = [&](int k, double c, int ev) { myc[k] = (float)c; };
        if (q == 0) {
            SharedModel mdl{s_lay};
            const int fail_k = surfdisp_column(mdl, rmax, s_per, K, a.tol, out);
            if (a.status) a.status[post] = fail_k < 0 ? 0 : fail_k + 1;
        } else {
            const int r = q - 1;
            const int node = r / 6, par = (r % 6) / 2, sgn = r & 1;
            const float* nv = par == 0 ? s_vs : (par == 1 ? s_vp : s_rho);
            const float x = nv[node];
            const float delta = __fmul_rn(__fmul_rn(0.5f, a.dln), x);
            PerturbedModel mdl;
            mdl.lay = s_lay; mdl.g = g; mdl.node_val = nv; mdl.pnode = node; mdl.par = par;
            mdl.pval = sgn ? __fadd_rn(x, delta) : __fsub_rn(x, delta);
            mdl.lo = node >= 1 ? s_first[node - 1] : 0;
            mdl.hi = node <= nz - 2 ? s_first[node + 1] - 1 : rmax - 1;
            surfdisp_column(mdl, rmax, s_per, K, a.tol, out);
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
            const float* nv = par == 0 ? s_vs : (par == 1 ? s_vp : s_rho);
            const double cm = (double)cbuf[(size_t)base * K + k];
            const double cp = (double)cbuf[(size_t)(base + 1) * K + k];
            const double div = (double)__fmul_rn(a.dln, nv[i]);
            double* dst = par == 0 ? a.sen_vs : (par == 1 ? a.sen_vp : a.sen_rho);
            dst[post + ncol * ((long long)k + (long long)K * i)] = (cp - cm) / div;
        }
    }
}

size_t fd_smem_bytes()
{
    return sizeof(float4) * NL + sizeof(float) * 3 * NZMAX + sizeof(int) * (NZMAX + 2) +
           sizeof(double) * NP;
}

// One thread per column: the base-model root search only (pv and the FP64
// roots the adjoint form differentiates).
struct GlobalModel {
    const float4* lay;
    __device__ __forceinline__ float4 layer(int m) const { return __ldg(lay + m); }
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
    float4* dst = a.layers + c * (long long)NL;
    for (int m = 0; m < g->rmax; ++m) dst[m] = flat_layer(*g, m, vp, vs, rho);
}

__global__ void root_kernel(RootArgs a)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncols) return;
    const long long post = a.col0 + c;
    const int K = a.kmax;
    GlobalModel mdl{a.layers + c * (long long)NL};
    auto out = [&](int k, double cval, int ev) {
        a.pv[post + a.ncol * k] = (double)(float)cval;
        if (a.croot) a.croot[c * K + k] = cval;
        if (a.evals) a.evals[post + a.ncol * k] = ev;
    };
    const int fk = surfdisp_column(mdl, a.geo->rmax, a.periods, K, a.tol, out);
    if (a.status) a.status[post] = fk < 0 ? 0 : fk + 1;
}

}  // namespace dk
