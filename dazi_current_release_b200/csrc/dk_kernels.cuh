// Kernel argument blocks and launch entry points shared by the C-ABI layer.
#pragma once
#include <cuda_runtime.h>
#include "dk_table.cuh"

namespace dk {

struct FdArgs {
    const Geometry* geo;
    int nz, kmax;
    long long ncol;      // nx*ny (column stride of the Fortran arrays)
    long long col0;      // first column (0-based) of this launch
    const float* vel;    // (nx, ny, nz) Fortran order
    const float* vp;     // optional explicit Vp (same layout) or nullptr
    const float* rho;    // optional explicit rho or nullptr
    const double* periods;
    double* pv;          // (ncol, K)
    double* sen_vs;      // (ncol, K, nz) or nullptr
    double* sen_vp;
    double* sen_rho;
    int* status;         // (ncol) first failing period (1-based) or 0
    float* cscratch;     // [columns in launch][fd_model_count(nz, sen_vs != nullptr)][K]
    unsigned long long* nevals;  // secular evaluations (accumulated), or nullptr
    float dln;
    double tol;
};

struct PrepOut {
    const long long* sen_off;   // ragged: first kernel entry of each column
    const long long* ls_off;    // ragged: first Lsen entry of each column
    unsigned long long* work;   // [0] sum of K_c * rmax_c (layer items), [1] sum of K_c
};

struct RootArgs {
    Tables T;
    const double* periods;
    double tol;
    double* pv;             // FP32-valued phase velocities (reference output)
    double* croot;          // [task * 32 + lane] FP64 roots for the adjoint, or nullptr
    double* croot_b = nullptr;   // group velocity: roots at t1b (croot: at t1a)
    int* status;            // [status_i] first failing period (1-based) or 0
    unsigned long long* nevals;  // secular evaluations (accumulated), or nullptr
    int scan32;             // FP32 coarse scan (with FP64 verification)
};

struct AdjArgs {
    Tables T;
    const double* periods;
    const double* croot;    // [task * 32 + lane]
    double* sen_vs;
    double* sen_vp;
    double* sen_rho;
    double* scratch;        // per warp [scr_layers][6][32 lanes]
    long long scr_layers;   // layer capacity of a warp's scratch block
    unsigned* queue;        // work-queue counter (zeroed before the launch)
    const double* croot_b = nullptr;   // group velocity: roots at t1b (0: none)
    const int* order = nullptr;        // phase velocity, or nullptr: [task * 32 + lane]
                                       // (key << 16) | (period * 32 + column lane),
                                       // written by adj_order_kernel (key: adj_pair_key)
};

// Doubles per refined layer in each persistent thread's Gc/Gs scratch: the
// up-sweep's compound vector and exponent sum (6); the down-sweep forms the
// layer's eigen-solution and waves again and overwrites entries 0..2 with
// the layer's raw partials once the vector is consumed.
constexpr int TI_SCR_Q = 6;

struct TiArgs {
    Tables T;
    const double* periods;
    const double* pv;       // phase velocities (FP32-valued)
    float* lsen;
    double* scratch;        // per warp [scr_layers][TI_SCR_Q][32 lanes]
    long long scr_layers;   // layer capacity of a warp's scratch block
    unsigned* queue;        // work-queue counter (zeroed before the launch)
    int* errflag;           // set to 1 when an Lsen_Gsc value is not finite
    int* order;             // [task * 32 + lane]: (key << 16) | (period * 32 + column lane),
                            // written by ti_order_kernel (key: ti_pair_key)
    int cut = 1;            // 0: every pair sweeps its whole stack (no depth cut)
};

// G-row epilogue (k_grows.cu): kernels of the grid interface to sparse
// rows of the LSMR system.
struct GrowsArgs {
    int nvx, nvz, nz, K;
    const float* vels;              // (nvx+2, nvz+2, nz) real*4
    const double* svs;              // (nxy, K, nz) real*8
    const double* svp;
    const double* srh;
    const float* lsen;              // (nxy, K, nz-1) real*4, or nullptr (isotropic rows)
    long long nrays;
    const int* ray_period;          // 0-based period index of each ray
    const int* ray_id;              // data-row id of each ray (iw)
    const long long* cell_off;      // CSR over rays
    const int* cell;                // (jj-1)*nvx + kk-1, ascending within a ray
    const float* fdm;
    const float* fdmc;
    const float* fdms;
    float ftol;
    long long* nnz_ray;             // count pass: entries per ray
    const long long* off;           // fill pass: first entry of each ray
    float* rw;
    int* iw;
    int* col;
    int* err;                       // bit 1: invalid ray
};
template <bool FILL> __global__ void grows_kernel(GrowsArgs a);

// Azimuthal phase-velocity maps (k_epilogue.cu).
struct AzimapArgs {
    int nvx, nvz, nz, K;
    const float* lsen;              // (nxy, K, nz-1) of the (nvx+2) x (nvz+2) grid
    const float* gc;                // (nvx, nvz, nz-1)
    const float* gs;
    const double* ciso;             // (nvx*nvz, K) isotropic phase velocity (tRcV)
    float* cosr;                    // (nvx*nvz, K) outputs
    float* sinr;
    float* amp;
    float* rela;
    float* ang;
};
__global__ void azimap_kernel(AzimapArgs a);

// Column source: regular grid (Fortran (nx,ny,nz) arrays, shared depz and
// periods) or ragged batch (CSR node and period arrays).
struct ColSrc {
    bool ragged;
    long long ncol, col0;          // grid: column stride and first column
    const float* vel;              // grid: vel(nx,ny,nz); ragged: vs by node_off
    const float* vp;
    const float* rho;
    const float* depz;             // grid: depz(nz); ragged: by node_off
    const long long* node_off;     // ragged
    const long long* per_off;      // ragged
    int nz, K;                     // grid
    float minthk;
    int ifunc;                     // 1 Love, 2 Rayleigh: sphere()'s density factor
    __device__ __forceinline__ int col_nz(long long c) const
    {
        return ragged ? (int)(node_off[c + 1] - node_off[c]) : nz;
    }
    __device__ __forceinline__ int col_K(long long c) const
    {
        return ragged ? (int)(per_off[c + 1] - per_off[c]) : K;
    }
    __device__ __forceinline__ float dep(long long c, int i) const
    {
        return ragged ? depz[node_off[c] + i] : depz[i];
    }
    __device__ __forceinline__ void node(long long c, int i, float& vs, float& vpo, float& rh) const
    {
        const long long idx = ragged ? node_off[c] + i : (col0 + c) + ncol * i;
        vs = vel[idx];
        if (vp) { vpo = vp[idx]; rh = rho[idx]; }
        else brocher(vs, vpo, rh);
    }
};

__global__ void prep_count_kernel(ColSrc src, long long ncols, unsigned* keys, int* colidx,
                                  int* rmax_out, int* err);
__global__ void prep_tile_kernel(long long ncols, const int* sorted_col, const int* rmax,
                                 ColSrc src, long long* tile_recs, long long* tile_tasks);
__global__ void prep_tasks_kernel(long long ntiles, const long long* tile_tasks,
                                  const long long* tile_tbase, int2* tasks);
__global__ void prep_build_kernel(ColSrc src, PrepOut o, Tables T, const int* sorted_col,
                                  const long long* tile_tbase);
// Rayleigh phase: (64|128|256, 0), (128, 5), (64, 10), each with the
// reference's nevill() refinement or (FAST) Brent's; the other wave and
// velocity types (IFUNC 1 Love / 2 Rayleigh, GROUP): (128, 0), nevill().
template <int BT, int MINB, int IFUNC = 2, bool GROUP = false, bool FAST = false>
__global__ void root_kernel(RootArgs a);
template <int MINB> __global__ void adjoint_kernel(AdjArgs a);    // MINB in {2, 3, 4}
template <int MINB> __global__ void adjoint_love_kernel(AdjArgs a);   // MINB = 3
// Group velocity (surfdisp96's igr > 0): the derivative of the reference's
// quotient of the roots at t1a and t1b, from the phase adjoint at both.
template <int MINB> __global__ void adjoint_group_kernel(AdjArgs a);        // MINB = 3
template <int MINB> __global__ void adjoint_love_group_kernel(AdjArgs a);   // MINB = 3
template <int MINB> __global__ void ti_kernel(TiArgs a);          // MINB in {2, 3, 4, 6, 8}
// One block per tile: the order of the tile's (column, period) pairs for
// ti_kernel's tasks (a.order), by the depth at which each pair's sweep stops.
__global__ void ti_order_kernel(TiArgs a, const long long* tile_tbase, const long long* tile_tasks);
__global__ void adj_order_kernel(AdjArgs a, int* order, const long long* tile_tbase, const long long* tile_tasks);

// Gives back the LSMR entries' device memory pools (k_lsmr.cu).
void lsmr_release();
constexpr int TI_ORDER_THREADS = 256;

__global__ void geometry_kernel(const float* depz, int nz, float minthk, Geometry* g);
// Models one column of the finite-difference kernel solves: the base model
// and, when kernels are requested, 6 perturbed models per node.  Its FP32
// phase velocities take fd_model_count * K scratch floats.
__host__ __device__ inline int fd_model_count(int nz, bool kernels) { return kernels ? 1 + 6 * nz : 1; }
// IFUNC 1 (Love) / 2 (Rayleigh), GROUP: all four combinations.
template <int IFUNC, bool GROUP> __global__ void fd_column_kernel(FdArgs a);
size_t fd_smem_bytes();

// Ragged batch source of the finite-difference kernel.
struct FdBatch {
    const long long* node_off;
    const long long* per_off;
    const float* depz;
    float minthk;
    const long long* sen_off;     // first kernel entry of each column
    const long long* cbuf_off;    // scratch offset (floats) of each column
};
template <int IFUNC, bool GROUP> __global__ void fd_batch_kernel(FdArgs a, FdBatch b);
size_t fd_batch_smem_bytes();

}  // namespace dk
