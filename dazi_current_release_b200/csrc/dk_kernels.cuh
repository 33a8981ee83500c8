// Kernel argument blocks and launch entry points shared by the C-ABI layer.
#pragma once
#include <cuda_runtime.h>
#include "dk_model.cuh"

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
    float* cscratch;     // [columns in launch][1 + 6 nz][K]
    unsigned long long* nevals;  // secular evaluations (accumulated), or nullptr
    float dln;
    double tol;
};

struct BuildArgs {
    const Geometry* geo;
    int nz;
    long long ncol, col0, ncols;
    const float* vel;
    const float* vp;
    const float* rho;
    float4* layers;      // [rmax][ncols] flattened (d, a, b, rho)
    LayerD* layersd;     // [rmax][ncols] FP64 per-layer constants
    float4* tilayers;    // [rmax][ncols] unflattened refined (vp, vs, rho), or nullptr
};

struct RootArgs {
    const Geometry* geo;
    int kmax;
    long long ncol, col0, ncols;
    const float4* layers;
    const LayerD* layersd;
    const double* periods;
    double tol;
    double* pv;          // (ncol, K) FP32-valued like the reference
    double* croot;       // [ncols][K] FP64 roots, or nullptr
    int* evals;          // (ncol, K) secular evaluations, or nullptr
    int* status;
    unsigned long long* nevals;  // secular evaluations (accumulated), or nullptr
};

struct AdjArgs {
    const Geometry* geo;
    int nz, kmax;
    long long ncol, col0, ncols;
    const float4* layers;   // [rmax][ncols]
    const double* periods;
    const double* croot;    // [K][ncols] roots (0 where no root)
    double* sen_vs;         // (ncol, K, nz) Fortran layout
    double* sen_vp;
    double* sen_rho;
    double* scratch;        // [(rmax-1)*6][grid threads]
};

__global__ void adjoint_kernel(AdjArgs a);

struct TiArgs {
    const Geometry* geo;
    int nz, kmax;
    long long ncol, col0, ncols;
    const float4* tilayers; // [rmax][ncols] refined (vp, vs, rho)
    const double* periods;
    const double* pv;       // (ncol, K) phase velocities (FP32-valued)
    float* lsen;            // (ncol, K, nz-1) Fortran layout
    double* scratch;        // [rmax*6][grid threads]
    int* errflag;           // set to 1 when an Lsen_Gsc value is not finite
};

__global__ void ti_kernel(TiArgs a);

__global__ void geometry_kernel(const float* depz, int nz, float minthk, Geometry* g);
__global__ void fd_column_kernel(FdArgs a);
__global__ void build_layers_kernel(BuildArgs a);
__global__ void root_kernel(RootArgs a);
size_t fd_smem_bytes();

}  // namespace dk
