// Per-layer tables and per-column metadata shared by the root-search,
// adjoint and TI kernels.
//
// Columns are sorted by (refined layer count, period count) and grouped in
// tiles of 32 -- one warp.  A tile's layer records are stored layer-major,
// lane-minor: record (tile t, layer m, lane l) sits at
//     tile_lbase[t] + m * 32 + l,
// so the 32 lanes of a warp, which walk their layer stacks in lock-step,
// read one layer with coalesced loads.  The same tables serve the regular
// grid interface (every column shares one depth grid and period list, the
// reference's depthkernel/depthkernelTI) and the ragged batch (each column
// its own grid and periods).
#pragma once
#include "dk_model.cuh"

namespace dk {

constexpr int TILE = 32;

// TI model of one refined layer as tregn96 holds it: real*4 stores of the
// flattened A = C, L = N and density, TF (from the unflattened values) and
// the flattened thickness, widened to double.  The Gc/Gs kernel forms the
// combinations its formulas divide by (1/TA, TF/TA, sqrt(TA/rho), eta, ...)
// from these when it reads a layer: 40 bytes per layer item instead of 120.
struct TiRec {
    double TA, TL, rho, TF;   // TF = TA - 2 TL of the unflattened values
    double td;                // flattened thickness (0 for the half-space)
};

// The Lsen_Gsc splice of one refined layer (depthkernelTI.f90:152-162, real*4):
//   dA = cA1 dcdah - cA2 dcdn,  dL = cL1 dcdbv + cL2 dcdn,
//   Lsen += dA TA + dL TL   (unflattened TA, TL), and sprayl's vtp.
struct SpRec {
    float vtp, cA1, cA2, cL1, cL2, TA, TL, pad;
};

// What the adjoint needs to chain layer derivatives to node derivatives.
struct ChainRec {
    double tmp;               // surfdisp96 flattening factor of Vp, Vs
    float rhofac;             // density factor btp**-2.275
    short node, sub, den;     // interval i, 2j-1, 2*nsublay (half-space: nz-1, 0, 1)
    short pad;
};

struct ColMeta {
    int col;                  // original column index (0-based, within the call's range)
    int rmax, K, nz;
    long long per_b;          // first period of the column in `periods`
    long long pv_b;           // pv index of period 0 (stride: pv_sk)
    long long sen_b;          // kernel index of (period 0, node 0)
    long long sen_is;         // kernel stride between nodes (period stride: sen_sk)
    long long ls_b;           // Lsen index of (period 0, interval 0)
    long long ls_is;          // Lsen stride between intervals (period stride: ls_sk)
    long long cr_b;           // root of period k at croot[cr_b + 32 k] (task-major)
    long long status_i;       // index into the status array
};

struct Tables {
    float4* flat;             // (d, a, b, rho) flattened, surfdisp96
    LayerD* ld;               // secular-function constants
    TiRec* ti;                // tregn96 model
    SpRec* sp;                // Lsen_Gsc splice
    ChainRec* ch;             // adjoint chain rule
    ColMeta* meta;            // [sorted position]
    long long* tile_lbase;    // [tile] first record of the tile
    int2* tasks;              // [task] (tile, period) for the per-(column, period) kernels
    long long ntasks;
    long long ncols;
    long long pv_sk, sen_sk, ls_sk;   // period strides of the outputs
};

__device__ __forceinline__ long long rec_index(const Tables& T, long long s, int m)
{
    const long long t = s / TILE;
    return T.tile_lbase[t] + (long long)m * TILE + (s % TILE);
}

}  // namespace dk
