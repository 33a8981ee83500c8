// Allocation-free entry point of the plain (perturb-and-recompute) form.
//
// Some callers cannot let a library call cudaMalloc: a Fortran or C driver
// that runs inside a framework owning the device through its own caching
// allocator or a fixed memory budget, or a pipeline that must not insert the
// device-wide synchronisation that cudaMalloc/cudaFree can cause between its
// kernels.  dazi_dk_iso_noalloc_dev serves them: the caller passes device
// inputs and outputs, and the only other device memory used is the file-scope
// static arrays below, which exist on every GPU that loads this library
// until the process exits:
//   g_na_scratch  per-model FP32 phase velocities, kNoAllocFloats floats
//                 (16 MiB); columns are processed in tiles that fit it
//   g_na_geo      the refined-layer geometry of the call's depth grid
// Every call reuses (and overwrites) both arrays: calls whose GPU work
// overlaps -- on different streams, or from different threads -- race on
// them and must be ordered by the caller.  Nothing needs clearing between
// calls: the geometry is rebuilt by each call and each model writes all of
// its scratch entries before they are read.
//
// The first call on a device looks up the arrays' device addresses there
// (cudaGetSymbolAddress, which also loads the module on that device); make
// that first call before any stream capture.
//
// Each call waits on `stream` twice: it reads the depth grid and periods
// back to validate them, then the refined layer count of the grid.  So it
// returns only after the work queued on `stream` before it has finished and
// the geometry is built; the finite-difference launches themselves are
// queued and not waited for.  With sen_* NULL only the base model of each
// column runs (phase velocities alone).
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/dazi_dk.h"
#include "dk_kernels.cuh"

namespace dk {
void set_last_error(const char* msg);
}

namespace {

constexpr size_t kNoAllocFloats = size_t(4) << 20;   // 16 MiB of FP32 scratch
static __device__ __align__(256) float g_na_scratch[kNoAllocFloats];
static __device__ __align__(256) dk::Geometry g_na_geo;

constexpr int kMaxDevices = 64;
struct NaDevice {
    bool ready;
    float* scratch;
    dk::Geometry* geo;
};
NaDevice g_na[kMaxDevices];   // zero-initialised: no device set up yet
std::mutex g_na_mu;

int fail(int code, const char* msg)
{
    dk::set_last_error(msg);
    return code;
}

}  // namespace

extern "C" int dazi_dk_iso_noalloc_dev(int nx, int ny, int nz, const float* vel, const float* vp,
                                       const float* rho, double* pvRc, double* sen_vsRc,
                                       double* sen_vpRc, double* sen_rhoRc, int kmaxRc,
                                       const double* tRc, const float* depz, float minthk,
                                       int col_start, int col_count, int* status, void* stream)
{
    using namespace dk;
    // An error left pending by the caller's earlier work is reported as
    // such and left pending, rather than being taken for one of ours.
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        char m[200];
        snprintf(m, sizeof m, "a CUDA error was already pending before this call: %s",
                 cudaGetErrorString(pending));
        return fail(DAZI_ERR_CUDA, m);
    }
    if (!vel || !pvRc || !tRc || !depz) return fail(DAZI_ERR_BADARG, "null argument");
    if ((sen_vsRc == nullptr) != (sen_vpRc == nullptr) || (sen_vsRc == nullptr) != (sen_rhoRc == nullptr))
        return fail(DAZI_ERR_BADARG, "sen_* must be all set or all NULL");
    if ((vp == nullptr) != (rho == nullptr))
        return fail(DAZI_ERR_BADARG, "vp and rho must both be set or both NULL");
    if (nx < 1 || ny < 1) return fail(DAZI_ERR_BADARG, "nx, ny must be >= 1");
    if (nz < 2 || nz > NZMAX) return fail(DAZI_ERR_LIMITS, "nz outside [2, 200]");
    if (kmaxRc < 1 || kmaxRc > NP) return fail(DAZI_ERR_LIMITS, "kmaxRc outside [1, 160]");
    const long long ncol = (long long)nx * ny;
    if (col_start < 1 || col_count < 0 || (long long)col_start - 1 + col_count > ncol)
        return fail(DAZI_ERR_BADARG, "column range outside the grid");
    if (!(minthk > 0.f) || !std::isfinite(minthk)) return fail(DAZI_ERR_BADARG, "minthk must be > 0");
    // one column's models (1 + 6 nz with kernels, 1 without) must fit the
    // static scratch at least once
    const int nmod = fd_model_count(nz, sen_vsRc != nullptr);
    const size_t per_col = (size_t)nmod * (size_t)kmaxRc;
    if (per_col > kNoAllocFloats) {
        char m[160];
        snprintf(m, sizeof m, "one column needs %zu scratch floats; the static array holds %zu",
                 per_col, kNoAllocFloats);
        return fail(DAZI_ERR_LIMITS, m);
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return fail(DAZI_ERR_NODEVICE, "no CUDA device"); }
    if (dev < 0 || dev >= kMaxDevices) return fail(DAZI_ERR_LIMITS, "device index beyond 63");
    std::lock_guard<std::mutex> lk(g_na_mu);
    NaDevice& D = g_na[dev];
    if (!D.ready) {
        // set-up, once per device, with that device current
        cudaError_t e1 = cudaGetSymbolAddress((void**)&D.scratch, g_na_scratch);
        cudaError_t e2 = cudaGetSymbolAddress((void**)&D.geo, g_na_geo);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            cudaGetLastError();
            return fail(DAZI_ERR_CUDA, "cudaGetSymbolAddress of the static scratch failed");
        }
        D.ready = true;
    }
    cudaStream_t st = (cudaStream_t)stream;   // NULL: the legacy default stream
    // validate the depth grid and periods (fixed-size host copies)
    float hd[NZMAX];
    double ht[NP];
    if (cudaMemcpyAsync(hd, depz, sizeof(float) * nz, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(ht, tRc, sizeof(double) * kmaxRc, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return fail(DAZI_ERR_CUDA, "reading depz/tRc failed");
    }
    for (int i = 0; i < nz; ++i)
        if (!std::isfinite(hd[i]) || (i > 0 && !(hd[i] > hd[i - 1])))
            return fail(DAZI_ERR_BADARG, "depz must be finite and strictly increasing");
    for (int k = 0; k < kmaxRc; ++k)
        if (!(ht[k] > 0.0) || !std::isfinite(ht[k])) return fail(DAZI_ERR_BADARG, "periods must be positive");
    if (col_count == 0) return DAZI_OK;
    geometry_kernel<<<1, 1, 0, st>>>(depz, nz, minthk, D.geo);
    int rmax = 0;
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(&rmax, &D.geo->rmax, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return fail(DAZI_ERR_CUDA, "geometry kernel failed");
    }
    if (rmax <= 0) return fail(DAZI_ERR_LIMITS, "refined layer count exceeds 200");
    const long long tile = (long long)(kNoAllocFloats / per_col);
    int threads = ((nmod + 31) / 32) * 32;
    if (threads > 256) threads = 256;
    for (long long c0 = 0; c0 < col_count; c0 += tile) {
        const long long n = (col_count - c0 < tile) ? col_count - c0 : tile;
        FdArgs a;
        a.geo = D.geo; a.nz = nz; a.kmax = kmaxRc; a.ncol = ncol;
        a.col0 = (long long)col_start - 1 + c0;
        a.vel = vel; a.vp = vp; a.rho = rho; a.periods = tRc;
        a.pv = pvRc; a.sen_vs = sen_vsRc; a.sen_vp = sen_vpRc; a.sen_rho = sen_rhoRc;
        a.status = status; a.cscratch = D.scratch; a.nevals = nullptr;
        a.dln = 0.01f; a.tol = 1.0e-6;
        fd_column_kernel<2, false><<<(unsigned)n, threads, fd_smem_bytes(), st>>>(a);
        if (cudaGetLastError() != cudaSuccess) return fail(DAZI_ERR_CUDA, "launch failed");
    }
    return DAZI_OK;
}
