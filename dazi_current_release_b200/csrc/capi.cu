// C-ABI of libdazi_dk.so: argument checks, device buffers, launches.
//
// The host entries mirror the reference's Fortran interfaces
// (code/src_inv_iso_joint/CalSurfG.f90:1-15 depthkernel,
//  code/src_inv_iso_joint/depthkernelTI.f90:2-14 depthkernelTI) and the
// column-range contract of the tile worker
// (code/depthkernel_lab/depthkernel_ti_worker.f90:19-38).
#include <cuda_runtime.h>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/dazi_dk.h"
#include "dk_kernels.cuh"

using namespace dk;

namespace {

char g_err[512] = "no error";

void set_err(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

#define CK(call)                                                                   \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            set_err("CUDA error %s at %s:%d (%s)", cudaGetErrorString(e_),        \
                    __FILE__, __LINE__, #call);                                    \
            return DAZI_ERR_CUDA;                                                  \
        }                                                                          \
    } while (0)

// Grow-only device buffer.
struct DBuf {
    void* p = nullptr;
    size_t n = 0;
    int ensure(size_t bytes)
    {
        if (bytes <= n) return 0;
        if (p) cudaFree(p);
        p = nullptr; n = 0;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            set_err("device allocation of %zu bytes failed", bytes);
            return DAZI_ERR_NOMEM;
        }
        n = bytes;
        return 0;
    }
    void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

struct Context {
    bool ready = false;
    int device = -1;
    cudaStream_t stream = nullptr;
    // host-entry staging
    DBuf vel, vp, rho, per, depz, pv, svs, svp, srh, status;
    // work buffers
    DBuf geo, cscratch, layers, layersd, tilayers, croot, counters, adjscr, tiscr, lsen;
    int last_launches = 0;
    int last_rmax = 0;
    // geometry cache key
    std::vector<float> geo_depz;
    float geo_minthk = -1.f;
    int geo_rmax = 0;
    std::vector<int> last_status;
    long long last_ncol = 0;
};

Context g_ctx;
std::mutex g_mu;

int ensure_context()
{
    if (g_ctx.ready) return 0;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        set_err("no CUDA device visible (%s)", cudaGetErrorString(e));
        return DAZI_ERR_NODEVICE;
    }
    CK(cudaGetDevice(&g_ctx.device));
    CK(cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamNonBlocking));
    g_ctx.ready = true;
    return 0;
}

// Geometry of the depth grid on the device (cached by content).
int prepare_geometry(const float* h_depz, int nz, float minthk, cudaStream_t st)
{
    if (g_ctx.geo.p && g_ctx.geo_minthk == minthk && (int)g_ctx.geo_depz.size() == nz &&
        std::memcmp(g_ctx.geo_depz.data(), h_depz, sizeof(float) * nz) == 0)
        return 0;
    int r;
    if ((r = g_ctx.geo.ensure(sizeof(Geometry)))) return r;
    if ((r = g_ctx.depz.ensure(sizeof(float) * nz))) return r;
    CK(cudaMemcpyAsync(g_ctx.depz.p, h_depz, sizeof(float) * nz, cudaMemcpyHostToDevice, st));
    geometry_kernel<<<1, 1, 0, st>>>(g_ctx.depz.as<float>(), nz, minthk, g_ctx.geo.as<Geometry>());
    CK(cudaGetLastError());
    int rmax = 0;
    CK(cudaMemcpyAsync(&rmax, &g_ctx.geo.as<Geometry>()->rmax, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (rmax <= 0) {
        g_ctx.geo_minthk = -1.f;
        set_err("refined layer count exceeds %d (nz=%d, minthk=%g)", NL, nz, (double)minthk);
        return DAZI_ERR_LIMITS;
    }
    g_ctx.geo_depz.assign(h_depz, h_depz + nz);
    g_ctx.geo_minthk = minthk;
    g_ctx.geo_rmax = rmax;
    return 0;
}

int check_grid(int nx, int ny, int nz, int kmax, const float* depz, float minthk,
               long long col_start, long long col_count)
{
    if (nx < 1 || ny < 1) { set_err("nx, ny must be >= 1"); return DAZI_ERR_BADARG; }
    if (nz < 2 || nz > NZMAX) { set_err("nz=%d outside [2, %d]", nz, NZMAX); return DAZI_ERR_LIMITS; }
    if (kmax < 1 || kmax > NP) { set_err("kmaxRc=%d outside [1, %d]", kmax, NP); return DAZI_ERR_LIMITS; }
    if (!(minthk > 0.f) || !std::isfinite(minthk)) { set_err("minthk must be > 0"); return DAZI_ERR_BADARG; }
    for (int i = 0; i < nz; ++i)
        if (!std::isfinite(depz[i]) || (i > 0 && !(depz[i] > depz[i - 1]))) {
            set_err("depz must be finite and strictly increasing (node %d)", i + 1);
            return DAZI_ERR_BADARG;
        }
    const long long ncol = (long long)nx * ny;
    if (col_start < 1 || col_count < 0 || col_start - 1 + col_count > ncol) {
        set_err("column range [%lld, %lld) outside 1..%lld", col_start, col_start + col_count, ncol);
        return DAZI_ERR_BADARG;
    }
    return 0;
}

int check_periods(const double* t, int kmax)
{
    for (int k = 0; k < kmax; ++k)
        if (!(t[k] > 0.0) || !std::isfinite(t[k])) {
            set_err("period %d is not a positive finite number", k + 1);
            return DAZI_ERR_BADARG;
        }
    return 0;
}

// Outputs of one stage call (device pointers; any kernel output may be null).
struct StageOut {
    double* pv;
    double* svs;
    double* svp;
    double* srh;
    float* lsen;
    int* status;
};

int launch_persistent_grid(const void* fn, long long nitems, int threads, long long& nblk)
{
    int dev = 0, sms = 0, per_sm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0));
    if (per_sm < 1) per_sm = 1;
    nblk = (long long)sms * per_sm;
    const long long need = (nitems + threads - 1) / threads;
    if (nblk > need) nblk = need;
    if (nblk < 1) nblk = 1;
    return 0;
}

// The stage on device pointers (stream-ordered, no host synchronisation).
//   plain   + kernels: one CTA per column runs the 1 + 6 nz models (FD)
//   adjoint + kernels: per-column root search, then per-(column, period)
//                      adjoint sweeps
//   Lsen requested   : per-(column, period) TI sweeps from the phase velocity
int stage_device(int nx, int ny, int nz, const float* vel, const float* vp, const float* rho,
                 const StageOut& o, int kmax, const double* per, long long col_start,
                 long long col_count, int form, cudaStream_t st)
{
    const long long ncol = (long long)nx * ny;
    if (col_count == 0) return 0;
    const Geometry* geo = g_ctx.geo.as<Geometry>();
    const double tol = 1.0e-6;   // surfdisp96.f:608
    const int rmax = g_ctx.geo_rmax;
    int r;
    if ((r = g_ctx.counters.ensure(sizeof(unsigned long long) * 4))) return r;
    CK(cudaMemsetAsync(g_ctx.counters.p, 0, sizeof(unsigned long long) * 4, st));
    g_ctx.last_rmax = rmax;
    unsigned long long* nevals = g_ctx.counters.as<unsigned long long>();
    int* errflag = reinterpret_cast<int*>(nevals + 1);
    g_ctx.last_launches = 0;
    const bool fd = o.svs && form == DAZI_FORM_PLAIN;
    if (fd) {
        const int nmod = 1 + 6 * nz;
        const size_t per_col = sizeof(float) * (size_t)nmod * kmax;
        const long long cap = 512ll << 20;
        long long tile = (long long)(cap / per_col);
        if (tile < 1) tile = 1;
        if (tile > col_count) tile = col_count;
        if ((r = g_ctx.cscratch.ensure(per_col * tile))) return r;
        int threads = ((nmod + 31) / 32) * 32;
        if (threads > 256) threads = 256;
        const size_t smem = fd_smem_bytes();
        for (long long c0 = 0; c0 < col_count; c0 += tile) {
            const long long n = (col_count - c0 < tile) ? col_count - c0 : tile;
            FdArgs a;
            a.geo = geo; a.nz = nz; a.kmax = kmax; a.ncol = ncol;
            a.col0 = col_start - 1 + c0;
            a.vel = vel; a.vp = vp; a.rho = rho; a.periods = per;
            a.pv = o.pv; a.sen_vs = o.svs; a.sen_vp = o.svp; a.sen_rho = o.srh;
            a.status = o.status; a.cscratch = g_ctx.cscratch.as<float>();
            a.dln = 0.01f; a.tol = tol; a.nevals = nevals;
            fd_column_kernel<<<(unsigned)n, threads, smem, st>>>(a);
            CK(cudaGetLastError());
            ++g_ctx.last_launches;
        }
        if (!o.lsen) return 0;
    }
    // per-column layer tables
    const size_t nl = (size_t)rmax * (size_t)col_count;
    if ((r = g_ctx.layers.ensure(sizeof(float4) * nl))) return r;
    if ((r = g_ctx.layersd.ensure(sizeof(LayerD) * nl))) return r;
    if (o.lsen && (r = g_ctx.tilayers.ensure(sizeof(float4) * nl))) return r;
    BuildArgs b;
    b.geo = geo; b.nz = nz; b.ncol = ncol; b.col0 = col_start - 1; b.ncols = col_count;
    b.vel = vel; b.vp = vp; b.rho = rho; b.layers = g_ctx.layers.as<float4>();
    b.layersd = g_ctx.layersd.as<LayerD>();
    b.tilayers = o.lsen ? g_ctx.tilayers.as<float4>() : nullptr;
    const int bt = 128;
    const unsigned nb = (unsigned)((col_count + bt - 1) / bt);
    build_layers_kernel<<<nb, bt, 0, st>>>(b);
    CK(cudaGetLastError());
    ++g_ctx.last_launches;
    const bool adj = o.svs && form == DAZI_FORM_ADJOINT;
    if (!fd) {
        RootArgs a;
        a.geo = geo; a.kmax = kmax; a.ncol = ncol; a.col0 = col_start - 1; a.ncols = col_count;
        a.layers = g_ctx.layers.as<float4>(); a.layersd = g_ctx.layersd.as<LayerD>();
        a.periods = per; a.tol = tol;
        a.pv = o.pv; a.croot = nullptr; a.evals = nullptr; a.status = o.status; a.nevals = nevals;
        if (adj) {
            if ((r = g_ctx.croot.ensure(sizeof(double) * (size_t)kmax * (size_t)col_count))) return r;
            a.croot = g_ctx.croot.as<double>();
        }
        root_kernel<<<nb, bt, 0, st>>>(a);
        CK(cudaGetLastError());
        ++g_ctx.last_launches;
    }
    const long long nitems = col_count * (long long)kmax;
    if (adj) {
        // adjoint sweeps: one thread per (column, period) on a persistent
        // grid, so the per-thread scratch slots are bounded by residency
        const int at = 128;
        long long nblk;
        if ((r = launch_persistent_grid((const void*)adjoint_kernel, nitems, at, nblk))) return r;
        const long long nslots = nblk * at;
        const size_t scr = sizeof(double) * 6 * (size_t)(rmax > 1 ? rmax - 1 : 1) * (size_t)nslots;
        if ((r = g_ctx.adjscr.ensure(scr))) return r;
        AdjArgs j;
        j.geo = geo; j.nz = nz; j.kmax = kmax; j.ncol = ncol; j.col0 = col_start - 1;
        j.ncols = col_count; j.layers = g_ctx.layers.as<float4>(); j.periods = per;
        j.croot = g_ctx.croot.as<double>(); j.sen_vs = o.svs; j.sen_vp = o.svp; j.sen_rho = o.srh;
        j.scratch = g_ctx.adjscr.as<double>();
        adjoint_kernel<<<(unsigned)nblk, at, 0, st>>>(j);
        CK(cudaGetLastError());
        ++g_ctx.last_launches;
    }
    if (o.lsen) {
        const int at = 128;
        long long nblk;
        if ((r = launch_persistent_grid((const void*)ti_kernel, nitems, at, nblk))) return r;
        const long long nslots = nblk * at;
        const size_t scr = sizeof(double) * 6 * (size_t)rmax * (size_t)nslots;
        if ((r = g_ctx.tiscr.ensure(scr))) return r;
        TiArgs t;
        t.geo = geo; t.nz = nz; t.kmax = kmax; t.ncol = ncol; t.col0 = col_start - 1;
        t.ncols = col_count; t.tilayers = g_ctx.tilayers.as<float4>(); t.periods = per;
        t.pv = o.pv; t.lsen = o.lsen; t.scratch = g_ctx.tiscr.as<double>(); t.errflag = errflag;
        ti_kernel<<<(unsigned)nblk, at, 0, st>>>(t);
        CK(cudaGetLastError());
        ++g_ctx.last_launches;
    }
    return 0;
}

int check_values(const float* vel, const float* vp, const float* rho, long long ncol, int nz,
                 long long col_start, long long col_count)
{
    for (long long c = col_start - 1; c < col_start - 1 + col_count; ++c)
        for (int i = 0; i < nz; ++i) {
            const float v = vel[c + ncol * i];
            if (!(v > 0.f) || !std::isfinite(v)) {
                set_err("vel(column %lld, node %d) = %g is not a positive finite velocity", c + 1, i + 1, (double)v);
                return DAZI_ERR_BADARG;
            }
            if (vp && (!(vp[c + ncol * i] > 0.f) || !(rho[c + ncol * i] > 0.f) ||
                       !std::isfinite(vp[c + ncol * i]) || !std::isfinite(rho[c + ncol * i]))) {
                set_err("vp/rho(column %lld, node %d) not positive finite", c + 1, i + 1);
                return DAZI_ERR_BADARG;
            }
        }
    return 0;
}

// Host-pointer stage: argument checks, copies in, stage_device, copies out.
int stage_host(const int* pnx, const int* pny, const int* pnz, const float* vel, const float* vp,
               const float* rho, double* pv, double* svs, double* svp, double* srh, float* lsen,
               const int* iwave, const int* igr, const int* pkmax, const double* tRc,
               const float* depz, const float* pminthk, int col_start, int col_count, int form)
{
    if (!pnx || !pny || !pnz || !vel || !pv || !iwave || !igr || !pkmax || !tRc || !depz || !pminthk) {
        set_err("null argument");
        return DAZI_ERR_BADARG;
    }
    if (*iwave != 2 || *igr != 0) {
        set_err("only Rayleigh (iwave=2) phase velocity (igr=0) is supported (got %d, %d)", *iwave, *igr);
        return DAZI_ERR_BADARG;
    }
    if ((svs == nullptr) != (svp == nullptr) || (svs == nullptr) != (srh == nullptr)) {
        set_err("sen_vsRc, sen_vpRc, sen_rhoRc must be all set or all NULL");
        return DAZI_ERR_BADARG;
    }
    if ((vp == nullptr) != (rho == nullptr)) { set_err("vp and rho must both be set or both NULL"); return DAZI_ERR_BADARG; }
    if (form != DAZI_FORM_PLAIN && form != DAZI_FORM_ADJOINT) { set_err("unknown form %d", form); return DAZI_ERR_BADARG; }
    const int nx = *pnx, ny = *pny, nz = *pnz, kmax = *pkmax;
    const float minthk = *pminthk;
    int r;
    if ((r = check_grid(nx, ny, nz, kmax, depz, minthk, col_start, col_count))) return r;
    if ((r = check_periods(tRc, kmax))) return r;
    const long long ncol = (long long)nx * ny;
    if ((r = check_values(vel, vp, rho, ncol, nz, col_start, col_count))) return r;
    const size_t nvel = (size_t)ncol * nz;
    std::lock_guard<std::mutex> lk(g_mu);
    if ((r = ensure_context())) return r;
    cudaStream_t st = g_ctx.stream;
    if ((r = prepare_geometry(depz, nz, minthk, st))) return r;
    const bool kern = svs != nullptr;
    const size_t npv = (size_t)ncol * kmax, nsen = npv * nz, nls = npv * (nz - 1);
    if ((r = g_ctx.vel.ensure(sizeof(float) * nvel))) return r;
    if (vp && ((r = g_ctx.vp.ensure(sizeof(float) * nvel)) || (r = g_ctx.rho.ensure(sizeof(float) * nvel)))) return r;
    if ((r = g_ctx.per.ensure(sizeof(double) * kmax))) return r;
    if ((r = g_ctx.pv.ensure(sizeof(double) * npv))) return r;
    if ((r = g_ctx.status.ensure(sizeof(int) * ncol))) return r;
    if (kern && ((r = g_ctx.svs.ensure(sizeof(double) * nsen)) || (r = g_ctx.svp.ensure(sizeof(double) * nsen)) ||
                 (r = g_ctx.srh.ensure(sizeof(double) * nsen))))
        return r;
    if (lsen && (r = g_ctx.lsen.ensure(sizeof(float) * nls))) return r;
    CK(cudaMemcpyAsync(g_ctx.vel.p, vel, sizeof(float) * nvel, cudaMemcpyHostToDevice, st));
    if (vp) {
        CK(cudaMemcpyAsync(g_ctx.vp.p, vp, sizeof(float) * nvel, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(g_ctx.rho.p, rho, sizeof(float) * nvel, cudaMemcpyHostToDevice, st));
    }
    CK(cudaMemcpyAsync(g_ctx.per.p, tRc, sizeof(double) * kmax, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(g_ctx.status.p, 0, sizeof(int) * ncol, st));
    StageOut o;
    o.pv = g_ctx.pv.as<double>();
    o.svs = kern ? g_ctx.svs.as<double>() : nullptr;
    o.svp = kern ? g_ctx.svp.as<double>() : nullptr;
    o.srh = kern ? g_ctx.srh.as<double>() : nullptr;
    o.lsen = lsen ? g_ctx.lsen.as<float>() : nullptr;
    o.status = g_ctx.status.as<int>();
    r = stage_device(nx, ny, nz, g_ctx.vel.as<float>(), vp ? g_ctx.vp.as<float>() : nullptr,
                     vp ? g_ctx.rho.as<float>() : nullptr, o, kmax, g_ctx.per.as<double>(),
                     col_start, col_count, form, st);
    if (r) return r;
    // Copy back only the written columns: every (k[, i]) slab holds the
    // column range contiguously.
    const size_t c0 = (size_t)(col_start - 1), cn = (size_t)col_count;
    CK(cudaMemcpy2DAsync(pv + c0, sizeof(double) * ncol, g_ctx.pv.as<double>() + c0, sizeof(double) * ncol,
                         sizeof(double) * cn, kmax, cudaMemcpyDeviceToHost, st));
    if (kern) {
        double* hs[3] = {svs, svp, srh};
        DBuf* ds[3] = {&g_ctx.svs, &g_ctx.svp, &g_ctx.srh};
        for (int q = 0; q < 3; ++q)
            CK(cudaMemcpy2DAsync(hs[q] + c0, sizeof(double) * ncol, ds[q]->as<double>() + c0,
                                 sizeof(double) * ncol, sizeof(double) * cn, (size_t)kmax * nz,
                                 cudaMemcpyDeviceToHost, st));
    }
    if (lsen)
        CK(cudaMemcpy2DAsync(lsen + c0, sizeof(float) * ncol, g_ctx.lsen.as<float>() + c0,
                             sizeof(float) * ncol, sizeof(float) * cn, (size_t)kmax * (nz - 1),
                             cudaMemcpyDeviceToHost, st));
    g_ctx.last_status.resize(ncol);
    CK(cudaMemcpyAsync(g_ctx.last_status.data(), g_ctx.status.p, sizeof(int) * ncol, cudaMemcpyDeviceToHost, st));
    int hflag[2] = {0, 0};
    CK(cudaMemcpyAsync(hflag, g_ctx.counters.as<unsigned long long>() + 1, sizeof(int) * 2,
                       cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    g_ctx.last_ncol = ncol;
    if (hflag[0]) {
        set_err("non-finite Lsen_Gsc value (degenerate layer: Vp <= Vs?)");
        return DAZI_ERR_MODEL;
    }
    for (long long c = col_start - 1; c < col_start - 1 + col_count; ++c)
        if (g_ctx.last_status[c] != 0) return DAZI_WARN_NOROOT;
    return DAZI_OK;
}

int check_dev_common(int nz, int kmaxRc, int form, const void* vp, const void* rho,
                     const void* svs, const void* svp, const void* srh)
{
    if ((svs == nullptr) != (svp == nullptr) || (svs == nullptr) != (srh == nullptr)) {
        set_err("sen_* must be all set or all NULL");
        return DAZI_ERR_BADARG;
    }
    if ((vp == nullptr) != (rho == nullptr)) { set_err("vp and rho must both be set or both NULL"); return DAZI_ERR_BADARG; }
    if (form != DAZI_FORM_PLAIN && form != DAZI_FORM_ADJOINT) { set_err("unknown form %d", form); return DAZI_ERR_BADARG; }
    if (nz < 2 || nz > NZMAX) { set_err("nz=%d outside [2, %d]", nz, NZMAX); return DAZI_ERR_LIMITS; }
    if (kmaxRc < 1 || kmaxRc > NP) { set_err("kmaxRc=%d outside [1, %d]", kmaxRc, NP); return DAZI_ERR_LIMITS; }
    return 0;
}

int stage_dev(int nx, int ny, int nz, const float* vel, const float* vp, const float* rho,
              double* pvRc, double* svs, double* svp, double* srh, float* lsen, int kmaxRc,
              const double* tRc, const float* depz, float minthk, int col_start, int col_count,
              int form, int* status, void* stream)
{
    if (!vel || !pvRc || !tRc || !depz) { set_err("null argument"); return DAZI_ERR_BADARG; }
    int r;
    if ((r = check_dev_common(nz, kmaxRc, form, vp, rho, svs, svp, srh))) return r;
    std::lock_guard<std::mutex> lk(g_mu);
    if ((r = ensure_context())) return r;
    cudaStream_t st = (cudaStream_t)stream;   // NULL: the legacy default stream
    std::vector<float> hd(nz);
    std::vector<double> ht(kmaxRc);
    CK(cudaMemcpyAsync(hd.data(), depz, sizeof(float) * nz, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(ht.data(), tRc, sizeof(double) * kmaxRc, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if ((r = check_grid(nx, ny, nz, kmaxRc, hd.data(), minthk, col_start, col_count))) return r;
    if ((r = check_periods(ht.data(), kmaxRc))) return r;
    if ((r = prepare_geometry(hd.data(), nz, minthk, st))) return r;
    StageOut o;
    o.pv = pvRc; o.svs = svs; o.svp = svp; o.srh = srh; o.lsen = lsen; o.status = status;
    return stage_device(nx, ny, nz, vel, vp, rho, o, kmaxRc, tRc, col_start, col_count, form, st);
}

}  // namespace

namespace dk {
// Error message hook for entry points defined in other translation units.
void set_last_error(const char* msg) { set_err("%s", msg); }
}  // namespace dk

extern "C" {

int dazi_dk_iso(const int* nx, const int* ny, const int* nz, const float* vel, double* pvRc,
                double* sen_vsRc, double* sen_vpRc, double* sen_rhoRc, const int* iwave,
                const int* igr, const int* kmaxRc, const double* tRc, const float* depz,
                const float* minthk, int col_start, int col_count, int form)
{
    return stage_host(nx, ny, nz, vel, nullptr, nullptr, pvRc, sen_vsRc, sen_vpRc, sen_rhoRc,
                      nullptr, iwave, igr, kmaxRc, tRc, depz, minthk, col_start, col_count, form);
}

int dazi_dk_iso_vpvsrho(const int* nx, const int* ny, const int* nz, const float* vel,
                        const float* vp, const float* rho, double* pvRc, double* sen_vsRc,
                        double* sen_vpRc, double* sen_rhoRc, const int* iwave, const int* igr,
                        const int* kmaxRc, const double* tRc, const float* depz,
                        const float* minthk, int col_start, int col_count, int form)
{
    if (!vp || !rho) { set_err("vp and rho are required"); return DAZI_ERR_BADARG; }
    return stage_host(nx, ny, nz, vel, vp, rho, pvRc, sen_vsRc, sen_vpRc, sen_rhoRc, nullptr,
                      iwave, igr, kmaxRc, tRc, depz, minthk, col_start, col_count, form);
}

int dazi_dk_ti(const int* nx, const int* ny, const int* nz, const float* vel, double* pvRc,
               const int* iwave, const int* igr, const int* kmaxRc, const double* tRc,
               const float* depz, const float* minthk, float* Lsen_Gsc, int col_start,
               int col_count)
{
    if (!Lsen_Gsc) { set_err("Lsen_Gsc is required"); return DAZI_ERR_BADARG; }
    return stage_host(nx, ny, nz, vel, nullptr, nullptr, pvRc, nullptr, nullptr, nullptr,
                      Lsen_Gsc, iwave, igr, kmaxRc, tRc, depz, minthk, col_start, col_count,
                      DAZI_FORM_PLAIN);
}

int dazi_dk_fused(const int* nx, const int* ny, const int* nz, const float* vel, const float* vp,
                  const float* rho, double* pvRc, double* sen_vsRc, double* sen_vpRc,
                  double* sen_rhoRc, float* Lsen_Gsc, const int* iwave, const int* igr,
                  const int* kmaxRc, const double* tRc, const float* depz, const float* minthk,
                  int col_start, int col_count, int form)
{
    return stage_host(nx, ny, nz, vel, vp, rho, pvRc, sen_vsRc, sen_vpRc, sen_rhoRc, Lsen_Gsc,
                      iwave, igr, kmaxRc, tRc, depz, minthk, col_start, col_count, form);
}

int dazi_dk_last_status(int* status, long long n)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_ctx.last_status.empty() || !status) { set_err("no status available"); return DAZI_ERR_BADARG; }
    const long long m = n < (long long)g_ctx.last_status.size() ? n : (long long)g_ctx.last_status.size();
    std::memcpy(status, g_ctx.last_status.data(), sizeof(int) * (size_t)m);
    return 0;
}

int dazi_dk_iso_dev(int nx, int ny, int nz, const float* vel, const float* vp, const float* rho,
                    double* pvRc, double* sen_vsRc, double* sen_vpRc, double* sen_rhoRc, int kmaxRc,
                    const double* tRc, const float* depz, float minthk, int col_start, int col_count,
                    int form, int* status, void* stream)
{
    return stage_dev(nx, ny, nz, vel, vp, rho, pvRc, sen_vsRc, sen_vpRc, sen_rhoRc, nullptr,
                     kmaxRc, tRc, depz, minthk, col_start, col_count, form, status, stream);
}

int dazi_dk_fused_dev(int nx, int ny, int nz, const float* vel, const float* vp, const float* rho,
                      double* pvRc, double* sen_vsRc, double* sen_vpRc, double* sen_rhoRc,
                      float* Lsen_Gsc, int kmaxRc, const double* tRc, const float* depz,
                      float minthk, int col_start, int col_count, int form, int* status,
                      void* stream)
{
    return stage_dev(nx, ny, nz, vel, vp, rho, pvRc, sen_vsRc, sen_vpRc, sen_rhoRc, Lsen_Gsc,
                     kmaxRc, tRc, depz, minthk, col_start, col_count, form, status, stream);
}

int dazi_dk_last_launches(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_ctx.last_launches;
}

int dazi_dk_last_work(long long* secular_evals, long long* layer_evals)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx.ready || !g_ctx.counters.p) { set_err("no call made yet"); return DAZI_ERR_BADARG; }
    unsigned long long h[4] = {0, 0, 0, 0};
    CK(cudaMemcpy(h, g_ctx.counters.p, sizeof(h), cudaMemcpyDeviceToHost));
    if (secular_evals) *secular_evals = (long long)h[0];
    if (layer_evals) *layer_evals = (long long)h[0] * (long long)g_ctx.last_rmax;
    return 0;
}

const char* dazi_dk_last_error(void) { return g_err; }

int dazi_dk_version(void) { return 100; }

void dazi_dk_finalize(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx.ready) return;
    DBuf* all[] = {&g_ctx.vel, &g_ctx.vp, &g_ctx.rho, &g_ctx.per, &g_ctx.depz, &g_ctx.pv,
                   &g_ctx.svs, &g_ctx.svp, &g_ctx.srh, &g_ctx.status, &g_ctx.geo,
                   &g_ctx.cscratch, &g_ctx.layers, &g_ctx.layersd, &g_ctx.croot, &g_ctx.counters, &g_ctx.adjscr, &g_ctx.tilayers,
                   &g_ctx.tiscr, &g_ctx.lsen};
    for (DBuf* b : all) b->release();
    if (g_ctx.stream) cudaStreamDestroy(g_ctx.stream);
    g_ctx = Context();
}

}  // extern "C"
