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
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/dazi_dk.h"
#include <cub/cub.cuh>

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

// Device buffers of one table-driven computation: the layer tables, the
// task list, the counters and the sweep scratch (the global entries share
// one; every plan owns one).
struct Work {
    DBuf croot, crootb, counters, adjscr, adjord, tiscr, tiord;
    DBuf keys, keys2, cidx, cidx2, rmaxb, trecs, ttasks, tlbase, ttbase, cubtmp;
    DBuf tflat, tld, tti, tsp, tch, tmeta, ttasklist;
    void release()
    {
        DBuf* all[] = {&croot, &crootb, &counters, &adjscr, &adjord, &tiscr, &tiord, &keys, &keys2, &cidx, &cidx2, &rmaxb,
                       &trecs, &ttasks, &tlbase, &ttbase, &cubtmp, &tflat, &tld, &tti, &tsp,
                       &tch, &tmeta, &ttasklist};
        for (DBuf* b : all) b->release();
    }
};

// Kernel variants of the table-driven phases (chosen by the autotuner of a
// plan; the global entries use the defaults).
struct LaunchCfg {
    int root_bt = 128;      // root_kernel threads per block: 64, 128, 256
    int root_minb = 0;      // root_kernel blocks per SM of the register budget: 0, 5 (128), 10 (64)
    int adj_minb = 3;       // adjoint_kernel blocks per SM: 2, 3, 4
    int ti_minb = 4;        // ti_kernel blocks per SM: 2, 3, 4, 6, 8
    bool cut = true;        // depth cut of the Rayleigh phase adjoint and Gc/Gs sweeps
                            // (off with DAZI_FORM_FULL_STACK)
};

// Root-search variants (threads per block, register-budget blocks per SM).
constexpr int kRootVariants[5][2] = {{64, 0}, {128, 0}, {256, 0}, {128, 5}, {64, 10}};

// Launch configuration of the per-call entries: the defaults, or
// DAZI_DK_LAUNCH="root=BT[xMINB],adj=MINB,ti=MINB" (values outside the
// instantiated variants are ignored).
LaunchCfg default_cfg()
{
    static LaunchCfg cfg;
    static bool done = false;
    if (done) return cfg;
    done = true;
    const char* e = std::getenv("DAZI_DK_LAUNCH");
    if (!e) return cfg;
    int a = 0, b = 0;
    const char* r = std::strstr(e, "root=");
    if (r && std::sscanf(r + 5, "%dx%d", &a, &b) >= 1) {
        for (const auto& v : kRootVariants)
            if (v[0] == a && v[1] == b) { cfg.root_bt = a; cfg.root_minb = b; }
    }
    const char* j = std::strstr(e, "adj=");
    if (j && std::sscanf(j + 4, "%d", &a) == 1 && a >= 2 && a <= 4) cfg.adj_minb = a;
    const char* t = std::strstr(e, "ti=");
    if (t && std::sscanf(t + 3, "%d", &a) == 1 && (a == 2 || a == 3 || a == 4 || a == 6 || a == 8))
        cfg.ti_minb = a;
    return cfg;
}

// Optional per-phase timing with CUDA events on the call's stream.
struct PhaseTimer {
    bool on = false;
    int n = 0;
    const char* name[16];
    cudaEvent_t ev[17];
    bool made = false;
};

struct Context {
    bool ready = false;
    PhaseTimer timer;
    int device = -1;
    cudaStream_t stream = nullptr;
    // host entries: results that are final before the Gc/Gs sweep (pv and
    // the sensitivity kernels) are copied to the host on cstream, after
    // outs_ready, while the sweep runs on stream
    cudaStream_t cstream = nullptr;
    cudaEvent_t outs_ready = nullptr;
    // host-entry staging
    DBuf vel, vp, rho, per, depz, pv, svs, svp, srh, status;
    // work buffers
    DBuf geo, cscratch, lsen;
    // per-call layer tables, counters and sweep scratch
    Work w;
    DBuf cbufoff;
    // G-row epilogue: ray offsets, scan storage, error flag
    DBuf goff, gtmp, gerr;
    // batch staging (host entry)
    DBuf bnode, bper, bdep, bvs, bvp, brho, bperiods, bsenoff, blsoff, bpv, bsvs, bsvp, bsrh, blsen, bstatus;
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

// A form is DAZI_FORM_PLAIN or DAZI_FORM_ADJOINT plus flags.  Both forms
// (and a phase-velocity-only call) take Love waves and group velocity; the
// FP32 scan and Lsen_Gsc are Rayleigh phase.
constexpr int kWaveFlags = DAZI_FORM_LOVE | DAZI_FORM_GROUP;

int check_form(int form, bool lsen)
{
    constexpr int known = DAZI_FORM_ADJOINT | DAZI_FORM_SCAN_FP32 | kWaveFlags | DAZI_FORM_FAST_ROOT |
                          DAZI_FORM_FULL_STACK;
    if (form & ~known) { set_err("unknown form %d", form); return DAZI_ERR_BADARG; }
    if (form & DAZI_FORM_FAST_ROOT) {
        if (form & kWaveFlags) {
            set_err("the Brent root refinement runs with Rayleigh phase velocity only (form %d)", form);
            return DAZI_ERR_BADARG;
        }
    }
    if (form & kWaveFlags) {
        if (form & DAZI_FORM_SCAN_FP32) {
            set_err("the FP32 scan runs with Rayleigh phase velocity only (form %d)", form);
            return DAZI_ERR_BADARG;
        }
        if (lsen) {
            set_err("Lsen_Gsc is a Rayleigh phase-velocity kernel (form %d)", form);
            return DAZI_ERR_BADARG;
        }
    }
    return 0;
}

int form_ifunc(int form) { return (form & DAZI_FORM_LOVE) ? 1 : 2; }
bool form_group(int form) { return (form & DAZI_FORM_GROUP) != 0; }

void phase_begin(cudaStream_t st)
{
    PhaseTimer& T = g_ctx.timer;
    T.n = 0;
    if (!T.on) return;
    if (!T.made) {
        for (int i = 0; i < 17; ++i) cudaEventCreate(&T.ev[i]);
        T.made = true;
    }
    cudaEventRecord(T.ev[0], st);
}

void phase_mark(const char* name, cudaStream_t st)
{
    PhaseTimer& T = g_ctx.timer;
    if (!T.on || T.n >= 16) return;
    T.name[T.n] = name;
    cudaEventRecord(T.ev[T.n + 1], st);
    ++T.n;
}

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
    CK(cudaStreamCreateWithFlags(&g_ctx.cstream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&g_ctx.outs_ready, cudaEventDisableTiming));
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

// Build the per-layer tables of a call (dk_table.cuh): count layers,
// sort the columns by (layers, periods), lay out 32-column tiles, build.
// One host synchronisation (to size the tables).
int build_tables(const ColSrc& src, long long ncols, const PrepOut& po, long long pv_sk,
                 long long sen_sk, long long ls_sk, cudaStream_t st, Tables& T, Work& W)
{
    int r;
    const long long ntiles = (ncols + TILE - 1) / TILE;
    if ((r = W.keys.ensure(sizeof(unsigned) * ncols)) || (r = W.keys2.ensure(sizeof(unsigned) * ncols)) ||
        (r = W.cidx.ensure(sizeof(int) * ncols)) || (r = W.cidx2.ensure(sizeof(int) * ncols)) ||
        (r = W.rmaxb.ensure(sizeof(int) * ncols + 16)) ||
        (r = W.trecs.ensure(sizeof(long long) * ntiles)) || (r = W.ttasks.ensure(sizeof(long long) * ntiles)) ||
        (r = W.tlbase.ensure(sizeof(long long) * ntiles)) || (r = W.ttbase.ensure(sizeof(long long) * ntiles)))
        return r;
    int* err = reinterpret_cast<int*>(W.rmaxb.as<char>() + sizeof(int) * ncols);
    CK(cudaMemsetAsync(err, 0, sizeof(int), st));
    const int bt = 128;
    const unsigned nb = (unsigned)((ncols + bt - 1) / bt);
    prep_count_kernel<<<nb, bt, 0, st>>>(src, ncols, W.keys.as<unsigned>(), W.cidx.as<int>(),
                                         W.rmaxb.as<int>(), err);
    CK(cudaGetLastError());
    size_t tb1 = 0, tb2 = 0, tb3 = 0;
    CK(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb1, W.keys.as<unsigned>(), W.keys2.as<unsigned>(),
                                                 W.cidx.as<int>(), W.cidx2.as<int>(), (int)ncols, 0, 16, st));
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tb2, W.trecs.as<long long>(), W.tlbase.as<long long>(),
                                     (int)ntiles, st));
    tb3 = tb1 > tb2 ? tb1 : tb2;
    if ((r = W.cubtmp.ensure(tb3 + 16))) return r;
    CK(cub::DeviceRadixSort::SortPairsDescending(W.cubtmp.p, tb3, W.keys.as<unsigned>(), W.keys2.as<unsigned>(),
                                                 W.cidx.as<int>(), W.cidx2.as<int>(), (int)ncols, 0, 16, st));
    const unsigned ntb = (unsigned)((ntiles + bt - 1) / bt);
    prep_tile_kernel<<<ntb, bt, 0, st>>>(ncols, W.cidx2.as<int>(), W.rmaxb.as<int>(), src,
                                         W.trecs.as<long long>(), W.ttasks.as<long long>());
    CK(cudaGetLastError());
    size_t tbs = tb3;
    CK(cub::DeviceScan::ExclusiveSum(W.cubtmp.p, tbs, W.trecs.as<long long>(), W.tlbase.as<long long>(),
                                     (int)ntiles, st));
    tbs = tb3;
    CK(cub::DeviceScan::ExclusiveSum(W.cubtmp.p, tbs, W.ttasks.as<long long>(), W.ttbase.as<long long>(),
                                     (int)ntiles, st));
    long long last[4] = {0, 0, 0, 0};
    int herr = 0;
    CK(cudaMemcpyAsync(&last[0], W.tlbase.as<long long>() + ntiles - 1, sizeof(long long), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&last[1], W.trecs.as<long long>() + ntiles - 1, sizeof(long long), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&last[2], W.ttbase.as<long long>() + ntiles - 1, sizeof(long long), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&last[3], W.ttasks.as<long long>() + ntiles - 1, sizeof(long long), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (herr) {
        set_err("invalid column (%s%s%s%s%s)", (herr & 1) ? "nz outside [2,200] " : "",
                (herr & 2) ? "period count outside [1,160] " : "", (herr & 4) ? "depths not increasing " : "",
                (herr & 8) ? "more than 200 refined layers " : "", (herr & 16) ? "non-positive velocity/density" : "");
        return (herr & (1 | 2 | 8)) ? DAZI_ERR_LIMITS : DAZI_ERR_BADARG;
    }
    const long long nrec = last[0] + last[1], ntask = last[2] + last[3];
    if ((r = W.tflat.ensure(sizeof(float4) * nrec)) || (r = W.tld.ensure(sizeof(LayerD) * nrec)) ||
        (r = W.tti.ensure(sizeof(TiRec) * nrec)) || (r = W.tsp.ensure(sizeof(SpRec) * nrec)) || (r = W.tch.ensure(sizeof(ChainRec) * nrec)) ||
        (r = W.tmeta.ensure(sizeof(ColMeta) * ncols)) || (r = W.ttasklist.ensure(sizeof(int2) * ntask)))
        return r;
    T.flat = W.tflat.as<float4>(); T.ld = W.tld.as<LayerD>(); T.ti = W.tti.as<TiRec>(); T.sp = W.tsp.as<SpRec>();
    T.ch = W.tch.as<ChainRec>(); T.meta = W.tmeta.as<ColMeta>();
    T.tile_lbase = W.tlbase.as<long long>(); T.tasks = W.ttasklist.as<int2>();
    T.ntasks = ntask; T.ncols = ncols; T.pv_sk = pv_sk; T.sen_sk = sen_sk; T.ls_sk = ls_sk;
    prep_tasks_kernel<<<ntb, bt, 0, st>>>(ntiles, W.ttasks.as<long long>(), W.ttbase.as<long long>(),
                                          T.tasks);
    CK(cudaGetLastError());
    prep_build_kernel<<<nb, bt, 0, st>>>(src, po, T, W.cidx2.as<int>(), W.ttbase.as<long long>());
    CK(cudaGetLastError());
    g_ctx.last_launches += 5;
    phase_mark("prep", st);
    return 0;
}

// Kernel variants (instantiations of the templated kernels).
const void* adjoint_fn(int minb)
{
    return minb == 2 ? (const void*)adjoint_kernel<2> : minb == 4 ? (const void*)adjoint_kernel<4>
                                                                  : (const void*)adjoint_kernel<3>;
}
const void* ti_fn(int minb)
{
    switch (minb) {
    case 2: return (const void*)ti_kernel<2>;
    case 3: return (const void*)ti_kernel<3>;
    case 6: return (const void*)ti_kernel<6>;
    case 8: return (const void*)ti_kernel<8>;
    default: return (const void*)ti_kernel<4>;
    }
}

// Largest refined layer count of the tables (first sorted column): one
// small read-back, done once per call (plans keep it).
int table_maxr(const Tables& T, cudaStream_t st, long long& maxr)
{
    ColMeta m0;
    CK(cudaMemcpyAsync(&m0, T.meta, sizeof(ColMeta), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    maxr = m0.rmax;
    return 0;
}

// Scratch of the sweeps, sized for the persistent grids of the chosen
// variants (allocation happens here, never inside a graph capture).
int ensure_sweep_scratch(const Tables& T, bool adj, bool ti, long long maxr, const LaunchCfg& cfg,
                         Work& W, bool group = false)
{
    int r;
    const long long nitems = T.ntasks * TILE;
    if (adj) {
        long long nblk;
        if ((r = W.croot.ensure(sizeof(double) * TILE * (size_t)T.ntasks))) return r;
        if (group && (r = W.crootb.ensure(sizeof(double) * TILE * (size_t)T.ntasks))) return r;
        if ((r = launch_persistent_grid(adjoint_fn(cfg.adj_minb), nitems, 128, nblk))) return r;
        const size_t scr = sizeof(double) * 6 * (size_t)(maxr > 1 ? maxr - 1 : 1) * (size_t)(nblk * 128);
        if ((r = W.adjscr.ensure(scr))) return r;
        if ((r = W.adjord.ensure(sizeof(int) * (size_t)nitems))) return r;
    }
    if (ti) {
        long long nblk;
        if ((r = launch_persistent_grid(ti_fn(cfg.ti_minb), nitems, 128, nblk))) return r;
        const size_t scr = sizeof(double) * TI_SCR_Q * (size_t)maxr * (size_t)(nblk * 128);
        if ((r = W.tiscr.ensure(scr))) return r;
        if ((r = W.tiord.ensure(sizeof(int) * (size_t)nitems))) return r;
    }
    return 0;
}

int run_root(const Tables& T, const double* per, const StageOut& o, int form, bool adj, Work& W,
             const LaunchCfg& cfg, cudaStream_t st)
{
    RootArgs a;
    a.T = T; a.periods = per; a.tol = 1.0e-6;   // surfdisp96.f:608
    a.pv = o.pv; a.croot = adj ? W.croot.as<double>() : nullptr; a.status = o.status;
    a.croot_b = adj && form_group(form) ? W.crootb.as<double>() : nullptr;
    a.nevals = W.counters.as<unsigned long long>();
    a.scan32 = (form & DAZI_FORM_SCAN_FP32) ? 1 : 0;
    const int ifunc = form_ifunc(form);
    const bool grp = form_group(form);
    if (ifunc == 1 || grp) {
        // Love and/or group velocity: one launch shape
        const unsigned nb = (unsigned)((T.ncols + 127) / 128);
        if (ifunc == 1 && grp) root_kernel<128, 0, 1, true><<<nb, 128, 0, st>>>(a);
        else if (ifunc == 1) root_kernel<128, 0, 1, false><<<nb, 128, 0, st>>>(a);
        else root_kernel<128, 0, 2, true><<<nb, 128, 0, st>>>(a);
    } else if (form & DAZI_FORM_FAST_ROOT) {
        const int bt = cfg.root_bt, mb = cfg.root_minb;
        const unsigned nb = (unsigned)((T.ncols + bt - 1) / bt);
        if (bt == 64 && mb == 10) root_kernel<64, 10, 2, false, true><<<nb, 64, 0, st>>>(a);
        else if (bt == 64) root_kernel<64, 0, 2, false, true><<<nb, 64, 0, st>>>(a);
        else if (bt == 256) root_kernel<256, 0, 2, false, true><<<nb, 256, 0, st>>>(a);
        else if (mb == 5) root_kernel<128, 5, 2, false, true><<<nb, 128, 0, st>>>(a);
        else root_kernel<128, 0, 2, false, true><<<nb, 128, 0, st>>>(a);
    } else {
        const int bt = cfg.root_bt, mb = cfg.root_minb;
        const unsigned nb = (unsigned)((T.ncols + bt - 1) / bt);
        if (bt == 64 && mb == 10) root_kernel<64, 10><<<nb, 64, 0, st>>>(a);
        else if (bt == 64) root_kernel<64, 0><<<nb, 64, 0, st>>>(a);
        else if (bt == 256) root_kernel<256, 0><<<nb, 256, 0, st>>>(a);
        else if (mb == 5) root_kernel<128, 5><<<nb, 128, 0, st>>>(a);
        else root_kernel<128, 0><<<nb, 128, 0, st>>>(a);
    }
    CK(cudaGetLastError());
    ++g_ctx.last_launches;
    phase_mark("root", st);
    return 0;
}

// love: Love waves (adjoint_love_kernel); group: group velocity, from the
// roots at t1a and t1b (adjoint_group_kernel, adjoint_love_group_kernel).
// All run on the grid and scratch of the Rayleigh phase kernel's variant.
int run_adjoint(const Tables& T, const double* per, const StageOut& o, long long maxr, Work& W,
                const LaunchCfg& cfg, cudaStream_t st, bool love = false, bool group = false)
{
    int r;
    long long nblk;
    if ((r = launch_persistent_grid(adjoint_fn(cfg.adj_minb), T.ntasks * TILE, 128, nblk))) return r;
    unsigned* queues = reinterpret_cast<unsigned*>(W.counters.as<unsigned long long>() + 2);
    CK(cudaMemsetAsync(queues, 0, sizeof(unsigned), st));
    AdjArgs j;
    j.T = T; j.periods = per; j.croot = W.croot.as<double>();
    j.sen_vs = o.svs; j.sen_vp = o.svp; j.sen_rho = o.srh;
    j.scratch = W.adjscr.as<double>(); j.scr_layers = maxr > 1 ? maxr - 1 : 1; j.queue = queues;
    j.croot_b = group ? W.crootb.as<double>() : nullptr;
    if (!love && !group && cfg.cut) {
        // Rayleigh phase velocity: the pairs of each tile by the depth their
        // sweep reaches (adj_order_kernel)
        const long long ntiles = (T.ncols + TILE - 1) / TILE;
        adj_order_kernel<<<(unsigned)ntiles, TI_ORDER_THREADS, 0, st>>>(j, W.adjord.as<int>(), W.ttbase.as<long long>(),
                                                                      W.ttasks.as<long long>());
        CK(cudaGetLastError());
        ++g_ctx.last_launches;
        j.order = W.adjord.as<int>();
    }
    if (love && group) adjoint_love_group_kernel<3><<<(unsigned)nblk, 128, 0, st>>>(j);
    else if (group) adjoint_group_kernel<3><<<(unsigned)nblk, 128, 0, st>>>(j);
    else if (love) adjoint_love_kernel<3><<<(unsigned)nblk, 128, 0, st>>>(j);
    else if (cfg.adj_minb == 2) adjoint_kernel<2><<<(unsigned)nblk, 128, 0, st>>>(j);
    else if (cfg.adj_minb == 4) adjoint_kernel<4><<<(unsigned)nblk, 128, 0, st>>>(j);
    else adjoint_kernel<3><<<(unsigned)nblk, 128, 0, st>>>(j);
    CK(cudaGetLastError());
    ++g_ctx.last_launches;
    phase_mark("adjoint", st);
    return 0;
}

int run_ti(const Tables& T, const double* per, const StageOut& o, long long maxr, Work& W,
           const LaunchCfg& cfg, cudaStream_t st)
{
    int r;
    long long nblk;
    if ((r = launch_persistent_grid(ti_fn(cfg.ti_minb), T.ntasks * TILE, 128, nblk))) return r;
    unsigned long long* c = W.counters.as<unsigned long long>();
    unsigned* queues = reinterpret_cast<unsigned*>(c + 2);
    CK(cudaMemsetAsync(queues + 1, 0, sizeof(unsigned), st));
    TiArgs t;
    t.T = T; t.periods = per; t.pv = o.pv; t.lsen = o.lsen;
    t.scratch = W.tiscr.as<double>(); t.scr_layers = maxr; t.queue = queues + 1;
    t.errflag = reinterpret_cast<int*>(c + 1);
    t.order = W.tiord.as<int>();
    t.cut = cfg.cut ? 1 : 0;
    const long long ntiles = (T.ncols + TILE - 1) / TILE;
    ti_order_kernel<<<(unsigned)ntiles, TI_ORDER_THREADS, 0, st>>>(t, W.ttbase.as<long long>(),
                                                                 W.ttasks.as<long long>());
    CK(cudaGetLastError());
    ++g_ctx.last_launches;
    if (cfg.ti_minb == 2) ti_kernel<2><<<(unsigned)nblk, 128, 0, st>>>(t);
    else if (cfg.ti_minb == 3) ti_kernel<3><<<(unsigned)nblk, 128, 0, st>>>(t);
    else if (cfg.ti_minb == 4) ti_kernel<4><<<(unsigned)nblk, 128, 0, st>>>(t);
    else if (cfg.ti_minb == 6) ti_kernel<6><<<(unsigned)nblk, 128, 0, st>>>(t);
    else ti_kernel<8><<<(unsigned)nblk, 128, 0, st>>>(t);
    CK(cudaGetLastError());
    ++g_ctx.last_launches;
    phase_mark("ti", st);
    return 0;
}

// The per-(column, period) kernels and the root search over built tables.
// outs_ready (optional) is recorded once pv and the sensitivity kernels are
// final, before the Gc/Gs sweep.
int run_tables(const Tables& T, const double* per, const StageOut& o, int form, bool fd_done,
               cudaStream_t st, Work& W, const LaunchCfg& cfg, cudaEvent_t outs_ready = nullptr)
{
    int r;
    const bool adj = o.svs && (form & 1) == DAZI_FORM_ADJOINT;
    LaunchCfg cf = cfg;
    cf.cut = (form & DAZI_FORM_FULL_STACK) == 0;
    long long maxr = 0;
    if ((r = table_maxr(T, st, maxr))) return r;
    if ((r = ensure_sweep_scratch(T, adj, o.lsen != nullptr, maxr, cfg, W, form_group(form)))) return r;
    if (!fd_done && (r = run_root(T, per, o, form, adj, W, cf, st))) return r;
    if (adj && (r = run_adjoint(T, per, o, maxr, W, cf, st, form_ifunc(form) == 1, form_group(form))))
        return r;
    if (outs_ready) CK(cudaEventRecord(outs_ready, st));
    if (o.lsen && (r = run_ti(T, per, o, maxr, W, cf, st))) return r;
    return 0;
}

// The stage on device pointers (stream-ordered; one small host sync sizes
// the layer tables).
//   plain   + kernels: one CTA per column runs the 1 + 6 nz models (FD)
//   adjoint + kernels: per-column root search, then per-(column, period)
//                      adjoint sweeps
//   Lsen requested   : per-(column, period) TI sweeps from the phase velocity
int stage_device(int nx, int ny, int nz, const float* vel, const float* vp, const float* rho,
                 const StageOut& o, int kmax, const double* per, long long col_start,
                 long long col_count, int form, cudaStream_t st, cudaEvent_t outs_ready = nullptr)
{
    const long long ncol = (long long)nx * ny;
    if (col_count == 0) return 0;
    const Geometry* geo = g_ctx.geo.as<Geometry>();
    int r;
    if ((r = g_ctx.w.counters.ensure(sizeof(unsigned long long) * 8))) return r;
    CK(cudaMemsetAsync(g_ctx.w.counters.p, 0, sizeof(unsigned long long) * 8, st));
    g_ctx.last_rmax = g_ctx.geo_rmax;
    g_ctx.last_launches = 0;
    phase_begin(st);
    const bool fd = o.svs && (form & 1) == DAZI_FORM_PLAIN;
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
            a.dln = 0.01f; a.tol = 1.0e-6; a.nevals = g_ctx.w.counters.as<unsigned long long>();
            const int ifunc = form_ifunc(form);
            const bool grp = form_group(form);
            if (ifunc == 1 && grp) fd_column_kernel<1, true><<<(unsigned)n, threads, smem, st>>>(a);
            else if (ifunc == 1) fd_column_kernel<1, false><<<(unsigned)n, threads, smem, st>>>(a);
            else if (grp) fd_column_kernel<2, true><<<(unsigned)n, threads, smem, st>>>(a);
            else fd_column_kernel<2, false><<<(unsigned)n, threads, smem, st>>>(a);
            CK(cudaGetLastError());
            ++g_ctx.last_launches;
        }
        phase_mark("fd", st);
        if (!o.lsen) {
            if (outs_ready) CK(cudaEventRecord(outs_ready, st));
            return 0;
        }
    }
    ColSrc src;
    src.ragged = false; src.ncol = ncol; src.col0 = col_start - 1;
    src.vel = vel; src.vp = vp; src.rho = rho; src.depz = g_ctx.depz.as<float>();
    src.node_off = nullptr; src.per_off = nullptr; src.nz = nz; src.K = kmax;
    src.minthk = g_ctx.geo_minthk;
    src.ifunc = form_ifunc(form);
    PrepOut po{nullptr, nullptr, g_ctx.w.counters.as<unsigned long long>() + 4};
    Tables T;
    if ((r = build_tables(src, col_count, po, ncol, ncol, ncol, st, T, g_ctx.w))) return r;
    return run_tables(T, per, o, form, fd, st, g_ctx.w, default_cfg(), outs_ready);
}

// Ragged batch on device pointers.
struct BatchIn {
    long long ncols;
    const long long* node_off;
    const float* depz;
    const float* vs;
    const float* vp;
    const float* rho;
    const long long* per_off;
    const double* periods;
    float minthk;
    const long long* sen_off;
    const long long* ls_off;
};

int batch_device(const BatchIn& B, const StageOut& o, int form, cudaStream_t st,
                 cudaEvent_t outs_ready = nullptr)
{
    if (B.ncols == 0) return 0;
    int r;
    if ((r = g_ctx.w.counters.ensure(sizeof(unsigned long long) * 8))) return r;
    CK(cudaMemsetAsync(g_ctx.w.counters.p, 0, sizeof(unsigned long long) * 8, st));
    g_ctx.last_launches = 0;
    g_ctx.last_rmax = 0;
    phase_begin(st);
    ColSrc src;
    src.ragged = true; src.ncol = 0; src.col0 = 0;
    src.vel = B.vs; src.vp = B.vp; src.rho = B.rho; src.depz = B.depz;
    src.node_off = B.node_off; src.per_off = B.per_off; src.nz = 0; src.K = 0;
    src.minthk = B.minthk;
    src.ifunc = form_ifunc(form);
    PrepOut po{B.sen_off, B.ls_off, g_ctx.w.counters.as<unsigned long long>() + 4};
    Tables T;
    if ((r = build_tables(src, B.ncols, po, 1, 1, 1, st, T, g_ctx.w))) return r;
    const bool fd = o.svs && (form & 1) == DAZI_FORM_PLAIN;
    if (fd) {
        // plain form: one CTA per column, scratch offsets per column
        std::vector<long long> hoff(B.ncols + 1), hn(B.ncols + 1), hp(B.ncols + 1);
        CK(cudaMemcpyAsync(hn.data(), B.node_off, sizeof(long long) * (B.ncols + 1), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hp.data(), B.per_off, sizeof(long long) * (B.ncols + 1), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        hoff[0] = 0;
        long long maxcol = 0;
        for (long long c = 0; c < B.ncols; ++c) {
            const long long need = (1 + 6 * (hn[c + 1] - hn[c])) * (hp[c + 1] - hp[c]);
            hoff[c + 1] = hoff[c] + need;
            if (need > maxcol) maxcol = need;
        }
        if ((r = g_ctx.cbufoff.ensure(sizeof(long long) * (B.ncols + 1)))) return r;
        CK(cudaMemcpyAsync(g_ctx.cbufoff.p, hoff.data(), sizeof(long long) * (B.ncols + 1), cudaMemcpyHostToDevice, st));
        const long long capf = std::max<long long>(maxcol, (512ll << 20) / 4);
        if ((r = g_ctx.cscratch.ensure(sizeof(float) * capf))) return r;
        long long c0 = 0;
        while (c0 < B.ncols) {
            long long c1 = c0;
            while (c1 < B.ncols && hoff[c1 + 1] - hoff[c0] <= capf) ++c1;
            FdArgs a;
            a.geo = nullptr; a.nz = 0; a.kmax = 0; a.ncol = 0; a.col0 = c0;
            a.vel = B.vs; a.vp = B.vp; a.rho = B.rho; a.periods = B.periods;
            a.pv = o.pv; a.sen_vs = o.svs; a.sen_vp = o.svp; a.sen_rho = o.srh;
            a.status = o.status; a.cscratch = g_ctx.cscratch.as<float>();
            a.dln = 0.01f; a.tol = 1.0e-6; a.nevals = g_ctx.w.counters.as<unsigned long long>();
            FdBatch fb;
            fb.node_off = B.node_off; fb.per_off = B.per_off; fb.depz = B.depz; fb.minthk = B.minthk;
            fb.sen_off = B.sen_off; fb.cbuf_off = g_ctx.cbufoff.as<long long>();
            const unsigned nb = (unsigned)(c1 - c0);
            const size_t sm = fd_batch_smem_bytes();
            const int ifunc = form_ifunc(form);
            const bool grp = form_group(form);
            if (ifunc == 1 && grp) fd_batch_kernel<1, true><<<nb, 256, sm, st>>>(a, fb);
            else if (ifunc == 1) fd_batch_kernel<1, false><<<nb, 256, sm, st>>>(a, fb);
            else if (grp) fd_batch_kernel<2, true><<<nb, 256, sm, st>>>(a, fb);
            else fd_batch_kernel<2, false><<<nb, 256, sm, st>>>(a, fb);
            CK(cudaGetLastError());
            ++g_ctx.last_launches;
            c0 = c1;
        }
        phase_mark("fd", st);
    }
    return run_tables(T, B.periods, o, form, fd, st, g_ctx.w, default_cfg(), outs_ready);
}

// ------------------------------------------------------------------ plans
// A plan binds a ragged batch (structure and device buffers) once: the
// structure part of the tables (refined layer counts, sort, tiles, tasks)
// is built at creation, the kernel variants are picked by timing them on
// this batch, and the per-run sequence -- layer values from the current
// velocities, counters, root search, adjoint and Gc/Gs sweeps -- is
// captured in a CUDA graph.  A run is one graph launch, with no host
// synchronisation.
struct Plan {
    int device = -1;
    cudaStream_t cs = nullptr;       // private stream (build, tuning, capture)
    Work w;
    ColSrc src;
    PrepOut po;
    Tables T;
    StageOut o;
    const double* periods = nullptr;
    int form = DAZI_FORM_ADJOINT;
    bool adj = false;
    long long maxr = 0;
    LaunchCfg cfg;
    float best_ms[3] = {0.f, 0.f, 0.f};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    void release()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr; graph = nullptr;
        w.release();
        if (cs) cudaStreamDestroy(cs);
        cs = nullptr;
    }
};

// Time one phase launcher on the plan's stream (best of two after a warm-up).
template <class F>
int time_phase(Plan& P, F launch, float& ms)
{
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    int r = launch();
    float best = 1e30f;
    for (int rep = 0; rep < 2 && !r; ++rep) {
        cudaEventRecord(a, P.cs);
        r = launch();
        cudaEventRecord(b, P.cs);
        if (!r && cudaEventSynchronize(b) == cudaSuccess) {
            float t = 0.f;
            cudaEventElapsedTime(&t, a, b);
            if (t < best) best = t;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    ms = best;
    return r;
}

int plan_tune(Plan& P)
{
    int r;
    const int adj_c[3] = {2, 3, 4}, ti_c[5] = {2, 3, 4, 6, 8};
    LaunchCfg c = P.cfg;
    float best = 1e30f;
    for (const auto& v : kRootVariants) {
        c.root_bt = v[0];
        c.root_minb = v[1];
        float ms;
        if ((r = time_phase(P, [&] { return run_root(P.T, P.periods, P.o, P.form, P.adj, P.w, c, P.cs); }, ms)))
            return r;
        if (ms < best) { best = ms; P.cfg.root_bt = v[0]; P.cfg.root_minb = v[1]; }
    }
    P.best_ms[0] = best;
    c.root_bt = P.cfg.root_bt;
    c.root_minb = P.cfg.root_minb;
    if (P.adj) {
        best = 1e30f;
        for (int mb : adj_c) {
            c.adj_minb = mb;
            float ms;
            if ((r = ensure_sweep_scratch(P.T, true, false, P.maxr, c, P.w))) return r;
            if ((r = time_phase(P, [&] { return run_adjoint(P.T, P.periods, P.o, P.maxr, P.w, c, P.cs); }, ms)))
                return r;
            if (ms < best) { best = ms; P.cfg.adj_minb = mb; }
        }
        P.best_ms[1] = best;
        c.adj_minb = P.cfg.adj_minb;
    }
    if (P.o.lsen) {
        best = 1e30f;
        for (int mb : ti_c) {
            c.ti_minb = mb;
            float ms;
            if ((r = ensure_sweep_scratch(P.T, false, true, P.maxr, c, P.w))) return r;
            if ((r = time_phase(P, [&] { return run_ti(P.T, P.periods, P.o, P.maxr, P.w, c, P.cs); }, ms)))
                return r;
            if (ms < best) { best = ms; P.cfg.ti_minb = mb; }
        }
        P.best_ms[2] = best;
    }
    return 0;
}

// The per-run sequence on the plan's stream (captured).
int plan_enqueue(Plan& P)
{
    int r;
    CK(cudaMemsetAsync(P.w.counters.p, 0, sizeof(unsigned long long) * 8, P.cs));
    const unsigned nb = (unsigned)((P.T.ncols + 127) / 128);
    prep_build_kernel<<<nb, 128, 0, P.cs>>>(P.src, P.po, P.T, P.w.cidx2.as<int>(), P.w.ttbase.as<long long>());
    CK(cudaGetLastError());
    if ((r = run_root(P.T, P.periods, P.o, P.form, P.adj, P.w, P.cfg, P.cs))) return r;
    if (P.adj && (r = run_adjoint(P.T, P.periods, P.o, P.maxr, P.w, P.cfg, P.cs))) return r;
    if (P.o.lsen && (r = run_ti(P.T, P.periods, P.o, P.maxr, P.w, P.cfg, P.cs))) return r;
    return 0;
}

int plan_create(const BatchIn& B, const StageOut& o, int form, bool tune, cudaStream_t user, Plan& P)
{
    int r;
    CK(cudaGetDevice(&P.device));
    CK(cudaStreamSynchronize(user));   // the inputs are ready
    CK(cudaStreamCreateWithFlags(&P.cs, cudaStreamNonBlocking));
    if ((r = P.w.counters.ensure(sizeof(unsigned long long) * 8))) return r;
    CK(cudaMemsetAsync(P.w.counters.p, 0, sizeof(unsigned long long) * 8, P.cs));
    P.src.ragged = true; P.src.ncol = 0; P.src.col0 = 0;
    P.src.vel = B.vs; P.src.vp = B.vp; P.src.rho = B.rho; P.src.depz = B.depz;
    P.src.node_off = B.node_off; P.src.per_off = B.per_off; P.src.nz = 0; P.src.K = 0;
    P.src.minthk = B.minthk;
    P.src.ifunc = 2;
    P.po = PrepOut{B.sen_off, B.ls_off, P.w.counters.as<unsigned long long>() + 4};
    P.o = o;
    P.form = form;
    P.cfg.cut = (form & DAZI_FORM_FULL_STACK) == 0;
    P.periods = B.periods;
    P.adj = o.svs != nullptr;
    if ((r = build_tables(P.src, B.ncols, P.po, 1, 1, 1, P.cs, P.T, P.w))) return r;
    if ((r = table_maxr(P.T, P.cs, P.maxr))) return r;
    if ((r = ensure_sweep_scratch(P.T, P.adj, o.lsen != nullptr, P.maxr, P.cfg, P.w))) return r;
    if (tune && (r = plan_tune(P))) return r;
    if ((r = ensure_sweep_scratch(P.T, P.adj, o.lsen != nullptr, P.maxr, P.cfg, P.w))) return r;
    CK(cudaStreamSynchronize(P.cs));
    // capture (per-phase timing stays out of the graph)
    const bool timing = g_ctx.timer.on;
    g_ctx.timer.on = false;
    CK(cudaStreamBeginCapture(P.cs, cudaStreamCaptureModeThreadLocal));
    r = plan_enqueue(P);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(P.cs, &g);
    g_ctx.timer.on = timing;
    if (r) { if (g) cudaGraphDestroy(g); return r; }
    if (e != cudaSuccess) { set_err("graph capture failed: %s", cudaGetErrorString(e)); return DAZI_ERR_CUDA; }
    P.graph = g;
    CK(cudaGraphInstantiate(&P.exec, P.graph, 0ULL));
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
    if (*iwave != 1 && *iwave != 2) {
        set_err("iwave must be 1 (Love) or 2 (Rayleigh), got %d", *iwave);
        return DAZI_ERR_BADARG;
    }
    if (form & kWaveFlags) {
        set_err("pass the wave and velocity type as iwave/igr, not as form flags (form %d)", form);
        return DAZI_ERR_BADARG;
    }
    // surfdisp96: ifunc = 1 for iwave = 1; group velocity for igr > 0
    form |= (*iwave == 1 ? DAZI_FORM_LOVE : 0) | (*igr > 0 ? DAZI_FORM_GROUP : 0);
    if ((svs == nullptr) != (svp == nullptr) || (svs == nullptr) != (srh == nullptr)) {
        set_err("sen_vsRc, sen_vpRc, sen_rhoRc must be all set or all NULL");
        return DAZI_ERR_BADARG;
    }
    if ((vp == nullptr) != (rho == nullptr)) { set_err("vp and rho must both be set or both NULL"); return DAZI_ERR_BADARG; }
    int r;
    if ((r = check_form(form, lsen != nullptr))) return r;
    const int nx = *pnx, ny = *pny, nz = *pnz, kmax = *pkmax;
    const float minthk = *pminthk;
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
                     col_start, col_count, form, st, g_ctx.outs_ready);
    if (r) return r;
    // Copy back only the written columns: every (k[, i]) slab holds the
    // column range contiguously.  pv and the sensitivity kernels go on the
    // copy stream as soon as they are final, overlapping the Gc/Gs sweep.
    const size_t c0 = (size_t)(col_start - 1), cn = (size_t)col_count;
    cudaStream_t cs = g_ctx.cstream;
    CK(cudaStreamWaitEvent(cs, g_ctx.outs_ready, 0));
    CK(cudaMemcpy2DAsync(pv + c0, sizeof(double) * ncol, g_ctx.pv.as<double>() + c0, sizeof(double) * ncol,
                         sizeof(double) * cn, kmax, cudaMemcpyDeviceToHost, cs));
    if (kern) {
        double* hs[3] = {svs, svp, srh};
        DBuf* ds[3] = {&g_ctx.svs, &g_ctx.svp, &g_ctx.srh};
        for (int q = 0; q < 3; ++q)
            CK(cudaMemcpy2DAsync(hs[q] + c0, sizeof(double) * ncol, ds[q]->as<double>() + c0,
                                 sizeof(double) * ncol, sizeof(double) * cn, (size_t)kmax * nz,
                                 cudaMemcpyDeviceToHost, cs));
    }
    if (lsen)
        CK(cudaMemcpy2DAsync(lsen + c0, sizeof(float) * ncol, g_ctx.lsen.as<float>() + c0,
                             sizeof(float) * ncol, sizeof(float) * cn, (size_t)kmax * (nz - 1),
                             cudaMemcpyDeviceToHost, st));
    g_ctx.last_status.resize(ncol);
    CK(cudaMemcpyAsync(g_ctx.last_status.data(), g_ctx.status.p, sizeof(int) * ncol, cudaMemcpyDeviceToHost, st));
    int hflag[2] = {0, 0};
    CK(cudaMemcpyAsync(hflag, g_ctx.w.counters.as<unsigned long long>() + 1, sizeof(int) * 2,
                       cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaStreamSynchronize(cs));
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
                     const void* svs, const void* svp, const void* srh, const void* lsen)
{
    if ((svs == nullptr) != (svp == nullptr) || (svs == nullptr) != (srh == nullptr)) {
        set_err("sen_* must be all set or all NULL");
        return DAZI_ERR_BADARG;
    }
    if ((vp == nullptr) != (rho == nullptr)) { set_err("vp and rho must both be set or both NULL"); return DAZI_ERR_BADARG; }
    if (int r = check_form(form, lsen != nullptr)) return r;
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
    if ((r = check_dev_common(nz, kmaxRc, form, vp, rho, svs, svp, srh, lsen))) return r;
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

int dazi_dk_batch_dev(long long ncols, const long long* node_off, const float* depz, const float* vs,
                      const float* vp, const float* rho, const long long* per_off,
                      const double* periods, float minthk, double* pv, const long long* sen_off,
                      double* sen_vs, double* sen_vp, double* sen_rho, const long long* ls_off,
                      float* lsen, int form, int* status, void* stream)
{
    if (ncols < 0 || (ncols > 0 && (!node_off || !depz || !vs || !per_off || !periods || !pv))) {
        set_err("null argument");
        return DAZI_ERR_BADARG;
    }
    if ((sen_vs == nullptr) != (sen_vp == nullptr) || (sen_vs == nullptr) != (sen_rho == nullptr) ||
        (sen_vs && !sen_off) || (lsen && !ls_off)) {
        set_err("kernel outputs need sen_off / ls_off and all three sen arrays");
        return DAZI_ERR_BADARG;
    }
    if ((vp == nullptr) != (rho == nullptr)) { set_err("vp and rho must both be set or both NULL"); return DAZI_ERR_BADARG; }
    if (int r = check_form(form, lsen != nullptr)) return r;
    if (!(minthk > 0.f) || !std::isfinite(minthk)) { set_err("minthk must be > 0"); return DAZI_ERR_BADARG; }
    std::lock_guard<std::mutex> lk(g_mu);
    int r;
    if ((r = ensure_context())) return r;
    BatchIn B{ncols, node_off, depz, vs, vp, rho, per_off, periods, minthk, sen_off, ls_off};
    StageOut o;
    o.pv = pv; o.svs = sen_vs; o.svp = sen_vp; o.srh = sen_rho; o.lsen = lsen; o.status = status;
    return batch_device(B, o, form, (cudaStream_t)stream);
}

int dazi_dk_batch(long long ncols, const long long* node_off, const float* depz, const float* vs,
                  const float* vp, const float* rho, const long long* per_off, const double* periods,
                  float minthk, double* pv, const long long* sen_off, double* sen_vs, double* sen_vp,
                  double* sen_rho, const long long* ls_off, float* lsen, int form, int* status)
{
    if (ncols < 0 || (ncols > 0 && (!node_off || !depz || !vs || !per_off || !periods || !pv))) {
        set_err("null argument");
        return DAZI_ERR_BADARG;
    }
    if ((sen_vs == nullptr) != (sen_vp == nullptr) || (sen_vs == nullptr) != (sen_rho == nullptr) ||
        (sen_vs && !sen_off) || (lsen && !ls_off)) {
        set_err("kernel outputs need sen_off / ls_off and all three sen arrays");
        return DAZI_ERR_BADARG;
    }
    if ((vp == nullptr) != (rho == nullptr)) { set_err("vp and rho must both be set or both NULL"); return DAZI_ERR_BADARG; }
    if (int r = check_form(form, lsen != nullptr)) return r;
    if (!(minthk > 0.f) || !std::isfinite(minthk)) { set_err("minthk must be > 0"); return DAZI_ERR_BADARG; }
    if (ncols == 0) return DAZI_OK;
    for (long long c = 0; c < ncols; ++c)
        if (node_off[c + 1] < node_off[c] || per_off[c + 1] < per_off[c]) {
            set_err("offsets must be non-decreasing (column %lld)", c);
            return DAZI_ERR_BADARG;
        }
    for (long long c = 0; c < ncols; ++c)
        for (long long p = per_off[c]; p < per_off[c + 1]; ++p)
            if (!(periods[p] > 0.0) || !std::isfinite(periods[p])) {
                set_err("period %lld is not a positive finite number", p);
                return DAZI_ERR_BADARG;
            }
    const long long nn = node_off[ncols], np_ = per_off[ncols];
    const long long ns = sen_vs ? sen_off[ncols] : 0, nl = lsen ? ls_off[ncols] : 0;
    std::lock_guard<std::mutex> lk(g_mu);
    int r;
    if ((r = ensure_context())) return r;
    cudaStream_t st = g_ctx.stream;
    const size_t o1 = sizeof(long long) * (ncols + 1);
    if ((r = g_ctx.bnode.ensure(o1)) || (r = g_ctx.bper.ensure(o1)) || (r = g_ctx.bdep.ensure(sizeof(float) * nn)) ||
        (r = g_ctx.bvs.ensure(sizeof(float) * nn)) || (r = g_ctx.bperiods.ensure(sizeof(double) * np_)) ||
        (r = g_ctx.bpv.ensure(sizeof(double) * np_)) || (r = g_ctx.bstatus.ensure(sizeof(int) * ncols)))
        return r;
    if (vp && ((r = g_ctx.bvp.ensure(sizeof(float) * nn)) || (r = g_ctx.brho.ensure(sizeof(float) * nn)))) return r;
    if (sen_vs && ((r = g_ctx.bsenoff.ensure(o1)) || (r = g_ctx.bsvs.ensure(sizeof(double) * ns)) ||
                   (r = g_ctx.bsvp.ensure(sizeof(double) * ns)) || (r = g_ctx.bsrh.ensure(sizeof(double) * ns))))
        return r;
    if (lsen && ((r = g_ctx.blsoff.ensure(o1)) || (r = g_ctx.blsen.ensure(sizeof(float) * nl)))) return r;
    CK(cudaMemcpyAsync(g_ctx.bnode.p, node_off, o1, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(g_ctx.bper.p, per_off, o1, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(g_ctx.bdep.p, depz, sizeof(float) * nn, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(g_ctx.bvs.p, vs, sizeof(float) * nn, cudaMemcpyHostToDevice, st));
    if (vp) {
        CK(cudaMemcpyAsync(g_ctx.bvp.p, vp, sizeof(float) * nn, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(g_ctx.brho.p, rho, sizeof(float) * nn, cudaMemcpyHostToDevice, st));
    }
    CK(cudaMemcpyAsync(g_ctx.bperiods.p, periods, sizeof(double) * np_, cudaMemcpyHostToDevice, st));
    if (sen_vs) CK(cudaMemcpyAsync(g_ctx.bsenoff.p, sen_off, o1, cudaMemcpyHostToDevice, st));
    if (lsen) CK(cudaMemcpyAsync(g_ctx.blsoff.p, ls_off, o1, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(g_ctx.bstatus.p, 0, sizeof(int) * ncols, st));
    BatchIn B{ncols, g_ctx.bnode.as<long long>(), g_ctx.bdep.as<float>(), g_ctx.bvs.as<float>(),
              vp ? g_ctx.bvp.as<float>() : nullptr, vp ? g_ctx.brho.as<float>() : nullptr,
              g_ctx.bper.as<long long>(), g_ctx.bperiods.as<double>(), minthk,
              sen_vs ? g_ctx.bsenoff.as<long long>() : nullptr, lsen ? g_ctx.blsoff.as<long long>() : nullptr};
    StageOut o;
    o.pv = g_ctx.bpv.as<double>();
    o.svs = sen_vs ? g_ctx.bsvs.as<double>() : nullptr;
    o.svp = sen_vs ? g_ctx.bsvp.as<double>() : nullptr;
    o.srh = sen_vs ? g_ctx.bsrh.as<double>() : nullptr;
    o.lsen = lsen ? g_ctx.blsen.as<float>() : nullptr;
    o.status = g_ctx.bstatus.as<int>();
    // the kernels are queued first; pv and the sensitivity kernels then go to
    // the host on the copy stream while the Gc/Gs sweep runs
    if ((r = batch_device(B, o, form, st, g_ctx.outs_ready))) return r;
    cudaStream_t cs = g_ctx.cstream;
    CK(cudaStreamWaitEvent(cs, g_ctx.outs_ready, 0));
    CK(cudaMemcpyAsync(pv, o.pv, sizeof(double) * np_, cudaMemcpyDeviceToHost, cs));
    if (sen_vs) {
        CK(cudaMemcpyAsync(sen_vs, o.svs, sizeof(double) * ns, cudaMemcpyDeviceToHost, cs));
        CK(cudaMemcpyAsync(sen_vp, o.svp, sizeof(double) * ns, cudaMemcpyDeviceToHost, cs));
        CK(cudaMemcpyAsync(sen_rho, o.srh, sizeof(double) * ns, cudaMemcpyDeviceToHost, cs));
    }
    if (lsen) CK(cudaMemcpyAsync(lsen, o.lsen, sizeof(float) * nl, cudaMemcpyDeviceToHost, st));
    std::vector<int> hst(ncols);
    CK(cudaMemcpyAsync(hst.data(), o.status, sizeof(int) * ncols, cudaMemcpyDeviceToHost, st));
    int hflag = 0;
    CK(cudaMemcpyAsync(&hflag, g_ctx.w.counters.as<unsigned long long>() + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaStreamSynchronize(cs));
    if (status) std::memcpy(status, hst.data(), sizeof(int) * ncols);
    if (hflag) { set_err("non-finite Lsen_Gsc value (degenerate layer: Vp <= Vs?)"); return DAZI_ERR_MODEL; }
    for (long long c = 0; c < ncols; ++c)
        if (hst[c] != 0) return DAZI_WARN_NOROOT;
    return DAZI_OK;
}

int dazi_dk_set_timing(int on)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_ctx.timer.on = on != 0;
    return 0;
}

int dazi_dk_last_timing(const char** names, double* ms, int cap)
{
    std::lock_guard<std::mutex> lk(g_mu);
    PhaseTimer& T = g_ctx.timer;
    if (!T.on || !T.made) return 0;
    if (cudaEventSynchronize(T.ev[T.n]) != cudaSuccess) { cudaGetLastError(); set_err("event sync failed"); return DAZI_ERR_CUDA; }
    const int n = T.n < cap ? T.n : cap;
    for (int i = 0; i < n; ++i) {
        float f = 0.f;
        cudaEventElapsedTime(&f, T.ev[i], T.ev[i + 1]);
        if (names) names[i] = T.name[i];
        if (ms) ms[i] = f;
    }
    return n;
}

int dazi_dk_last_launches(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_ctx.last_launches;
}

int dazi_dk_last_work(long long* secular_evals, long long* layer_evals)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx.ready || !g_ctx.w.counters.p) { set_err("no call made yet"); return DAZI_ERR_BADARG; }
    unsigned long long h[4] = {0, 0, 0, 0};
    CK(cudaMemcpy(h, g_ctx.w.counters.p, sizeof(h), cudaMemcpyDeviceToHost));
    if (secular_evals) *secular_evals = (long long)h[0];
    if (layer_evals) *layer_evals = (long long)h[3];
    return 0;
}

int dazi_dk_last_items(long long* column_periods, long long* layer_items)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx.ready || !g_ctx.w.counters.p) { set_err("no call made yet"); return DAZI_ERR_BADARG; }
    unsigned long long h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    CK(cudaMemcpy(h, g_ctx.w.counters.p, sizeof(h), cudaMemcpyDeviceToHost));
    if (column_periods) *column_periods = (long long)h[5];
    if (layer_items) *layer_items = (long long)h[4];
    return 0;
}

int dazi_dk_plan_create(long long ncols, const long long* node_off, const float* depz, const float* vs,
                        const float* vp, const float* rho, const long long* per_off,
                        const double* periods, float minthk, double* pv, const long long* sen_off,
                        double* sen_vs, double* sen_vp, double* sen_rho, const long long* ls_off,
                        float* lsen, int form, int* status, int tune, void* stream, void** plan)
{
    if (!plan) { set_err("null plan pointer"); return DAZI_ERR_BADARG; }
    *plan = nullptr;
    if (ncols < 1 || !node_off || !depz || !vs || !per_off || !periods || !pv || !status) {
        set_err("null argument or empty batch");
        return DAZI_ERR_BADARG;
    }
    if ((sen_vs == nullptr) != (sen_vp == nullptr) || (sen_vs == nullptr) != (sen_rho == nullptr) ||
        (sen_vs && !sen_off) || (lsen && !ls_off)) {
        set_err("kernel outputs need sen_off / ls_off and all three sen arrays");
        return DAZI_ERR_BADARG;
    }
    if ((vp == nullptr) != (rho == nullptr)) { set_err("vp and rho must both be set or both NULL"); return DAZI_ERR_BADARG; }
    if (check_form(form, lsen != nullptr) || (form & 1) != DAZI_FORM_ADJOINT || (form & kWaveFlags)) {
        set_err("plans run the adjoint form of Rayleigh phase velocity (form %d)", form);
        return DAZI_ERR_BADARG;
    }
    if (!(minthk > 0.f) || !std::isfinite(minthk)) { set_err("minthk must be > 0"); return DAZI_ERR_BADARG; }
    std::lock_guard<std::mutex> lk(g_mu);
    int r;
    if ((r = ensure_context())) return r;
    Plan* P = new Plan;
    BatchIn B{ncols, node_off, depz, vs, vp, rho, per_off, periods, minthk, sen_off, ls_off};
    StageOut o;
    o.pv = pv; o.svs = sen_vs; o.svp = sen_vp; o.srh = sen_rho; o.lsen = lsen; o.status = status;
    if ((r = plan_create(B, o, form, tune != 0, (cudaStream_t)stream, *P))) {
        P->release();
        delete P;
        return r;
    }
    *plan = P;
    return 0;
}

int dazi_dk_plan_launch(void* plan, void* stream)
{
    if (!plan) { set_err("null plan"); return DAZI_ERR_BADARG; }
    Plan* P = static_cast<Plan*>(plan);
    int cur = -1;
    CK(cudaGetDevice(&cur));
    if (cur != P->device) CK(cudaSetDevice(P->device));
    CK(cudaGraphLaunch(P->exec, (cudaStream_t)stream));
    if (cur != P->device) CK(cudaSetDevice(cur));
    return 0;
}

int dazi_dk_plan_status(void* plan)
{
    if (!plan) { set_err("null plan"); return DAZI_ERR_BADARG; }
    Plan* P = static_cast<Plan*>(plan);
    int flag = 0;
    CK(cudaMemcpy(&flag, P->w.counters.as<unsigned long long>() + 1, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) { set_err("non-finite Lsen_Gsc value (degenerate layer: Vp <= Vs?)"); return DAZI_ERR_MODEL; }
    return 0;
}

int dazi_dk_plan_config(void* plan, int* root_block, int* adjoint_blocks_per_sm,
                        int* ti_blocks_per_sm, float* tuned_ms)
{
    if (!plan) { set_err("null plan"); return DAZI_ERR_BADARG; }
    const Plan* P = static_cast<const Plan*>(plan);
    if (root_block) *root_block = P->cfg.root_bt * 100 + P->cfg.root_minb;
    if (adjoint_blocks_per_sm) *adjoint_blocks_per_sm = P->cfg.adj_minb;
    if (ti_blocks_per_sm) *ti_blocks_per_sm = P->cfg.ti_minb;
    if (tuned_ms) for (int i = 0; i < 3; ++i) tuned_ms[i] = P->best_ms[i];
    return 0;
}

int dazi_dk_plan_destroy(void* plan)
{
    if (!plan) return 0;
    Plan* P = static_cast<Plan*>(plan);
    std::lock_guard<std::mutex> lk(g_mu);
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != P->device) cudaSetDevice(P->device);
    P->release();
    if (cur != P->device) cudaSetDevice(cur);
    delete P;
    return 0;
}

int dazi_dk_grows_dev(int nvx, int nvz, int nz, int kmaxRc, const float* vels, const double* sen_vsRc,
                      const double* sen_vpRc, const double* sen_rhoRc, const float* Lsen_Gsc,
                      long long nrays, const int* ray_period, const int* ray_id,
                      const long long* cell_off, const int* cell, const float* fdm,
                      const float* fdmc, const float* fdms, float ftol, long long cap, float* rw,
                      int* iw, int* col, long long* nnz_ray, long long* nnz_total, void* stream)
{
    if (nvx < 1 || nvz < 1 || nz < 2 || nz > NZMAX || kmaxRc < 1 || kmaxRc > NP || nrays < 0) {
        set_err("grid or ray count out of range");
        return DAZI_ERR_BADARG;
    }
    if (!vels || !sen_vsRc || !sen_vpRc || !sen_rhoRc || !ray_period || !ray_id || !cell_off ||
        !cell || !fdm || !nnz_ray || !nnz_total || (Lsen_Gsc && (!fdmc || !fdms)) ||
        (cap > 0 && (!rw || !iw || !col))) {
        set_err("null argument");
        return DAZI_ERR_BADARG;
    }
    if (!(ftol >= 0.f) || !std::isfinite(ftol)) { set_err("ftol must be >= 0"); return DAZI_ERR_BADARG; }
    *nnz_total = 0;
    if (nrays == 0) return 0;
    std::lock_guard<std::mutex> lk(g_mu);
    int r;
    if ((r = ensure_context())) return r;
    cudaStream_t st = (cudaStream_t)stream;
    if ((r = g_ctx.goff.ensure(sizeof(long long) * (nrays + 1))) || (r = g_ctx.gerr.ensure(sizeof(int) * 4)))
        return r;
    CK(cudaMemsetAsync(g_ctx.gerr.p, 0, sizeof(int), st));
    GrowsArgs a;
    a.nvx = nvx; a.nvz = nvz; a.nz = nz; a.K = kmaxRc;
    a.vels = vels; a.svs = sen_vsRc; a.svp = sen_vpRc; a.srh = sen_rhoRc; a.lsen = Lsen_Gsc;
    a.nrays = nrays; a.ray_period = ray_period; a.ray_id = ray_id; a.cell_off = cell_off; a.cell = cell;
    a.fdm = fdm; a.fdmc = fdmc; a.fdms = fdms; a.ftol = ftol;
    a.nnz_ray = nnz_ray; a.off = g_ctx.goff.as<long long>();
    a.rw = rw; a.iw = iw; a.col = col; a.err = g_ctx.gerr.as<int>();
    const unsigned nb = (unsigned)((nrays * 32 + 127) / 128);
    grows_kernel<false><<<nb, 128, 0, st>>>(a);
    CK(cudaGetLastError());
    size_t tb = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, nnz_ray, g_ctx.goff.as<long long>(), (int)nrays, st));
    if ((r = g_ctx.gtmp.ensure(tb + 16))) return r;
    CK(cub::DeviceScan::ExclusiveSum(g_ctx.gtmp.p, tb, nnz_ray, g_ctx.goff.as<long long>(), (int)nrays, st));
    long long last[2] = {0, 0};
    int herr = 0;
    CK(cudaMemcpyAsync(&last[0], g_ctx.goff.as<long long>() + nrays - 1, sizeof(long long), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&last[1], nnz_ray + nrays - 1, sizeof(long long), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&herr, g_ctx.gerr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (herr) { set_err("invalid ray: period index, or cells not ascending inside the grid"); return DAZI_ERR_BADARG; }
    *nnz_total = last[0] + last[1];
    if (*nnz_total > cap) {
        set_err("%lld entries exceed the capacity %lld", *nnz_total, cap);
        return DAZI_ERR_LIMITS;
    }
    grows_kernel<true><<<nb, 128, 0, st>>>(a);
    CK(cudaGetLastError());
    return 0;
}

int dazi_dk_azimuthal_map_dev(int nx, int ny, int nz, int kmaxRc, const float* Lsen_Gsc,
                              const float* gcf, const float* gsf, const double* tRcV, float* cosRc,
                              float* sinRc, float* amp, float* amp_rel, float* angle, void* stream)
{
    if (nx < 3 || ny < 3 || nz < 2 || nz > NZMAX || kmaxRc < 1 || kmaxRc > NP) {
        set_err("grid out of range");
        return DAZI_ERR_BADARG;
    }
    if (!Lsen_Gsc || !gcf || !gsf || !tRcV || !cosRc || !sinRc || !amp || !amp_rel || !angle) {
        set_err("null argument");
        return DAZI_ERR_BADARG;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    int r;
    if ((r = ensure_context())) return r;
    AzimapArgs a;
    a.nvx = nx - 2; a.nvz = ny - 2; a.nz = nz; a.K = kmaxRc;
    a.lsen = Lsen_Gsc; a.gc = gcf; a.gs = gsf; a.ciso = tRcV;
    a.cosr = cosRc; a.sinr = sinRc; a.amp = amp; a.rela = amp_rel; a.ang = angle;
    const long long n = (long long)a.nvx * a.nvz * kmaxRc;
    azimap_kernel<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(a);
    CK(cudaGetLastError());
    return 0;
}

const char* dazi_dk_last_error(void) { return g_err; }

int dazi_dk_version(void) { return 100; }

void dazi_dk_finalize(void)
{
    lsmr_release();
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx.ready) return;
    DBuf* all[] = {&g_ctx.vel, &g_ctx.vp, &g_ctx.rho, &g_ctx.per, &g_ctx.depz, &g_ctx.pv,
                   &g_ctx.svs, &g_ctx.svp, &g_ctx.srh, &g_ctx.status, &g_ctx.geo,
                   &g_ctx.cscratch, &g_ctx.w.croot, &g_ctx.w.crootb, &g_ctx.w.counters, &g_ctx.w.adjscr, &g_ctx.w.adjord,
                   &g_ctx.w.tiscr, &g_ctx.w.tiord, &g_ctx.lsen, &g_ctx.w.keys, &g_ctx.w.keys2, &g_ctx.w.cidx, &g_ctx.w.cidx2,
                   &g_ctx.w.rmaxb, &g_ctx.w.trecs, &g_ctx.w.ttasks, &g_ctx.w.tlbase, &g_ctx.w.ttbase,
                   &g_ctx.w.cubtmp, &g_ctx.w.tflat, &g_ctx.w.tld, &g_ctx.w.tti, &g_ctx.w.tsp, &g_ctx.w.tch, &g_ctx.w.tmeta,
                   &g_ctx.w.ttasklist, &g_ctx.cbufoff, &g_ctx.bnode, &g_ctx.bper, &g_ctx.bdep,
                   &g_ctx.bvs, &g_ctx.bvp, &g_ctx.brho, &g_ctx.bperiods, &g_ctx.bsenoff,
                   &g_ctx.blsoff, &g_ctx.bpv, &g_ctx.bsvs, &g_ctx.bsvp, &g_ctx.bsrh, &g_ctx.blsen,
                   &g_ctx.bstatus, &g_ctx.goff, &g_ctx.gtmp, &g_ctx.gerr};
    for (DBuf* b : all) b->release();
    if (g_ctx.outs_ready) cudaEventDestroy(g_ctx.outs_ready);
    if (g_ctx.cstream) cudaStreamDestroy(g_ctx.cstream);
    if (g_ctx.stream) cudaStreamDestroy(g_ctx.stream);
    g_ctx = Context();
}

}  // extern "C"
