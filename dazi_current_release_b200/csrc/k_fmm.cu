// Host side of the traveltime solver (fmm_device.cuh): the propagation
// grid, the per-instance layout and ri*sin tables, the workspace and the
// C-ABI entries dazi_fmm_batch, dazi_fmm_batch_dev and dazi_fmm_times.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/dazi_dk.h"
#include "fmm_device.cuh"

namespace dk {
void set_last_error(const char* msg);
}

namespace {

using namespace dk::fmm;

#define FK(call)                                                                  \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) {                                                  \
            char m_[200];                                                         \
            snprintf(m_, sizeof m_, "FMM: CUDA error %s (%s)", cudaGetErrorString(e_), #call); \
            dk::set_last_error(m_);                                               \
            return DAZI_ERR_CUDA;                                                 \
        }                                                                         \
    } while (0)

int fail(int code, const char* msg)
{
    dk::set_last_error(msg);
    return code;
}

// grow-only device buffer
struct FBuf {
    void* p = nullptr;
    size_t n = 0;
    int ensure(size_t bytes)
    {
        if (bytes <= n) return 0;
        if (p) cudaFree(p);
        p = nullptr; n = 0;
        if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
            cudaGetLastError();
            return fail(DAZI_ERR_NOMEM, "FMM: device allocation failed");
        }
        n = bytes;
        return 0;
    }
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

struct FWork {
    FBuf velv, veln, slow, inst, risti_c, risti_r, sin_rcx, wnode, wrnode, wvr, wsr, wh, ctl;
    FBuf pv, rcx, rcz, times, ttn, scx, scz, per, off;   // copies of host inputs
};

std::mutex g_fmm_mu;
FWork g_fmm;

// The whole batch on `st`: maps -> velv -> coarse grids, instances on a
// persistent grid of warps, receivers; inputs pv, rcx, rcz and outputs
// times, ttn in device memory, the instance tables from the host.
int run_fmm(const dazi_fmm_params& p, const double* pv, int nper, int ninst, const int* per,
            const float* scx, const float* scz, const long long* rc_off, const float* rcx_host,
            const float* rcx, const float* rcz, float* times, float* ttn, cudaStream_t st)
{
    FWork& W = g_fmm;
    const FGrid g = grid_of(p);
    std::vector<FInst> inst;
    std::vector<float> risti_r;
    long long wr = 1;
    int wh = 1;
    int r;
    const char* msg = "";
    if ((r = layout(p, g, nper, ninst, per, scx, scz, rc_off, inst, risti_r, wr, wh, &msg)))
        return fail(r, msg);
    const long long nrc = rc_off[ninst];
    std::vector<float> risti_c(g.nnx), sin_rcx(nrc > 0 ? nrc : 1);
    for (int ix = 1; ix <= g.nnx; ++ix) risti_c[ix - 1] = p.earth * sinf(g.gox + (float)(ix - 1) * g.dnx);
    for (long long q = 0; q < nrc; ++q) sin_rcx[q] = sinf(rcx_host[q]);
    // persistent grid: as many warps as fit, at most one per instance
    int dev = 0, sms = 0, per_sm = 0;
    FK(cudaGetDevice(&dev));
    FK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    FK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fmm_kernel, 32 * kWarpsPerBlock, 0));
    if (per_sm < 1) per_sm = 1;
    long long nblk = (long long)sms * per_sm;
    const long long need = (ninst + kWarpsPerBlock - 1) / kWarpsPerBlock;
    if (nblk > need) nblk = need;
    if (nblk < 1) nblk = 1;
    const long long slots = nblk * kWarpsPerBlock;
    const long long nc = (long long)g.nnx * g.nnz;
    const long long nv = (long long)p.nx * p.ny;
    if ((r = W.velv.ensure(sizeof(float) * nv * nper)) || (r = W.veln.ensure(sizeof(float) * nc * nper)) ||
        (r = W.slow.ensure(sizeof(float) * nc * nper)) ||
        (r = W.inst.ensure(sizeof(FInst) * inst.size())) || (r = W.risti_c.ensure(sizeof(float) * g.nnx)) ||
        (r = W.risti_r.ensure(sizeof(float) * risti_r.size())) ||
        (r = W.sin_rcx.ensure(sizeof(float) * sin_rcx.size())) ||
        (r = W.wnode.ensure(sizeof(Node) * nc * slots)) || (r = W.wrnode.ensure(sizeof(Node) * wr * slots)) ||
        (r = W.wvr.ensure(sizeof(float) * wr * slots)) || (r = W.wsr.ensure(sizeof(float) * wr * slots)) ||
        (r = W.wh.ensure(sizeof(HeapE) * (size_t)wh * slots)) || (r = W.ctl.ensure(16)))
        return r;
    FK(cudaMemcpyAsync(W.inst.p, inst.data(), sizeof(FInst) * inst.size(), cudaMemcpyHostToDevice, st));
    FK(cudaMemcpyAsync(W.risti_c.p, risti_c.data(), sizeof(float) * g.nnx, cudaMemcpyHostToDevice, st));
    FK(cudaMemcpyAsync(W.risti_r.p, risti_r.data(), sizeof(float) * risti_r.size(), cudaMemcpyHostToDevice, st));
    FK(cudaMemcpyAsync(W.sin_rcx.p, sin_rcx.data(), sizeof(float) * sin_rcx.size(), cudaMemcpyHostToDevice, st));
    FK(cudaMemsetAsync(W.ctl.p, 0, 16, st));
    const int bt = 256;
    fmm_velv_kernel<<<(unsigned)((nv * nper + bt - 1) / bt), bt, 0, st>>>(pv, p.nx, p.ny, nper, W.velv.as<float>());
    FK(cudaGetLastError());
    fmm_gridder_kernel<<<(unsigned)((nc * nper + bt - 1) / bt), bt, 0, st>>>(W.velv.as<float>(), g.nvx, g.nvz,
                                                                             p.gdx, p.gdz, nper, W.veln.as<float>(),
                                                                             W.slow.as<float>());
    FK(cudaGetLastError());
    FArgs a;
    a.ninst = ninst; a.inst = W.inst.as<FInst>();
    a.nnx = g.nnx; a.nnz = g.nnz; a.nvx = g.nvx; a.nvz = g.nvz; a.gdx = p.gdx; a.gdz = p.gdz;
    a.sgdl = p.sgdl; a.fom = p.fom; a.asgr = p.asgr;
    a.gox = g.gox; a.goz = g.goz; a.dnx = g.dnx; a.dnz = g.dnz; a.drnx = g.drnx; a.drnz = g.drnz;
    a.earth = p.earth; a.dpl = g.dpl;
    a.velv = W.velv.as<float>(); a.veln = W.veln.as<float>(); a.slow = W.slow.as<float>();
    a.risti_c = W.risti_c.as<float>(); a.risti_r = W.risti_r.as<float>();
    a.rcx = rcx; a.rcz = rcz; a.sin_rcx = W.sin_rcx.as<float>();
    a.times = times; a.ttn_out = ttn;
    a.w_node = W.wnode.as<Node>(); a.w_rnode = W.wrnode.as<Node>(); a.w_vr = W.wvr.as<float>(); a.w_sr = W.wsr.as<float>();
    a.w_heap = W.wh.as<HeapE>();
    a.wc = nc; a.wr = wr; a.wh = wh;
    a.queue = W.ctl.as<unsigned>(); a.err = W.ctl.as<int>() + 1; a.err_inst = W.ctl.as<int>() + 2;
    fmm_kernel<<<(unsigned)nblk, 32 * kWarpsPerBlock, 0, st>>>(a);
    FK(cudaGetLastError());
    int herr[2] = {0, 0};
    FK(cudaMemcpyAsync(herr, W.ctl.as<int>() + 1, sizeof(herr), cudaMemcpyDeviceToHost, st));
    FK(cudaStreamSynchronize(st));
    if (herr[0]) {
        char m[256];
        snprintf(m, sizeof m, "FMM: instance %d: %s", herr[1],
                 herr[0] == kErrOutside ? "source or receiver outside the grid"
                 : herr[0] == kErrBand  ? "narrow band beyond snb of the nodes"
                 : herr[0] == kErrNoSol ? "node without an upwind solution"
                 : herr[0] == kErrNoBand
                     ? "source in the last cell before the right or bottom side: the refined sweep "
                       "stops before it reaches a coarse node (the reference's field is undefined)"
                     : "marching did not end");
        return fail(herr[0] == kErrBand ? DAZI_ERR_LIMITS : herr[0] == kErrOutside ? DAZI_ERR_BADARG
                                                                                   : DAZI_ERR_MODEL, m);
    }
    return 0;
}

int check_batch(const dazi_fmm_params* p, const void* pv, int nper, int ninst, const void* per,
                const void* scx, const void* scz, const void* rc_off, const void* rcx, const void* rcz,
                const void* times)
{
    int r;
    const char* msg = "";
    if ((r = check_params(p, &msg))) return fail(r, msg);
    if (nper < 1 || ninst < 0 || !pv || !rc_off || (ninst > 0 && (!per || !scx || !scz)))
        return fail(DAZI_ERR_BADARG, "FMM: missing input");
    (void)rcx; (void)rcz; (void)times;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return fail(DAZI_ERR_NODEVICE, "FMM: no CUDA device");
    }
    return 0;
}

}  // namespace

extern "C" {

void dazi_fmm_default_params(dazi_fmm_params* p, int nx, int ny, float goxd, float gozd, float dvxd,
                             float dvzd)
{
    if (!p) return;
    p->nx = nx; p->ny = ny;
    p->goxd = goxd; p->gozd = gozd; p->dvxd = dvxd; p->dvzd = dvzd;
    p->gdx = 5; p->gdz = 5;
    p->asgr = 1; p->sgdl = 8; p->sgs = 8;
    p->fom = 1;
    p->snb = 0.5f;
    p->earth = 6371.0f;
}

int dazi_fmm_batch(const dazi_fmm_params* p, const double* pv, int nper, int ninst, const int* inst_period,
                   const float* scx, const float* scz, const long long* rc_off, const float* rcx,
                   const float* rcz, float* times, float* ttn)
{
    int r;
    if ((r = check_batch(p, pv, nper, ninst, inst_period, scx, scz, rc_off, rcx, rcz, times))) return r;
    std::lock_guard<std::mutex> lk(g_fmm_mu);
    FWork& W = g_fmm;
    const long long nrc = rc_off[ninst];
    if (nrc > 0 && (!rcx || !rcz || !times)) return fail(DAZI_ERR_BADARG, "FMM: missing receivers");
    const long long nv = (long long)p->nx * p->ny;
    const long long nc = (long long)((p->nx - 3) * p->gdx + 1) * ((p->ny - 3) * p->gdz + 1);
    if ((r = W.pv.ensure(sizeof(double) * nv * nper)) || (r = W.rcx.ensure(sizeof(float) * (nrc + 1))) ||
        (r = W.rcz.ensure(sizeof(float) * (nrc + 1))) || (r = W.times.ensure(sizeof(float) * (nrc + 1))) ||
        (ttn && (r = W.ttn.ensure(sizeof(float) * nc * (ninst > 0 ? ninst : 1)))))
        return r;
    cudaStream_t st = 0;
    FK(cudaMemcpyAsync(W.pv.p, pv, sizeof(double) * nv * nper, cudaMemcpyHostToDevice, st));
    if (nrc > 0) {
        FK(cudaMemcpyAsync(W.rcx.p, rcx, sizeof(float) * nrc, cudaMemcpyHostToDevice, st));
        FK(cudaMemcpyAsync(W.rcz.p, rcz, sizeof(float) * nrc, cudaMemcpyHostToDevice, st));
    }
    if (ninst == 0) return 0;
    if ((r = run_fmm(*p, W.pv.as<double>(), nper, ninst, inst_period, scx, scz, rc_off, rcx, W.rcx.as<float>(),
                     W.rcz.as<float>(), W.times.as<float>(), ttn ? W.ttn.as<float>() : nullptr, st)))
        return r;
    if (nrc > 0) FK(cudaMemcpyAsync(times, W.times.p, sizeof(float) * nrc, cudaMemcpyDeviceToHost, st));
    if (ttn) FK(cudaMemcpyAsync(ttn, W.ttn.p, sizeof(float) * nc * ninst, cudaMemcpyDeviceToHost, st));
    FK(cudaStreamSynchronize(st));
    return 0;
}

int dazi_fmm_batch_dev(const dazi_fmm_params* p, const double* pv, int nper, int ninst,
                       const int* inst_period, const float* scx, const float* scz, const long long* rc_off,
                       const float* rcx, const float* rcz, float* times, float* ttn, void* stream)
{
    int r;
    if ((r = check_batch(p, pv, nper, ninst, inst_period, scx, scz, rc_off, rcx, rcz, times))) return r;
    std::lock_guard<std::mutex> lk(g_fmm_mu);
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<int> per(ninst > 0 ? ninst : 1);
    std::vector<float> hx(ninst > 0 ? ninst : 1), hz(ninst > 0 ? ninst : 1);
    std::vector<long long> off(ninst + 1);
    FK(cudaMemcpyAsync(off.data(), rc_off, sizeof(long long) * (ninst + 1), cudaMemcpyDeviceToHost, st));
    if (ninst > 0) {
        FK(cudaMemcpyAsync(per.data(), inst_period, sizeof(int) * ninst, cudaMemcpyDeviceToHost, st));
        FK(cudaMemcpyAsync(hx.data(), scx, sizeof(float) * ninst, cudaMemcpyDeviceToHost, st));
        FK(cudaMemcpyAsync(hz.data(), scz, sizeof(float) * ninst, cudaMemcpyDeviceToHost, st));
    }
    FK(cudaStreamSynchronize(st));
    const long long nrc = off[ninst];
    if (nrc > 0 && (!rcx || !rcz || !times)) return fail(DAZI_ERR_BADARG, "FMM: missing receivers");
    std::vector<float> hrx(nrc > 0 ? nrc : 1);
    if (nrc > 0) {
        FK(cudaMemcpyAsync(hrx.data(), rcx, sizeof(float) * nrc, cudaMemcpyDeviceToHost, st));
        FK(cudaStreamSynchronize(st));
    }
    if (ninst == 0) return 0;
    return run_fmm(*p, pv, nper, ninst, per.data(), hx.data(), hz.data(), off.data(), hrx.data(), rcx, rcz,
                   times, ttn, st);
}

int dazi_fmm_times(const int* nx, const int* ny, const int* kmax, const int* nsrc, const int* nrc,
                   const int* nper, const double* pv, const int* periods, const int* nsrc1, const int* nrc1,
                   const float* scxf, const float* sczf, const float* rcxf, const float* rczf,
                   const float* goxd, const float* gozd, const float* dvxd, const float* dvzd,
                   const long long* dall, float* dsurf)
{
    if (!nx || !ny || !kmax || !nsrc || !nrc || !nper || !pv || !periods || !nsrc1 || !nrc1 || !scxf ||
        !sczf || !rcxf || !rczf || !goxd || !gozd || !dvxd || !dvzd || !dall || !dsurf)
        return fail(DAZI_ERR_BADARG, "FMM: NULL argument");
    const int K = *kmax, NS = *nsrc, NR = *nrc;
    if (K < 1 || NS < 1 || NR < 1) return fail(DAZI_ERR_BADARG, "FMM: empty tables");
    dazi_fmm_params p;
    dazi_fmm_default_params(&p, *nx, *ny, *goxd, *gozd, *dvxd, *dvzd);
    // instances in countsurf order (FmmBackend.f90:64-72)
    std::vector<int> per;
    std::vector<float> sx, sz, rx, rz;
    std::vector<long long> off(1, 0);
    for (int k = 0; k < K; ++k) {
        if (nsrc1[k] < 0 || nsrc1[k] > NS) return fail(DAZI_ERR_BADARG, "FMM: nsrc1 outside [0, nsrc]");
        for (int s = 0; s < nsrc1[k]; ++s) {
            const long long sk = (long long)k * NS + s;
            const int n = nrc1[sk];
            if (n < 0 || n > NR) return fail(DAZI_ERR_BADARG, "FMM: nrc1 outside [0, nrc]");
            per.push_back(periods[sk] - 1);
            sx.push_back(scxf[sk]);
            sz.push_back(sczf[sk]);
            for (int q = 0; q < n; ++q) {
                const long long i = ((long long)k * NS + s) * NR + q;
                rx.push_back(rcxf[i]);
                rz.push_back(rczf[i]);
            }
            off.push_back(off.back() + n);
        }
    }
    if (off.back() != *dall) return fail(DAZI_ERR_BADARG, "FMM: dall differs from the receiver count");
    return dazi_fmm_batch(&p, pv, *nper, (int)per.size(), per.data(), sx.data(), sz.data(), off.data(),
                          rx.data(), rz.data(), dsurf, nullptr);
}

}  // extern "C"
