// TEST INFRASTRUCTURE ONLY: the table build (k_prep.cu), the root search
// (root_kernel, k_plain.cu), the adjoint sweeps (k_adjoint.cu) and the
// Gc/Gs sweep (k_ti.cu) and the traveltime solver (fmm_device.cuh) of the
// library
// compiled as host code and driven in the order the library drives them
// (build_tables, run_tables in csrc/capi.cu: columns sorted by (refined
// layers, periods), 32-column tiles, one task per (tile, period), one lane
// per column; one root-search thread per column).  Used by the
// tests/test_host_emu_*.py suites to check the device arithmetic against
// the oracle on the CPU; the shipped library never uses it.
#include "emu_shim.h"
#include <algorithm>
#include <numeric>
#include <vector>
namespace dk { alignas(16) unsigned char smem_raw[1 << 16]; }
#include "../../dazi_current_release_b200/csrc/k_prep.cu"
#include "../../dazi_current_release_b200/csrc/k_plain.cu"
#include "../../dazi_current_release_b200/csrc/k_ti.cu"
#include "../../dazi_current_release_b200/csrc/k_adjoint.cu"
#include "../../dazi_current_release_b200/csrc/fmm_device.cuh"
using namespace dk;

namespace {

struct HostTables {
    std::vector<int> sorted;
    std::vector<long long> lbase, tbase, ttask;
    std::vector<int2> tasks;
    std::vector<float4> flat;
    std::vector<LayerD> ld;
    std::vector<TiRec> ti;
    std::vector<SpRec> sp;
    std::vector<ChainRec> ch;
    std::vector<ColMeta> meta;
    Tables T;
    int maxr = 1;
};

// build_tables (capi.cu) on the host.  Returns false for an invalid column.
bool build_host(const ColSrc& src, long long ncols, const PrepOut& po, HostTables& H)
{
    std::vector<unsigned> keys(ncols);
    std::vector<int> colidx(ncols), rmax(ncols);
    int err = 0;
    for (long long c = 0; c < ncols; ++c) prep_count_one(src, c, keys.data(), colidx.data(), rmax.data(), &err);
    if (err) return false;
    // stable descending order, as the library's radix sort of the keys
    H.sorted.resize(ncols);
    std::iota(H.sorted.begin(), H.sorted.end(), 0);
    std::stable_sort(H.sorted.begin(), H.sorted.end(), [&](int a, int b) { return keys[a] > keys[b]; });
    const long long ntiles = (ncols + TILE - 1) / TILE;
    H.lbase.resize(ntiles); H.tbase.resize(ntiles);
    std::vector<long long> trec(ntiles);
    std::vector<long long>& ttask = H.ttask;
    ttask.resize(ntiles);
    for (long long t = 0; t < ntiles; ++t) {
        int rm = 0, km = 0;
        for (int l = 0; l < TILE && t * TILE + l < ncols; ++l) {
            const int c = H.sorted[t * TILE + l];
            rm = std::max(rm, rmax[c]);
            km = std::max(km, src.col_K(c));
        }
        trec[t] = (long long)rm * TILE;
        ttask[t] = km;
        H.maxr = std::max(H.maxr, rm);
    }
    long long nrec = 0, ntask = 0;
    for (long long t = 0; t < ntiles; ++t) {
        H.lbase[t] = nrec; nrec += trec[t];
        H.tbase[t] = ntask; ntask += ttask[t];
    }
    H.tasks.resize(ntask);
    for (long long t = 0; t < ntiles; ++t)
        for (long long k = 0; k < ttask[t]; ++k) H.tasks[H.tbase[t] + k] = make_int2((int)t, (int)k);
    H.flat.resize(nrec); H.ld.resize(nrec); H.ti.resize(nrec); H.sp.resize(nrec); H.ch.resize(nrec);
    H.meta.resize(ncols);
    Tables& T = H.T;
    T.flat = H.flat.data(); T.ld = H.ld.data(); T.ti = H.ti.data(); T.sp = H.sp.data(); T.ch = H.ch.data();
    T.meta = H.meta.data(); T.tile_lbase = H.lbase.data(); T.tasks = H.tasks.data();
    T.ntasks = ntask; T.ncols = ncols; T.pv_sk = 1; T.sen_sk = 1; T.ls_sk = 1;
    for (long long s = 0; s < ncols; ++s) prep_build_one(src, po, T, H.sorted.data(), H.tbase.data(), s);
    return true;
}

ColSrc ragged_src(const long long* node_off, const float* depz, const float* vs,
                  const long long* per_off, float minthk, int ifunc = 2)
{
    ColSrc src;
    src.ragged = true; src.ncol = 0; src.col0 = 0;
    src.vel = vs; src.vp = nullptr; src.rho = nullptr; src.depz = depz;
    src.node_off = node_off; src.per_off = per_off; src.nz = 0; src.K = 0; src.minthk = minthk;
    src.ifunc = ifunc;
    return src;
}

}  // namespace

// Root search of a ragged batch (root_kernel, one thread per sorted
// column): pv[per_off[c] + k] (sngl(c), as the library writes it), status
// per column, the secular evaluations in *evals.  scan32 selects the FP32
// coarse scan; ifunc 1 (Love) / 2 (Rayleigh) and group select the
// root_kernel instantiation the library launches for that form; fast the
// Brent refinement (Rayleigh phase).
extern "C" int emu_root_batch(long long ncols, const long long* node_off, const float* depz,
                              const float* vs, const long long* per_off, const double* periods,
                              float minthk, int scan32, int ifunc, int group, int fast,
                              double* pv, int* status, long long* evals)
{
    if (ifunc != 1 && ifunc != 2) return -2;
    if (fast && (ifunc != 2 || group)) return -2;
    const ColSrc src = ragged_src(node_off, depz, vs, per_off, minthk, ifunc);
    HostTables H;
    PrepOut po{nullptr, nullptr, nullptr};
    if (!build_host(src, ncols, po, H)) return -1;
    unsigned long long counters[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    RootArgs a;
    a.T = H.T; a.periods = periods; a.tol = 1.0e-6; a.pv = pv; a.croot = nullptr;
    a.status = status; a.nevals = counters; a.scan32 = scan32;
    blockDim.x = 128;
    for (long long s = 0; s < ncols; ++s) {
        blockIdx.x = (unsigned)(s / 128);
        threadIdx.x = (unsigned)(s % 128);
        if (fast) root_kernel<128, 0, 2, false, true>(a);
        else if (ifunc == 1 && group) root_kernel<128, 0, 1, true>(a);
        else if (ifunc == 1) root_kernel<128, 0, 1, false>(a);
        else if (group) root_kernel<128, 0, 2, true>(a);
        else root_kernel<128, 0>(a);
    }
    *evals = (long long)counters[0];
    return 0;
}

// Ragged batch (CSR layout of dazi_dk_batch) with given phase velocities pv;
// writes lsen in the batch layout.  Returns 0, -1 for an invalid column,
// -2 for a non-finite Lsen value.
extern "C" int emu_ti_batch(long long ncols, const long long* node_off, const float* depz,
                            const float* vs, const long long* per_off, const double* periods,
                            float minthk, const double* pv, const long long* ls_off, float* lsen)
{
    const ColSrc src = ragged_src(node_off, depz, vs, per_off, minthk);
    HostTables H;
    PrepOut po{nullptr, ls_off, nullptr};
    if (!build_host(src, ncols, po, H)) return -1;
    std::vector<double> scratch((size_t)H.maxr * TI_SCR_Q * TILE);
    unsigned queue = 0;
    int errflag = 0;
    TiArgs a;
    a.T = H.T; a.periods = periods; a.pv = pv; a.lsen = lsen; a.scratch = scratch.data();
    a.scr_layers = H.maxr; a.queue = &queue; a.errflag = &errflag;
    // ti_order_kernel: per tile, the pairs in ascending key order (a
    // stable sort here; the device's counting sort may order equal keys
    // differently, which changes no result)
    std::vector<int> order((size_t)H.T.ntasks * TILE);
    a.order = order.data();
    for (long long t = 0; t < (long long)H.ttask.size(); ++t) {
        const int np = (int)H.ttask[t] * TILE;
        std::vector<int> pk(np);
        for (int p = 0; p < np; ++p) pk[p] = (ti_pair_key(a, t, p & 31, p >> 5) << 16) | p;
        std::stable_sort(pk.begin(), pk.end(), [](int x, int y) { return (x >> 16) < (y >> 16); });
        std::copy(pk.begin(), pk.end(), order.begin() + H.tbase[t] * TILE);
    }
    for (long long task = 0; task < H.T.ntasks; ++task)
        for (int lane = 0; lane < TILE; ++lane) ti_task(a, task, lane, scratch.data() + lane);
    return errflag ? -2 : 0;
}

// Adjoint form of a ragged batch (the root search with FP64 roots, then the
// adjoint sweep of every (column, period), as run_tables drives them):
// pv, status and the three kernels in the dazi_dk_batch layout (sen_off).
// ifunc 1 (Love) / 2 (Rayleigh); group selects group velocity.  A test may
// plant the group fallback (the second root search found no root): with
// drop_every > 0 every drop_every-th root at t1b is set to 0 before the
// sweep, and dropped[pv index] = 1 marks those (column, period) entries.
extern "C" int emu_adjoint_batch(long long ncols, const long long* node_off, const float* depz,
                                 const float* vs, const long long* per_off, const double* periods,
                                 float minthk, int ifunc, int group, int drop_every, int fast,
                                 double* pv, int* status, const long long* sen_off, double* svs,
                                 double* svp, double* srh, unsigned char* dropped)
{
    if (ifunc != 1 && ifunc != 2) return -2;
    if (fast && (ifunc != 2 || group)) return -2;
    const ColSrc src = ragged_src(node_off, depz, vs, per_off, minthk, ifunc);
    HostTables H;
    PrepOut po{sen_off, nullptr, nullptr};
    if (!build_host(src, ncols, po, H)) return -1;
    const size_t nroots = (size_t)H.T.ntasks * TILE;
    std::vector<double> croot(nroots, 0.0), crootb(nroots, 0.0);
    unsigned long long counters[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    RootArgs a;
    a.T = H.T; a.periods = periods; a.tol = 1.0e-6; a.pv = pv; a.croot = croot.data();
    a.croot_b = group ? crootb.data() : nullptr;
    a.status = status; a.nevals = counters; a.scan32 = 0;
    blockDim.x = 128;
    for (long long s = 0; s < ncols; ++s) {
        blockIdx.x = (unsigned)(s / 128);
        threadIdx.x = (unsigned)(s % 128);
        if (fast) root_kernel<128, 0, 2, false, true>(a);
        else if (ifunc == 1 && group) root_kernel<128, 0, 1, true>(a);
        else if (ifunc == 1) root_kernel<128, 0, 1, false>(a);
        else if (group) root_kernel<128, 0, 2, true>(a);
        else root_kernel<128, 0>(a);
    }
    for (long long task = 0; task < H.T.ntasks; ++task)
        for (int lane = 0; lane < TILE; ++lane) {
            const size_t i = (size_t)task * TILE + lane;
            const long long s = (long long)H.T.tasks[task].x * TILE + lane;
            const int k = H.T.tasks[task].y;
            if (!group || drop_every <= 0 || i % (size_t)drop_every != 0) continue;
            if (s >= H.T.ncols || k >= H.T.meta[s].K || !(croot[i] > 0.0)) continue;
            crootb[i] = 0.0;
            dropped[H.T.meta[s].pv_b + H.T.pv_sk * k] = 1;
        }
    std::vector<double> scratch((size_t)H.maxr * 6 * TILE);
    AdjArgs j;
    j.T = H.T; j.periods = periods; j.croot = croot.data(); j.sen_vs = svs; j.sen_vp = svp;
    j.sen_rho = srh; j.scratch = scratch.data(); j.scr_layers = H.maxr > 1 ? H.maxr - 1 : 1;
    j.queue = nullptr; j.croot_b = group ? crootb.data() : nullptr;
    // adj_order_kernel (Rayleigh phase velocity): per tile, the pairs in
    // ascending key order, as for the Gc/Gs sweep
    std::vector<int> order;
    if (ifunc == 2 && !group) {
        order.resize((size_t)H.T.ntasks * TILE);
        for (long long t = 0; t < (long long)H.ttask.size(); ++t) {
            const int np = (int)H.ttask[t] * TILE;
            std::vector<int> pk(np);
            for (int p = 0; p < np; ++p) pk[p] = (adj_pair_key(j, t, p & 31, p >> 5) << 16) | p;
            std::stable_sort(pk.begin(), pk.end(), [](int x, int y) { return (x >> 16) < (y >> 16); });
            std::copy(pk.begin(), pk.end(), order.begin() + H.tbase[t] * TILE);
        }
        j.order = order.data();
    }
    for (long long task = 0; task < H.T.ntasks; ++task)
        for (int lane = 0; lane < TILE; ++lane) {
            double* scr = scratch.data() + lane;
            if (ifunc == 1 && group) adjoint_love_task<true>(j, task, lane, scr);
            else if (ifunc == 1) adjoint_love_task<false>(j, task, lane, scr);
            else if (group) adjoint_rayleigh_task<true>(j, task, lane, scr);
            else adjoint_rayleigh_task<false>(j, task, lane, scr);
        }
    return 0;
}

// Traveltimes of a batch (dazi_fmm_batch's inputs) through the library's
// traveltime device code, driven as run_fmm (k_fmm.cu) drives it: the maps'
// vertex values and coarse grids by the gridding kernels' thread bodies,
// then per instance the lane-shared steps for lanes 0..31 in turn around
// the marching's phases in the order the GPU's warps run them
// (travel_four: after each pop the four neighbours' times, then their
// commits), one workspace slot.  times and, when not NULL, the
// coarse fields ttn (as dazi_fmm_batch).  Returns 0, or the library's error
// code with *code the instance's error.
extern "C" int emu_fmm_batch(const dazi_fmm_params* p, const double* pv, int nper, int ninst,
                             const int* per, const float* scx, const float* scz,
                             const long long* rc_off, const float* rcx, const float* rcz,
                             float* times, float* ttn, int* code)
{
    using namespace dk::fmm;
    const char* msg = "";
    int r;
    if ((r = check_params(p, &msg))) return r;
    const FGrid g = grid_of(*p);
    std::vector<FInst> inst;
    std::vector<float> risti_r;
    long long wr = 1;
    int wh = 1;
    if ((r = layout(*p, g, nper, ninst, per, scx, scz, rc_off, inst, risti_r, wr, wh, &msg))) return r;
    const long long nrc = rc_off[ninst], nc = (long long)g.nnx * g.nnz, nv = (long long)p->nx * p->ny;
    std::vector<float> risti_c(g.nnx), sin_rcx(nrc > 0 ? nrc : 1);
    for (int ix = 1; ix <= g.nnx; ++ix) risti_c[ix - 1] = p->earth * sinf(g.gox + (float)(ix - 1) * g.dnx);
    for (long long q = 0; q < nrc; ++q) sin_rcx[q] = sinf(rcx[q]);
    std::vector<float> velv(nv * nper), veln(nc * nper), slow(nc * nper);
    blockDim.x = 256;
    for (long long t = 0; t < nv * nper; ++t) {
        blockIdx.x = (unsigned)(t / 256); threadIdx.x = (unsigned)(t % 256);
        fmm_velv_kernel(pv, p->nx, p->ny, nper, velv.data());
    }
    for (long long t = 0; t < nc * nper; ++t) {
        blockIdx.x = (unsigned)(t / 256); threadIdx.x = (unsigned)(t % 256);
        fmm_gridder_kernel(velv.data(), g.nvx, g.nvz, p->gdx, p->gdz, nper, veln.data(), slow.data());
    }
    std::vector<Node> wnode(nc), wrnode(wr);
    std::vector<float> wvr(wr), wsr(wr);
    std::vector<int> ctl(4, 0);
    std::vector<HeapE> hglobal(wh), hshared(kHeapShared);
    const Heap heap{hshared.data(), hglobal.data()};
    FArgs a;
    a.ninst = ninst; a.inst = inst.data();
    a.nnx = g.nnx; a.nnz = g.nnz; a.nvx = g.nvx; a.nvz = g.nvz; a.gdx = p->gdx; a.gdz = p->gdz;
    a.sgdl = p->sgdl; a.fom = p->fom; a.asgr = p->asgr;
    a.gox = g.gox; a.goz = g.goz; a.dnx = g.dnx; a.dnz = g.dnz; a.drnx = g.drnx; a.drnz = g.drnz;
    a.earth = p->earth; a.dpl = g.dpl;
    a.velv = velv.data(); a.veln = veln.data(); a.slow = slow.data(); a.risti_c = risti_c.data(); a.risti_r = risti_r.data();
    a.rcx = rcx; a.rcz = rcz; a.sin_rcx = sin_rcx.data(); a.times = times; a.ttn_out = ttn;
    a.w_node = wnode.data(); a.w_rnode = wrnode.data(); a.w_vr = wvr.data(); a.w_sr = wsr.data();
    a.w_heap = hglobal.data(); a.wc = nc; a.wr = wr; a.wh = wh;
    a.queue = nullptr; a.err = &ctl[1]; a.err_inst = &ctl[2];
    for (int s = 0; s < ninst; ++s) {
        const FInst& I = inst[s];
        FField C, R;
        inst_fields(a, I, 0, C, R);
        const Box B = inst_box(I);
        for (int lane = 0; lane < 32; ++lane) step_init(a, I, C, R, lane, 32);
        if (p->asgr) {
            if ((r = travel_four(R, 1, I.scx, I.scz, B, heap, I.cap))) {
                *code = r;
                return -1;
            }
            for (int lane = 0; lane < 32; ++lane) step_map(a, I, C, R, lane, 32);
            for (int base = 0; base < box_nodes(I); base += 32 * 32) {
                unsigned mask[32];
                for (int lane = 0; lane < 32; ++lane) mask[lane] = step_band_decide(a, I, C, base, lane, 32);
                for (int lane = 0; lane < 32; ++lane) step_band_write(a, I, C, base, lane, 32, mask[lane]);
            }
            r = travel_four(C, 2, I.scx, I.scz, B, heap, I.cap);
        } else {
            r = travel_four(C, 0, I.scx, I.scz, B, heap, I.cap);
        }
        if (r) { *code = r; return -1; }
        for (int lane = 0; lane < 32; ++lane) step_receivers(a, I, C, s, lane, 32);
        if (ctl[1]) { *code = ctl[1]; return -1; }
    }
    return 0;
}
