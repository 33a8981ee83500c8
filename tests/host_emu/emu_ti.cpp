// TEST INFRASTRUCTURE ONLY: the Gc/Gs path of the library (table build of
// k_prep.cu, per-(column, period) sweep of k_ti.cu) compiled as host code
// and driven in the order the library drives it (build_tables, run_tables
// in csrc/capi.cu: columns sorted by (refined layers, periods), 32-column
// tiles, one task per (tile, period), one lane per column).  Used by
// tests/test_host_emu_ti.py to check the device arithmetic against the
// oracle on the CPU; the shipped library never uses it.
#include "emu_shim.h"
#include <numeric>
#include <vector>
#include "../../dazi_current_release_b200/csrc/k_prep.cu"
#include "../../dazi_current_release_b200/csrc/k_ti.cu"
using namespace dk;

// Ragged batch (CSR layout of dazi_dk_batch) with given phase velocities pv;
// writes lsen in the batch layout.  Returns 0, -1 for an invalid column,
// -2 for a non-finite Lsen value.
extern "C" int emu_ti_batch(long long ncols, const long long* node_off, const float* depz,
                            const float* vs, const long long* per_off, const double* periods,
                            float minthk, const double* pv, const long long* ls_off, float* lsen)
{
    ColSrc src;
    src.ragged = true; src.ncol = 0; src.col0 = 0;
    src.vel = vs; src.vp = nullptr; src.rho = nullptr; src.depz = depz;
    src.node_off = node_off; src.per_off = per_off; src.nz = 0; src.K = 0; src.minthk = minthk;
    std::vector<unsigned> keys(ncols);
    std::vector<int> colidx(ncols), rmax(ncols);
    int err = 0;
    for (long long c = 0; c < ncols; ++c) prep_count_one(src, c, keys.data(), colidx.data(), rmax.data(), &err);
    if (err) return -1;
    // stable descending order, as the library's radix sort of the keys
    std::vector<int> sorted(ncols);
    std::iota(sorted.begin(), sorted.end(), 0);
    std::stable_sort(sorted.begin(), sorted.end(), [&](int a, int b) { return keys[a] > keys[b]; });
    const long long ntiles = (ncols + TILE - 1) / TILE;
    std::vector<long long> lbase(ntiles), tbase(ntiles), trec(ntiles), ttask(ntiles);
    int maxr = 1;
    for (long long t = 0; t < ntiles; ++t) {
        int rm = 0, km = 0;
        for (int l = 0; l < TILE && t * TILE + l < ncols; ++l) {
            const int c = sorted[t * TILE + l];
            rm = std::max(rm, rmax[c]);
            km = std::max(km, src.col_K(c));
        }
        trec[t] = (long long)rm * TILE;
        ttask[t] = km;
        maxr = std::max(maxr, rm);
    }
    long long nrec = 0, ntask = 0;
    for (long long t = 0; t < ntiles; ++t) {
        lbase[t] = nrec; nrec += trec[t];
        tbase[t] = ntask; ntask += ttask[t];
    }
    std::vector<int2> tasks(ntask);
    for (long long t = 0; t < ntiles; ++t)
        for (long long k = 0; k < ttask[t]; ++k) tasks[tbase[t] + k] = make_int2((int)t, (int)k);
    std::vector<float4> flat(nrec);
    std::vector<LayerD> ld(nrec);
    std::vector<TiRec> ti(nrec);
    std::vector<SpRec> sp(nrec);
    std::vector<ChainRec> ch(nrec);
    std::vector<ColMeta> meta(ncols);
    Tables T;
    T.flat = flat.data(); T.ld = ld.data(); T.ti = ti.data(); T.sp = sp.data(); T.ch = ch.data();
    T.meta = meta.data(); T.tile_lbase = lbase.data(); T.tasks = tasks.data();
    T.ntasks = ntask; T.ncols = ncols; T.pv_sk = 1; T.sen_sk = 1; T.ls_sk = 1;
    PrepOut po{nullptr, ls_off, nullptr};
    for (long long s = 0; s < ncols; ++s) prep_build_one(src, po, T, sorted.data(), tbase.data(), s);
    std::vector<double> scratch((size_t)maxr * TI_SCR_Q * TILE);
    unsigned queue = 0;
    int errflag = 0;
    TiArgs a;
    a.T = T; a.periods = periods; a.pv = pv; a.lsen = lsen; a.scratch = scratch.data();
    a.scr_layers = maxr; a.queue = &queue; a.errflag = &errflag;
    for (long long task = 0; task < ntask; ++task)
        for (int lane = 0; lane < TILE; ++lane) ti_task(a, task, lane, scratch.data() + lane);
    return errflag ? -2 : 0;
}
