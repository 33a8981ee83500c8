// Preparation of the per-layer tables (dk_table.cuh) for a call.
//
// Per column: node values (Vs, and Vp/rho either given or from the Brocher
// relations, DepthKernel1D.f90:187-200), the layer split
// (refineGrid2LayerMdl, CalSurfG.f90:2490-2549), surfdisp96's Earth
// flattening (sphere, surfdisp96.f:480-547, R = 6370 km) and tregn96's own
// flattening and sphericity factors (sphere_tdisp96 / bldsph,
// tregn96.f:774-841, 1301-1383, R = 6371 / 6370 km).  The arithmetic is the
// same as build_geometry + flat_layer (dk_model.cuh), streamed layer by layer
// so that no per-column geometry array is kept.
#include "dk_table.cuh"
#include "dk_kernels.cuh"

namespace dk {

__device__ __forceinline__ int nsub_of(float thk, float minthk0)
{
    const float minthk = __fdiv_rn(thk, minthk0);
    return (int)__fdiv_rn(__fadd_rn(thk, 1.0e-4f), minthk) + 1;
}

// rmax of column c, validation and the sort key.
__device__ __forceinline__ void prep_count_one(const ColSrc& src, long long c, unsigned* keys, int* colidx,
                               int* rmax_out, int* err)
{
    const int nz = src.col_nz(c), K = src.col_K(c);
    int r = 0, bad = 0;
    if (nz < 2 || nz > NZMAX) bad |= 1;
    if (K < 1 || K > NP) bad |= 2;
    if (!bad) {
        for (int i = 0; i < nz - 1; ++i) {
            const float d0 = src.dep(c, i), d1 = src.dep(c, i + 1);
            if (!(d1 > d0)) { bad |= 4; break; }
            r += nsub_of(__fsub_rn(d1, d0), src.minthk);
        }
        r += 1;
        if (r > NL) bad |= 8;
        for (int i = 0; i < nz && !bad; ++i) {
            float vs, vp, rh;
            src.node(c, i, vs, vp, rh);
            if (!(vs > 0.f) || !(vp > 0.f) || !(rh > 0.f) || !isfinite(vs) || !isfinite(vp) || !isfinite(rh))
                bad |= 16;
        }
    }
    if (bad) { atomicOr(err, bad); r = 1; }
    rmax_out[c] = r;
    keys[c] = ((unsigned)r << 8) | (unsigned)(K > 255 ? 255 : K);
    colidx[c] = (int)c;
}

__global__ void prep_count_kernel(ColSrc src, long long ncols, unsigned* keys, int* colidx,
                                  int* rmax_out, int* err)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncols) return;
    prep_count_one(src, c, keys, colidx, rmax_out, err);
}

// Per tile (after sorting): its layer count, period count and record count.
__global__ void prep_tile_kernel(long long ncols, const int* sorted_col, const int* rmax,
                                 ColSrc src, long long* tile_recs, long long* tile_tasks)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long ntiles = (ncols + TILE - 1) / TILE;
    if (t >= ntiles) return;
    int rm = 0, km = 0;
    for (int l = 0; l < TILE; ++l) {
        const long long s = t * TILE + l;
        if (s >= ncols) break;
        const int c = sorted_col[s];
        rm = max(rm, rmax[c]);
        km = max(km, src.col_K(c));
    }
    tile_recs[t] = (long long)rm * TILE;
    tile_tasks[t] = km;
}

__global__ void prep_tasks_kernel(long long ntiles, const long long* tile_tasks,
                                  const long long* tile_tbase, int2* tasks)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    const long long b = tile_tbase[t];
    for (long long k = 0; k < tile_tasks[t]; ++k) tasks[b + k] = make_int2((int)t, (int)k);
}

// Build the layer records and metadata of the column at sorted position s.
// Output addressing of the column goes into its ColMeta.
__device__ __forceinline__ void prep_build_one(const ColSrc& src, const PrepOut& o, const Tables& T,
                               const int* sorted_col, const long long* tile_tbase, long long s)
{
    const int c = sorted_col[s];
    const int nz = src.col_nz(c), K = src.col_K(c);
    ColMeta M;
    M.col = c; M.nz = nz; M.K = K;
    if (src.ragged) {
        M.per_b = src.per_off[c];
        M.pv_b = src.per_off[c];
        M.sen_b = o.sen_off ? o.sen_off[c] : 0;
        M.sen_is = K;
        M.ls_b = o.ls_off ? o.ls_off[c] : 0;
        M.ls_is = K;
    } else {
        const long long post = src.col0 + c;
        M.per_b = 0;
        M.pv_b = post;
        M.sen_b = post;
        M.sen_is = src.ncol * (long long)K;
        M.ls_b = post;
        M.ls_is = src.ncol * (long long)K;
    }
    const long long t = s / TILE;
    M.cr_b = tile_tbase[t] * TILE + (s % TILE);
    M.status_i = src.ragged ? (long long)c : src.col0 + c;
    // streaming geometry
    const double ar = 6370.0, ar2 = (double)6371.0f;
    double dr = 0.0, r0 = ar, q0 = ar2, p0 = ar;
    int m = 0;
    float vs0, vp0, rh0, vs1, vp1, rh1;
    src.node(c, 0, vs0, vp0, rh0);
    for (int i = 0; i < nz; ++i) {
        const bool half = (i == nz - 1);
        int ns = 1;
        float newthk = 0.0f;
        if (!half) {
            src.node(c, i + 1, vs1, vp1, rh1);
            const float thk = __fsub_rn(src.dep(c, i + 1), src.dep(c, i));
            ns = nsub_of(thk, src.minthk);
            newthk = __fdiv_rn(thk, (float)ns);
        }
        for (int j = 1; j <= ns; ++j, ++m) {
            float rvp, rvs, rrh;
            ChainRec ch;
            if (half) {
                rvp = vp0; rvs = vs0; rrh = rh0;
                ch.node = (short)i; ch.sub = 0; ch.den = 1;
            } else {
                const int sub = 2 * j - 1, den = 2 * ns;
                rvp = sublayer_value(vp0, vp1, sub, den);
                rvs = sublayer_value(vs0, vs1, sub, den);
                rrh = sublayer_value(rh0, rh1, sub, den);
                ch.node = (short)i; ch.sub = (short)sub; ch.den = (short)den;
            }
            ch.pad = 0;
            // surfdisp96 sphere(): thickness, velocity factor, density factor
            const float dm = half ? 1.0f : newthk;
            dr = __dadd_rn(dr, (double)dm);
            const double r1 = __dsub_rn(ar, dr);
            const double z0 = __dmul_rn(ar, log(__ddiv_rn(ar, r0)));
            const double z1 = __dmul_rn(ar, log(__ddiv_rn(ar, r1)));
            const float dflat = half ? 0.0f : (float)__dsub_rn(z1, z0);
            const double tmp = __ddiv_rn(__dadd_rn(ar, ar), __dadd_rn(r0, r1));
            const float btp = (float)tmp;
            const float rhofac = src.ifunc == 1 ? love_rhofac(btp)
                                                : (float)pow((double)btp, (double)(-2.275f));
            r0 = r1;
            float4 L;
            L.x = dflat;
            L.y = (float)__dmul_rn((double)rvp, tmp);
            L.z = (float)__dmul_rn((double)rvs, tmp);
            L.w = __fmul_rn(rrh, rhofac);
            ch.tmp = tmp;
            ch.rhofac = rhofac;
            // tregn96 sphere_tdisp96() and bldsph()
            const double q1 = __dsub_rn(q0, (double)dm);
            const double y0 = __dmul_rn(ar2, log(__ddiv_rn(ar2, q0)));
            const double y1 = __dmul_rn(ar2, log(__ddiv_rn(ar2, q1)));
            const float td = (float)__dsub_rn(y1, y0);
            const double t2 = __ddiv_rn(__dadd_rn(ar2, ar2), __dadd_rn(q0, q1));
            q0 = q1;
            const double zd = half ? 1.0 : (double)td;
            const double p1 = __dmul_rn(p0, exp(-__ddiv_rn(zd, ar)));
            const float vtp = (float)__ddiv_rn(__dadd_rn(ar, ar), __dadd_rn(p0, p1));
            p0 = p1;
            const float TAu = __fmul_rn(rrh, __fmul_rn(rvp, rvp));
            const float TLu = __fmul_rn(rrh, __fmul_rn(rvs, rvs));
            // tregn96's model: A, L and rho flattened (real*4 stores), F
            // left unmapped (depthkernelTI.f90:124-131 with sphere_tdisp96)
            const float fTA = (float)__dmul_rn((double)TAu, pow(t2, (double)(-0.2750f)));
            const float fTL = (float)__dmul_rn((double)TLu, pow(t2, (double)(-0.2750f)));
            const float frh = (float)__dmul_rn((double)rrh, pow(t2, (double)(-2.275f)));
            TiRec tr;
            tr.TA = (double)fTA;
            tr.TL = (double)fTL;
            tr.rho = (double)frh;
            tr.TF = (double)__fsub_rn(TAu, __fmul_rn(2.0f, TLu));
            tr.td = half ? 0.0 : (double)td;
            // splice coefficients, real*4 as depthkernelTI.f90:152-162
            SpRec sr;
            const float TFs = __fmul_rn(1.0f, __fsub_rn(TAu, __fmul_rn(2.0f, TLu)));
            const float den = __fsub_rn(TAu, __fmul_rn(2.0f, TLu));
            const float den2 = __fmul_rn(den, den);
            sr.vtp = vtp;
            sr.cA1 = __fdiv_rn(0.5f, __fmul_rn(rrh, rvp));
            sr.cA2 = __fdiv_rn(TFs, den2);
            sr.cL1 = __fdiv_rn(0.5f, __fmul_rn(rrh, rvs));
            sr.cL2 = __fdiv_rn(__fmul_rn(2.0f, TFs), den2);
            sr.TA = TAu;
            sr.TL = TLu;
            sr.pad = 0.0f;
            const long long ix = rec_index(T, s, m);
            T.flat[ix] = L;
            T.ld[ix] = make_layerd(L);
            T.ti[ix] = tr;
            T.sp[ix] = sr;
            T.ch[ix] = ch;
        }
        vs0 = vs1; vp0 = vp1; rh0 = rh1;
    }
    M.rmax = m;
    T.meta[s] = M;
    if (o.work) {
        atomicAdd(o.work, (unsigned long long)K * (unsigned long long)m);
        atomicAdd(o.work + 1, (unsigned long long)K);
    }
}

// One thread per sorted position.
__global__ void prep_build_kernel(ColSrc src, PrepOut o, Tables T, const int* sorted_col,
                                  const long long* tile_tbase)
{
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= T.ncols) return;
    prep_build_one(src, o, T, sorted_col, tile_tbase, s);
}

}  // namespace dk
