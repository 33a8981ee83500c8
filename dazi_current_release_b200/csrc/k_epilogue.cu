// Epilogues of the stage: the G rows of the LSMR system and the azimuthal
// phase-velocity maps.
//
// G rows of the LSMR system from the depth kernels (the consumer of the
// stage, CalSurfG_parallel.f90:2363-2400, iso_phase_only with
// use_aniso_active).  For each ray (a data row) and each model cell of its
// path with |fdm| >= ftol, the reference fills a dense real*4 parameter row
//   row(i, cell)          = (sen_vp coe_a + sen_rho coe_rho + sen_vs) fdm
//   row(nparpi + i, cell) = Lsen fdmc,   row(2 nparpi + i, cell) = Lsen fdms
// (i = 1 .. nz-1; coe_a, coe_rho the Brocher derivatives at the node
// velocity, real*4) and appends the entries |row| > ftol in parameter order.
// Here one warp builds one ray's entries straight from the kernel arrays,
// in the same order, without the dense row: a counting pass, a scan of the
// counts, and a filling pass that compacts each group of 32 entries with a
// ballot.
#include "dk_kernels.cuh"

namespace dk {

// real*4 Brocher derivatives as the reference writes them (x**2 = x*x,
// x**3 = x**2*x, x**4 = x**2*x**2; products of constants folded in real*4)
__device__ __forceinline__ float grow_coe_a(float v)
{
    constexpr float a1 = 0.8206f * 2.0f, a2 = 0.2683f * 3.0f, a3 = 0.0251f * 4.0f;
    const float v2 = __fmul_rn(v, v), v3 = __fmul_rn(v2, v);
    return __fsub_rn(__fadd_rn(__fsub_rn(2.0947f, __fmul_rn(a1, v)), __fmul_rn(a2, v2)), __fmul_rn(a3, v3));
}

__device__ __forceinline__ float grow_coe_rho(float v, float ca)
{
    constexpr float b1 = 0.4721f * 2.0f, b2 = 0.0671f * 3.0f, b3 = 0.0043f * 4.0f, b4 = 0.000106f * 5.0f;
    const float v2 = __fmul_rn(v, v), v3 = __fmul_rn(v2, v), v4 = __fmul_rn(v2, v2);
    const float vp = __fsub_rn(__fadd_rn(__fsub_rn(__fadd_rn(0.9409f, __fmul_rn(2.0947f, v)), __fmul_rn(0.8206f, v2)),
                                         __fmul_rn(0.2683f, v3)), __fmul_rn(0.0251f, v4));
    const float p2 = __fmul_rn(vp, vp), p3 = __fmul_rn(p2, vp), p4 = __fmul_rn(p2, p2);
    const float poly = __fadd_rn(__fsub_rn(__fadd_rn(__fsub_rn(1.6612f, __fmul_rn(b1, vp)), __fmul_rn(b2, p2)),
                                           __fmul_rn(b3, p3)), __fmul_rn(b4, p4));
    return __fmul_rn(ca, poly);
}

// Value of entry e (a path cell) of interval i in block b (0 iso, 1 Gc, 2 Gs)
// of ray r; `keep` = the cell passes the fdm test.
__device__ __forceinline__ float grow_value(const GrowsArgs& a, int b, int i, long long e, int k, bool& keep)
{
    const float w = a.fdm[e];
    keep = fabsf(w) >= a.ftol;
    if (!keep) return 0.0f;
    const int c = a.cell[e];
    const int nx = a.nvx + 2;
    const long long nxy = (long long)nx * (a.nvz + 2);
    const long long post = (long long)(c / a.nvx + 1) * nx + (c % a.nvx + 1);
    const long long ks = post + nxy * (k + (long long)a.K * i);
    if (b == 0) {
        const float v = a.vels[post + nxy * i];
        const float ca = grow_coe_a(v), cr = grow_coe_rho(v, ca);
        const double s = __dadd_rn(__dadd_rn(__dmul_rn(a.svp[ks], (double)ca), __dmul_rn(a.srh[ks], (double)cr)),
                                   a.svs[ks]);
        return (float)__dmul_rn(s, (double)w);
    }
    const float L = a.lsen[ks];
    return __fmul_rn(L, b == 1 ? a.fdmc[e] : a.fdms[e]);
}

// fill == false: count the entries of every ray (and check its cells);
// fill == true: write them at off[ray] in parameter order.
template <bool FILL>
__global__ void __launch_bounds__(128) grows_kernel(GrowsArgs a)
{
    const long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= a.nrays) return;
    const long long e0 = a.cell_off[r], e1 = a.cell_off[r + 1];
    const int k = a.ray_period[r];
    const int ncell = a.nvx * a.nvz;
    if (!FILL) {
        bool bad = (k < 0 || k >= a.K || e1 < e0);
        for (long long e = e0 + lane; e < e1 && !bad; e += 32) {
            const int c = a.cell[e];
            if (c < 0 || c >= ncell || (e > e0 && a.cell[e - 1] >= c)) bad = true;
        }
        if (__any_sync(0xffffffffu, bad)) {
            if (lane == 0) { atomicOr(a.err, 1); a.nnz_ray[r] = 0; }
            return;
        }
    }
    const int nblk = a.lsen ? 3 : 1;
    long long base = FILL ? a.off[r] : 0;
    long long cnt = 0;
    for (int b = 0; b < nblk; ++b) {
        for (int i = 0; i < a.nz - 1; ++i) {
            for (long long e = e0; e < e1; e += 32) {
                const long long ee = e + lane;
                bool keep = false;
                float v = 0.0f;
                if (ee < e1) v = grow_value(a, b, i, ee, k, keep);
                const bool put = keep && fabsf(v) > a.ftol;
                const unsigned m = __ballot_sync(0xffffffffu, put);
                if (FILL && put) {
                    const long long pos = base + __popc(m & ((1u << lane) - 1u));
                    const int c = a.cell[ee];
                    a.rw[pos] = v;
                    a.iw[pos] = a.ray_id[r];
                    a.col[pos] = (int)((long long)b * ncell * (a.nz - 1) + (long long)i * ncell + c + 1);
                }
                base += __popc(m);
                cnt += __popc(m);
            }
        }
    }
    if (!FILL && lane == 0) a.nnz_ray[r] = cnt;
}

template __global__ void grows_kernel<false>(GrowsArgs);
template __global__ void grows_kernel<true>(GrowsArgs);

// Azimuthal phase-velocity maps, FwdAzimuthalAniMap.f90:43-86: per inner
// column (ii, jj) and period tt,
//   cos = sum_k Lsen(k) gc(k),  sin = sum_k Lsen(k) gs(k)   (real*4, k ascending)
//   amp = 0.5 sqrt(cos^2 + sin^2),  rela = amp / c_iso,
//   ang = 0.5 (atan2(sin, cos) / pi * 180, + 360 when negative)
// with the reference's real*4 / real*8 mix (pi real*8, the angle stored
// real*4).  Outputs indexed (jj-1)*nvx + ii-1 + nvx*nvz*(tt-1).
__global__ void __launch_bounds__(128) azimap_kernel(AzimapArgs a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long ncell = (long long)a.nvx * a.nvz;
    if (t >= ncell * a.K) return;
    const int tt = (int)(t / ncell);
    const long long c = t % ncell;
    const int ii = (int)(c % a.nvx) + 1, jj = (int)(c / a.nvx) + 1;
    const int nx = a.nvx + 2;
    const long long nxy = (long long)nx * (a.nvz + 2);
    const long long post = (long long)jj * nx + ii;
    float cs = 0.0f, sn = 0.0f;
    for (int k = 0; k < a.nz - 1; ++k) {
        const float L = a.lsen[post + nxy * (tt + (long long)a.K * k)];
        const long long g = (ii - 1) + (long long)a.nvx * ((jj - 1) + (long long)a.nvz * k);
        cs = __fadd_rn(cs, __fmul_rn(L, a.gc[g]));
        sn = __fadd_rn(sn, __fmul_rn(L, a.gs[g]));
    }
    const float amp = __fmul_rn(0.5f, __fsqrt_rn(__fadd_rn(__fmul_rn(cs, cs), __fmul_rn(sn, sn))));
    const float iso = (float)a.ciso[c + ncell * tt];
    const double pi = 3.1415926535898;
    float ang = (float)__dmul_rn(__ddiv_rn((double)atan2f(sn, cs), pi), 180.0);
    if (ang < 0.0f) ang = __fadd_rn(ang, 360.0f);
    ang = __fmul_rn(0.5f, ang);
    a.cosr[t] = cs;
    a.sinr[t] = sn;
    a.amp[t] = amp;
    a.rela[t] = __fdiv_rn(amp, iso);
    a.ang[t] = ang;
}

}  // namespace dk
