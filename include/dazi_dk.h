/*
 * dazi_dk.h — C-ABI of the B200 depth-kernel library (libdazi_dk.so).
 *
 * Drop-in replacement for DAzi's per-column dispersion and depth-kernel
 * stage.  All arrays use the reference's Fortran layouts:
 *   vel, vp, rho   (nx, ny, nz)            real*4, column-major
 *   pvRc           (nx*ny, kmaxRc)         real*8
 *   sen_*Rc        (nx*ny, kmaxRc, nz)     real*8
 *   Lsen_Gsc       (nx*ny, kmaxRc, nz-1)   real*4
 *   tRc            (kmaxRc)                real*8, ascending periods (s)
 *   depz           (nz)                    real*4, node depths (km)
 * Column index post = ii + (jj-1)*nx (1-based), as in the reference.
 * Scalars that the reference passes by reference stay pointers so the
 * Fortran side can bind them without the VALUE attribute; the column range
 * and the form selector are passed by value.
 *
 * Wave and velocity type: iwave = 2 (Rayleigh) or 1 (Love), igr = 0 (phase)
 * or > 0 (group), as surfdisp96 takes them (DepthKernel1D.f90 passes both
 * through; DAzi's inversion calls Rayleigh phase, CalSurfG_parallel.f90:
 * 1967-1976, and holds the other three calls at CalSurfG.f90:1227-1245).
 * The plain form, the adjoint form and phase-velocity-only calls take all
 * four (Love: the adjoint differentiates dltar1's 2x2 Haskell-Thomson chain
 * and dc/dVp is zero; group velocity: the adjoint differentiates the
 * reference's quotient of the roots at t/(1+h) and t/(1-h)); Lsen_Gsc is
 * Rayleigh phase only.  Other values return DAZI_ERR_BADARG.
 *
 * Depth cut: the Lsen_Gsc sweep and the adjoint form's Rayleigh
 * phase-velocity sweep stop at the first layer below which the shear wave
 * has decayed by exp(-16) (E = sum of nu_b d >= 16, nu_b = sqrt(k^2 -
 * (omega/Vs)^2)); that layer is the sweep's half-space and the kernels of
 * the nodes below it are zero (their values are of relative order
 * exp(-32)); DAZI_FORM_FULL_STACK turns it off.  Love waves, group
 * velocity and the plain form's finite differences sweep the whole stack.
 *
 * Limits (the reference's compiled limits, surfdisp96.f:57-59):
 *   nz <= 200, kmaxRc <= 160, refined layers <= 200.
 *
 * Errors: 0 on success; DAZI_WARN_NOROOT (> 0) when at least one column had
 * a period without a fundamental-mode root — that period and every later one
 * of the column are zero in pvRc and in the kernels, as surfdisp96.f:1700-1770
 * leaves them; negative codes are errors and leave the outputs unspecified.
 * The library never exits or aborts; device code never traps.
 *
 * Threading: one host thread at a time (the reference calls the stage from
 * one thread outside its OpenMP regions, CalSurfG_parallel.f90:1967-1976).
 * The library owns its device buffers and stream; dazi_dk_finalize() frees
 * them.
 */
#ifndef DAZI_DK_H
#define DAZI_DK_H

#ifdef __cplusplus
extern "C" {
#endif

#define DAZI_OK            0
#define DAZI_WARN_NOROOT   1
#define DAZI_ERR_BADARG   -1
#define DAZI_ERR_LIMITS   -2
#define DAZI_ERR_CUDA     -3
#define DAZI_ERR_TIMEOUT  -4
#define DAZI_ERR_NOMEM    -5
#define DAZI_ERR_NODEVICE -6
#define DAZI_ERR_MODEL    -7   /* non-finite kernel (degenerate layer)     */

/* form selector */
#define DAZI_FORM_PLAIN    0   /* perturb-and-recompute, as the reference */
#define DAZI_FORM_ADJOINT  1   /* implicit differentiation of the root     */
/* flag, OR-ed into the form: the root search of the adjoint form (and of
 * the Lsen-only entry) scans for the bracket with the secular function in
 * FP32, re-evaluating near-zero values and both bracket ends in FP64 (same
 * roots as the default all-FP64 search).  The plain form always evaluates
 * in FP64. */
#define DAZI_FORM_SCAN_FP32 2
/* flags, OR-ed into the form (plain or adjoint, or a phase-velocity-only
 * call; no Lsen_Gsc output): Love instead of Rayleigh waves
 * (surfdisp96's iwave = 1, dltar1) and group instead of phase velocity
 * (igr > 0; pvRc and the kernels are then the group velocity and its
 * derivatives).  The entries with iwave/igr arguments set them from those
 * (and reject them in form); the device and uneven-column entries take
 * them here.  Both forms take them.  DAZI_FORM_SCAN_FP32, Lsen_Gsc and
 * plans are Rayleigh phase velocity only: combining them with these flags
 * returns DAZI_ERR_BADARG. */
#define DAZI_FORM_LOVE     4
#define DAZI_FORM_GROUP    8
/* flag, OR-ed into the form: the root search (adjoint form, phase-velocity-
 * or Lsen-only calls, plans) keeps the reference's getsol scan, point for
 * point, so each period's bracket and mode are the reference's, but refines
 * the bracket by Brent's method to 1e-10 c instead of nevill() to 1e-6 c
 * (about 3.5 instead of 12 evaluations per period).  pvRc is then the
 * float32 of the exact root, within the reference's own 1e-6 c of its
 * value; the default search reproduces its value bit for bit.  Rayleigh
 * phase velocity; with DAZI_FORM_LOVE or DAZI_FORM_GROUP it returns
 * DAZI_ERR_BADARG.  The plain form's finite differences ignore it. */
#define DAZI_FORM_FAST_ROOT 16
/* flag, OR-ed into the form (adjoint form, Lsen_Gsc, plans): the Lsen_Gsc
 * sweep and the adjoint form's Rayleigh phase-velocity sweep run over the
 * whole layer stack, without the depth cut described above (slower; the
 * kernels below the cut are then their exp(-32)-small values instead of
 * zero). */
#define DAZI_FORM_FULL_STACK 32

/* Replaces depthkernel() of code/src_inv_iso_joint/CalSurfG.f90:1-15
 * (default_fortran_fd backend, CalSurfG.f90:86-107), for the 1-based column
 * range [col_start, col_start + col_count).  Writes pvRc and the three
 * kernels of those columns.  sen_* may all be NULL to compute pvRc only
 * (depthkernel_column_phase_fd, DepthKernel1D.f90:1-23). */
int dazi_dk_iso(const int *nx, const int *ny, const int *nz, const float *vel,
                double *pvRc, double *sen_vsRc, double *sen_vpRc,
                double *sen_rhoRc, const int *iwave, const int *igr,
                const int *kmaxRc, const double *tRc, const float *depz,
                const float *minthk, int col_start, int col_count, int form);

/* As dazi_dk_iso with explicit Vp and rho arrays in place of the Brocher
 * relations (depthkernel_empirical_vp_rho, DepthKernel1D.f90:187-200);
 * the finite differences still perturb Vs, Vp and rho independently. */
int dazi_dk_iso_vpvsrho(const int *nx, const int *ny, const int *nz,
                        const float *vel, const float *vp, const float *rho,
                        double *pvRc, double *sen_vsRc, double *sen_vpRc,
                        double *sen_rhoRc, const int *iwave, const int *igr,
                        const int *kmaxRc, const double *tRc,
                        const float *depz, const float *minthk,
                        int col_start, int col_count, int form);

/* Replaces depthkernelTI() of code/src_inv_iso_joint/depthkernelTI.f90:2-14
 * (default_fortran_tregn96 backend, depthkernelTI.f90:86-169): pvRc and
 * the Gc/Gs kernel Lsen_Gsc(nx*ny, kmaxRc, nz-1) of the column range.
 * Periods without a root leave their Lsen_Gsc entries at zero. */
int dazi_dk_ti(const int *nx, const int *ny, const int *nz, const float *vel,
               double *pvRc, const int *iwave, const int *igr,
               const int *kmaxRc, const double *tRc, const float *depz,
               const float *minthk, float *Lsen_Gsc, int col_start,
               int col_count);

/* Both stages in one call: pvRc computed once (the reference computes it in
 * depthkernelTI and again in depthkernel, CalSurfG_parallel.f90:1972-1975).
 * vp/rho may be NULL (Brocher relations); sen_* may all be NULL; Lsen_Gsc
 * may be NULL. */
int dazi_dk_fused(const int *nx, const int *ny, const int *nz,
                  const float *vel, const float *vp, const float *rho,
                  double *pvRc, double *sen_vsRc, double *sen_vpRc,
                  double *sen_rhoRc, float *Lsen_Gsc, const int *iwave,
                  const int *igr, const int *kmaxRc, const double *tRc,
                  const float *depz, const float *minthk, int col_start,
                  int col_count, int form);

/* Per-column status of the last call: first period (1-based) without a root,
 * 0 when all periods have one.  status has nx*ny entries; only the columns
 * of the last call's range are written.  Returns 0, or DAZI_ERR_BADARG if no
 * call was made yet. */
int dazi_dk_last_status(int *status, long long n);

/* Device-pointer entry of the iso stage for callers that already hold the
 * data in HBM (the PyTorch binding).  All array pointers are device
 * pointers; vp/rho may be NULL (Brocher); sen_* may be NULL; status (nx*ny
 * ints, device) may be NULL.  stream is a cudaStream_t; NULL means the
 * legacy default stream.  Work is stream-ordered and the call returns
 * without waiting for it (only the tiny depz/tRc read-back synchronises). */
int dazi_dk_iso_dev(int nx, int ny, int nz, const float *vel, const float *vp,
                    const float *rho, double *pvRc, double *sen_vsRc,
                    double *sen_vpRc, double *sen_rhoRc, int kmaxRc,
                    const double *tRc, const float *depz, float minthk,
                    int col_start, int col_count, int form, int *status,
                    void *stream);

/* Device-pointer form of dazi_dk_fused (same conventions as
 * dazi_dk_iso_dev). */
int dazi_dk_fused_dev(int nx, int ny, int nz, const float *vel, const float *vp,
                      const float *rho, double *pvRc, double *sen_vsRc,
                      double *sen_vpRc, double *sen_rhoRc, float *Lsen_Gsc,
                      int kmaxRc, const double *tRc, const float *depz,
                      float minthk, int col_start, int col_count, int form,
                      int *status, void *stream);

/* Allocation-free variant of dazi_dk_iso_dev for the plain form.  No
 * counterpart in the reference.  For callers that cannot let a library call
 * cudaMalloc (a driver under another framework's allocator or a fixed memory
 * budget, or a pipeline that must avoid cudaMalloc's device-wide
 * synchronisation): the caller passes device inputs and outputs; the only
 * other device memory is a file-scope static array of 4 Mi floats (16 MiB)
 * plus the depth-grid geometry, held on every GPU that loads the library
 * until exit.  Columns run in tiles of 16 MiB / (4 M kmaxRc) bytes, with
 * M = 1 + 6 nz models per column when sen_* are given and M = 1 (phase
 * velocities only) when they are NULL; a column whose scratch exceeds the
 * array is rejected with DAZI_ERR_LIMITS.  All calls share the array: calls
 * whose GPU work overlaps race and must be ordered by the caller.  The first
 * call on a device does that device's set-up (cudaGetSymbolAddress); make it
 * before any stream capture.  Each call synchronises `stream` (NULL = legacy
 * default stream) twice, to read back the depth grid, the periods and the
 * refined layer count for validation; the finite-difference launches that
 * follow are queued and not waited for.  A CUDA error already pending when
 * the call starts is reported (DAZI_ERR_CUDA) and left pending.  No-root
 * periods are reported through `status`. */
int dazi_dk_iso_noalloc_dev(int nx, int ny, int nz, const float *vel,
                            const float *vp, const float *rho, double *pvRc,
                            double *sen_vsRc, double *sen_vpRc,
                            double *sen_rhoRc, int kmaxRc, const double *tRc,
                            const float *depz, float minthk, int col_start,
                            int col_count, int *status, void *stream);

/* Ragged batch: columns with their own depth grids and period lists (for
 * instance the cells of many Voronoi realisations), the extension that
 * replaces the reference's fixed column tiles (pdsurf_tile_columns /
 * ti_tile_columns, depthkernel_ti_process_batch.py:17-28).  CSR layout:
 * column c has nodes node_off[c] .. node_off[c+1]-1 (depz, vs and optional
 * vp, rho) and periods per_off[c] .. per_off[c+1]-1 (ascending).  Outputs:
 * pv[per_off[c] + k]; sen_*[sen_off[c] + k + K_c i] (K_c periods x nz_c
 * nodes, column-major as one column of the reference's arrays);
 * lsen[ls_off[c] + k + K_c j] (K_c x (nz_c - 1)).  sen_* / lsen may be NULL
 * (with their offsets).  status[c] as dazi_dk_last_status.  minthk is the
 * common sublayer count.  Host-pointer form: */
int dazi_dk_batch(long long ncols, const long long *node_off,
                  const float *depz, const float *vs, const float *vp,
                  const float *rho, const long long *per_off,
                  const double *periods, float minthk, double *pv,
                  const long long *sen_off, double *sen_vs, double *sen_vp,
                  double *sen_rho, const long long *ls_off, float *lsen,
                  int form, int *status);

/* Device-pointer form of dazi_dk_batch (all arrays in device memory,
 * stream-ordered on `stream`; one small synchronisation sizes the tables). */
int dazi_dk_batch_dev(long long ncols, const long long *node_off,
                      const float *depz, const float *vs, const float *vp,
                      const float *rho, const long long *per_off,
                      const double *periods, float minthk, double *pv,
                      const long long *sen_off, double *sen_vs,
                      double *sen_vp, double *sen_rho, const long long *ls_off,
                      float *lsen, int form, int *status, void *stream);

/* Plans: the uneven-column batch bound once, run many times.  No
 * counterpart in the reference (its per-call drivers rebuild everything);
 * this replaces the fixed tile pipelines for the inversion loop, where the
 * column structure (node depths, periods) stays while the velocities
 * change.  dazi_dk_plan_create takes the arguments of dazi_dk_batch_dev
 * (device pointers, adjoint form only; sen_* and/or lsen may be NULL), builds
 * the structure of the layer tables, picks the kernel variants by timing
 * them on this batch when tune != 0 (root-search block size; register
 * budgets of the adjoint and Gc/Gs sweeps), and captures the per-run
 * sequence in a CUDA graph.  The buffers stay bound: dazi_dk_plan_launch
 * recomputes everything from the current contents of vs (vp, rho) and
 * writes the same output buffers, as one graph launch on `stream` with no
 * host synchronisation.  Velocities are validated at creation only; a
 * non-finite Lsen_Gsc of a later run is reported by dazi_dk_plan_status
 * (which reads the device flag; call it after the run completes).  A plan
 * owns its device buffers and stream until dazi_dk_plan_destroy.  Creation
 * synchronises with `stream` and takes several runs' time (tuning). */
int dazi_dk_plan_create(long long ncols, const long long *node_off,
                        const float *depz, const float *vs, const float *vp,
                        const float *rho, const long long *per_off,
                        const double *periods, float minthk, double *pv,
                        const long long *sen_off, double *sen_vs,
                        double *sen_vp, double *sen_rho,
                        const long long *ls_off, float *lsen, int form,
                        int *status, int tune, void *stream, void **plan);
int dazi_dk_plan_launch(void *plan, void *stream);
int dazi_dk_plan_status(void *plan);
/* The tuner's choice: root-search variant (100 x threads per block +
 * register-budget blocks per SM, 0 = unconstrained), blocks per SM of the
 * adjoint and Gc/Gs sweeps, and their tuned phase times (ms, 3 floats).
 * The per-call entries use 128x0 / 3 / 8, or the environment variable
 * DAZI_DK_LAUNCH="root=BT[xMINB],adj=MINB,ti=MINB" when set. */
int dazi_dk_plan_config(void *plan, int *root_block, int *adjoint_blocks_per_sm,
                        int *ti_blocks_per_sm, float *tuned_ms);
int dazi_dk_plan_destroy(void *plan);

/* G rows of the LSMR system from the kernels: the consumer of the stage,
 * CalSurfG_parallel.f90:2363-2400 (iso_phase_only, use_aniso_active), on
 * device pointers.  Grid interface: nvx x nvz inner model cells, kernel
 * arrays of the (nvx+2) x (nvz+2) grid in the reference's layouts
 * (sen_*Rc (nxy, kmaxRc, nz) real*8, Lsen_Gsc (nxy, kmaxRc, nz-1) real*4, or
 * NULL for isotropic rows), vels (nvx+2, nvz+2, nz) real*4.  Rays in CSR:
 * ray r (data row ray_id[r], period index ray_period[r], 0-based) crosses
 * cells cell[cell_off[r] .. cell_off[r+1]-1] ((jj-1)*nvx + kk-1, strictly
 * ascending) with path weights fdm (and fdmc, fdms for Gc, Gs).  Writes
 * the entries |row| > ftol in the reference's order: rw (real*4), iw (ray
 * id), col (1-based parameter: iso block, then Gc, then Gs, each ordered
 * by depth interval then cell), the count of every ray in nnz_ray
 * (device) and the total in *nnz_total (host).  Returns DAZI_ERR_LIMITS
 * (with *nnz_total set) when the total exceeds cap; one small
 * synchronisation sizes the output. */
int dazi_dk_grows_dev(int nvx, int nvz, int nz, int kmaxRc, const float *vels,
                      const double *sen_vsRc, const double *sen_vpRc,
                      const double *sen_rhoRc, const float *Lsen_Gsc,
                      long long nrays, const int *ray_period, const int *ray_id,
                      const long long *cell_off, const int *cell,
                      const float *fdm, const float *fdmc, const float *fdms,
                      float ftol, long long cap, float *rw, int *iw, int *col,
                      long long *nnz_ray, long long *nnz_total, void *stream);

/* Azimuthal phase-velocity maps, replacing the computation of
 * FwdAzimuthalAniMap (code/src_inv_iso_joint/FwdAzimuthalAniMap.f90:43-86),
 * device pointers: from Lsen_Gsc (nx*ny, kmaxRc, nz-1) real*4, the Gc/Gs
 * model gcf, gsf (nx-2, ny-2, nz-1) real*4 and the isotropic phase velocity
 * tRcV ((nx-2)*(ny-2), kmaxRc) real*8, every inner column and period gets
 * cosRc = sum Lsen gc, sinRc = sum Lsen gs, amp = 0.5 sqrt(cos^2 + sin^2),
 * amp_rel = amp / tRcV and the fast-axis angle (degrees, [0, 180)), all
 * ((nx-2)*(ny-2), kmaxRc) real*4.  Stream-ordered on `stream`. */
int dazi_dk_azimuthal_map_dev(int nx, int ny, int nz, int kmaxRc,
                              const float *Lsen_Gsc, const float *gcf,
                              const float *gsf, const double *tRcV,
                              float *cosRc, float *sinRc, float *amp,
                              float *amp_rel, float *angle, void *stream);

/* LSMR least squares on the system the G rows fill: replaces LSMR(m, n,
 * leniw, lenrw, iw, rw, b, damp, atol, btol, conlim, itnlim, localSize,
 * nout, x, istop, itn, normA, condA, normr, normAr, normx) of
 * code/src_inv_iso_joint/lsmrModule.f90:36 (the matrix as aprod.f90 reads
 * it: row indices iw(1:lenrw), column indices iw(lenrw+1:2*lenrw),
 * 1-based, values rw(1:lenrw) real*4; b, x real*8), all arguments by
 * reference as the Fortran passes them.  Solves min ||(A; damp I) x -
 * (b; 0)|| by LSMR (Fong & Saunders 2011) in FP64 on the GPU with the
 * stopping rules atol, btol, conlim, itnlim and the outputs istop (0..7),
 * itn and the estimates normA, condA, normr, normAr, normx.  Like the
 * reference's SciPy backend (scipy_lsmr_solve, which calls
 * scipy.sparse.linalg.lsmr), it does no local reorthogonalization:
 * localSize and nout are accepted and not used.  Duplicate (row, col)
 * entries add. */
int dazi_lsmr(const int *m, const int *n, const long long *leniw,
              const long long *lenrw, const int *iw, const float *rw,
              const double *b, const double *damp, const double *atol,
              const double *btol, const double *conlim, const int *itnlim,
              const int *localSize, const int *nout, double *x, int *istop,
              int *itn, double *normA, double *condA, double *normr,
              double *normAr, double *normx);

/* Device-pointer form: nnz triplets (row, col, val) with 0- or 1-based
 * indices (index_base), b (m) and x (n) real*8 in device memory;
 * norms[0..4] (host, may be NULL) = normA, condA, normr, normAr, normx.
 * Stream-ordered on `stream`; the host reads the stop flag once per 16
 * iterations (with the next 16 already queued), and returns when the solve
 * has finished.  Device memory comes from a private pool per device that
 * keeps it between calls; dazi_dk_finalize gives it back. */
int dazi_lsmr_dev(int m, int n, long long nnz, const int *row, const int *col,
                  const float *val, int index_base, const double *b,
                  double damp, double atol, double btol, double conlim,
                  int itnlim, double *x, int *istop, int *itn, double *norms,
                  void *stream);

/* First-arrival traveltimes (the FMM eikonal solver).
 *
 * The reference computes, per (period, source), the traveltime field on the
 * propagation grid by fast marching and interpolates it at the receivers:
 * the OpenMP loop of code/src_inv_iso_joint/CalSurfG_parallel.f90:2061-2340
 * (gridder_parallel :811 on the period's phase-velocity map, source-grid
 * refinement with bsplrefine_parallel :918 and travel_parallel :125 with
 * urg = 1, then travel_parallel with urg = 2 on the coarse grid, and
 * srtimes_parallel :997 per receiver).  These entries run that loop on the
 * GPU for all instances at once, with the reference's arithmetic (real*4,
 * its operation order, its binary-heap narrow band), so that every field
 * and time is the reference's value.  Ray paths (rpaths) are not part of
 * it. */
typedef struct {
    int nx, ny;                     /* model grid: pv maps are nx*ny, x fastest */
    float goxd, gozd, dvxd, dvzd;   /* first inner vertex (lat, lon) and spacing, degrees */
    int gdx, gdz;                   /* grid dicing (CalSurfG_parallel.f90:1900-1911: 5, 5) */
    int asgr, sgdl, sgs;            /* source-grid refinement on, dicing, extent (1, 8, 8) */
    int fom;                        /* 0 first-order, 1 mixed-order upwind scheme (1) */
    float snb;                      /* narrow-band capacity as a fraction of the nodes (0.5) */
    float earth;                    /* Earth radius, km (6371) */
} dazi_fmm_params;

/* The reference's settings for a model grid. */
void dazi_fmm_default_params(dazi_fmm_params *p, int nx, int ny, float goxd, float gozd,
                             float dvxd, float dvzd);

/* Traveltimes of ninst (period, source) instances: pv (nx*ny, nper) real*8
 * phase-velocity maps; instance s uses column inst_period[s] (0-based), its
 * source at (scx[s], scz[s]) and receivers rc_off[s] .. rc_off[s+1]-1 at
 * (rcx, rcz), all in radians as colatitude and longitude (real*4, as
 * Main_Jt.f90:412-431 converts them).  times (rc_off[ninst]) real*4 out;
 * ttn, when not NULL, receives each instance's coarse field as the
 * reference's ttn(nnz, nnx) (nnx = (nx-3)*gdx+1, nnz = (ny-3)*gdz+1).
 * Host arrays; returns DAZI_ERR_BADARG for a source or receiver outside
 * the grid, DAZI_ERR_LIMITS when a narrow band outgrows snb of the nodes
 * (the reference's array bound). */
int dazi_fmm_batch(const dazi_fmm_params *p, const double *pv, int nper, int ninst,
                   const int *inst_period, const float *scx, const float *scz,
                   const long long *rc_off, const float *rcx, const float *rcz,
                   float *times, float *ttn);

/* Device-pointer form of dazi_fmm_batch (all arrays in device memory),
 * stream-ordered on `stream`; the host reads the instances' sources and
 * receiver offsets once to lay out the work. */
int dazi_fmm_batch_dev(const dazi_fmm_params *p, const double *pv, int nper, int ninst,
                       const int *inst_period, const float *scx, const float *scz,
                       const long long *rc_off, const float *rcx, const float *rcz,
                       float *times, float *ttn, void *stream);

/* The reference's own arrays, by reference (Fortran-callable): the source
 * and receiver tables of CalSurfG_parallel.f90:1745-1850 (scxf, sczf
 * (nsrc, kmax); rcxf, rczf (nrc, nsrc, kmax); nrc1 (nsrc, kmax); nsrc1
 * (kmax); periods (nsrc, kmax), the 1-based column of pv for each source),
 * pv (nx*ny, nper) real*8 and the grid of para.in; writes dsurf (dall) in
 * the row order of countsurf (FmmBackend.f90:64-72: period, source,
 * receiver). */
int dazi_fmm_times(const int *nx, const int *ny, const int *kmax, const int *nsrc,
                   const int *nrc, const int *nper, const double *pv, const int *periods,
                   const int *nsrc1, const int *nrc1, const float *scxf, const float *sczf,
                   const float *rcxf, const float *rczf, const float *goxd,
                   const float *gozd, const float *dvxd, const float *dvzd,
                   const long long *dall, float *dsurf);

/* Per-phase timing: with dazi_dk_set_timing(1), each call records CUDA
 * events on its stream around its phases ("prep", "fd", "root", "adjoint",
 * "ti"); dazi_dk_last_timing fills up to cap (name, milliseconds) pairs of
 * the last call (waiting for its events) and returns their number. */
int dazi_dk_set_timing(int on);
int dazi_dk_last_timing(const char **names, double *ms, int cap);

/* Number of kernel launches the last call issued (all on its stream). */
int dazi_dk_last_launches(void);

/* Work done by the last call, for roofline accounting: the number of
 * Rayleigh secular-function evaluations of the root searches (each one a
 * pass over a refined layer stack) and the sum of evaluations x layers.
 * Synchronises with the device. */
int dazi_dk_last_work(long long *secular_evals, long long *layer_evals);

/* Size of the last call's per-(column, period) work: the number of
 * column-periods (sum of K_c) and of layer items (sum of K_c x refined layer
 * count of the column), the units of the adjoint and Gc/Gs sweeps.  Counted
 * when the layer tables are built (adjoint form, or Lsen requested); 0
 * otherwise.  Synchronises with the device. */
int dazi_dk_last_items(long long *column_periods, long long *layer_items);

/* Diagnostic: measured FP64 FMA throughput of the current device in
 * GFLOP/s (best of 5 launches of an FMA-chain kernel).  The stage's kernels
 * run on the FP64 CUDA-core pipe; this is their roofline denominator. */
int dazi_dk_fp64_peak(double *gflops);

/* Message of the last error (static storage, never NULL). */
const char *dazi_dk_last_error(void);

/* Library version as 10000*major + 100*minor + patch. */
int dazi_dk_version(void);

/* Releases every device buffer and stream the library created. */
void dazi_dk_finalize(void);

#ifdef __cplusplus
}
#endif
#endif /* DAZI_DK_H */
