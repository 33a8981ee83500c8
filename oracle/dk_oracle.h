/* CPU oracle (test infrastructure only): C restatement of the reference
 * depth-kernel stage.  See dk_oracle.c and tregn_oracle.c for citations. */
#ifndef DK_ORACLE_H
#define DK_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif
void or_brocher(int nz, const float *vs, float *vp, float *rho);
int or_refine(float minthk0, int nz, const float *dep, const float *vp,
              const float *vs, const float *rho, float *rthk, float *rvp,
              float *rvs, float *rrho, int *nsublay);
int or_surfdisp96(const float *thkm, const float *vpm, const float *vsm,
                  const float *rhom, int nlayer, int iflsph, int iwave,
                  int mode, int igr, int kmax, const double *t, double *cg);
int or_surfdisp96_ex(const float *thkm, const float *vpm, const float *vsm,
                     const float *rhom, int nlayer, int iflsph, int iwave,
                     int mode, int igr, int kmax, const double *t, double *cg,
                     double tol, int round_f32, int *evals_per_period);
int or_column_fd(int nz, const float *vs, const float *vp, const float *rho,
                 int kmax, const double *periods, int iwave, int igr,
                 const float *depz, float minthk, float dlnvs, float dlnvp,
                 float dlnrho, double tol, int precision, double *pv,
                 double *sen_vs, double *sen_vp, double *sen_rho, long *evals);
int or_depthkernel(int nx, int ny, int nz, const float *vel,
                   const float *vp_in, const float *rho_in, double *pvRc,
                   double *sen_vs, double *sen_vp, double *sen_rho, int iwave,
                   int igr, int kmax, const double *tRc, const float *depz,
                   float minthk, int col_start, int col_count, int nthreads,
                   double tol, int precision, float dln, int *status_out,
                   long *evals_out);
int or_phase(int nx, int ny, int nz, const float *vel, const float *vp_in,
             const float *rho_in, double *pvRc, int iwave, int igr, int kmax,
             const double *tRc, const float *depz, float minthk, int nthreads,
             double tol, int round_f32, int *evals_cp, int *status_out);
int or_surfdisp96_split(const float *thkm, const float *vpm, const float *vsm,
                        const float *rhom, int nlayer, int kmax, const double *t, double *cg,
                        int *evals_per_period, int *scan_per_period);
int or_surfdisp96_d(const double *thkm, const double *vpm, const double *vsm,
                    const double *rhom, int nlayer, int iflsph, int kmax,
                    const double *t, double *cg, double tol);
int or_tregn96(int nl, const float *d_in, const float *TA_in, const float *TC_in,
               const float *TF_in, const float *TL_in, const float *TN_in,
               const float *TRho_in, const float *qai_in, const float *qbi_in,
               const float *etapi_in, const float *etasi_in, const float *frefpi_in,
               const float *frefsi_in, int nt, const float *t_in, const float *cp_in,
               float *dcdah_out, float *dcdbv_out, float *dcdn_out);
int or_tregn96_ex(int nl, const float *d_in, const float *TA_in, const float *TC_in,
                  const float *TF_in, const float *TL_in, const float *TN_in,
                  const float *TRho_in, const float *qai_in, const float *qbi_in,
                  const float *etapi_in, const float *etasi_in, const float *frefpi_in,
                  const float *frefsi_in, int nt, const float *t_in, const float *cp_in,
                  float *dcdah_out, float *dcdbv_out, float *dcdn_out, int nsph, int dogam,
                  double *full);
int or_tregn96_cd(int nl, const float *d_in, const float *TA_in, const float *TC_in,
                  const float *TF_in, const float *TL_in, const float *TN_in,
                  const float *TRho_in, const float *qai_in, const float *qbi_in,
                  const float *etapi_in, const float *etasi_in, const float *frefpi_in,
                  const float *frefsi_in, int nt, const float *t_in, const double *cp_d,
                  float *dcdah_out, float *dcdbv_out, float *dcdn_out, int nsph, int dogam,
                  double *full);
double or_ti_secular_d(int nl, const double *d, const double *TA, const double *TC,
                       const double *TF, const double *TL, const double *TN, const double *rho,
                       double omega, double c);
int or_ti_root_d(int nl, const double *d, const double *TA, const double *TC, const double *TF,
                 const double *TL, const double *TN, const double *rho, double omega, double c0,
                 double xtol, double *root);
int or_ti_root_fd(int nl, const double *d, const double *TA, const double *TC, const double *TF,
                  const double *TL, const double *TN, const double *rho, double omega,
                  double c0, double h, double xtol, int npert, const int *lo, const int *hi,
                  const int *kind, double *dcdp, int nthreads);
int or_depthkernelTI(int nx, int ny, int nz, const float *vel, const float *vp_in,
                     const float *rho_in, double *pvRc, int iwave, int igr, int kmax,
                     const double *tRc, const float *depz, float minthk, float *Lsen,
                     int col_start, int col_count, int nthreads, int *status_out);
int or_batch(long ncols, const long *node_off, const float *depz, const float *vs_all,
             const long *per_off, const double *periods, float minthk, double *pv,
             const long *sen_off, double *svs, double *svp, double *srh, const long *ls_off,
             float *lsen, int nthreads);
int or_batch_ti(long ncols, const long *node_off, const float *depz, const float *vs_all,
                const long *per_off, const double *periods, float minthk, const double *pv_in,
                double root_tol, double *pv_out, const long *ls_off, float *lsen, int nthreads);
int or_batch_fd(long ncols, const long *node_off, const float *depz, const float *vs_all,
                const long *per_off, const double *periods, float minthk, double *pv,
                const long *sen_off, double *svs, double *svp, double *srh, int precision,
                double tol, float dln, int *status, int nthreads);
long or_grows(int nvx, int nvz, int nz, int K, const float *vels, const double *svs,
              const double *svp, const double *srh, const float *lsen, long nrays,
              const int *ray_period, const int *ray_id, const long *cell_off, const int *cell,
              const float *fdm, const float *fdmc, const float *fdms, float ftol, long cap,
              float *rw, int *iw, int *col, long *nnz_ray);
void or_azimap(int nx, int ny, int nz, int K, const float *lsen, const float *gc, const float *gs,
               const double *ciso, float *cosr, float *sinr, float *amp, float *rela, float *ang);
/* First-arrival traveltimes (fmm_oracle.c).  The model grid is nx x ny
 * (x = latitude from goxd, z = longitude from gozd, degrees, spacing
 * dvxd x dvzd); the propagation grid is (nx-3)*gdx+1 x (ny-3)*gdz+1 nodes. */
typedef struct {
    int nx, ny;             /* phase-velocity map (model grid) */
    float goxd, gozd, dvxd, dvzd;
    int gdx, gdz;           /* grid dicing (5, 5) */
    int asgr, sgdl, sgs;    /* source-grid refinement (1, 8, 8) */
    int fom;                /* 0 first order, 1 mixed order (1) */
    float snb;              /* narrow-band capacity fraction (0.5) */
    float earth;            /* 6371 */
} OrFmmParams;
int or_fmm_batch(const OrFmmParams *P, const double *pv, int ninst, const int *inst_period,
                 const float *scx, const float *scz, const long *rc_off, const float *rcx,
                 const float *rcz, float *times, float *ttn_out, int nthreads);
int or_fmm_travel(int nnx, int nnz, float gox, float goz, float dnx, float dnz, float earth, int fom,
                  float snb, const float *veln, float scx, float scz, float *ttn, int *nsts_out);
#ifdef __cplusplus
}
#endif
#endif
