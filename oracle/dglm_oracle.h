/* ORACLE -- test infrastructure only (see dglm_oracle.c). */
#ifndef DGLM_ORACLE_H
#define DGLM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_ADVECTION = 0, ORC_EULER = 1 };

typedef struct {
    int N, Np, Nfp, nvar, K, physics;
    double cfl, gamma, tau_scale, tmax;
    const double *WDr, *WDs, *WDt, *LIFT;          /* row-major */
    const double *rx, *ry, *rz, *sx, *sy, *sz, *tx, *ty, *tz;
    const double *Fscale, *nx, *ny, *nz;
    const int *EtoB, *vmapF, *vmapP, *Fmask;
    const double *vx, *vy, *vz;                     /* advection only */
} orc_mesh;

typedef struct {
    double t, dt;
    int tstep, last;
} orc_clock;

void orc_rk_coefficients(double *a, double *b, double *c);
void orc_calc_maxv(const orc_mesh *m, const double *u, double *maxv, double *maxv_fs);
double orc_calc_dt(const orc_mesh *m, const double *maxv_fs);
void orc_update_tau(const orc_mesh *m, const double *maxv, double *tau);
void orc_update_ub(const orc_mesh *m, const double *u, double *ub);
void orc_calc_fluxLM(const orc_mesh *m, const double *u, const double *ub, const double *tau,
                     double *fluxLM);
void orc_calc_fluxes(const orc_mesh *m, const double *u, double *fR, double *fS, double *fT);
void orc_update_rhs(const orc_mesh *m, const double *fR, const double *fS, const double *fT,
                    const double *fLM, double *utmp);
void orc_lserk_stage(const orc_mesh *m, double dt, double a, double b, const double *utmp,
                     double *k, double *u);
double orc_rhs(const orc_mesh *m, const double *u, double *maxv, double *tau, double *ub,
               double *fluxLM, double *fR, double *fS, double *fT, double *utmp);
int orc_run(const orc_mesh *m, double *u, double *k, orc_clock *clk, int nsteps, double dt_fixed,
            double *dt_hist);
int orc_num_threads(void);
void orc_rhs_adjoint(const orc_mesh *m, const double *u, const double *tau, const double *mu,
                     double *lam);
int orc_run_record(const orc_mesh *m, double *u, double *k, int nsteps, double *dt_hist,
                   double *tau_hist);
void orc_run_frozen(const orc_mesh *m, double *u, double *k, int nsteps, const double *dt_hist,
                    const double *tau_hist);
void orc_adjoint(const orc_mesh *m, const double *u0, int nsteps, const double *dt_hist,
                 const double *tau_hist, double *lam);

#ifdef __cplusplus
}
#endif
#endif
