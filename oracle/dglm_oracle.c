/*
 * ORACLE -- test infrastructure only.
 *
 * A CPU restatement, in plain C with OpenMP, of the reference's explicit
 * DGLM right-hand side and 5-stage low-storage Runge-Kutta step for linear
 * advection (Nvar = 1) and compressible Euler (Nvar = 5).  Only the tests,
 * the smoke check and the CPU-baseline leg of the benchmark load it, and
 * only as the checker; the product path never calls it.
 *
 * It follows dim3/src/cpp/euler_dglm.cpp, euler_time.cpp (Euler) and
 * advec_dglm.cpp, advec_time.cpp (advection) line by line in arithmetic, with
 * the compile-time macros of the reference (N, NP, NFP, NVAR, CFL, GAMMA,
 * TAU_SCALE, TMAX) turned into run-time fields of orc_mesh.  It is pinned to
 * the reference by tests/test_oracle.py: against the reference solver
 * compiled from its sources (oracle/_ref) and against committed golden
 * vectors generated from it.
 *
 * Layouts (reference datain, CPU flavour):
 *   WDr/WDs/WDt  Np x Np, row-major ('c' order, launcher :144-147)
 *   LIFT         Np x 4Nfp, row-major
 *   u, k, utmp   nvar blocks of K*Np doubles, element-major (idx = e*Np + i)
 *   ub, fluxLM   nvar blocks of K*4*Nfp doubles (idx = (e*4 + f)*Nfp + j)
 *   rx..tz       K;  Fscale, nx, ny, nz, tau, maxv   K*4
 *   vmapP        K*4*Nfp;  vmapF, EtoB  K*4;  Fmask 4*Nfp
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "dglm_oracle.h"

/* Carpenter & Kennedy (1994) 5-stage, 4th-order 2N-storage coefficients,
 * the values the reference stores (euler_data.cpp:41-60). */
static const double RKA[5] = {0.0,
                              -567301805773.0 / 1357537059087.0,
                              -2404267990393.0 / 2016746695238.0,
                              -3550918686646.0 / 2091501179385.0,
                              -1275806237668.0 / 842570457699.0};
static const double RKB[5] = {1432997174477.0 / 9575080441755.0,
                              5161836677717.0 / 13612068292357.0,
                              1720146321549.0 / 2090206949498.0,
                              3134564353537.0 / 4481467310338.0,
                              2277821191437.0 / 14882151754819.0};
static const double RKC[5] = {0.0,
                              1432997174477.0 / 9575080441755.0,
                              2526269341429.0 / 6820363962896.0,
                              2006345519317.0 / 3224310063776.0,
                              2802321613138.0 / 2924317926251.0};

void orc_rk_coefficients(double *a, double *b, double *c) {
    for (int s = 0; s < 5; s++) { a[s] = RKA[s]; b[s] = RKB[s]; c[s] = RKC[s]; }
}

/* euler_dglm.cpp:6-50 (Euler) and advec_dglm.cpp:6-35 (advection) */
void orc_calc_maxv(const orc_mesh *m, const double *u, double *maxv, double *maxv_fs) {
    const long K = m->K, Np = m->Np, Nfp = m->Nfp, n = K * Np;
    const double g = m->gamma;
#pragma omp parallel for
    for (long fidx = 0; fidx < K * 4; fidx++) {
        long ei = fidx / 4, fi = fidx % 4;
        double max_v2 = 0, max_c2 = 0;
        for (long j = 0; j < Nfp; j++) {
            long idxM = ei * Np + m->Fmask[fi * Nfp + j];
            if (m->physics == ORC_EULER) {
                double u1 = u[idxM], u2 = u[n + idxM], u3 = u[2 * n + idxM];
                double u4 = u[3 * n + idxM], u5 = u[4 * n + idxM];
                double vx = u2 / u1, vy = u3 / u1, vz = u4 / u1;
                double v2 = vx * vx + vy * vy + vz * vz;
                if (v2 > max_v2) max_v2 = v2;
                double pres = (g - 1) * (u5 - 0.5 * u1 * v2);
                double c2 = fabs(g * pres / u1);
                if (c2 > max_c2) max_c2 = c2;
            } else {
                double vx = m->vx[idxM], vy = m->vy[idxM], vz = m->vz[idxM];
                double v2 = vx * vx + vy * vy + vz * vz;
                if (v2 > max_v2) max_v2 = v2;
            }
        }
        double mv = (m->physics == ORC_EULER) ? sqrt(max_v2) + sqrt(max_c2) : sqrt(max_v2);
        maxv[fidx] = mv;
        maxv_fs[fidx] = mv * m->Fscale[fidx];
    }
}

/* euler_dglm.cpp:53-69 */
double orc_calc_dt(const orc_mesh *m, const double *maxv_fs) {
    double max_v = 0;
#pragma omp parallel for reduction(max : max_v)
    for (long f = 0; f < (long)m->K * 4; f++)
        if (maxv_fs[f] > max_v) max_v = maxv_fs[f];
    return (m->cfl / (2 * m->N + 1)) * (1 / max_v);
}

/* euler_dglm.cpp:72-84 */
void orc_update_tau(const orc_mesh *m, const double *maxv, double *tau) {
#pragma omp parallel for
    for (long f = 0; f < (long)m->K * 4; f++)
        tau[f] = 0.25 * (maxv[f] + maxv[m->vmapF[f]]) * m->tau_scale;
}

/* euler_dglm.cpp:87-107 */
void orc_update_ub(const orc_mesh *m, const double *u, double *ub) {
    const long K = m->K, Np = m->Np, Nfp = m->Nfp, n = K * Np, nf = K * 4 * Nfp;
#pragma omp parallel for
    for (long idx = 0; idx < nf; idx++) {
        long ei = idx / (4 * Nfp), fi = (idx / Nfp) % 4;
        long idxM = ei * Np + m->Fmask[fi * Nfp + idx % Nfp];
        long idxP = m->vmapP[idx];
        for (int v = 0; v < m->nvar; v++)
            ub[v * nf + idx] = 0.5 * (u[v * n + idxM] + u[v * n + idxP]);
    }
}

/* Euler flux (F, G, W) of the state q, written as in euler_dglm.cpp:152-168.
 * vb2 is |m|^2 (momentum, not velocity), as in the reference. */
static inline void euler_flux(double g, const double q[5], double F[5], double G[5], double W[5]) {
    double u1 = q[0], u2 = q[1], u3 = q[2], u4 = q[3], u5 = q[4];
    double v2 = u2 * u2 + u3 * u3 + u4 * u4;
    F[0] = u2;
    F[1] = (u2 * u2) / u1 + (g - 1) * (u5 - 0.5 * v2 / u1);
    F[2] = (u2 * u3) / u1;
    F[3] = (u2 * u4) / u1;
    F[4] = (u5 + (g - 1) * (u5 - 0.5 * v2 / u1)) * (u2 / u1);
    G[0] = u3;
    G[1] = u2 * u3 / u1;
    G[2] = (u3 * u3) / u1 + (g - 1) * (u5 - 0.5 * v2 / u1);
    G[3] = u3 * u4 / u1;
    G[4] = (u5 + (g - 1) * (u5 - 0.5 * v2 / u1)) * (u3 / u1);
    W[0] = u4;
    W[1] = u2 * u4 / u1;
    W[2] = u3 * u4 / u1;
    W[3] = (u4 * u4) / u1 + (g - 1) * (u5 - 0.5 * v2 / u1);
    W[4] = (u5 + (g - 1) * (u5 - 0.5 * v2 / u1)) * (u4 / u1);
}

/* euler_dglm.cpp:110-183 and advec_dglm.cpp:88-133.  Faces with EtoB == 1
 * (Dirichlet) are an empty branch in the reference, which leaves the trace
 * uninitialised; here they use the stored trace ub like every other face. */
void orc_calc_fluxLM(const orc_mesh *m, const double *u, const double *ub, const double *tau,
                     double *fluxLM) {
    const long K = m->K, Np = m->Np, Nfp = m->Nfp, n = K * Np, nf = K * 4 * Nfp;
    const int nvar = m->nvar;
#pragma omp parallel for
    for (long fidx = 0; fidx < K * 4; fidx++) {
        double nx = m->nx[fidx], ny = m->ny[fidx], nz = m->nz[fidx], fs = m->Fscale[fidx];
        long ei = fidx / 4, fi = fidx % 4;
        for (long j = 0; j < Nfp; j++) {
            long idx = fidx * Nfp + j;
            long idxM = ei * Np + m->Fmask[fi * Nfp + j];
            if (m->physics == ORC_EULER) {
                double q[5], F[5], G[5], W[5];
                for (int v = 0; v < 5; v++) q[v] = ub[v * nf + idx];
                euler_flux(m->gamma, q, F, G, W);
                for (int v = 0; v < 5; v++) {
                    double nf_v = nx * F[v] + ny * G[v] + nz * W[v];
                    fluxLM[v * nf + idx] = (nf_v - tau[fidx] * (q[v] - u[v * n + idxM])) * fs;
                }
            } else {
                double b = ub[idx];
                double F = m->vx[idxM] * b, G = m->vy[idxM] * b, W = m->vz[idxM] * b;
                double nd = nx * F + ny * G + nz * W;
                fluxLM[idx] = (nd - tau[fidx] * (b - u[idxM])) * fs;
            }
        }
    }
    (void)nvar;
}

/* euler_dglm.cpp:186-251 and advec_dglm.cpp:136-169 */
void orc_calc_fluxes(const orc_mesh *m, const double *u, double *fR, double *fS, double *fT) {
    const long K = m->K, Np = m->Np, n = K * Np;
#pragma omp parallel for
    for (long ei = 0; ei < K; ei++) {
        double rx = m->rx[ei], ry = m->ry[ei], rz = m->rz[ei];
        double sx = m->sx[ei], sy = m->sy[ei], sz = m->sz[ei];
        double tx = m->tx[ei], ty = m->ty[ei], tz = m->tz[ei];
        for (long i = 0; i < Np; i++) {
            long idx = ei * Np + i;
            if (m->physics == ORC_EULER) {
                double q[5], F[5], G[5], W[5];
                for (int v = 0; v < 5; v++) q[v] = u[v * n + idx];
                euler_flux(m->gamma, q, F, G, W);
                for (int v = 0; v < 5; v++) {
                    fR[v * n + idx] = rx * F[v] + ry * G[v] + rz * W[v];
                    fS[v * n + idx] = sx * F[v] + sy * G[v] + sz * W[v];
                    fT[v * n + idx] = tx * F[v] + ty * G[v] + tz * W[v];
                }
            } else {
                double F = m->vx[idx] * u[idx], G = m->vy[idx] * u[idx], W = m->vz[idx] * u[idx];
                fR[idx] = rx * F + ry * G + rz * W;
                fS[idx] = sx * F + sy * G + sz * W;
                fT[idx] = tx * F + ty * G + tz * W;
            }
        }
    }
}

/* euler_dglm.cpp:254-302: utmp = WDr fR + WDs fS + WDt fT - LIFT fluxLM,
 * summed per output node in the reference's order. */
void orc_update_rhs(const orc_mesh *m, const double *fR, const double *fS, const double *fT,
                    const double *fLM, double *utmp) {
    const long K = m->K, Np = m->Np, NF = 4 * (long)m->Nfp, n = K * Np, nf = K * NF;
    const int nvar = m->nvar;
#pragma omp parallel for
    for (long ei = 0; ei < K; ei++) {
        for (long i = 0; i < Np; i++) {
            for (int v = 0; v < nvar; v++) {
                const double *r = fR + v * n + ei * Np, *s = fS + v * n + ei * Np;
                const double *t = fT + v * n + ei * Np, *l = fLM + v * nf + ei * NF;
                double rhs = 0;
                for (long j = 0; j < Np; j++)
                    rhs += m->WDr[i * Np + j] * r[j] + m->WDs[i * Np + j] * s[j] +
                           m->WDt[i * Np + j] * t[j];
                for (long j = 0; j < NF; j++) rhs -= m->LIFT[i * NF + j] * l[j];
                utmp[v * n + ei * Np + i] = rhs;
            }
        }
    }
}

/* euler_time.cpp:15-38 */
void orc_lserk_stage(const orc_mesh *m, double dt, double a, double b, const double *utmp,
                     double *k, double *u) {
    const long n = (long)m->nvar * m->K * m->Np;
#pragma omp parallel for
    for (long idx = 0; idx < n; idx++) {
        k[idx] = a * k[idx] + dt * utmp[idx];
        u[idx] += b * k[idx];
    }
}

static void *xmalloc(size_t n) {
    void *p = malloc(n ? n : 1);
    return p;
}

/* One right-hand side with dt/tau taken from the state (maxv, dt, tau, ub,
 * fluxLM, fluxes, utmp); every out-pointer may be NULL except utmp. */
double orc_rhs(const orc_mesh *m, const double *u, double *maxv, double *tau, double *ub,
               double *fluxLM, double *fR, double *fS, double *fT, double *utmp) {
    const size_t nF = (size_t)m->K * 4, nT = (size_t)m->nvar * m->K * 4 * m->Nfp;
    const size_t nV = (size_t)m->nvar * m->K * m->Np;
    double *own[7] = {0};
    if (!maxv) maxv = own[0] = xmalloc(nF * 8);
    if (!tau) tau = own[1] = xmalloc(nF * 8);
    if (!ub) ub = own[2] = xmalloc(nT * 8);
    if (!fluxLM) fluxLM = own[3] = xmalloc(nT * 8);
    if (!fR) fR = own[4] = xmalloc(nV * 8);
    if (!fS) fS = own[5] = xmalloc(nV * 8);
    if (!fT) fT = own[6] = xmalloc(nV * 8);
    double *maxv_fs = xmalloc(nF * 8);
    orc_calc_maxv(m, u, maxv, maxv_fs);
    double dt = orc_calc_dt(m, maxv_fs);
    orc_update_tau(m, maxv, tau);
    orc_update_ub(m, u, ub);
    orc_calc_fluxLM(m, u, ub, tau, fluxLM);
    orc_calc_fluxes(m, u, fR, fS, fT);
    orc_update_rhs(m, fR, fS, fT, fluxLM, utmp);
    free(maxv_fs);
    for (int i = 0; i < 7; i++) free(own[i]);
    return dt;
}

/* euler_time.cpp:41-107 (runRK) for nsteps steps, stopping once t reaches
 * tmax.  u (state) and k (RK register) are updated in place; clk carries t,
 * the last dt and the step counter.  When dt_fixed > 0 it replaces the CFL
 * dt (the TMAX clip still applies).  dt_hist, if not NULL, receives the dt
 * of each step taken.  Returns the number of steps taken. */
int orc_run(const orc_mesh *m, double *u, double *k, orc_clock *clk, int nsteps, double dt_fixed,
            double *dt_hist) {
    const size_t nF = (size_t)m->K * 4, nT = (size_t)m->nvar * m->K * 4 * m->Nfp;
    const size_t nV = (size_t)m->nvar * m->K * m->Np;
    double *maxv = xmalloc(nF * 8), *maxv_fs = xmalloc(nF * 8), *tau = xmalloc(nF * 8);
    double *ub = xmalloc(nT * 8), *fLM = xmalloc(nT * 8);
    double *fR = xmalloc(nV * 8), *fS = xmalloc(nV * 8), *fT = xmalloc(nV * 8);
    double *utmp = xmalloc(nV * 8);
    int done = 0;
    for (; done < nsteps && clk->t < m->tmax; done++) {
        orc_calc_maxv(m, u, maxv, maxv_fs);
        double dt = dt_fixed > 0 ? dt_fixed : orc_calc_dt(m, maxv_fs);
        if (clk->t + dt > m->tmax) {
            dt = m->tmax - clk->t;
            clk->last = 1;
        }
        orc_update_tau(m, maxv, tau);
        for (int s = 0; s < 5; s++) {
            orc_update_ub(m, u, ub);
            orc_calc_fluxLM(m, u, ub, tau, fLM);
            orc_calc_fluxes(m, u, fR, fS, fT);
            orc_update_rhs(m, fR, fS, fT, fLM, utmp);
            orc_lserk_stage(m, dt, RKA[s], RKB[s], utmp, k, u);
        }
        if (dt_hist) dt_hist[done] = dt;
        clk->dt = dt;
        clk->t += dt;
        clk->tstep += 1;
    }
    free(maxv); free(maxv_fs); free(tau); free(ub); free(fLM);
    free(fR); free(fS); free(fT); free(utmp);
    return done;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---------------------------------------------------------------------------
 * Discrete adjoint (test infrastructure): the transpose of the derivative of
 * runRK with dt and tau frozen (recorded in the forward run and replayed),
 * for checking the GPU adjoint.  The reference has no adjoint; this is the
 * exact derivative of the oracle's own step above.
 * ------------------------------------------------------------------------- */

/* w = A_n(q)^T g for the Euler flux in direction n (the Jacobian of
 * F.n with p = (gamma-1)(E - |m|^2/(2 rho)), the reference's flux). */
static void euler_jac_t(double gm, const double q[5], const double n[3], const double g[5],
                        double w[5]) {
    double ir = 1.0 / q[0], u[3] = {q[1] * ir, q[2] * ir, q[3] * ir};
    double q2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    double p = (gm - 1) * (q[4] - 0.5 * q[0] * q2);
    double H = (q[4] + p) * ir;
    double un = u[0] * n[0] + u[1] * n[1] + u[2] * n[2];
    double gu = g[1] * u[0] + g[2] * u[1] + g[3] * u[2];
    double gn = g[1] * n[0] + g[2] * n[1] + g[3] * n[2];
    double phi = 0.5 * (gm - 1) * q2;
    w[0] = -un * gu + phi * gn + g[4] * un * (phi - H);
    for (int j = 0; j < 3; j++)
        w[1 + j] = g[0] * n[j] + un * g[1 + j] + gu * n[j] - (gm - 1) * gn * u[j] +
                   g[4] * (H * n[j] - (gm - 1) * un * u[j]);
    w[4] = (gm - 1) * gn + gm * un * g[4];
}

/* lam += R'(u)^T mu with tau frozen. */
void orc_rhs_adjoint(const orc_mesh *m, const double *u, const double *tau, const double *mu,
                     double *lam) {
    const long K = m->K, Np = m->Np, Nfp = m->Nfp, NF = 4 * Nfp, n = K * Np;
    const int nv = m->nvar;
    double *nu = malloc(sizeof(double) * 3 * Np * nv), *phi = malloc(sizeof(double) * NF * nv);
    for (long e = 0; e < K; e++) {
        /* nu_d = WD_d^T mu, phi = -LIFT^T mu (per variable) */
        for (int v = 0; v < nv; v++) {
            const double *mv = mu + v * n + e * Np;
            for (long j = 0; j < Np; j++) {
                double a0 = 0, a1 = 0, a2 = 0;
                for (long i = 0; i < Np; i++) {
                    a0 += m->WDr[i * Np + j] * mv[i];
                    a1 += m->WDs[i * Np + j] * mv[i];
                    a2 += m->WDt[i * Np + j] * mv[i];
                }
                nu[(v * 3 + 0) * Np + j] = a0;
                nu[(v * 3 + 1) * Np + j] = a1;
                nu[(v * 3 + 2) * Np + j] = a2;
            }
            for (long f = 0; f < NF; f++) {
                double s = 0;
                for (long i = 0; i < Np; i++) s -= m->LIFT[i * NF + f] * mv[i];
                phi[v * NF + f] = s;
            }
        }
        /* volume: lam_j += sum_x A_x(u_j)^T G_x, G_x = r_x nu_r + s_x nu_s + t_x nu_t */
        const double mt[3][3] = {{m->rx[e], m->ry[e], m->rz[e]},
                                 {m->sx[e], m->sy[e], m->sz[e]},
                                 {m->tx[e], m->ty[e], m->tz[e]}};
        for (long j = 0; j < Np; j++) {
            long idx = e * Np + j;
            for (int x = 0; x < 3; x++) {
                double G[5];
                for (int v = 0; v < nv; v++)
                    G[v] = mt[0][x] * nu[(v * 3 + 0) * Np + j] + mt[1][x] * nu[(v * 3 + 1) * Np + j] +
                           mt[2][x] * nu[(v * 3 + 2) * Np + j];
                if (m->physics == ORC_EULER) {
                    double q[5], w[5], dir[3] = {0, 0, 0};
                    dir[x] = 1;
                    for (int v = 0; v < 5; v++) q[v] = u[v * n + idx];
                    euler_jac_t(m->gamma, q, dir, G, w);
                    for (int v = 0; v < 5; v++) lam[v * n + idx] += w[v];
                } else {
                    const double *vel = x == 0 ? m->vx : x == 1 ? m->vy : m->vz;
                    lam[idx] += vel[idx] * G[0];
                }
            }
        }
        /* faces: d fluxLM/du- = fs (A_n(ub)/2 + tau/2), d fluxLM/du+ = fs (A_n(ub)/2 - tau/2) */
        for (long fj = 0; fj < NF; fj++) {
            long f = fj / Nfp, gf = e * 4 + f, idx = e * NF + fj;
            long iM = e * Np + m->Fmask[fj], iP = m->vmapP[idx];
            double fs = m->Fscale[gf], ta = tau[gf];
            double nrm[3] = {m->nx[gf], m->ny[gf], m->nz[gf]};
            if (m->physics == ORC_EULER) {
                double qb[5], g[5], w[5];
                for (int v = 0; v < 5; v++) {
                    qb[v] = 0.5 * (u[v * n + iM] + u[v * n + iP]);
                    g[v] = phi[v * NF + fj];
                }
                euler_jac_t(m->gamma, qb, nrm, g, w);
                for (int v = 0; v < 5; v++) {
                    lam[v * n + iM] += fs * (0.5 * w[v] + 0.5 * ta * g[v]);
                    lam[v * n + iP] += fs * (0.5 * w[v] - 0.5 * ta * g[v]);
                }
            } else {
                double an = nrm[0] * m->vx[iM] + nrm[1] * m->vy[iM] + nrm[2] * m->vz[iM];
                double g = phi[fj];
                lam[iM] += fs * (0.5 * an + 0.5 * ta) * g;
                lam[iP] += fs * (0.5 * an - 0.5 * ta) * g;
            }
        }
    }
    free(nu);
    free(phi);
}

/* One LSERK step from u with the given dt and tau (no tmax clipping);
 * stage_in (5 states) receives the input state of every stage. */
static void frozen_step(const orc_mesh *m, double *u, double *k, double dt, const double *tau,
                        double *stage_in) {
    const size_t nV = (size_t)m->nvar * m->K * m->Np, nT = (size_t)m->nvar * m->K * 4 * m->Nfp;
    double *ub = xmalloc(nT * 8), *fLM = xmalloc(nT * 8), *fR = xmalloc(nV * 8),
           *fS = xmalloc(nV * 8), *fT = xmalloc(nV * 8), *ut = xmalloc(nV * 8);
    for (int s = 0; s < 5; s++) {
        if (stage_in) memcpy(stage_in + s * nV, u, nV * 8);
        orc_update_ub(m, u, ub);
        orc_calc_fluxLM(m, u, ub, tau, fLM);
        orc_calc_fluxes(m, u, fR, fS, fT);
        orc_update_rhs(m, fR, fS, fT, fLM, ut);
        orc_lserk_stage(m, dt, RKA[s], RKB[s], ut, k, u);
    }
    free(ub); free(fLM); free(fR); free(fS); free(fT); free(ut);
}

/* Forward run recording dt and tau of every step (tau_hist: nsteps x 4K). */
int orc_run_record(const orc_mesh *m, double *u, double *k, int nsteps, double *dt_hist,
                   double *tau_hist) {
    const size_t nF = (size_t)m->K * 4;
    double *maxv = xmalloc(nF * 8), *maxv_fs = xmalloc(nF * 8);
    for (int st = 0; st < nsteps; st++) {
        orc_calc_maxv(m, u, maxv, maxv_fs);
        dt_hist[st] = orc_calc_dt(m, maxv_fs);
        orc_update_tau(m, maxv, tau_hist + st * nF);
        frozen_step(m, u, k, dt_hist[st], tau_hist + st * nF, NULL);
    }
    free(maxv); free(maxv_fs);
    return nsteps;
}

/* Forward run replaying recorded dt and tau. */
void orc_run_frozen(const orc_mesh *m, double *u, double *k, int nsteps, const double *dt_hist,
                    const double *tau_hist) {
    const size_t nF = (size_t)m->K * 4;
    for (int st = 0; st < nsteps; st++) frozen_step(m, u, k, dt_hist[st], tau_hist + st * nF, NULL);
}

/* Reverse sweep: lam holds dJ/du(T) on entry and dJ/du(0) on return, for the
 * frozen run of nsteps from u0. */
void orc_adjoint(const orc_mesh *m, const double *u0, int nsteps, const double *dt_hist,
                 const double *tau_hist, double *lam) {
    const size_t nV = (size_t)m->nvar * m->K * m->Np, nF = (size_t)m->K * 4;
    double *starts = xmalloc(nV * 8 * (size_t)nsteps), *u = xmalloc(nV * 8), *k = xmalloc(nV * 8);
    double *stage_in = xmalloc(nV * 8 * 5), *lk = xmalloc(nV * 8), *mu = xmalloc(nV * 8);
    memcpy(u, u0, nV * 8);
    memset(k, 0, nV * 8);
    for (int st = 0; st < nsteps; st++) {
        memcpy(starts + st * nV, u, nV * 8);
        frozen_step(m, u, k, dt_hist[st], tau_hist + st * nF, NULL);
    }
    for (int st = nsteps - 1; st >= 0; st--) {
        memcpy(u, starts + st * nV, nV * 8);
        memset(k, 0, nV * 8);      /* k is reset by rka[0] = 0 */
        frozen_step(m, u, k, dt_hist[st], tau_hist + st * nF, stage_in);
        memset(lk, 0, nV * 8);
        for (int s = 4; s >= 0; s--) {
            for (size_t i = 0; i < nV; i++) mu[i] = lk[i] + RKB[s] * lam[i];
            for (size_t i = 0; i < nV; i++) lk[i] = RKA[s] * mu[i];
            for (size_t i = 0; i < nV; i++) mu[i] *= dt_hist[st];
            orc_rhs_adjoint(m, stage_in + s * nV, tau_hist + st * nF, mu, lam);
        }
    }
    free(starts); free(u); free(k); free(stage_in); free(lk); free(mu);
}
