// Per-kernel entry points: one C function per reference kernel, with the
// reference's argument meaning, on caller-owned device arrays.  They keep the
// reference's decomposition (one launch per kernel, intermediates in HBM) and
// exist so each piece of the fused stage can be checked on its own; the
// solver handle never uses them.
//
// Per-variable pointer tables come in as HOST arrays of device pointers (the
// reference's p_u vectors) and are passed to the kernels by value.
#include <cuda_runtime.h>

#include <cmath>

#include "dglm_common.cuh"

namespace dglm {
namespace {

struct P5 {
  const double *p[5];
};
struct W5 {
  double *p[5];
};

inline P5 pack(const double *const *src, int nvar) {
  P5 r{};
  for (int v = 0; v < nvar; v++) r.p[v] = src[v];
  return r;
}
inline W5 packw(double *const *src, int nvar) {
  W5 r{};
  for (int v = 0; v < nvar; v++) r.p[v] = src[v];
  return r;
}

inline unsigned blocks_for(long n, int tpb) { return (unsigned)((n + tpb - 1) / tpb); }

bool bad_order(int N) { return N < 1 || N > kMaxOrder; }

// euler_nopad_dglm.cu:7-76 / advec_nopad_dglm.cu:7-62 (one thread per face;
// the reference's shared-memory tree has an early return before a barrier)
__global__ void calc_maxv_k(int physics, int Np, int Nfp, long nfaces, double gamma,
                            const int *__restrict__ Fmask, const double *__restrict__ Fscale,
                            P5 u, const double *vx, const double *vy, const double *vz,
                            double *maxv, double *maxv_fs) {
  const long f = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (f >= nfaces) return;
  const double mv = face_max_speed(physics, Np, Nfp, gamma, Fmask, u, vx, vy, vz, f / 4,
                                   (int)(f % 4));
  maxv[f] = mv;
  maxv_fs[f] = mv * Fscale[f];
}

// euler_nopad_dglm.cu:79-96 without the host round trip: one CTA reduces
// and writes dt to device memory.
__global__ void calc_dt_k(int N, long n, double cfl, const double *__restrict__ maxv_fs,
                          double *dt) {
  __shared__ unsigned long long s[32];
  unsigned long long b = 0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) {
    const unsigned long long x = dbits(maxv_fs[i]);
    b = x > b ? x : b;
  }
  b = warp_max_bits(b);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = b;
  __syncthreads();
  if (threadIdx.x < 32) {
    b = threadIdx.x < blockDim.x / 32 ? s[threadIdx.x] : 0ull;
    b = warp_max_bits(b);
    if (threadIdx.x == 0) {
      const double m = __longlong_as_double((long long)b);
      *dt = (cfl / (2 * N + 1)) * (1 / m);
    }
  }
}

__global__ void update_tau_k(long nfaces, double tau_scale, const int *__restrict__ vmapF,
                             const double *__restrict__ maxv, double *tau) {
  const long f = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (f < nfaces) tau[f] = 0.25 * (maxv[f] + maxv[vmapF[f]]) * tau_scale;
}

// euler_nopad_dglm.cu:115-135
__global__ void update_ub_k(int Np, int Nfp, int nvar, long n, const int *__restrict__ Fmask,
                            const int *__restrict__ vmapP, P5 u, W5 ub) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const long e = idx / (4 * Nfp);
  const long fj = idx % (4 * Nfp);
  const long iM = e * Np + Fmask[fj];
  const long iP = vmapP[idx];
  for (int v = 0; v < nvar; v++) ub.p[v][idx] = 0.5 * (u.p[v][iM] + u.p[v][iP]);
}

// euler_nopad_dglm.cu:138-210 / advec_nopad_dglm.cu:120-165
__global__ void calc_fluxLM_k(int physics, int Np, int Nfp, long n, double gamma,
                              const int *__restrict__ Fmask, const double *nx, const double *ny,
                              const double *nz, const double *tau, const double *Fscale,
                              const double *vx, const double *vy, const double *vz, P5 ub, P5 u,
                              W5 flm) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const long e = idx / (4 * Nfp);
  const long fj = idx % (4 * Nfp);
  const long f = e * 4 + fj / Nfp;
  const long iM = e * Np + Fmask[fj];
  const double fs = Fscale[f], ta = tau[f];
  if (physics == DGLM_EULER) {
    double q[5], F[5], G[5], W[5];
    for (int v = 0; v < 5; v++) q[v] = ub.p[v][idx];
    euler_flux(gamma, q, F, G, W);
    for (int v = 0; v < 5; v++) {
      const double nd = nx[f] * F[v] + ny[f] * G[v] + nz[f] * W[v];
      flm.p[v][idx] = (nd - ta * (q[v] - u.p[v][iM])) * fs;
    }
  } else {
    const double b = ub.p[0][idx];
    const double nd = nx[f] * (vx[iM] * b) + ny[f] * (vy[iM] * b) + nz[f] * (vz[iM] * b);
    flm.p[0][idx] = (nd - ta * (b - u.p[0][iM])) * fs;
  }
}

struct Geo9 {
  const double *g[9];
};

// euler_nopad_dglm.cu:213-266 / advec_nopad_dglm.cu:168-189
__global__ void calc_fluxes_k(int physics, int Np, long n, double gamma, Geo9 geo,
                              const double *vx, const double *vy, const double *vz, P5 u, W5 fR,
                              W5 fS, W5 fT) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const long e = idx / Np;
  double g[9];
  for (int m = 0; m < 9; m++) g[m] = geo.g[m][e];
  if (physics == DGLM_EULER) {
    double q[5], F[5], G[5], W[5];
    for (int v = 0; v < 5; v++) q[v] = u.p[v][idx];
    euler_flux(gamma, q, F, G, W);
    for (int v = 0; v < 5; v++) {
      fR.p[v][idx] = g[0] * F[v] + g[1] * G[v] + g[2] * W[v];
      fS.p[v][idx] = g[3] * F[v] + g[4] * G[v] + g[5] * W[v];
      fT.p[v][idx] = g[6] * F[v] + g[7] * G[v] + g[8] * W[v];
    }
  } else {
    const double uu = u.p[0][idx];
    const double F = vx[idx] * uu, G = vy[idx] * uu, W = vz[idx] * uu;
    fR.p[0][idx] = g[0] * F + g[1] * G + g[2] * W;
    fS.p[0][idx] = g[3] * F + g[4] * G + g[5] * W;
    fT.p[0][idx] = g[6] * F + g[7] * G + g[8] * W;
  }
}

// euler_nopad_dglm.cu:269-300: one thread per output (var, node).
__global__ void update_rhs_k(int Np, int NF, long nnodes, int nvar, const double *WDr,
                             const double *WDs, const double *WDt, const double *LIFT,
                             int col_major, P5 fR, P5 fS, P5 fT, P5 fLM, W5 ut) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= nnodes * nvar) return;
  const int v = (int)(idx / nnodes);
  const long n = idx % nnodes;
  const long e = n / Np;
  const int i = (int)(n % Np);
  const double *r = fR.p[v] + e * Np, *s = fS.p[v] + e * Np, *t = fT.p[v] + e * Np;
  const double *l = fLM.p[v] + e * NF;
  double acc = 0;
  for (int j = 0; j < Np; j++) {
    const long a = col_major ? (long)j * Np + i : (long)i * Np + j;
    acc += WDr[a] * r[j] + WDs[a] * s[j] + WDt[a] * t[j];
  }
  for (int j = 0; j < NF; j++) {
    const long a = col_major ? (long)j * Np + i : (long)i * NF + j;
    acc -= LIFT[a] * l[j];
  }
  ut.p[v][n] = acc;
}

// euler_nopad_time.cu:15-29
__global__ void lserk_k(long n, int nvar, double dt, double a, double b, P5 ut, W5 k, W5 u) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= n) return;
  for (int v = 0; v < nvar; v++) {
    const double kn = a * k.p[v][idx] + dt * ut.p[v][idx];
    k.p[v][idx] = kn;
    u.p[v][idx] += b * kn;
  }
}

dglm_status launched(const char *what) { return cuda_check(cudaGetLastError(), what); }

}  // namespace
}  // namespace dglm

using namespace dglm;

extern "C" {

dglm_status dglm_calc_maxv(int physics, int N, int nelem, double gamma, const int *Fmask,
                           const double *Fscale, const double *const *u, const double *vx,
                           const double *vy, const double *vz, double *maxv, double *maxv_fs,
                           void *stream) {
  if (bad_order(N) || nelem < 0 || !Fmask || !Fscale || !maxv || !maxv_fs)
    return set_error(DGLM_ERR_INVALID, "dglm_calc_maxv: bad argument");
  P5 up{};
  if (physics == DGLM_EULER) {
    if (!u) return set_error(DGLM_ERR_INVALID, "dglm_calc_maxv: u is NULL");
    up = pack(u, 5);
  } else if (!vx || !vy || !vz) {
    return set_error(DGLM_ERR_INVALID, "dglm_calc_maxv: velocity is NULL");
  }
  const long nf = 4L * nelem;
  if (nf == 0) return DGLM_OK;
  calc_maxv_k<<<blocks_for(nf, 256), 256, 0, (cudaStream_t)stream>>>(
      physics, np_of(N), nfp_of(N), nf, gamma, Fmask, Fscale, up, vx, vy, vz, maxv, maxv_fs);
  return launched("calc_maxv");
}

dglm_status dglm_calc_dt(int N, int nelem, double cfl, const double *maxv_fs, double *dt_dev,
                         void *stream) {
  if (bad_order(N) || nelem <= 0 || !maxv_fs || !dt_dev)
    return set_error(DGLM_ERR_INVALID, "dglm_calc_dt: bad argument");
  calc_dt_k<<<1, 1024, 0, (cudaStream_t)stream>>>(N, 4L * nelem, cfl, maxv_fs, dt_dev);
  return launched("calc_dt");
}

dglm_status dglm_update_tau(int nelem, double tau_scale, const int *vmapF, const double *maxv,
                            double *tau, void *stream) {
  if (nelem < 0 || !vmapF || !maxv || !tau)
    return set_error(DGLM_ERR_INVALID, "dglm_update_tau: bad argument");
  const long nf = 4L * nelem;
  if (nf == 0) return DGLM_OK;
  update_tau_k<<<blocks_for(nf, 256), 256, 0, (cudaStream_t)stream>>>(nf, tau_scale, vmapF,
                                                                       maxv, tau);
  return launched("update_tau");
}

dglm_status dglm_update_ub(int N, int nvar, int nelem, const int *Fmask, const int *vmapP,
                           const double *const *u, double *const *ub, void *stream) {
  if (bad_order(N) || (nvar != 1 && nvar != 5) || nelem < 0 || !Fmask || !vmapP || !u || !ub)
    return set_error(DGLM_ERR_INVALID, "dglm_update_ub: bad argument");
  const long n = 4L * nelem * nfp_of(N);
  if (n == 0) return DGLM_OK;
  update_ub_k<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
      np_of(N), nfp_of(N), nvar, n, Fmask, vmapP, pack(u, nvar), packw(ub, nvar));
  return launched("update_ub");
}

dglm_status dglm_calc_fluxLM(int physics, int N, int nelem, double gamma, const int *Fmask,
                             const double *nx, const double *ny, const double *nz,
                             const double *tau, const double *Fscale, const double *vx,
                             const double *vy, const double *vz, const double *const *ub,
                             const double *const *u, double *const *fluxLM, void *stream) {
  const int nvar = physics == DGLM_EULER ? 5 : 1;
  if (bad_order(N) || nelem < 0 || !Fmask || !nx || !ny || !nz || !tau || !Fscale || !ub || !u ||
      !fluxLM || (physics != DGLM_EULER && (!vx || !vy || !vz)))
    return set_error(DGLM_ERR_INVALID, "dglm_calc_fluxLM: bad argument");
  const long n = 4L * nelem * nfp_of(N);
  if (n == 0) return DGLM_OK;
  calc_fluxLM_k<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
      physics, np_of(N), nfp_of(N), n, gamma, Fmask, nx, ny, nz, tau, Fscale, vx, vy, vz,
      pack(ub, nvar), pack(u, nvar), packw(fluxLM, nvar));
  return launched("calc_fluxLM");
}

dglm_status dglm_calc_fluxes(int physics, int N, int nelem, double gamma,
                             const double *const *geo, const double *vx, const double *vy,
                             const double *vz, const double *const *u, double *const *fluxR,
                             double *const *fluxS, double *const *fluxT, void *stream) {
  const int nvar = physics == DGLM_EULER ? 5 : 1;
  if (bad_order(N) || nelem < 0 || !geo || !u || !fluxR || !fluxS || !fluxT ||
      (physics != DGLM_EULER && (!vx || !vy || !vz)))
    return set_error(DGLM_ERR_INVALID, "dglm_calc_fluxes: bad argument");
  Geo9 g{};
  for (int m = 0; m < 9; m++) g.g[m] = geo[m];
  const long n = (long)nelem * np_of(N);
  if (n == 0) return DGLM_OK;
  calc_fluxes_k<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
      physics, np_of(N), n, gamma, g, vx, vy, vz, pack(u, nvar), packw(fluxR, nvar),
      packw(fluxS, nvar), packw(fluxT, nvar));
  return launched("calc_fluxes");
}

dglm_status dglm_update_rhs(int N, int nvar, int nelem, const double *WDr, const double *WDs,
                            const double *WDt, const double *LIFT, char matrix_order,
                            const double *const *fluxR, const double *const *fluxS,
                            const double *const *fluxT, const double *const *fluxLM,
                            double *const *utmp, void *stream) {
  if (bad_order(N) || (nvar != 1 && nvar != 5) || nelem < 0 || !WDr || !WDs || !WDt || !LIFT ||
      !fluxR || !fluxS || !fluxT || !fluxLM || !utmp ||
      (matrix_order != 'c' && matrix_order != 'f'))
    return set_error(DGLM_ERR_INVALID, "dglm_update_rhs: bad argument");
  const long nn = (long)nelem * np_of(N);
  if (nn == 0) return DGLM_OK;
  update_rhs_k<<<blocks_for(nn * nvar, 128), 128, 0, (cudaStream_t)stream>>>(
      np_of(N), 4 * nfp_of(N), nn, nvar, WDr, WDs, WDt, LIFT, matrix_order == 'f',
      pack(fluxR, nvar), pack(fluxS, nvar), pack(fluxT, nvar), pack(fluxLM, nvar),
      packw(utmp, nvar));
  return launched("update_rhs");
}

dglm_status dglm_lserk_stage(int N, int nvar, int nelem, double dt, double rka, double rkb,
                             const double *const *utmp, double *const *k, double *const *u,
                             void *stream) {
  if (bad_order(N) || (nvar != 1 && nvar != 5) || nelem < 0 || !utmp || !k || !u)
    return set_error(DGLM_ERR_INVALID, "dglm_lserk_stage: bad argument");
  const long n = (long)nelem * np_of(N);
  if (n == 0) return DGLM_OK;
  lserk_k<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
      n, nvar, dt, rka, rkb, pack(utmp, nvar), packw(k, nvar), packw(u, nvar));
  return launched("lserk_stage");
}

}  // extern "C"
