// Discrete adjoint of the DGLM right-hand side and of the LSERK step.
//
// The reference has no adjoint; this is the exact transpose of the
// derivative of this library's own forward step with the step size dt and
// the face penalty tau frozen at the values of the forward run (both are
// non-smooth functions of u: a global max and a per-face max).
//
// One LSERK stage s maps (u, k) to
//     k' = a_s k + dt R(u),   u' = u + b_s k'.
// Its transpose, for adjoints (lam, lk) of (u', k'), is
//     mu  = lk + b_s lam
//     lk  = a_s mu
//     lam = lam + dt R'(u)^T mu
// and a step is the five stages in reverse order.  R = WD_d (geo.F) - LIFT
// fluxLM, so with phi = -LIFT^T mu (a face-point field):
//   volume: lam_j += sum_x A_x(u_j)^T G_x,  G_x = sum_d geo[d][x] (WD_d^T mu)_j
//   faces:  for face point p with own node M(p) and partner node P(p)
//           d fluxLM_p/du_M = fs (A_n(ub)/2 + tau/2),
//           d fluxLM_p/du_P = fs (A_n(ub)/2 - tau/2).
// The second term scatters to the neighbour.  On a conforming mesh the face
// points pair up (mapP: the partner face point p' with vmapP[p'] == M(p), an
// involution), so node M(p) gathers it from p' instead:
//   lam_M += fs (A_n^T phi_p + tau phi_p)/2 + fs' (A_n'^T phi_p' - tau' phi_p')/2
// with fs', n', tau' the partner face's values.  No atomics.
//
// Kernel layout.  phi of a stage is needed by the neighbours, so it is
// produced one launch ahead: the launch for stage s reads phi_s (phi_in),
// updates lam and lk, then forms mu of the next stage in reverse order and
// writes phi of it (phi_out).  One launch per adjoint stage plus one
// phi-only launch at the start of a sweep.
//
// A CTA owns E elements.  Both contractions are register-tiled DFMA over the
// k = Np nodes with the output rows interleaved so that a thread ends with
// everything one node needs: rows (3j + d) of [WD_r^T; WD_s^T; WD_t^T] for
// RJ nodes j and all NV variables of one element, so the Euler Jacobian
// transposes run in registers on the contraction's output.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dglm_common.cuh"
#include "dglm_handle.cuh"

namespace dglm {

struct AdjArgs {
  const double *AV;      // [Np][IPV]: AV[i*IPV + 3j + d] = WD_d(i, j)
  const double *AL;      // [Np][IPL]: AL[i*IPL + fj] = -LIFT(i, fj)
  const double *geo;     // 9 x gstride
  const double *fscale;  // 4 K
  const double *nrm;     // 3 x 4 gstride
  const double *tau;     // 4 K (frozen)
  const int *vmapP;      // K NFF
  const int *vmapF;      // 4 K
  const int *mapP;       // K NFF: partner face point
  const int *Fmask;      // NFF
  const double *vel;     // advection velocity, stride vs
  const double *u;       // state at the stage's input
  double *lam, *lk;      // adjoints of u and k (updated in place, own tile only)
  const double *phi_in;  // phi of this stage, nvar x vsF
  double *phi_out;       // phi of the next stage in reverse order
  double *fw;            // face terms of this stage (split variants), nvar x vsF
  long vs, vsF, gstride;
  int K;
  double gamma, dt, rka, rkb, rkb_next;
  int update;            // 1: apply the stage's transpose; 0: only form phi_out
  int phi_next;          // 1: write phi_out
};

enum { A_ADV = 0, A_EUL = 1 };

template <int PHYS, int N, int E_, int MINB_ = 1>
struct ACfg {
  static constexpr int NV = PHYS == A_EUL ? 5 : 1;
  static constexpr int Np = np_of(N), Nfp = nfp_of(N), NFF = 4 * Nfp;
  static constexpr int E = E_, EP = E_ + 1;
  static constexpr int RJ = (E * Np + 767) / 768;     // nodes per thread
  static constexpr int G = (Np + RJ - 1) / RJ;        // row groups
  static constexpr int T = E * G;                     // threads
  static constexpr int RF = (NFF + G - 1) / G;        // lift rows per thread
  static constexpr int IPV = 3 * G * RJ, IPL = G * RF;
  static constexpr int BLD = NV * E;
  static constexpr int VMLD = NFF + 1;
  static constexpr int S_U = NV * Np * EP, S_MU = Np * BLD, S_FC = NV * NFF * EP;
  static constexpr size_t SMEM =
      sizeof(double) * (2 * S_U + S_MU + S_FC + 9 * E + 40 * E) +
      sizeof(int) * (2 * E * VMLD + NFF + 4 * Np);
  static_assert(T <= 1024, "block too large");
};

// Shared part of A_n(q)^T for the Euler flux with p = (gamma-1)(E - |m|^2/(2 rho)).
struct JacPre {
  double u[3], H, phi;
};

__device__ __forceinline__ JacPre jac_pre(double gm, const double q[5]) {
  JacPre P;
  const double ir = 1.0 / q[0];
  P.u[0] = q[1] * ir;
  P.u[1] = q[2] * ir;
  P.u[2] = q[3] * ir;
  const double q2 = P.u[0] * P.u[0] + P.u[1] * P.u[1] + P.u[2] * P.u[2];
  const double p = (gm - 1) * (q[4] - 0.5 * q[0] * q2);
  P.H = (q[4] + p) * ir;
  P.phi = 0.5 * (gm - 1) * q2;
  return P;
}

// w += s * A_n(q)^T g
__device__ __forceinline__ void jac_t_add(const JacPre &P, double gm, double nx, double ny,
                                          double nz, const double g[5], double s, double w[5]) {
  const double un = P.u[0] * nx + P.u[1] * ny + P.u[2] * nz;
  const double gu = g[1] * P.u[0] + g[2] * P.u[1] + g[3] * P.u[2];
  const double gn = g[1] * nx + g[2] * ny + g[3] * nz;
  const double n3[3] = {nx, ny, nz};
  w[0] += s * (-un * gu + P.phi * gn + g[4] * un * (P.phi - P.H));
#pragma unroll
  for (int j = 0; j < 3; j++)
    w[1 + j] += s * (g[0] * n3[j] + un * g[1 + j] + gu * n3[j] - (gm - 1) * gn * P.u[j] +
                     g[4] * (P.H * n3[j] - (gm - 1) * un * P.u[j]));
  w[4] += s * ((gm - 1) * gn + gm * un * g[4]);
}

template <int PHYS, int N, int E_, int MINB>
__global__ void __launch_bounds__(ACfg<PHYS, N, E_>::T, MINB)
    adjoint_stage_kernel(const AdjArgs a) {
  using C = ACfg<PHYS, N, E_>;
  constexpr int NV = C::NV, Np = C::Np, Nfp = C::Nfp, NFF = C::NFF, E = C::E, EP = C::EP,
                BLD = C::BLD, T = C::T, RJ = C::RJ, RF = C::RF, VMLD = C::VMLD;
  extern __shared__ __align__(16) double smem[];
  double *sU = smem;                   // [v][i][EP] stage state, later lk'
  double *sLam = sU + C::S_U;          // [v][i][EP]
  double *sMu = sLam + C::S_U;         // [i][BLD], col = v*E + e
  double *sFc = sMu + C::S_MU;         // [v][fj][EP] face terms, later phi'
  double *sGeo = sFc + C::S_FC;        // [9][E]
  double *sFace = sGeo + 9 * E;        // [10][4][E]: n fs tau, partner n fs tau
  int *sVm = reinterpret_cast<int *>(sFace + 40 * E);   // [E][VMLD]
  int *sMp = sVm + E * VMLD;           // [E][VMLD]
  int *sFm = sMp + E * VMLD;           // [NFF]
  int *sNF = sFm + NFF;                // [Np][4] face points of each node

  const int tid = threadIdx.x;
  const long e0 = (long)blockIdx.x * E;
  const int ne = (int)min((long)E, (long)a.K - e0);
  const long vs = a.vs, vsF = a.vsF;
  const bool upd = a.update != 0;

  // ---- staging ------------------------------------------------------------
  for (int i = tid; i < NFF; i += T) sFm[i] = __ldg(a.Fmask + i);
  for (int i = tid; i < Np; i += T) {
    int c = 0;
    for (int fj = 0; fj < NFF; fj++)
      if (__ldg(a.Fmask + fj) == i && c < 4) sNF[i * 4 + c++] = fj;
    for (; c < 4; c++) sNF[i * 4 + c] = -1;
  }
  const double bm = upd ? a.rkb : a.rkb_next;
  for (int v = 0; v < NV; v++) {
    const long base = v * vs + e0 * Np;
    for (int g = tid; g < E * Np; g += T) {
      const int e = g / Np, i = g - e * Np;
      const bool ok = g < ne * Np;
      const double lam = ok ? a.lam[base + g] : 0.0;
      const double lk = ok ? a.lk[base + g] : 0.0;
      sLam[(v * Np + i) * EP + e] = lam;
      sMu[i * BLD + v * E + e] = lk + bm * lam;
      if (upd) sU[(v * Np + i) * EP + e] = ok ? __ldg(a.u + base + g) : (v == 0 ? 1.0 : 0.0);
    }
  }
  if (upd) {
    for (int g = tid; g < 9 * E; g += T) {
      const int m = g / E, e = g - m * E;
      sGeo[g] = e < ne ? __ldg(a.geo + (long)m * a.gstride + e0 + e) : 0.0;
    }
    for (int g = tid; g < 4 * E; g += T) {
      const int e = g >> 2, f = g & 3;
      const bool ok = e < ne;
      const long gf = (e0 + e) * 4 + f;
      const long gf2 = ok ? __ldg(a.vmapF + gf) : 0;
      const long gs = a.gstride;
      sFace[(0 * 4 + f) * E + e] = ok ? __ldg(a.nrm + gf) : 0.0;
      sFace[(1 * 4 + f) * E + e] = ok ? __ldg(a.nrm + 4 * gs + gf) : 0.0;
      sFace[(2 * 4 + f) * E + e] = ok ? __ldg(a.nrm + 8 * gs + gf) : 0.0;
      sFace[(3 * 4 + f) * E + e] = ok ? __ldg(a.fscale + gf) : 0.0;
      sFace[(4 * 4 + f) * E + e] = ok ? __ldg(a.tau + gf) : 0.0;
      sFace[(5 * 4 + f) * E + e] = ok ? __ldg(a.nrm + gf2) : 0.0;
      sFace[(6 * 4 + f) * E + e] = ok ? __ldg(a.nrm + 4 * gs + gf2) : 0.0;
      sFace[(7 * 4 + f) * E + e] = ok ? __ldg(a.nrm + 8 * gs + gf2) : 0.0;
      sFace[(8 * 4 + f) * E + e] = ok ? __ldg(a.fscale + gf2) : 0.0;
      sFace[(9 * 4 + f) * E + e] = ok ? __ldg(a.tau + gf2) : 0.0;
    }
    for (int g = tid; g < E * NFF; g += T) {
      const int e = g / NFF, fj = g - e * NFF;
      const bool ok = g < ne * NFF;
      sVm[e * VMLD + fj] = ok ? __ldg(a.vmapP + e0 * NFF + g) : 0;
      sMp[e * VMLD + fj] = ok ? __ldg(a.mapP + e0 * NFF + g) : 0;
    }
  }
  __syncthreads();

  const int cg = tid % E, rg = tid / E;
  double acc[3 * RJ][NV];
  if (upd) {
    // ---- face terms -> sFc ------------------------------------------------
    for (int it = tid; it < E * NFF; it += T) {
      const int e = it / NFF, fj = it - e * NFF, f = fj / Nfp;
      if (e >= ne) {
#pragma unroll
        for (int v = 0; v < NV; v++) sFc[(v * NFF + fj) * EP + e] = 0.0;
        continue;
      }
      const long p = (e0 + e) * NFF + fj;
      const long iP = sVm[e * VMLD + fj], p2 = sMp[e * VMLD + fj];
      const int nodeM = sFm[fj];
      const double *F4 = sFace + f * E + e;
      const double nx = F4[0], ny = F4[4 * E], nz = F4[8 * E], fs = F4[12 * E],
                   ta = F4[16 * E], nx2 = F4[20 * E], ny2 = F4[24 * E], nz2 = F4[28 * E],
                   fs2 = F4[32 * E], ta2 = F4[36 * E];
      if (PHYS == A_EUL) {
        double qb[5], g1[5], g2[5], w[5];
#pragma unroll
        for (int v = 0; v < 5; v++) {
          qb[v] = 0.5 * (sU[(v * Np + nodeM) * EP + e] + __ldg(a.u + v * vs + iP));
          g1[v] = a.phi_in[v * vsF + p];
          g2[v] = a.phi_in[v * vsF + p2];
          w[v] = 0.5 * (fs * ta * g1[v] - fs2 * ta2 * g2[v]);
        }
        const JacPre P = jac_pre(a.gamma, qb);
        jac_t_add(P, a.gamma, nx, ny, nz, g1, 0.5 * fs, w);
        jac_t_add(P, a.gamma, nx2, ny2, nz2, g2, 0.5 * fs2, w);
#pragma unroll
        for (int v = 0; v < 5; v++) sFc[(v * NFF + fj) * EP + e] = w[v];
      } else {
        const long nM = (e0 + e) * Np + nodeM;
        const double an = nx * __ldg(a.vel + nM) + ny * __ldg(a.vel + vs + nM) +
                          nz * __ldg(a.vel + 2 * vs + nM);
        const double an2 = nx2 * __ldg(a.vel + iP) + ny2 * __ldg(a.vel + vs + iP) +
                           nz2 * __ldg(a.vel + 2 * vs + iP);
        const double g1 = a.phi_in[p], g2 = a.phi_in[p2];
        sFc[fj * EP + e] = fs * (0.5 * an + 0.5 * ta) * g1 + fs2 * (0.5 * an2 - 0.5 * ta2) * g2;
      }
    }

    // ---- nu = [WD_r^T; WD_s^T; WD_t^T] mu, rows 3j + d ---------------------
#pragma unroll
    for (int r = 0; r < 3 * RJ; r++)
#pragma unroll
      for (int v = 0; v < NV; v++) acc[r][v] = 0.0;
    const double *Ab = a.AV + rg * 3 * RJ;
#pragma unroll 5
    for (int k = 0; k < Np; k++) {
      double bv[NV], av[3 * RJ];
#pragma unroll
      for (int v = 0; v < NV; v++) bv[v] = sMu[k * BLD + v * E + cg];
#pragma unroll
      for (int r = 0; r < 3 * RJ; r++) av[r] = __ldg(Ab + k * C::IPV + r);
#pragma unroll
      for (int r = 0; r < 3 * RJ; r++)
#pragma unroll
        for (int v = 0; v < NV; v++) acc[r][v] = fma(av[r], bv[v], acc[r][v]);
    }
  }
  __syncthreads();

  if (upd) {
    // ---- combine: lam' = lam + dt (volume + face terms), lk' = a mu ---------
    const double *gg = sGeo + cg;
#pragma unroll
    for (int r = 0; r < RJ; r++) {
      const int j = rg * RJ + r;
      if (j >= Np) continue;
      double w[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) w[v] = 0.0;
#pragma unroll
      for (int x = 0; x < 3; x++) {
        double Gx[NV];
#pragma unroll
        for (int v = 0; v < NV; v++)
          Gx[v] = gg[x * E] * acc[3 * r][v] + gg[(3 + x) * E] * acc[3 * r + 1][v] +
                  gg[(6 + x) * E] * acc[3 * r + 2][v];
        if (PHYS == A_EUL) {
          double q[5];
#pragma unroll
          for (int v = 0; v < 5; v++) q[v] = sU[(v * Np + j) * EP + cg];
          const JacPre P = jac_pre(a.gamma, q);
          jac_t_add(P, a.gamma, x == 0, x == 1, x == 2, Gx, 1.0, w);
        } else {
          const long n = (cg < ne) ? (e0 + cg) * Np + j : 0;
          w[0] += __ldg(a.vel + x * vs + n) * Gx[0];
        }
      }
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const int fj = sNF[j * 4 + c];
        if (fj < 0) break;
#pragma unroll
        for (int v = 0; v < NV; v++) w[v] += sFc[(v * NFF + fj) * EP + cg];
      }
#pragma unroll
      for (int v = 0; v < NV; v++) {
        const int s = (v * Np + j) * EP + cg;
        const double mu = sMu[j * BLD + v * E + cg];
        const double lamn = sLam[s] + a.dt * w[v];
        const double lkn = a.rka * mu;
        sLam[s] = lamn;
        sU[s] = lkn;
        sMu[j * BLD + v * E + cg] = lkn + a.rkb_next * lamn;
      }
    }
    __syncthreads();
  }

  if (a.phi_next) {
    // ---- phi' = -LIFT^T mu' -> sFc ------------------------------------------
    double acf[RF][NV];
#pragma unroll
    for (int r = 0; r < RF; r++)
#pragma unroll
      for (int v = 0; v < NV; v++) acf[r][v] = 0.0;
    const double *Ab = a.AL + rg * RF;
#pragma unroll 5
    for (int k = 0; k < Np; k++) {
      double bv[NV], av[RF];
#pragma unroll
      for (int v = 0; v < NV; v++) bv[v] = sMu[k * BLD + v * E + cg];
#pragma unroll
      for (int r = 0; r < RF; r++) av[r] = __ldg(Ab + k * C::IPL + r);
#pragma unroll
      for (int r = 0; r < RF; r++)
#pragma unroll
        for (int v = 0; v < NV; v++) acf[r][v] = fma(av[r], bv[v], acf[r][v]);
    }
#pragma unroll
    for (int r = 0; r < RF; r++) {
      const int fj = rg * RF + r;
      if (fj < NFF) {
#pragma unroll
        for (int v = 0; v < NV; v++) sFc[(v * NFF + fj) * EP + cg] = acf[r][v];
      }
    }
    __syncthreads();
    for (int v = 0; v < NV; v++) {
      const long base = v * vsF + e0 * NFF;
      for (int g = tid; g < ne * NFF; g += T) {
        const int e = g / NFF, fj = g - e * NFF;
        a.phi_out[base + g] = sFc[(v * NFF + fj) * EP + e];
      }
    }
  }

  if (upd) {
    for (int v = 0; v < NV; v++) {
      const long base = v * vs + e0 * Np;
      for (int g = tid; g < ne * Np; g += T) {
        const int e = g / Np, i = g - e * Np;
        const int s = (v * Np + i) * EP + e;
        a.lam[base + g] = sLam[s];
        a.lk[base + g] = sU[s];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// FP64 tensor-core variant: the two contractions on mma.sync.m8n8k4.f64.
//
// Rows of the volume operator are (d*Np + j) of [WD_r^T; WD_s^T; WD_t^T]
// (MTV m-tiles), rows of the lift operator are the face points of -LIFT^T
// (MTL m-tiles); k runs over the Np nodes (padded to KP).  Both are stored
// on the device as A fragments [kstep][mtile][lane] (row 8*mtile + lane/4,
// k 4*kstep + lane%4), one coalesced 256-byte load each.  The B operand is
// mu in shared memory, [k][v*E + e].  Warp w owns n-tile w % NT (8 columns)
// and the m-tiles of group w / NT.  Results go through shared memory to the
// element-local phases (Jacobians, faces, update), which use all threads.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void adj_dmma(double (&d)[2], double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

// Face terms of the adjoint stage, one thread per face point p = e NFF + fj
// (the face loop of the fused kernels, split out so that its gathers -- the
// partner trace u[vmapP], phi at p and at the partner point mapP[p], and the
// partner face's normal, fscale and tau -- run at full occupancy):
//   w = 1/2 (fs tau g1 - fs2 tau2 g2) + 1/2 fs A_n(qb)^T g1 + 1/2 fs2 A_n2(qb)^T g2
// with qb the face average of the stage state and g1, g2 = phi at p, mapP[p]
// (Euler); the upwind-flux transpose for advection.  Output fw[v vsF + p].
template <int PHYS, int N>
__global__ void __launch_bounds__(256) adjoint_face_kernel(const AdjArgs a) {
  constexpr int NV = PHYS == A_EUL ? 5 : 1;
  constexpr int Np = np_of(N), Nfp = nfp_of(N), NFF = 4 * Nfp;
  const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (p >= (long)a.K * NFF) return;
  const long e = p / NFF;
  const int fj = (int)(p - e * NFF), f = fj / Nfp;
  const long vs = a.vs, vsF = a.vsF, gs = a.gstride;
  const long gf = e * 4 + f, gf2 = __ldg(a.vmapF + gf);
  const long iP = __ldg(a.vmapP + p), p2 = __ldg(a.mapP + p);
  const long nM = e * Np + __ldg(a.Fmask + fj);
  const double nx = __ldg(a.nrm + gf), ny = __ldg(a.nrm + 4 * gs + gf),
               nz = __ldg(a.nrm + 8 * gs + gf), fs = __ldg(a.fscale + gf), ta = __ldg(a.tau + gf);
  const double nx2 = __ldg(a.nrm + gf2), ny2 = __ldg(a.nrm + 4 * gs + gf2),
               nz2 = __ldg(a.nrm + 8 * gs + gf2), fs2 = __ldg(a.fscale + gf2),
               ta2 = __ldg(a.tau + gf2);
  if (PHYS == A_EUL) {
    double qb[5], g1[5], g2[5], w[5];
#pragma unroll
    for (int v = 0; v < 5; v++) {
      qb[v] = 0.5 * (__ldg(a.u + v * vs + nM) + __ldg(a.u + v * vs + iP));
      g1[v] = a.phi_in[v * vsF + p];
      g2[v] = a.phi_in[v * vsF + p2];
      w[v] = 0.5 * (fs * ta * g1[v] - fs2 * ta2 * g2[v]);
    }
    const JacPre P = jac_pre(a.gamma, qb);
    jac_t_add(P, a.gamma, nx, ny, nz, g1, 0.5 * fs, w);
    jac_t_add(P, a.gamma, nx2, ny2, nz2, g2, 0.5 * fs2, w);
#pragma unroll
    for (int v = 0; v < 5; v++) a.fw[v * vsF + p] = w[v];
  } else {
    const double an = nx * __ldg(a.vel + nM) + ny * __ldg(a.vel + vs + nM) +
                      nz * __ldg(a.vel + 2 * vs + nM);
    const double an2 = nx2 * __ldg(a.vel + iP) + ny2 * __ldg(a.vel + vs + iP) +
                       nz2 * __ldg(a.vel + 2 * vs + iP);
    const double g1 = a.phi_in[p], g2 = a.phi_in[p2];
    a.fw[p] = fs * (0.5 * an + 0.5 * ta) * g1 + fs2 * (0.5 * an2 - 0.5 * ta2) * g2;
  }
  (void)NV;
}

template <int PHYS, int N, int E_, int MG_, bool SPLIT_ = false>
struct DCfg {
  static constexpr int NV = PHYS == A_EUL ? 5 : 1;
  static constexpr int Np = np_of(N), Nfp = nfp_of(N), NFF = 4 * Nfp;
  static constexpr int E = E_, EP = E_ + 1, NCOL = NV * E, NT = NCOL / 8;
  static constexpr int KP = (Np + 3) / 4 * 4, KS = KP / 4;
  static constexpr int MTV = (3 * Np + 7) / 8, MTL = (NFF + 7) / 8;
  static constexpr int MG = MG_;
  static constexpr int WMV = (MTV + MG - 1) / MG, WML = (MTL + MG - 1) / MG;
  static constexpr int WARPS = NT * MG, T = 32 * WARPS;
  // mu rows [k][BLD]: stride 8 (mod 16) doubles with column bit 2 flipped on
  // rows whose bit 1 is set (bcol), so that the m8n8k4 B-fragment loads and
  // stores to two neighbouring rows by a half-warp hit distinct bank pairs
  static constexpr int BLD = NCOL + (24 - NCOL % 16) % 16;
  static constexpr int VMLD = NFF + 1;
  static constexpr int ROWS = 8 * (MTV > MTL ? MTV : MTL);
  // per-(variable, element) rows with a stride of 2 (mod 4) doubles: node-
  // contiguous accesses, accesses by 8 elements x 2 nodes and the DMMA result
  // stores (4 rows x 4 column pairs) are all free of bank conflicts
  static constexpr int pad2(int n) { return n + (6 - n % 4) % 4; }
  static constexpr int IP = pad2(Np), RLD = pad2(ROWS), FRL = pad2(NFF);
  // SPLIT: the face terms come from adjoint_face_kernel through global
  // memory; no face buffers, face data or face-point maps in shared memory
  static constexpr bool SPLIT = SPLIT_;
  static constexpr int S_U = NV * E * IP, S_B = KP * BLD, S_OUT = NV * E * RLD,
                       S_FC = SPLIT ? 0 : NV * E * FRL, S_FACE = SPLIT ? 0 : 40 * E,
                       S_MAPS = SPLIT ? 0 : 2 * E * VMLD;
  static constexpr size_t SMEM =
      sizeof(double) * (2 * S_U + S_B + S_OUT + S_FC + 9 * E + S_FACE) +
      sizeof(int) * (S_MAPS + NFF + 4 * Np);
  static constexpr int AFV = KS * MTV * 32, AFL = KS * MTL * 32;   // fragment doubles
  static_assert(NCOL % 8 == 0, "columns must fill whole n-tiles");
  static_assert(T <= 1024, "block too large");
  static_assert(S_OUT >= S_U, "mu staging reuses the result buffer");
  __device__ static __forceinline__ int bcol(int row, int col) {
    return col ^ (((row >> 1) & 1) << 2);
  }
};

// Transposed-operator contraction with every warp on all NT n-tiles: warp w
// takes m-tiles w, w + WARPS, ... of the MTX m-tiles (A fragments [kstep]
// [mtile][lane] from global memory, one load per k-step for NT DMMAs), the B
// fragments come from the mu rows in shared memory; results for rows below
// `rows` go to sOut[(v E + e) RLD + row].
template <class C>
__device__ __forceinline__ void adj_contract_all_n(const double *A, int MTX, int rows,
                                                   const double *sB, double *sOut, int warp,
                                                   int lane) {
  constexpr int NT = C::NT, E = C::E;
  // rows k0 + (lane & 3), k0 % 4 == 0: the swizzle bit is lane bit 1
  const double *Bb = sB + (lane & 3) * C::BLD + C::bcol(lane & 3, lane >> 2);
  for (int mt = warp; mt < MTX; mt += C::WARPS) {
    double acc[NT][2];
#pragma unroll
    for (int j = 0; j < NT; j++) acc[j][0] = acc[j][1] = 0.0;
    const double *Ab = A + (long)mt * 32 + lane;
    double an = __ldg(Ab);
#pragma unroll 3
    for (int ks = 0; ks < C::KS; ks++) {
      const double av = an;
      if (ks + 1 < C::KS) an = __ldg(Ab + (long)(ks + 1) * MTX * 32);
#pragma unroll
      for (int j = 0; j < NT; j++) adj_dmma(acc[j], av, Bb[ks * 4 * C::BLD + j * 8]);
    }
    const int row = mt * 8 + (lane >> 2);
    if (row < rows) {
#pragma unroll
      for (int j = 0; j < NT; j++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int col = j * 8 + (lane & 3) * 2 + h, v = col / E, e = col - v * E;
          sOut[(v * E + e) * C::RLD + row] = acc[j][h];
        }
    }
  }
}

template <int PHYS, int N, int E_, int MG_, int MINB, bool SPLIT, bool ALLN = false>
__global__ void __launch_bounds__(DCfg<PHYS, N, E_, MG_, SPLIT>::T, MINB)
    adjoint_dmma_kernel(const AdjArgs a) {
  using C = DCfg<PHYS, N, E_, MG_, SPLIT>;
  constexpr int NV = C::NV, Np = C::Np, Nfp = C::Nfp, NFF = C::NFF, E = C::E,
                BLD = C::BLD, T = C::T, VMLD = C::VMLD, KP = C::KP;
  extern __shared__ __align__(16) double smem[];
  double *sU = smem;                   // [v][e][IP] stage state, later lk'
  double *sLam = sU + C::S_U;          // [v][e][IP]
  double *sB = sLam + C::S_U;          // [k][BLD] mu, col = v*E + e (swizzled)
  double *sOut = sB + C::S_B;          // [v][e][RLD] contraction results by row
  double *sFc = sOut + C::S_OUT;       // [v][e][FRL] face terms
  double *sGeo = sFc + C::S_FC;        // [9][E]
  double *sFace = sGeo + 9 * E;        // [10][4][E]
  int *sVm = reinterpret_cast<int *>(sFace + C::S_FACE);
  int *sMp = sVm + C::S_MAPS / 2;
  int *sFm = sVm + C::S_MAPS;
  int *sNF = sFm + NFF;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long e0 = (long)blockIdx.x * E;
  const int ne = (int)min((long)E, (long)a.K - e0);
  const long vs = a.vs, vsF = a.vsF;
  const bool upd = a.update != 0;
  const int ng = warp % C::NT, mg = warp / C::NT;

  // ---- staging ------------------------------------------------------------
  for (int i = tid; i < NFF; i += T) sFm[i] = __ldg(a.Fmask + i);
  for (int i = tid; i < Np; i += T) {
    int c = 0;
    for (int fj = 0; fj < NFF; fj++)
      if (__ldg(a.Fmask + fj) == i && c < 4) sNF[i * 4 + c++] = fj;
    for (; c < 4; c++) sNF[i * 4 + c] = -1;
  }
  const double bm = upd ? a.rkb : a.rkb_next;
  for (int v = 0; v < NV; v++) {
    const long base = v * vs + e0 * Np;
    for (int g = tid; g < E * Np; g += T) {
      const int e = g / Np, i = g - e * Np;
      const bool ok = g < ne * Np;
      const int s = (v * E + e) * C::IP + i;
      sLam[s] = ok ? a.lam[base + g] : 0.0;
      sOut[s] = ok ? a.lk[base + g] : 0.0;   // lk, until mu is formed below
      if (upd) sU[s] = ok ? __ldg(a.u + base + g) : (v == 0 ? 1.0 : 0.0);
    }
  }
  for (int g = tid; g < (KP - Np) * BLD; g += T) sB[Np * BLD + g] = 0.0;
  __syncthreads();
  // mu = lk + b lam -> sB; a half-warp takes 8 elements x 2 nodes
  for (int g = tid; g < NV * Np * E; g += T) {
    const int e = g % E, r = g / E, i = r % Np, v = r / Np;
    const int s = (v * E + e) * C::IP + i;
    sB[i * BLD + C::bcol(i, v * E + e)] = sOut[s] + bm * sLam[s];
  }
  if (upd) {
    for (int g = tid; g < 9 * E; g += T) {
      const int m = g / E, e = g - m * E;
      sGeo[g] = e < ne ? __ldg(a.geo + (long)m * a.gstride + e0 + e) : 0.0;
    }
    for (int g = tid; g < (SPLIT ? 0 : 4 * E); g += T) {
      const int e = g >> 2, f = g & 3;
      const bool ok = e < ne;
      const long gf = (e0 + e) * 4 + f;
      const long gf2 = ok ? __ldg(a.vmapF + gf) : 0;
      const long gs = a.gstride;
      sFace[(0 * 4 + f) * E + e] = ok ? __ldg(a.nrm + gf) : 0.0;
      sFace[(1 * 4 + f) * E + e] = ok ? __ldg(a.nrm + 4 * gs + gf) : 0.0;
      sFace[(2 * 4 + f) * E + e] = ok ? __ldg(a.nrm + 8 * gs + gf) : 0.0;
      sFace[(3 * 4 + f) * E + e] = ok ? __ldg(a.fscale + gf) : 0.0;
      sFace[(4 * 4 + f) * E + e] = ok ? __ldg(a.tau + gf) : 0.0;
      sFace[(5 * 4 + f) * E + e] = ok ? __ldg(a.nrm + gf2) : 0.0;
      sFace[(6 * 4 + f) * E + e] = ok ? __ldg(a.nrm + 4 * gs + gf2) : 0.0;
      sFace[(7 * 4 + f) * E + e] = ok ? __ldg(a.nrm + 8 * gs + gf2) : 0.0;
      sFace[(8 * 4 + f) * E + e] = ok ? __ldg(a.fscale + gf2) : 0.0;
      sFace[(9 * 4 + f) * E + e] = ok ? __ldg(a.tau + gf2) : 0.0;
    }
    for (int g = tid; g < (SPLIT ? 0 : E * NFF); g += T) {
      const int e = g / NFF, fj = g - e * NFF;
      const bool ok = g < ne * NFF;
      sVm[e * VMLD + fj] = ok ? __ldg(a.vmapP + e0 * NFF + g) : 0;
      sMp[e * VMLD + fj] = ok ? __ldg(a.mapP + e0 * NFF + g) : 0;
    }
  }
  __syncthreads();

  if (upd) {
    // ---- face terms -> sFc (as the SIMT variant; SPLIT: adjoint_face_kernel)
    for (int it = tid; it < (SPLIT ? 0 : E * NFF); it += T) {
      const int e = it / NFF, fj = it - e * NFF, f = fj / Nfp;
      if (e >= ne) {
#pragma unroll
        for (int v = 0; v < NV; v++) sFc[(v * E + e) * C::FRL + fj] = 0.0;
        continue;
      }
      const long p = (e0 + e) * NFF + fj;
      const long iP = sVm[e * VMLD + fj], p2 = sMp[e * VMLD + fj];
      const int nodeM = sFm[fj];
      const double *F4 = sFace + f * E + e;
      const double nx = F4[0], ny = F4[4 * E], nz = F4[8 * E], fs = F4[12 * E],
                   ta = F4[16 * E], nx2 = F4[20 * E], ny2 = F4[24 * E], nz2 = F4[28 * E],
                   fs2 = F4[32 * E], ta2 = F4[36 * E];
      if (PHYS == A_EUL) {
        double qb[5], g1[5], g2[5], w[5];
#pragma unroll
        for (int v = 0; v < 5; v++) {
          qb[v] = 0.5 * (sU[(v * E + e) * C::IP + nodeM] + __ldg(a.u + v * vs + iP));
          g1[v] = a.phi_in[v * vsF + p];
          g2[v] = a.phi_in[v * vsF + p2];
          w[v] = 0.5 * (fs * ta * g1[v] - fs2 * ta2 * g2[v]);
        }
        const JacPre P = jac_pre(a.gamma, qb);
        jac_t_add(P, a.gamma, nx, ny, nz, g1, 0.5 * fs, w);
        jac_t_add(P, a.gamma, nx2, ny2, nz2, g2, 0.5 * fs2, w);
#pragma unroll
        for (int v = 0; v < 5; v++) sFc[(v * E + e) * C::FRL + fj] = w[v];
      } else {
        const long nM = (e0 + e) * Np + nodeM;
        const double an = nx * __ldg(a.vel + nM) + ny * __ldg(a.vel + vs + nM) +
                          nz * __ldg(a.vel + 2 * vs + nM);
        const double an2 = nx2 * __ldg(a.vel + iP) + ny2 * __ldg(a.vel + vs + iP) +
                           nz2 * __ldg(a.vel + 2 * vs + iP);
        const double g1 = a.phi_in[p], g2 = a.phi_in[p2];
        sFc[e * C::FRL + fj] =
            fs * (0.5 * an + 0.5 * ta) * g1 + fs2 * (0.5 * an2 - 0.5 * ta2) * g2;
      }
    }

    // ---- nu = [WD^T] mu on the tensor cores --------------------------------
    if constexpr (ALLN) {
      adj_contract_all_n<C>(a.AV, C::MTV, 3 * Np, sB, sOut, warp, lane);
    } else {
    double acc[C::WMV][2];
#pragma unroll
    for (int i = 0; i < C::WMV; i++) acc[i][0] = acc[i][1] = 0.0;
    const int m0 = mg * C::WMV;
    const double *Ab = a.AV + (long)m0 * 32 + lane;
    // rows k0 + (lane & 3), k0 % 4 == 0: the swizzle bit is lane bit 1
    const double *Bb = sB + (lane & 3) * BLD + ng * 8 + C::bcol(lane & 3, lane >> 2);
#pragma unroll 3
    for (int ks = 0; ks < C::KS; ks++) {
      const double bv = Bb[ks * 4 * BLD];
#pragma unroll
      for (int i = 0; i < C::WMV; i++)
        if (m0 + i < C::MTV) adj_dmma(acc[i], __ldg(Ab + ((long)ks * C::MTV + i) * 32), bv);
    }
    // results -> sOut[row][v][e] (row = d*Np + j)
#pragma unroll
    for (int i = 0; i < C::WMV; i++) {
      const int row = (m0 + i) * 8 + (lane >> 2);
      if (m0 + i < C::MTV && row < 3 * Np) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int col = ng * 8 + (lane & 3) * 2 + h, v = col / E, e = col - v * E;
          sOut[(v * E + e) * C::RLD + row] = acc[i][h];
        }
      }
    }
    }
  }
  __syncthreads();

  if (upd) {
    // ---- combine: lam' = lam + dt (volume + face terms), lk' = a mu ---------
    for (int it = tid; it < E * Np; it += T) {
      const int j = it / E, e = it - j * E;
      const double *gg = sGeo + e;
      double w[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) w[v] = 0.0;
      double nu[3][NV];
#pragma unroll
      for (int d = 0; d < 3; d++)
#pragma unroll
        for (int v = 0; v < NV; v++) nu[d][v] = sOut[(v * E + e) * C::RLD + d * Np + j];
      JacPre P;
      if (PHYS == A_EUL) {
        double q[5];
#pragma unroll
        for (int v = 0; v < 5; v++) q[v] = sU[(v * E + e) * C::IP + j];
        P = jac_pre(a.gamma, q);
      }
#pragma unroll
      for (int x = 0; x < 3; x++) {
        double Gx[NV];
#pragma unroll
        for (int v = 0; v < NV; v++)
          Gx[v] = gg[x * E] * nu[0][v] + gg[(3 + x) * E] * nu[1][v] + gg[(6 + x) * E] * nu[2][v];
        if (PHYS == A_EUL) {
          jac_t_add(P, a.gamma, x == 0, x == 1, x == 2, Gx, 1.0, w);
        } else {
          const long n = (e < ne) ? (e0 + e) * Np + j : 0;
          w[0] += __ldg(a.vel + x * vs + n) * Gx[0];
        }
      }
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const int fj = sNF[j * 4 + c];
        if (fj < 0) break;
        if constexpr (SPLIT) {
          if (e < ne) {
#pragma unroll
            for (int v = 0; v < NV; v++) w[v] += a.fw[v * vsF + (e0 + e) * NFF + fj];
          }
        } else {
#pragma unroll
          for (int v = 0; v < NV; v++) w[v] += sFc[(v * E + e) * C::FRL + fj];
        }
      }
#pragma unroll
      for (int v = 0; v < NV; v++) {
        const int s = (v * E + e) * C::IP + j, bi = j * BLD + C::bcol(j, v * E + e);
        const double mu = sB[bi];
        const double lamn = sLam[s] + a.dt * w[v];
        const double lkn = a.rka * mu;
        sLam[s] = lamn;
        sU[s] = lkn;
        sB[bi] = lkn + a.rkb_next * lamn;
      }
    }
    __syncthreads();
  }

  if (a.phi_next) {
    // ---- phi' = -LIFT^T mu' on the tensor cores -> sOut[fj][v][e] -----------
    if constexpr (ALLN) {
      adj_contract_all_n<C>(a.AL, C::MTL, NFF, sB, sOut, warp, lane);
    } else {
    double acc[C::WML][2];
#pragma unroll
    for (int i = 0; i < C::WML; i++) acc[i][0] = acc[i][1] = 0.0;
    const int m0 = mg * C::WML;
    const double *Ab = a.AL + (long)m0 * 32 + lane;
    // rows k0 + (lane & 3), k0 % 4 == 0: the swizzle bit is lane bit 1
    const double *Bb = sB + (lane & 3) * BLD + ng * 8 + C::bcol(lane & 3, lane >> 2);
#pragma unroll 3
    for (int ks = 0; ks < C::KS; ks++) {
      const double bv = Bb[ks * 4 * BLD];
#pragma unroll
      for (int i = 0; i < C::WML; i++)
        if (m0 + i < C::MTL) adj_dmma(acc[i], __ldg(Ab + ((long)ks * C::MTL + i) * 32), bv);
    }
#pragma unroll
    for (int i = 0; i < C::WML; i++) {
      const int row = (m0 + i) * 8 + (lane >> 2);
      if (m0 + i < C::MTL && row < NFF) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int col = ng * 8 + (lane & 3) * 2 + h, v = col / E, e = col - v * E;
          sOut[(v * E + e) * C::RLD + row] = acc[i][h];
        }
      }
    }
    }
    __syncthreads();
    for (int v = 0; v < NV; v++) {
      const long base = v * vsF + e0 * NFF;
      for (int g = tid; g < ne * NFF; g += T) {
        const int e = g / NFF, fj = g - e * NFF;
        a.phi_out[base + g] = sOut[(v * E + e) * C::RLD + fj];
      }
    }
  }

  if (upd) {
    for (int v = 0; v < NV; v++) {
      const long base = v * vs + e0 * Np;
      for (int g = tid; g < ne * Np; g += T) {
        const int e = g / Np, i = g - e * Np;
        const int s = (v * E + e) * C::IP + i;
        a.lam[base + g] = sLam[s];
        a.lk[base + g] = sU[s];
      }
    }
  }
}

// Partner face point of every face point (see the file comment); flags a
// face point without exactly one partner or a pairing that is not an
// involution.
__global__ void adjoint_mapP_kernel(int K, int Np, int Nfp, const int *__restrict__ Fmask,
                                    const int *__restrict__ vmapP,
                                    const int *__restrict__ vmapF, int *__restrict__ mapP,
                                    int *bad) {
  const int NFF = 4 * Nfp;
  const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (p >= (long)K * NFF) return;
  const long e = p / NFF;
  const int fj = (int)(p - e * NFF), f = fj / Nfp;
  const long target = e * Np + Fmask[fj];
  const long gf2 = vmapF[e * 4 + f];
  long found = p;
  int cnt = 0;
  for (int j2 = 0; j2 < Nfp; j2++)
    if (vmapP[gf2 * Nfp + j2] == target) {
      found = gf2 * Nfp + j2;
      cnt++;
    }
  if (cnt != 1) atomicOr(bad, 1);
  mapP[p] = (int)found;
}

__global__ void adjoint_mapP_check_kernel(long n, const int *__restrict__ mapP, int *bad) {
  const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (p < n && mapP[mapP[p]] != p) atomicOr(bad, 2);
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------

struct AdjVariant {
  int kind;                  // 0: SIMT (k-major operators), 1: DMMA (A fragments)
  int E, T, minb;
  size_t smem;
  int IPV, IPL;              // SIMT: padded rows of the k-major operators
  int MTV, MTL, KS;          // DMMA: m-tiles and k-steps of the fragments
  cudaError_t (*launch)(const AdjArgs &, cudaStream_t);
  int split = 0;             // 1: face terms by adjoint_face_kernel into the tape's fw;
                             // 2: the same, every warp on all n-tiles of the contractions
};

template <int PHYS, int N, int E, int MINB>
cudaError_t launch_adj(const AdjArgs &a, cudaStream_t s) {
  using C = ACfg<PHYS, N, E>;
  auto k = adjoint_stage_kernel<PHYS, N, E, MINB>;
  cudaError_t e =
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
  if (e != cudaSuccess) return e;
  const int blocks = (a.K + E - 1) / E;
  k<<<blocks, C::T, C::SMEM, s>>>(a);
  return cudaGetLastError();
}

template <int PHYS, int N, int E, int MINB = 1>
AdjVariant adj_variant() {
  using C = ACfg<PHYS, N, E>;
  return AdjVariant{0, E, C::T, MINB, C::SMEM, C::IPV, C::IPL, 0, 0, 0,
                    launch_adj<PHYS, N, E, MINB>};
}

template <int PHYS, int N, int E, int MG, int MINB>
cudaError_t launch_adj_dmma(const AdjArgs &a, cudaStream_t s) {
  using C = DCfg<PHYS, N, E, MG>;
  auto k = adjoint_dmma_kernel<PHYS, N, E, MG, MINB, false>;
  cudaError_t e =
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
  if (e != cudaSuccess) return e;
  const int blocks = (a.K + E - 1) / E;
  k<<<blocks, C::T, C::SMEM, s>>>(a);
  return cudaGetLastError();
}

template <int PHYS, int N, int E, int MG, int MINB = 1>
AdjVariant adj_dmma_variant() {
  using C = DCfg<PHYS, N, E, MG>;
  return AdjVariant{1, E, C::T, MINB, C::SMEM, 0, 0, C::MTV, C::MTL, C::KS,
                    launch_adj_dmma<PHYS, N, E, MG, MINB>};
}

// face-point kernel, then the DMMA kernel without face buffers
template <int PHYS, int N, int E, int MG, int MINB, bool ALLN>
cudaError_t launch_adj_split(const AdjArgs &a, cudaStream_t s) {
  using C = DCfg<PHYS, N, E, MG, true>;
  if (a.update) {
    const long n = (long)a.K * C::NFF;
    adjoint_face_kernel<PHYS, N><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  auto k = adjoint_dmma_kernel<PHYS, N, E, MG, MINB, true, ALLN>;
  cudaError_t e =
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
  if (e != cudaSuccess) return e;
  const int blocks = (a.K + E - 1) / E;
  k<<<blocks, C::T, C::SMEM, s>>>(a);
  return cudaGetLastError();
}

template <int PHYS, int N, int E, int MG, int MINB = 1, bool ALLN = false>
AdjVariant adj_split_variant() {
  using C = DCfg<PHYS, N, E, MG, true>;
  return AdjVariant{1, E, C::T, MINB, C::SMEM, 0, 0, C::MTV, C::MTL, C::KS,
                    launch_adj_split<PHYS, N, E, MG, MINB, ALLN>, ALLN ? 2 : 1};
}

// Tile shapes per (physics, N); the first is the default.
const std::vector<AdjVariant> &adjoint_variants(int physics, int N) {
  static const std::vector<AdjVariant> none;
  static const std::vector<AdjVariant> eul[6] = {
      {adj_variant<A_EUL, 1, 16>()},
      {adj_variant<A_EUL, 2, 16>(), adj_dmma_variant<A_EUL, 2, 8, 1>()},
      {adj_variant<A_EUL, 3, 8>(), adj_dmma_variant<A_EUL, 3, 8, 2>()},
      {adj_split_variant<A_EUL, 4, 8, 2, 3, true>(), adj_split_variant<A_EUL, 4, 8, 2, 3>(),
       adj_dmma_variant<A_EUL, 4, 8, 2, 2>(),
       adj_variant<A_EUL, 4, 4, 4>(), adj_dmma_variant<A_EUL, 4, 8, 3>(),
       adj_split_variant<A_EUL, 4, 8, 2, 2>(), adj_split_variant<A_EUL, 4, 8, 2, 2, true>()},
      {adj_variant<A_EUL, 5, 8>(), adj_dmma_variant<A_EUL, 5, 8, 2>()},
      {adj_variant<A_EUL, 6, 4>()}};
  static const std::vector<AdjVariant> adv[6] = {
      {adj_variant<A_ADV, 1, 64>()},
      {adj_variant<A_ADV, 2, 32>(), adj_dmma_variant<A_ADV, 2, 32, 1>()},
      {adj_variant<A_ADV, 3, 32>(), adj_dmma_variant<A_ADV, 3, 32, 2>()},
      {adj_variant<A_ADV, 4, 32>(), adj_dmma_variant<A_ADV, 4, 32, 2>()},
      {adj_variant<A_ADV, 5, 16>(), adj_dmma_variant<A_ADV, 5, 16, 2>()},
      {adj_variant<A_ADV, 6, 16>()}};
  if (N < 1 || N > 6 || (physics != DGLM_EULER && physics != DGLM_ADVECTION)) return none;
  return physics == DGLM_EULER ? eul[N - 1] : adv[N - 1];
}

}  // namespace dglm

using namespace dglm;

// ---------------------------------------------------------------------------
// the tape of a recorded forward run
// ---------------------------------------------------------------------------

struct AdjointTape {
  AdjVariant var{};
  int var_index = 0;
  long state = 0;            // doubles per stored state (nvar * vs)
  long vsF = 0;              // doubles between variables of a face-point field
  int nsteps = 0, every = 0, nseg = 0, cap_ckpt = 0, cap_steps = 0, cap_store = 0;
  bool recorded = false;
  bool last_seg_stored = false;   // the store already holds the last segment's stage inputs
  std::vector<double> dt;    // dt of every recorded step
  double *AV = nullptr, *AL = nullptr;
  int *mapP = nullptr, *bad = nullptr;
  double *lam = nullptr, *lk = nullptr, *phi[2] = {nullptr, nullptr}, *kbuf = nullptr;
  double *fw = nullptr;      // face terms of one stage (split variants)
  double *dt_dev = nullptr;  // cap_steps
  double *tau = nullptr;     // cap_steps x 4Kp (Euler) or 4Kp (advection)
  double *ckpt = nullptr;    // cap_ckpt states
  double *store = nullptr;   // cap_store states: stage inputs of one segment
  std::vector<void *> fixed, sized;   // allocations: per mesh / per recording size
  size_t bytes = 0, sized_bytes = 0;
  // binomial (revolve) recording under a memory cap: chunks of `leaf`
  // steps, `slots` state checkpoints (slot 0: the initial state), the
  // checkpoints the recording placed (spine[q] = chunk held by slot q)
  bool capped = false, spine_valid = false;
  int leaf = 0, slots = 0, nchunk = 0;
  long long advance_steps = 0;   // forward steps recomputed by one backward pass
  std::vector<int> spine;
  std::vector<int> plan_split;   // split[n][free] of the schedule table
  int plan_f = 0;                // its free-slot columns - 1
  double *maxv_tmp = nullptr, *tau_tmp = nullptr;   // wave speeds / tau of a recomputed step
  DevScalars *sc_tmp = nullptr;
};

namespace dglm {

void free_tape(dglm_handle *h) {
  if (!h->tape) return;
  for (void *p : h->tape->fixed) cudaFree(p);
  for (void *p : h->tape->sized) cudaFree(p);
  delete h->tape;
  h->tape = nullptr;
}

}  // namespace dglm

namespace {

template <typename T>
dglm_status talloc(AdjointTape *t, std::vector<void *> &list, T **p, size_t count) {
  const bool sized = &list == &t->sized;
  void *q = nullptr;
  const size_t n = std::max<size_t>(count * sizeof(T), 16);
  cudaError_t e = cudaMalloc(&q, n);
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(DGLM_ERR_NOMEM, std::string("adjoint: cudaMalloc of ") +
                                         std::to_string(n) + " bytes failed: " +
                                         cudaGetErrorString(e));
  }
  list.push_back(q);
  t->bytes += n;
  if (sized) t->sized_bytes += n;
  *p = static_cast<T *>(q);
  return DGLM_OK;
}

// Per-mesh part of the tape: transposed operators, the face-point pairing
// and the adjoint fields.  Rebuilt after every mesh upload.
dglm_status tape_setup(dglm_handle *h) {
  if (h->d.precision != DGLM_PREC_FP64)
    return set_error(DGLM_ERR_UNSUPPORTED,
                     "adjoint: only FP64 handles (the adjoint is the transpose of the FP64 step)");
  if (h->tape && h->tape->AV) return DGLM_OK;
  free_tape(h);
  AdjointTape *t = new AdjointTape();
  h->tape = t;
  const std::vector<AdjVariant> &vl = adjoint_variants(h->d.physics, h->d.N);
  if (vl.empty()) {
    free_tape(h);
    return set_error(DGLM_ERR_UNSUPPORTED, "adjoint: order not built (1..6)");
  }
  t->var_index = h->adj_variant < (int)vl.size() ? h->adj_variant : 0;
  t->var = vl[t->var_index];
  const int Np = h->Np, NFF = h->NFF, KA = 3 * Np + NFF;
  const long K = h->d.K;
  t->state = (long)h->nvar * h->vs;
  t->vsF = (h->Kp * NFF + 31) / 32 * 32;
  dglm_status st = DGLM_OK;
  auto chk = [&](dglm_status s) {
    if (st == DGLM_OK) st = s;
  };
  const AdjVariant &v = t->var;
  const size_t nav = v.kind == 0 ? (size_t)Np * v.IPV : (size_t)v.KS * v.MTV * 32;
  const size_t nal = v.kind == 0 ? (size_t)Np * v.IPL : (size_t)v.KS * v.MTL * 32;
  chk(talloc(t, t->fixed, &t->AV, nav));
  chk(talloc(t, t->fixed, &t->AL, nal));
  chk(talloc(t, t->fixed, &t->mapP, (size_t)K * NFF));
  chk(talloc(t, t->fixed, &t->bad, 1));
  chk(talloc(t, t->fixed, &t->lam, (size_t)t->state));
  chk(talloc(t, t->fixed, &t->lk, (size_t)t->state));
  chk(talloc(t, t->fixed, &t->kbuf, (size_t)t->state));
  chk(talloc(t, t->fixed, &t->phi[0], (size_t)h->nvar * t->vsF));
  chk(talloc(t, t->fixed, &t->phi[1], (size_t)h->nvar * t->vsF));
  if (v.split) chk(talloc(t, t->fixed, &t->fw, (size_t)h->nvar * t->vsF));
  if (st != DGLM_OK) {
    free_tape(h);
    return st;
  }
  std::vector<double> av(nav, 0.0), al(nal, 0.0);
  auto WD = [&](int d, int i, int j) { return h->Ahost[(size_t)i * KA + d * Np + j]; };
  auto NL = [&](int i, int fj) { return h->Ahost[(size_t)i * KA + 3 * Np + fj]; };   // -LIFT
  if (v.kind == 0) {
    for (int i = 0; i < Np; i++) {
      for (int j = 0; j < Np; j++)
        for (int d = 0; d < 3; d++) av[(size_t)i * v.IPV + 3 * j + d] = WD(d, i, j);
      for (int fj = 0; fj < NFF; fj++) al[(size_t)i * v.IPL + fj] = NL(i, fj);
    }
  } else {
    // A fragments [kstep][mtile][lane]: row 8*mtile + lane/4, k 4*kstep + lane%4
    for (int ks = 0; ks < v.KS; ks++)
      for (int lane = 0; lane < 32; lane++) {
        const int k = 4 * ks + lane % 4;
        if (k >= Np) continue;
        for (int mt = 0; mt < v.MTV; mt++) {
          const int row = 8 * mt + lane / 4;
          if (row < 3 * Np) av[((size_t)ks * v.MTV + mt) * 32 + lane] = WD(row / Np, k, row % Np);
        }
        for (int mt = 0; mt < v.MTL; mt++) {
          const int row = 8 * mt + lane / 4;
          if (row < NFF) al[((size_t)ks * v.MTL + mt) * 32 + lane] = NL(k, row);
        }
      }
  }
  cudaStream_t s = h->stream;
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess)
    e = cudaMemcpy(t->AV, av.data(), sizeof(double) * av.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(t->AL, al.data(), sizeof(double) * al.size(), cudaMemcpyHostToDevice);
  // every later use of these buffers is on the handle's stream: zero them there
  for (double *p : {t->lam, t->lk, t->kbuf})
    if (e == cudaSuccess) e = cudaMemsetAsync(p, 0, sizeof(double) * t->state, s);
  for (double *p : t->phi)
    if (e == cudaSuccess) e = cudaMemsetAsync(p, 0, sizeof(double) * h->nvar * t->vsF, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(t->bad, 0, sizeof(int), s);
  const long nfp = K * NFF;
  if (e == cudaSuccess) {
    adjoint_mapP_kernel<<<(unsigned)((nfp + 255) / 256), 256, 0, s>>>(
        (int)K, Np, h->Nfp, h->Fmask, h->vmapP, h->vmapF, t->mapP, t->bad);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    adjoint_mapP_check_kernel<<<(unsigned)((nfp + 255) / 256), 256, 0, s>>>(nfp, t->mapP,
                                                                             t->bad);
    e = cudaGetLastError();
  }
  int bad = 0;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMemcpy(&bad, t->bad, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    free_tape(h);
    return cuda_check(e, "adjoint setup");
  }
  if (bad) {
    free_tape(h);
    return set_error(DGLM_ERR_UNSUPPORTED,
                     "adjoint: face points do not pair up one to one (non-conforming mesh)");
  }
  return DGLM_OK;
}

// Recording-size part: checkpoints, per-step tau and dt, one segment's store.
dglm_status tape_size(dglm_handle *h, int nsteps, int every) {
  AdjointTape *t = h->tape;
  const int nseg = (nsteps + every - 1) / every;
  const int seg_len = std::min(every, nsteps);
  const bool euler = h->d.physics == DGLM_EULER;
  if (nseg <= t->cap_ckpt && nsteps <= t->cap_steps && 5 * seg_len <= t->cap_store) return DGLM_OK;
  cudaStreamSynchronize(h->stream);
  for (void *p : t->sized) cudaFree(p);
  t->sized.clear();
  t->bytes -= t->sized_bytes;
  t->sized_bytes = 0;
  t->cap_ckpt = t->cap_steps = t->cap_store = 0;
  dglm_status st = DGLM_OK;
  auto chk = [&](dglm_status s) {
    if (st == DGLM_OK) st = s;
  };
  chk(talloc(t, t->sized, &t->ckpt, (size_t)nseg * t->state));
  chk(talloc(t, t->sized, &t->dt_dev, (size_t)nsteps));
  chk(talloc(t, t->sized, &t->tau, (size_t)(euler ? nsteps : 1) * 4 * h->Kp));
  // slot 0 of a segment is its checkpoint, slots 1..5*seg_len are stored here
  chk(talloc(t, t->sized, &t->store, (size_t)5 * seg_len * t->state));
  if (st != DGLM_OK) {
    for (void *p : t->sized) cudaFree(p);
    t->sized.clear();
    t->bytes -= t->sized_bytes;
    t->sized_bytes = 0;
    return st;
  }
  // zero-filled (on the handle's stream, ordered before the recording that
  // writes them) so the padded tail elements of every stored state stay zero
  cudaStream_t s = h->stream;
  cudaError_t e = cudaMemsetAsync(t->tau, 0, sizeof(double) * (euler ? nsteps : 1) * 4 * h->Kp, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(t->ckpt, 0, sizeof(double) * nseg * t->state, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(t->store, 0, sizeof(double) * 5 * seg_len * t->state, s);
  if (e != cudaSuccess) return cuda_check(e, "adjoint tape");
  t->cap_ckpt = nseg;
  t->cap_steps = nsteps;
  t->cap_store = 5 * seg_len;
  return DGLM_OK;
}

const double *tau_of(const dglm_handle *h, int step) {
  const AdjointTape *t = h->tape;
  return h->d.physics == DGLM_EULER ? t->tau + (size_t)step * 4 * h->Kp : t->tau;
}

AdjArgs adj_args(dglm_handle *h) {
  AdjointTape *t = h->tape;
  AdjArgs a{};
  a.AV = t->AV;
  a.AL = t->AL;
  a.geo = h->geo;
  a.fscale = h->fscale;
  a.nrm = h->nrm;
  a.vmapP = h->vmapP;
  a.vmapF = h->vmapF;
  a.mapP = t->mapP;
  a.Fmask = h->Fmask;
  a.vel = h->vel;
  a.lam = t->lam;
  a.lk = t->lk;
  a.fw = t->fw;
  a.vs = h->vs;
  a.vsF = t->vsF;
  a.gstride = h->Kp;
  a.K = h->d.K;
  a.gamma = h->d.gamma;
  return a;
}

// Forward stage with recorded dt and tau (no wave-speed side effects).
cudaError_t frozen_stage(dglm_handle *h, const double *u_in, double *u_out, double *k, int s,
                         double dt, const double *tau, cudaStream_t cs) {
  StageArgs a = stage_args(h, u_in, u_out, s);
  a.kreg = k;
  a.tau = tau;
  a.dt_override = dt;
  a.last_stage = 0;
  return launch_stage_fp64(h->d.physics, h->d.N, h->variant, a, cs);
}

// ---- binomial checkpointing under a memory cap ------------------------------
// Binomial checkpointing (Griewank and Walther, "Algorithm 799: revolve",
// ACM TOMS 26, 2000) over chunks of `leaf` LSERK steps.  A chunk is
// reversed by recomputing its stage inputs once from the state at its start
// (into the stage store) and sweeping it backwards; reaching that state from
// a checkpoint costs forward steps ("advances").  With the state of chunk c0
// in a slot and `free` further slots, n chunks are reversed by advancing m
// chunks, storing that state in a free slot, reversing the last n - m chunks
// with one slot fewer and then the first m with the same slots.  The fewest
// chunk advances follow from the recursion
//   cost[1][f] = 0,  cost[n][0] = n (n - 1) / 2,
//   cost[n][f] = min(cost[n][f-1], min_m  m + cost[n-m][f-1] + cost[m][f]),
// solved here as a table (the binomial optimum of revolve, computed instead
// of taken from its closed form).
struct RevolvePlan {
  int n = 0, f = 0;
  std::vector<long long> cost;
  std::vector<int> split;   // 0: the slot is not used for this (n, f)
  long long c(int a, int b) const { return cost[(size_t)a * (f + 1) + b]; }
  int m(int a, int b) const { return split[(size_t)a * (f + 1) + b]; }
};

void plan_revolve(RevolvePlan &p, int n, int f) {
  p.n = n;
  p.f = f;
  p.cost.assign((size_t)(n + 1) * (f + 1), 0);
  p.split.assign((size_t)(n + 1) * (f + 1), 0);
  for (int a = 1; a <= n; a++) {
    p.cost[(size_t)a * (f + 1)] = (long long)a * (a - 1) / 2;
    for (int b = 1; b <= f; b++) {
      long long best = p.c(a, b - 1);
      int bm = 0;
      for (int m = 1; m < a; m++) {
        const long long v = m + p.c(a - m, b - 1) + p.c(m, b);
        if (v < best) {
          best = v;
          bm = m;
        }
      }
      p.cost[(size_t)a * (f + 1) + b] = best;
      p.split[(size_t)a * (f + 1) + b] = bm;
    }
  }
}

// One action of a backward pass: advance `count` chunks from the state of
// chunk `chunk` (in slot src) into slot dst (-1: the scratch state), or
// reverse chunk `chunk` starting from slot src (-1: the scratch state).
struct RevAction {
  int kind, src, chunk, count, dst;   // kind 0: advance, 1: reverse a chunk
};

// checkpoints the recording places: spine[q] = chunk whose start state
// slot q holds (slot 0: chunk 0), the first path of the schedule
void revolve_spine(const RevolvePlan &p, int nchunk, int free, std::vector<int> &spine) {
  spine.assign(1, 0);
  int c0 = 0, n = nchunk;
  while (n > 1 && free > 0) {
    const int m = p.m(n, free);
    free--;
    if (m == 0) continue;
    c0 += m;
    n -= m;
    spine.push_back(c0);
  }
}

// actions reversing chunks [c0, c0 + n) from the state of c0 in `slot`;
// pre: the recording already stored this path's checkpoints
void revolve_actions(const RevolvePlan &p, int c0, int n, int slot, int free, bool pre,
                     std::vector<RevAction> &out) {
  if (n == 1) {
    out.push_back({1, slot, c0, 1, -1});
    return;
  }
  if (free == 0) {
    for (int j = n - 1; j >= 1; j--) {
      out.push_back({0, slot, c0, j, -1});
      out.push_back({1, -1, c0 + j, 1, -1});
    }
    out.push_back({1, slot, c0, 1, -1});
    return;
  }
  const int m = p.m(n, free);
  if (m == 0) {
    revolve_actions(p, c0, n, slot, free - 1, pre, out);
    return;
  }
  if (!pre) out.push_back({0, slot, c0, m, slot + 1});
  revolve_actions(p, c0 + m, n - m, slot + 1, free - 1, pre, out);
  revolve_actions(p, c0, m, slot, free, false, out);
}

// forward steps of the advances in a list of actions
long long revolve_advance_steps(const std::vector<RevAction> &acts, int leaf, int nsteps) {
  long long n = 0;
  for (const RevAction &a : acts)
    if (a.kind == 0)
      n += std::min((long long)(a.chunk + a.count) * leaf, (long long)nsteps) -
           (long long)a.chunk * leaf;
  return n;
}

// Largest chunk count the schedule table is built for (the table costs
// kMaxChunks^3 / 2 operations once per recording).
constexpr int kMaxChunks = 256;

// Bytes of a capped recording's sized part for a given leaf and slot count.
size_t capped_bytes(const dglm_handle *h, int nsteps, int leaf, int slots) {
  const AdjointTape *t = h->tape;
  const bool euler = h->d.physics == DGLM_EULER;
  auto rnd = [](size_t b) { return std::max<size_t>(b, 16); };
  size_t b = rnd(sizeof(double) * (size_t)slots * t->state);
  b += rnd(sizeof(double) * (size_t)5 * leaf * t->state);
  b += rnd(sizeof(double) * (size_t)nsteps);
  b += rnd(sizeof(double) * (size_t)(euler ? leaf : 1) * 4 * h->Kp);
  b += 2 * rnd(sizeof(double) * (size_t)4 * h->Kp);
  b += rnd(sizeof(DevScalars));
  return b;
}

// tau of one step from its input state u (Euler), as the forward step
// computed it: face wave speeds, then the per-face penalty
cudaError_t tau_from_state(dglm_handle *h, const double *u, double *tau, cudaStream_t s) {
  AdjointTape *t = h->tape;
  StageArgs a = stage_args(h, u, nullptr, -1);
  a.maxv = t->maxv_tmp;
  a.sc = t->sc_tmp;
  cudaError_t e = launch_face_maxv(h->d.physics, h->d.N, a, 0, s);
  if (e == cudaSuccess) e = launch_tau(h->d.K, h->d.tau_scale, h->vmapF, t->maxv_tmp, tau, s);
  h->launches += 2;
  return e;
}

// advance: the stages of `count` chunks from the state `src` of chunk c0,
// the last stage writing `dst`; stage outputs alternate between the first
// two states of the stage store, tau is recomputed from each step's input
cudaError_t capped_advance(dglm_handle *h, const double *src, int c0, int count, double *dst,
                           cudaStream_t s) {
  AdjointTape *t = h->tape;
  const bool euler = h->d.physics == DGLM_EULER;
  const int i0 = c0 * t->leaf, i1 = std::min((c0 + count) * t->leaf, t->nsteps);
  const int last = 5 * (i1 - i0) - 1;
  const double *in = src;
  cudaError_t e = cudaSuccess;
  int g = 0;
  for (int i = i0; i < i1 && e == cudaSuccess; i++)
    for (int k = 0; k < 5 && e == cudaSuccess; k++, g++) {
      if (k == 0 && euler) e = tau_from_state(h, in, t->tau_tmp, s);
      double *out = g == last ? dst : t->store + (size_t)(g & 1) * t->state;
      if (e == cudaSuccess)
        e = frozen_stage(h, in, out, t->kbuf, k, t->dt[i], euler ? t->tau_tmp : t->tau, s);
      h->launches++;
      in = out;
    }
  return e;
}

// reverse one chunk from the state `src` at its start: its stage inputs
// recomputed into the stage store (tau of each step beside them), then the
// adjoint stages in reverse order (phi ping-pong index p carried across)
cudaError_t capped_reverse_chunk(dglm_handle *h, AdjArgs &a, int &p, int c, const double *src,
                                 cudaStream_t s) {
  AdjointTape *t = h->tape;
  const bool euler = h->d.physics == DGLM_EULER;
  const int s0 = c * t->leaf, s1 = std::min(s0 + t->leaf, t->nsteps);
  auto slot = [&](int j) -> const double * {
    return j == 0 ? src : t->store + (size_t)(j - 1) * t->state;
  };
  auto tau_i = [&](int i) -> double * {
    return euler ? t->tau + (size_t)(i - s0) * 4 * h->Kp : t->tau;
  };
  cudaError_t e = cudaSuccess;
  for (int i = s0; i < s1 && e == cudaSuccess; i++)
    for (int k = 0; k < 5 && e == cudaSuccess; k++) {
      const int j = 5 * (i - s0) + k;
      if (i == s1 - 1 && k == 4) break;   // the last stage's output is not needed
      if (k == 0 && euler) e = tau_from_state(h, slot(j), tau_i(i), s);
      if (e == cudaSuccess)
        e = frozen_stage(h, slot(j), const_cast<double *>(slot(j + 1)), t->kbuf, k, t->dt[i],
                         tau_i(i), s);
      h->launches++;
    }
  for (int i = s1 - 1; i >= s0 && e == cudaSuccess; i--)
    for (int k = 4; k >= 0 && e == cudaSuccess; k--) {
      a.update = 1;
      a.u = slot(5 * (i - s0) + k);
      a.tau = tau_i(i);
      a.dt = t->dt[i];
      a.rka = RKA[k];
      a.rkb = RKB[k];
      a.phi_next = (i == 0 && k == 0) ? 0 : 1;
      a.rkb_next = k > 0 ? RKB[k - 1] : RKB[4];
      a.phi_in = t->phi[p];
      a.phi_out = t->phi[p ^ 1];
      e = t->var.launch(a, s);
      h->launches++;
      p ^= 1;
    }
  return e;
}

// the reverse sweep of a capped recording: the binomial schedule's actions
cudaError_t capped_sweep(dglm_handle *h, AdjArgs &a, int &p, cudaStream_t s) {
  AdjointTape *t = h->tape;
  RevolvePlan plan;
  plan.f = t->plan_f;
  plan.split = t->plan_split;
  std::vector<RevAction> acts;
  revolve_actions(plan, 0, t->nchunk, 0, t->slots - 1, t->spine_valid, acts);
  double *scratch = t->store + (size_t)(5 * t->leaf - 1) * t->state;
  auto ck = [&](int q) { return q < 0 ? scratch : t->ckpt + (size_t)q * t->state; };
  cudaError_t e = cudaSuccess;
  for (size_t x = 0; x < acts.size() && e == cudaSuccess; x++) {
    const RevAction &r = acts[x];
    if (r.kind == 0)
      e = capped_advance(h, ck(r.src), r.chunk, r.count, ck(r.dst), s);
    else
      e = capped_reverse_chunk(h, a, p, r.chunk, ck(r.src), s);
  }
  // the sweep overwrote the recording's checkpoints past slot 0
  t->spine_valid = false;
  return e;
}

dglm_status copy_fields(dglm_handle *h, double *dst, const double *const *src, int on_device,
                        const char *what) {
  const long n = (long)h->d.K * h->Np;
  cudaError_t e = cudaSuccess;
  for (int v = 0; v < h->nvar && e == cudaSuccess; v++) {
    if (!src[v]) return set_error(DGLM_ERR_INVALID, std::string(what) + ": NULL pointer");
    e = cudaMemcpyAsync(dst + (size_t)v * h->vs, src[v], sizeof(double) * n,
                        on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                        h->stream);
  }
  return cuda_check(e, what);
}

dglm_status fetch_fields(dglm_handle *h, double *const *dst, const double *src, int on_device,
                         const char *what) {
  const long n = (long)h->d.K * h->Np;
  cudaError_t e = cudaSuccess;
  for (int v = 0; v < h->nvar && e == cudaSuccess; v++) {
    if (!dst[v]) return set_error(DGLM_ERR_INVALID, std::string(what) + ": NULL pointer");
    e = cudaMemcpyAsync(dst[v], src + (size_t)v * h->vs, sizeof(double) * n,
                        on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        h->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  return cuda_check(e, what);
}

}  // namespace

extern "C" {

dglm_status dglm_adjoint_record(dglm_handle *h, int nsteps, int checkpoint_every) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_adjoint_record: NULL handle");
  if (!h->state_ready) return set_error(DGLM_ERR_STATE, "dglm_adjoint_record: set a state first");
  if (nsteps <= 0 || checkpoint_every <= 0)
    return set_error(DGLM_ERR_INVALID,
                     "dglm_adjoint_record: nsteps and checkpoint_every must be positive");
  DeviceGuard g(h->dev);
  dglm_status st = tape_setup(h);
  if (st == DGLM_OK) st = tape_size(h, nsteps, checkpoint_every);
  if (st != DGLM_OK) return st;
  AdjointTape *t = h->tape;
  t->recorded = false;
  t->capped = false;
  cudaStream_t s = h->stream;
  const double zero = 0.0;
  cudaError_t e = cudaMemcpyAsync(&h->sc->dt_fixed, &zero, sizeof(double),
                                  cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_check(e, "dglm_adjoint_record");
  h->launches = 0;
  const bool euler = h->d.physics == DGLM_EULER;
  const int last_s0 = (nsteps - 1) / checkpoint_every * checkpoint_every;
  for (int i = 0; i < nsteps; i++) {
    const size_t bytes = sizeof(double) * t->state;
    if (i % checkpoint_every == 0) {
      e = cudaMemcpyAsync(t->ckpt + (size_t)(i / checkpoint_every) * t->state, h->u[h->cur],
                          bytes, cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return cuda_check(e, "dglm_adjoint_record");
    }
    if (i < last_s0) {
      st = run_steps(h, 1);
    } else {
      // last segment: the stages write their outputs straight into the
      // segment store (slot j + 1 = output of stage j), so the reverse sweep
      // starts without recomputing it; the final stage writes the state back
      const double *ck = t->ckpt + (size_t)(i / checkpoint_every) * t->state;
      auto slot = [&](int j) -> double * {
        return j == 0 ? const_cast<double *>(ck) : t->store + (size_t)(j - 1) * t->state;
      };
      const double *in[5];
      double *out[5];
      for (int k = 0; k < 5; k++) {
        const int j = 5 * (i - last_s0) + k;
        in[k] = (i == last_s0 && k == 0) ? h->u[h->cur] : slot(j);
        out[k] = (i == nsteps - 1 && k == 4) ? h->u[h->cur ^ 1] : slot(j + 1);
      }
      st = issue_step_ptrs(h, in, out, s);
      h->launches += euler ? 8 : 7;
      h->cur ^= 1;
    }
    if (st != DGLM_OK) return st;
    if (euler || i == 0)
      e = cudaMemcpyAsync(const_cast<double *>(tau_of(h, i)), h->tau,
                          sizeof(double) * 4 * h->Kp, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(t->dt_dev + i, &h->sc->dt, sizeof(double), cudaMemcpyDeviceToDevice,
                          s);
    if (e != cudaSuccess) return cuda_check(e, "dglm_adjoint_record");
  }
  t->dt.assign(nsteps, 0.0);
  e = cudaMemcpyAsync(t->dt.data(), t->dt_dev, sizeof(double) * nsteps,
                      cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_check(e, "dglm_adjoint_record");
  for (double d : t->dt)
    if (!std::isfinite(d) || d < 0)
      return set_error(DGLM_ERR_NONFINITE, "dglm_adjoint_record: non-finite dt recorded");
  t->nsteps = nsteps;
  t->every = checkpoint_every;
  t->nseg = (nsteps + checkpoint_every - 1) / checkpoint_every;
  t->recorded = true;
  t->last_seg_stored = true;
  return DGLM_OK;
}

dglm_status dglm_adjoint_replay(dglm_handle *h) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_adjoint_replay: NULL handle");
  if (!h->state_ready) return set_error(DGLM_ERR_STATE, "dglm_adjoint_replay: set a state first");
  if (!h->tape || !h->tape->recorded)
    return set_error(DGLM_ERR_STATE, "dglm_adjoint_replay: record a forward run first");
  AdjointTape *t = h->tape;
  if (t->capped)
    return set_error(DGLM_ERR_STATE,
                     "dglm_adjoint_replay: a capped recording keeps no per-step tau; record "
                     "with dglm_adjoint_record to replay");
  DeviceGuard g(h->dev);
  cudaStream_t s = h->stream;
  cudaError_t e = cudaMemsetAsync(h->kreg, 0, sizeof(double) * t->state, s);
  h->launches = 0;
  for (int i = 0; i < t->nsteps && e == cudaSuccess; i++)
    for (int st = 0; st < 5 && e == cudaSuccess; st++) {
      e = frozen_stage(h, h->u[h->cur], h->u[h->cur ^ 1], h->kreg, st, t->dt[i], tau_of(h, i), s);
      h->cur ^= 1;
      h->launches++;
    }
  return cuda_check(e, "dglm_adjoint_replay");
}

dglm_status dglm_adjoint_backward(dglm_handle *h, const double *const *lam_T,
                                  double *const *lam_0, int on_device) {
  if (!h || !lam_T || !lam_0)
    return set_error(DGLM_ERR_INVALID, "dglm_adjoint_backward: NULL argument");
  if (!h->tape || !h->tape->recorded)
    return set_error(DGLM_ERR_STATE, "dglm_adjoint_backward: record a forward run first");
  DeviceGuard g(h->dev);
  AdjointTape *t = h->tape;
  cudaStream_t s = h->stream;
  dglm_status st = copy_fields(h, t->lam, lam_T, on_device, "dglm_adjoint_backward");
  if (st != DGLM_OK) return st;
  cudaError_t e = cudaMemsetAsync(t->lk, 0, sizeof(double) * t->state, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(t->kbuf, 0, sizeof(double) * t->state, s);
  h->launches = 0;
  AdjArgs a = adj_args(h);
  int p = 0;
  // phi of the first adjoint stage (stage 4 of the last step)
  a.update = 0;
  a.phi_next = 1;
  a.rkb_next = RKB[4];
  a.phi_out = t->phi[p];
  if (e == cudaSuccess) e = t->var.launch(a, s);
  h->launches++;
  if (t->capped && e == cudaSuccess) e = capped_sweep(h, a, p, s);
  for (int seg = t->capped ? -1 : t->nseg - 1; seg >= 0 && e == cudaSuccess; seg--) {
    const int s0 = seg * t->every, s1 = std::min(s0 + t->every, t->nsteps);
    double *ck = t->ckpt + (size_t)seg * t->state;
    auto slot = [&](int j) -> double * {
      return j == 0 ? ck : t->store + (size_t)(j - 1) * t->state;
    };
    // recompute the segment's stage inputs from its checkpoint (the last
    // segment's are still in the store from the recording, on the first sweep)
    const bool stored = seg == t->nseg - 1 && t->last_seg_stored;
    for (int i = s0; i < s1 && e == cudaSuccess && !stored; i++)
      for (int k = 0; k < 5 && e == cudaSuccess; k++) {
        const int j = 5 * (i - s0) + k;
        if (i == s1 - 1 && k == 4) break;   // the last stage's output is not needed
        e = frozen_stage(h, slot(j), slot(j + 1), t->kbuf, k, t->dt[i], tau_of(h, i), s);
        h->launches++;
      }
    // reverse sweep over the segment
    for (int i = s1 - 1; i >= s0 && e == cudaSuccess; i--)
      for (int k = 4; k >= 0 && e == cudaSuccess; k--) {
        a.update = 1;
        a.u = slot(5 * (i - s0) + k);
        a.tau = tau_of(h, i);
        a.dt = t->dt[i];
        a.rka = RKA[k];
        a.rkb = RKB[k];
        const bool last = (i == 0 && k == 0);
        a.phi_next = last ? 0 : 1;
        a.rkb_next = k > 0 ? RKB[k - 1] : RKB[4];
        a.phi_in = t->phi[p];
        a.phi_out = t->phi[p ^ 1];
        e = t->var.launch(a, s);
        h->launches++;
        p ^= 1;
      }
  }
  // the store now holds the first segment: a second sweep recomputes all
  if (!t->capped && t->nseg > 1) t->last_seg_stored = false;
  if (e != cudaSuccess) return cuda_check(e, "dglm_adjoint_backward");
  return fetch_fields(h, lam_0, t->lam, on_device, "dglm_adjoint_backward");
}

dglm_status dglm_adjoint_rhs(dglm_handle *h, const double *const *u, const double *const *mu,
                             double *const *out) {
  if (!h || !u || !mu || !out) return set_error(DGLM_ERR_INVALID, "dglm_adjoint_rhs: NULL argument");
  if (!h->mesh_ready) return set_error(DGLM_ERR_STATE, "dglm_adjoint_rhs: upload the mesh first");
  DeviceGuard g(h->dev);
  dglm_status st = tape_setup(h);
  if (st == DGLM_OK) st = ensure_rhs_scratch(h);
  if (st != DGLM_OK) return st;
  AdjointTape *t = h->tape;
  cudaStream_t s = h->stream;
  // tau of u, as dglm_rhs computes it
  st = copy_fields(h, h->rhs_in, u, 1, "dglm_adjoint_rhs");
  if (st == DGLM_OK) st = copy_fields(h, t->lk, mu, 1, "dglm_adjoint_rhs");
  if (st != DGLM_OK) return st;
  cudaError_t e = cudaMemsetAsync(h->sc_s, 0, sizeof(DevScalars), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(t->lam, 0, sizeof(double) * t->state, s);
  StageArgs sa = stage_args(h, h->rhs_in, h->rhs_out, -1);
  sa.maxv = h->maxv_s;
  sa.tau = h->tau_s;
  sa.sc = h->sc_s;
  if (e == cudaSuccess) e = launch_face_maxv(h->d.physics, h->d.N, sa, 0, s);
  if (e == cudaSuccess) e = launch_tau(h->d.K, h->d.tau_scale, h->vmapF, h->maxv_s, h->tau_s, s);
  AdjArgs a = adj_args(h);
  a.u = h->rhs_in;
  a.tau = h->tau_s;
  // phi of mu (mu = lk + 0 lam), then lam = 0 + 1 * R'(u)^T mu
  a.update = 0;
  a.phi_next = 1;
  a.rkb_next = 0.0;
  a.phi_out = t->phi[0];
  if (e == cudaSuccess) e = t->var.launch(a, s);
  a.update = 1;
  a.phi_next = 0;
  a.dt = 1.0;
  a.rka = 0.0;
  a.rkb = 0.0;
  a.phi_in = t->phi[0];
  a.phi_out = t->phi[1];
  if (e == cudaSuccess) e = t->var.launch(a, s);
  if (e != cudaSuccess) return cuda_check(e, "dglm_adjoint_rhs");
  return fetch_fields(h, out, t->lam, 1, "dglm_adjoint_rhs");
}

int dglm_adjoint_variant_count(int physics, int N) {
  return (int)adjoint_variants(physics, N).size();
}

dglm_status dglm_adjoint_variant_describe(int physics, int N, int variant, char *buf,
                                          size_t len) {
  const std::vector<AdjVariant> &vl = adjoint_variants(physics, N);
  if (!buf || len == 0 || variant < 0 || variant >= (int)vl.size())
    return set_error(DGLM_ERR_INVALID, "dglm_adjoint_variant_describe: no such variant");
  const AdjVariant &v = vl[variant];
  snprintf(buf, len, "adjoint-%s E=%d threads=%d minblocks=%d smem=%zu",
           v.kind == 0     ? "simt"
           : v.split == 2  ? "dmma-split-alln"
           : v.split       ? "dmma-split"
                           : "dmma",
           v.E, v.T, v.minb, v.smem);
  return DGLM_OK;
}

dglm_status dglm_adjoint_set_variant(dglm_handle *h, int variant) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_adjoint_set_variant: NULL handle");
  if (variant < 0 || variant >= dglm_adjoint_variant_count(h->d.physics, h->d.N))
    return set_error(DGLM_ERR_INVALID, "dglm_adjoint_set_variant: no such variant");
  if (variant == h->adj_variant) return DGLM_OK;
  DeviceGuard g(h->dev);
  cudaStreamSynchronize(h->stream);
  free_tape(h);   // operator layout depends on the tile shape; record again
  h->adj_variant = variant;
  return DGLM_OK;
}

dglm_status dglm_adjoint_record_capped(dglm_handle *h, int nsteps, size_t max_bytes) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_adjoint_record_capped: NULL handle");
  if (!h->state_ready)
    return set_error(DGLM_ERR_STATE, "dglm_adjoint_record_capped: set a state first");
  if (nsteps <= 0)
    return set_error(DGLM_ERR_INVALID, "dglm_adjoint_record_capped: nsteps must be positive");
  DeviceGuard g(h->dev);
  dglm_status st = tape_setup(h);
  if (st != DGLM_OK) return st;
  AdjointTape *t = h->tape;
  t->recorded = false;
  const size_t fixed = t->bytes - t->sized_bytes;
  const size_t sbytes = sizeof(double) * (size_t)t->state;
  // the leaf length and slot count with the fewest recomputed steps
  const int lmin = (nsteps + kMaxChunks - 1) / kMaxChunks;
  const int nmax = (nsteps + lmin - 1) / lmin;
  RevolvePlan plan;
  plan_revolve(plan, nmax, nmax - 1);
  int best_l = 0, best_free = 0;
  long long best_cost = -1;
  for (int L = lmin; L <= nsteps; L++) {
    const size_t need = fixed + capped_bytes(h, nsteps, L, 1);
    if (need > max_bytes) break;   // the store grows with L
    const int n = (nsteps + L - 1) / L;
    const long long extra = (long long)((max_bytes - need) / sbytes);
    const int free = (int)std::min<long long>(extra, n - 1);
    const long long cost = plan.c(n, free) * L;
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      best_l = L;
      best_free = free;
    }
  }
  if (best_cost < 0)
    return set_error(DGLM_ERR_NOMEM,
                     "dglm_adjoint_record_capped: the cap is below the minimum tape of " +
                         std::to_string(fixed + capped_bytes(h, nsteps, lmin, 1)) + " bytes");
  const int L = best_l, nchunk = (nsteps + L - 1) / L, slots = best_free + 1;
  const bool euler = h->d.physics == DGLM_EULER;
  // the sized part, reallocated for this recording
  cudaStreamSynchronize(h->stream);
  for (void *p : t->sized) cudaFree(p);
  t->sized.clear();
  t->bytes -= t->sized_bytes;
  t->sized_bytes = 0;
  t->cap_ckpt = t->cap_steps = t->cap_store = 0;
  auto chk = [&](dglm_status x) {
    if (st == DGLM_OK) st = x;
  };
  chk(talloc(t, t->sized, &t->ckpt, (size_t)slots * t->state));
  chk(talloc(t, t->sized, &t->store, (size_t)5 * L * t->state));
  chk(talloc(t, t->sized, &t->dt_dev, (size_t)nsteps));
  chk(talloc(t, t->sized, &t->tau, (size_t)(euler ? L : 1) * 4 * h->Kp));
  chk(talloc(t, t->sized, &t->maxv_tmp, (size_t)4 * h->Kp));
  chk(talloc(t, t->sized, &t->tau_tmp, (size_t)4 * h->Kp));
  chk(talloc(t, t->sized, &t->sc_tmp, 1));
  if (st != DGLM_OK) {
    for (void *p : t->sized) cudaFree(p);
    t->sized.clear();
    t->bytes -= t->sized_bytes;
    t->sized_bytes = 0;
    return st;
  }
  cudaStream_t s = h->stream;
  // zero-filled so the padded tail elements of every stored state stay zero
  cudaError_t e = cudaMemsetAsync(t->ckpt, 0, sbytes * slots, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(t->store, 0, sbytes * 5 * L, s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(t->tau, 0, sizeof(double) * (euler ? L : 1) * 4 * h->Kp, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(t->tau_tmp, 0, sizeof(double) * 4 * h->Kp, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(t->sc_tmp, 0, sizeof(DevScalars), s);
  // advection: the penalty is fixed at set-state time
  if (e == cudaSuccess && !euler)
    e = cudaMemcpyAsync(t->tau, h->tau, sizeof(double) * 4 * h->Kp, cudaMemcpyDeviceToDevice, s);
  const double zero = 0.0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&h->sc->dt_fixed, &zero, sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_check(e, "dglm_adjoint_record_capped");
  revolve_spine(plan, nchunk, slots - 1, t->spine);
  h->launches = 0;
  size_t q = 0;
  for (int i = 0; i < nsteps; i++) {
    if (q < t->spine.size() && i == t->spine[q] * L) {
      e = cudaMemcpyAsync(t->ckpt + q * t->state, h->u[h->cur], sbytes,
                          cudaMemcpyDeviceToDevice, s);
      q++;
      if (e != cudaSuccess) return cuda_check(e, "dglm_adjoint_record_capped");
    }
    st = run_steps(h, 1);
    if (st != DGLM_OK) return st;
    e = cudaMemcpyAsync(t->dt_dev + i, &h->sc->dt, sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return cuda_check(e, "dglm_adjoint_record_capped");
  }
  t->dt.assign(nsteps, 0.0);
  e = cudaMemcpyAsync(t->dt.data(), t->dt_dev, sizeof(double) * nsteps, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_check(e, "dglm_adjoint_record_capped");
  for (double d : t->dt)
    if (!std::isfinite(d) || d < 0)
      return set_error(DGLM_ERR_NONFINITE, "dglm_adjoint_record_capped: non-finite dt recorded");
  t->nsteps = nsteps;
  t->every = 0;
  t->nseg = 0;
  t->last_seg_stored = false;
  t->leaf = L;
  t->slots = slots;
  t->nchunk = nchunk;
  t->plan_f = plan.f;
  t->plan_split = plan.split;
  std::vector<RevAction> acts;
  revolve_actions(plan, 0, nchunk, 0, slots - 1, true, acts);
  t->advance_steps = revolve_advance_steps(acts, L, nsteps);
  t->capped = true;
  t->spine_valid = true;
  t->recorded = true;
  return DGLM_OK;
}

dglm_status dglm_adjoint_tape_plan(dglm_handle *h, int *leaf, int *slots,
                                   long long *advance_steps) {
  if (!h || !leaf || !slots || !advance_steps)
    return set_error(DGLM_ERR_INVALID, "dglm_adjoint_tape_plan: NULL argument");
  if (!h->tape || !h->tape->recorded)
    return set_error(DGLM_ERR_STATE, "dglm_adjoint_tape_plan: record a forward run first");
  const AdjointTape *t = h->tape;
  *leaf = t->capped ? t->leaf : t->every;
  *slots = t->capped ? t->slots : t->nseg;
  *advance_steps = t->capped ? t->advance_steps : 0;
  return DGLM_OK;
}

dglm_status dglm_adjoint_schedule(int nsteps, int leaf, int slots, int prestored, int *spine,
                                  int max_spine, int *n_spine, int *actions, int max_actions,
                                  int *n_actions, long long *advance_steps) {
  if (!n_spine || !n_actions || !advance_steps || (max_spine > 0 && !spine) ||
      (max_actions > 0 && !actions))
    return set_error(DGLM_ERR_INVALID, "dglm_adjoint_schedule: NULL argument");
  if (nsteps <= 0 || leaf <= 0 || slots <= 0)
    return set_error(DGLM_ERR_INVALID,
                     "dglm_adjoint_schedule: nsteps, leaf and slots must be positive");
  const int n = (nsteps + leaf - 1) / leaf;
  if (n > 4 * kMaxChunks)
    return set_error(DGLM_ERR_INVALID, "dglm_adjoint_schedule: more than " +
                                           std::to_string(4 * kMaxChunks) + " chunks");
  const int free = std::min(slots - 1, n - 1);
  RevolvePlan plan;
  plan_revolve(plan, n, free);
  std::vector<int> sp;
  revolve_spine(plan, n, free, sp);
  std::vector<RevAction> acts;
  revolve_actions(plan, 0, n, 0, free, prestored != 0, acts);
  *n_spine = (int)sp.size();
  *n_actions = (int)acts.size();
  *advance_steps = revolve_advance_steps(acts, leaf, nsteps);
  if ((int)sp.size() > max_spine || (int)acts.size() > max_actions)
    return set_error(DGLM_ERR_INVALID, "dglm_adjoint_schedule: output arrays too short");
  for (size_t q = 0; q < sp.size(); q++) spine[q] = sp[q];
  for (size_t x = 0; x < acts.size(); x++) {
    int *r = actions + 5 * x;
    r[0] = acts[x].kind;
    r[1] = acts[x].src;
    r[2] = acts[x].chunk;
    r[3] = acts[x].count;
    r[4] = acts[x].dst;
  }
  return DGLM_OK;
}

dglm_status dglm_adjoint_tape_bytes(dglm_handle *h, size_t *bytes) {
  if (!h || !bytes) return set_error(DGLM_ERR_INVALID, "dglm_adjoint_tape_bytes: NULL argument");
  *bytes = h->tape ? h->tape->bytes : 0;
  return DGLM_OK;
}

}  // extern "C"
