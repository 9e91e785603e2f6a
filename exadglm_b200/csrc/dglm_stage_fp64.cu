// Fused FP64 LSERK stage: one kernel per Runge-Kutta stage.
//
// The reference runs each stage as five launches that round-trip every
// intermediate through HBM (euler_nopad_time.cu:63-103): update_ub writes the
// trace average, calc_fluxLM the face flux, calc_fluxes three volume fluxes,
// four batched cuBLAS DGEMMs build utmp, lserk_stage updates k and u.  Here a
// CTA owns a tile of E elements and does all of it on chip:
//
//   0. the tile's state u (all variables) is staged in shared memory with
//      coalesced loads;
//   1. volume fluxes F, G, W at every node, combined with the element's affine
//      metrics into fluxR/S/T (calc_fluxes, euler_dglm.cpp:186-251), go to a
//      shared "column" buffer B with one column per (variable, element);
//   2. acc += [WDr WDs WDt] * [fluxR; fluxS; fluxT]: a register-tiled FP64
//      contraction, R output rows x CPT columns per thread, operators read
//      through L1 from a k-major stacked copy;
//   3. the trace average ub = (u- + u+)/2 (update_ub, euler_dglm.cpp:87-107)
//      with u+ gathered through vmapP, and the face flux
//      (n.F(ub) - tau (ub - u-)) Fscale (calc_fluxLM, :110-183) replace B;
//   4. acc -= LIFT * fluxLM (update_rhs, :254-302);
//   5. epilogue: k = a k + dt rhs, u_out = u_in + b k (lserk_stage,
//      euler_time.cpp:15-38) with coalesced stores; on the fifth stage the
//      per-face wave speed of the new state (calc_maxv, euler_dglm.cpp:6-50)
//      and a device-wide max of maxv*Fscale for the next dt are fused in.
//
// u is ping-ponged between two buffers (u_in -> u_out) because neighbouring
// tiles read u_in's face values while this tile writes its update.
#include <cuda_runtime.h>

#include "dglm_common.cuh"

namespace dglm {

enum { ADV = 0, EUL = 1 };

// Tile shape per (physics, N): E elements per CTA, R output rows per thread,
// CPT columns per thread (Euler: the 5 variables of one element; advection:
// CPT elements of the single variable).
template <int PHYS, int N>
struct Tile;

#define DGLM_TILE(P, NN, EE, RR, CC)             \
  template <>                                    \
  struct Tile<P, NN> {                           \
    static constexpr int E = EE, R = RR, CPT = CC; \
  };
DGLM_TILE(EUL, 1, 128, 4, 5)
DGLM_TILE(EUL, 2, 64, 5, 5)
DGLM_TILE(EUL, 3, 32, 5, 5)
DGLM_TILE(EUL, 4, 16, 5, 5)
DGLM_TILE(EUL, 5, 8, 7, 5)
DGLM_TILE(EUL, 6, 8, 7, 5)
DGLM_TILE(EUL, 7, 4, 8, 5)
DGLM_TILE(EUL, 8, 4, 8, 5)
DGLM_TILE(ADV, 1, 256, 4, 4)
DGLM_TILE(ADV, 2, 128, 5, 4)
DGLM_TILE(ADV, 3, 64, 5, 4)
DGLM_TILE(ADV, 4, 64, 5, 4)
DGLM_TILE(ADV, 5, 32, 7, 4)
DGLM_TILE(ADV, 6, 32, 7, 4)
DGLM_TILE(ADV, 7, 16, 8, 4)
DGLM_TILE(ADV, 8, 16, 8, 4)
#undef DGLM_TILE

template <int PHYS, int N>
struct Cfg {
  static constexpr int NV = PHYS == EUL ? 5 : 1;
  static constexpr int Np = np_of(N), Nfp = nfp_of(N), NFF = 4 * Nfp;
  static constexpr int E = Tile<PHYS, N>::E, R = Tile<PHYS, N>::R, CPT = Tile<PHYS, N>::CPT;
  static constexpr int G = (Np + R - 1) / R;       // row groups
  static constexpr int IP = G * R;                 // padded rows of AT
  static constexpr int NCOL = NV * E;              // columns of B
  static constexpr int CG = NCOL / CPT;            // column groups
  static constexpr int THREADS = CG * G;
  static constexpr int BROWS = (3 * Np > NFF) ? 3 * Np : NFF;
  static constexpr size_t SMEM =
      sizeof(double) * ((size_t)NV * E * Np + (size_t)BROWS * NCOL) + sizeof(int) * NFF;
  static_assert(NCOL % CPT == 0, "columns must split evenly");
  static_assert(NV * E * Np <= BROWS * NCOL, "epilogue reuses B for the rhs");
};

template <int PHYS, int N>
__global__ void __launch_bounds__(Cfg<PHYS, N>::THREADS)
    stage_fp64_kernel(const StageArgs a) {
  using C = Cfg<PHYS, N>;
  constexpr int NV = C::NV, Np = C::Np, Nfp = C::Nfp, NFF = C::NFF, E = C::E, R = C::R,
                CPT = C::CPT, CG = C::CG, NCOL = C::NCOL, IP = C::IP;
  extern __shared__ __align__(16) double smem[];
  double *sU = smem;                              // [NV][E][Np]
  double *sB = sU + NV * E * Np;                  // [BROWS][NCOL], col = v*E + e
  int *sFm = reinterpret_cast<int *>(sB + C::BROWS * NCOL);

  const int tid = threadIdx.x;
  const long e0 = (long)blockIdx.x * E;
  const int ne = (int)min((long)E, (long)a.K - e0);
  const long vs = a.vs;

  for (int i = tid; i < NFF; i += C::THREADS) sFm[i] = a.Fmask[i];
  // 0. stage the tile's state
  for (int v = 0; v < NV; v++) {
    const double *src = a.u_in + v * vs + e0 * Np;
    for (int i = tid; i < E * Np; i += C::THREADS)
      sU[v * E * Np + i] = (i < ne * Np) ? src[i] : (v == 0 ? 1.0 : 0.0);
  }
  __syncthreads();

  // 1. volume fluxes -> B rows [0, 3Np)
  for (int it = tid; it < E * Np; it += C::THREADS) {
    const int e = it / Np, i = it % Np;
    double g[9];
    if (e < ne) {
#pragma unroll
      for (int m = 0; m < 9; m++) g[m] = __ldg(a.geo + (long)m * a.K + e0 + e);
    } else {
#pragma unroll
      for (int m = 0; m < 9; m++) g[m] = 0.0;
    }
    if (PHYS == EUL) {
      double q[5], F[5], Gf[5], W[5];
#pragma unroll
      for (int v = 0; v < 5; v++) q[v] = sU[v * E * Np + e * Np + i];
      euler_flux(a.gamma, q, F, Gf, W);
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const int col = v * E + e;
        sB[(0 * Np + i) * NCOL + col] = g[0] * F[v] + g[1] * Gf[v] + g[2] * W[v];
        sB[(1 * Np + i) * NCOL + col] = g[3] * F[v] + g[4] * Gf[v] + g[5] * W[v];
        sB[(2 * Np + i) * NCOL + col] = g[6] * F[v] + g[7] * Gf[v] + g[8] * W[v];
      }
    } else {
      const long n = (e < ne) ? (e0 + e) * Np + i : 0;
      const double uu = sU[e * Np + i];
      const double F = __ldg(a.vel + n) * uu, Gf = __ldg(a.vel + vs + n) * uu,
                   W = __ldg(a.vel + 2 * vs + n) * uu;
      sB[(0 * Np + i) * NCOL + e] = g[0] * F + g[1] * Gf + g[2] * W;
      sB[(1 * Np + i) * NCOL + e] = g[3] * F + g[4] * Gf + g[5] * W;
      sB[(2 * Np + i) * NCOL + e] = g[6] * F + g[7] * Gf + g[8] * W;
    }
  }
  __syncthreads();

  // 2. volume contraction
  const int cg = tid % CG, rg = tid / CG;
  double acc[R][CPT];
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int j = 0; j < CPT; j++) acc[r][j] = 0.0;

  const double *Ab = a.AT + rg * R;
#pragma unroll 3
  for (int k = 0; k < 3 * Np; k++) {
    double bv[CPT], av[R];
#pragma unroll
    for (int j = 0; j < CPT; j++) bv[j] = sB[k * NCOL + cg + j * CG];
#pragma unroll
    for (int r = 0; r < R; r++) av[r] = __ldg(Ab + (long)k * IP + r);
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
      for (int j = 0; j < CPT; j++) acc[r][j] = fma(av[r], bv[j], acc[r][j]);
  }
  __syncthreads();

  // 3. face traces and fluxes -> B rows [0, NFF)
  for (int it = tid; it < E * NFF; it += C::THREADS) {
    const int e = it / NFF, fj = it % NFF, f = fj / Nfp;
    const int nodeM = sFm[fj];
    if (e >= ne) {
#pragma unroll
      for (int v = 0; v < NV; v++) sB[fj * NCOL + v * E + e] = 0.0;
      continue;
    }
    const long gf = (e0 + e) * 4 + f;
    const long idxP = __ldg(a.vmapP + (e0 + e) * NFF + fj);
    const double nx = __ldg(a.nrm + gf), ny = __ldg(a.nrm + 4L * a.K + gf),
                 nz = __ldg(a.nrm + 8L * a.K + gf);
    const double fs = __ldg(a.fscale + gf), tau = __ldg(a.tau + gf);
    if (PHYS == EUL) {
      double qm[5], qb[5], F[5], Gf[5], W[5];
#pragma unroll
      for (int v = 0; v < 5; v++) {
        qm[v] = sU[v * E * Np + e * Np + nodeM];
        qb[v] = 0.5 * (qm[v] + __ldg(a.u_in + v * vs + idxP));
      }
      euler_flux(a.gamma, qb, F, Gf, W);
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const double nd = nx * F[v] + ny * Gf[v] + nz * W[v];
        sB[fj * NCOL + v * E + e] = (nd - tau * (qb[v] - qm[v])) * fs;
      }
    } else {
      const double um = sU[e * Np + nodeM];
      const double ub = 0.5 * (um + __ldg(a.u_in + idxP));
      const long nM = (e0 + e) * Np + nodeM;
      const double F = __ldg(a.vel + nM) * ub, Gf = __ldg(a.vel + vs + nM) * ub,
                   W = __ldg(a.vel + 2 * vs + nM) * ub;
      const double nd = nx * F + ny * Gf + nz * W;
      sB[fj * NCOL + e] = (nd - tau * (ub - um)) * fs;
    }
  }
  __syncthreads();

  // 4. lift contraction (AT rows [3Np, 3Np+NFF) hold -LIFT^T)
  const double *Al = a.AT + (long)3 * Np * IP + rg * R;
#pragma unroll 3
  for (int k = 0; k < NFF; k++) {
    double bv[CPT], av[R];
#pragma unroll
    for (int j = 0; j < CPT; j++) bv[j] = sB[k * NCOL + cg + j * CG];
#pragma unroll
    for (int r = 0; r < R; r++) av[r] = __ldg(Al + (long)k * IP + r);
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
      for (int j = 0; j < CPT; j++) acc[r][j] = fma(av[r], bv[j], acc[r][j]);
  }
  __syncthreads();

  // 5. epilogue through shared memory: rhs as [v][e][i] in B
  double *sR = sB;
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int i = rg * R + r;
    if (i < Np) {
#pragma unroll
      for (int j = 0; j < CPT; j++) sR[(cg + j * CG) * Np + i] = acc[r][j];
    }
  }
  __syncthreads();

  const double dt = a.dt_override >= 0 ? a.dt_override : a.sc->dt;
  for (int v = 0; v < NV; v++) {
    const long base = v * vs + e0 * Np;
    for (int i = tid; i < ne * Np; i += C::THREADS) {
      const double rhs = sR[v * E * Np + i];
      if (a.rhs_only) {
        a.u_out[base + i] = rhs;
      } else {
        const double kn = a.rka * a.kreg[base + i] + dt * rhs;
        const double un = sU[v * E * Np + i] + a.rkb * kn;
        a.kreg[base + i] = kn;
        a.u_out[base + i] = un;
        sU[v * E * Np + i] = un;
      }
    }
  }
  if (PHYS != EUL || !a.last_stage || a.rhs_only) return;
  __syncthreads();

  // fused calc_maxv on the new state (Euler): per face max |v|^2 and c^2
  __shared__ unsigned long long sMax[32];
  unsigned long long local = 0ull;
  for (int it = tid; it < ne * 4; it += C::THREADS) {
    const int e = it / 4, f = it % 4;
    double mv2 = 0.0, mc2 = 0.0;
    bool bad = false;
    for (int j = 0; j < Nfp; j++) {
      const int nd = e * Np + sFm[f * Nfp + j];
      const double u1 = sU[nd], u2 = sU[E * Np + nd], u3 = sU[2 * E * Np + nd],
                   u4 = sU[3 * E * Np + nd], u5 = sU[4 * E * Np + nd];
      const double vx = u2 / u1, vy = u3 / u1, vz = u4 / u1;
      const double v2 = vx * vx + vy * vy + vz * vz;
      mv2 = v2 > mv2 ? v2 : mv2;
      const double pres = (a.gamma - 1) * (u5 - 0.5 * u1 * v2);
      const double c2 = fabs(a.gamma * pres / u1);
      mc2 = c2 > mc2 ? c2 : mc2;
      bad |= (v2 != v2) || (c2 != c2);
    }
    const long gf = (e0 + e) * 4 + f;
    double mv = sqrt(mv2) + sqrt(mc2);
    if (bad) mv = __longlong_as_double(0x7ff8000000000000LL);
    a.maxv[gf] = mv;
    const unsigned long long b = dbits(mv * __ldg(a.fscale + gf));
    local = b > local ? b : local;
  }
  local = warp_max_bits(local);
  if ((tid & 31) == 0) sMax[tid >> 5] = local;
  __syncthreads();
  if (tid < 32) {
    unsigned long long v = tid < (C::THREADS + 31) / 32 ? sMax[tid] : 0ull;
    v = warp_max_bits(v);
    if (tid == 0) atomicMax(&a.sc->acc[a.sc->parity ^ 1], v);
  }
}

// Standalone calc_maxv (initial state, advection velocity): maxv per face and
// a device-wide max of maxv*Fscale into sc->acc[slot].
template <int PHYS, int N>
__global__ void face_maxv_kernel(const StageArgs a, int slot) {
  constexpr int Np = np_of(N), Nfp = nfp_of(N);
  __shared__ unsigned long long sMax[32];
  unsigned long long local = 0ull;
  const long nF = 4L * a.K;
  for (long gf = blockIdx.x * (long)blockDim.x + threadIdx.x; gf < nF;
       gf += (long)gridDim.x * blockDim.x) {
    const long e = gf / 4;
    const int f = (int)(gf % 4);
    double mv2 = 0.0, mc2 = 0.0;
    bool bad = false;
    for (int j = 0; j < Nfp; j++) {
      const long nd = e * Np + a.Fmask[f * Nfp + j];
      if (PHYS == EUL) {
        const double u1 = a.u_in[nd], u2 = a.u_in[a.vs + nd], u3 = a.u_in[2 * a.vs + nd],
                     u4 = a.u_in[3 * a.vs + nd], u5 = a.u_in[4 * a.vs + nd];
        const double vx = u2 / u1, vy = u3 / u1, vz = u4 / u1;
        const double v2 = vx * vx + vy * vy + vz * vz;
        mv2 = v2 > mv2 ? v2 : mv2;
        const double pres = (a.gamma - 1) * (u5 - 0.5 * u1 * v2);
        const double c2 = fabs(a.gamma * pres / u1);
        mc2 = c2 > mc2 ? c2 : mc2;
        bad |= (v2 != v2) || (c2 != c2);
      } else {
        const double vx = a.vel[nd], vy = a.vel[a.vs + nd], vz = a.vel[2 * a.vs + nd];
        const double v2 = vx * vx + vy * vy + vz * vz;
        mv2 = v2 > mv2 ? v2 : mv2;
        bad |= (v2 != v2);
      }
    }
    double mv = (PHYS == EUL) ? sqrt(mv2) + sqrt(mc2) : sqrt(mv2);
    if (bad) mv = __longlong_as_double(0x7ff8000000000000LL);
    a.maxv[gf] = mv;
    const unsigned long long b = dbits(mv * a.fscale[gf]);
    local = b > local ? b : local;
  }
  local = warp_max_bits(local);
  if ((threadIdx.x & 31) == 0) sMax[threadIdx.x >> 5] = local;
  __syncthreads();
  if (threadIdx.x < 32) {
    unsigned long long v = threadIdx.x < (blockDim.x + 31) / 32 ? sMax[threadIdx.x] : 0ull;
    v = warp_max_bits(v);
    if (threadIdx.x == 0) atomicMax(&a.sc->acc[slot], v);
  }
}

// dt for the coming step: the CFL dt from the device max (or the prescribed
// dt), clipped so the step ends at tmax (euler_time.cpp:49-57); steps
// requested after t reached tmax get dt = 0 and leave u unchanged.  With a
// frozen wave speed (advection: the velocity field does not change) the max
// stays in acc[0]; otherwise the last stage of each step accumulates the max
// of the new state into the other slot.
__global__ void step_begin_kernel(int N, double cfl, double tmax, int frozen, DevScalars *sc,
                                  double *dt_hist) {
  if (threadIdx.x != 0) return;
  const int p = frozen ? 0 : sc->parity;
  const double m = __longlong_as_double((long long)sc->acc[p]);
  double dt = sc->dt_fixed > 0 ? sc->dt_fixed : (cfl / (2 * N + 1)) * (1 / m);
  if (!(dt > 0) || dt != dt || dt > 1e300) sc->flags |= 1;
  const int active = sc->t < tmax;
  if (active && sc->t + dt > tmax) dt = tmax - sc->t;
  if (!active) dt = 0.0;
  sc->dt = dt;
  sc->active = active;
  if (!frozen) sc->acc[p ^ 1] = 0ull;
  if (dt_hist && active) dt_hist[sc->tstep % kHistory] = dt;
}

// NaN/Inf scan of an uploaded state (sets flags bit 1)
__global__ void finite_check_kernel(const double *__restrict__ u, long vs, long n, int nvar,
                                    DevScalars *sc) {
  bool bad = false;
  for (int v = 0; v < nvar; v++)
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
      bad |= !isfinite(u[v * vs + i]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&sc->flags, 2);
}

__global__ void step_end_kernel(DevScalars *sc) {
  if (threadIdx.x != 0) return;
  if (sc->active) {
    sc->t += sc->dt;
    sc->tstep += 1;
  }
  sc->parity ^= 1;
}

// update_tau (euler_dglm.cpp:72-84)
__global__ void tau_kernel(int K, double tau_scale, const int *__restrict__ vmapF,
                           const double *__restrict__ maxv, double *__restrict__ tau) {
  const long f = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (f < 4L * K) tau[f] = 0.25 * (maxv[f] + maxv[vmapF[f]]) * tau_scale;
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------

template <int PHYS, int N>
static cudaError_t launch_one(const StageArgs &a, cudaStream_t s) {
  using C = Cfg<PHYS, N>;
  // set per call: the attribute belongs to the current device's context
  cudaError_t e = cudaFuncSetAttribute(stage_fp64_kernel<PHYS, N>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
  if (e != cudaSuccess) return e;
  const int blocks = (a.K + C::E - 1) / C::E;
  stage_fp64_kernel<PHYS, N><<<blocks, C::THREADS, C::SMEM, s>>>(a);
  return cudaGetLastError();
}

template <int PHYS, int N>
static cudaError_t launch_maxv_one(const StageArgs &a, int slot, cudaStream_t s) {
  const long nF = 4L * a.K;
  int blocks = (int)((nF + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  face_maxv_kernel<PHYS, N><<<blocks, 256, 0, s>>>(a, slot);
  return cudaGetLastError();
}

#define DGLM_DISPATCH(FN, PHYS, N, ...)                        \
  switch (N) {                                                 \
    case 1: return FN<PHYS, 1>(__VA_ARGS__);                   \
    case 2: return FN<PHYS, 2>(__VA_ARGS__);                   \
    case 3: return FN<PHYS, 3>(__VA_ARGS__);                   \
    case 4: return FN<PHYS, 4>(__VA_ARGS__);                   \
    case 5: return FN<PHYS, 5>(__VA_ARGS__);                   \
    case 6: return FN<PHYS, 6>(__VA_ARGS__);                   \
    case 7: return FN<PHYS, 7>(__VA_ARGS__);                   \
    case 8: return FN<PHYS, 8>(__VA_ARGS__);                   \
    default: return cudaErrorInvalidValue;                     \
  }

bool stage_fp64_supported(int physics, int N) {
  return (physics == DGLM_EULER || physics == DGLM_ADVECTION) && N >= 1 && N <= kMaxOrder;
}

template <int PHYS, int N>
static int ip_of() { return Cfg<PHYS, N>::IP; }

int stage_rows_padded(int physics, int N) {
  if (physics == DGLM_EULER) {
    switch (N) {
      case 1: return ip_of<EUL, 1>(); case 2: return ip_of<EUL, 2>();
      case 3: return ip_of<EUL, 3>(); case 4: return ip_of<EUL, 4>();
      case 5: return ip_of<EUL, 5>(); case 6: return ip_of<EUL, 6>();
      case 7: return ip_of<EUL, 7>(); case 8: return ip_of<EUL, 8>();
    }
  } else {
    switch (N) {
      case 1: return ip_of<ADV, 1>(); case 2: return ip_of<ADV, 2>();
      case 3: return ip_of<ADV, 3>(); case 4: return ip_of<ADV, 4>();
      case 5: return ip_of<ADV, 5>(); case 6: return ip_of<ADV, 6>();
      case 7: return ip_of<ADV, 7>(); case 8: return ip_of<ADV, 8>();
    }
  }
  return -1;
}

cudaError_t launch_stage_fp64(int physics, int N, const StageArgs &a, cudaStream_t s) {
  if (physics == DGLM_EULER) {
    DGLM_DISPATCH(launch_one, EUL, N, a, s)
  } else {
    DGLM_DISPATCH(launch_one, ADV, N, a, s)
  }
}

cudaError_t launch_face_maxv(int physics, int N, const StageArgs &a, int slot,
                             cudaStream_t s) {
  if (physics == DGLM_EULER) {
    DGLM_DISPATCH(launch_maxv_one, EUL, N, a, slot, s)
  } else {
    DGLM_DISPATCH(launch_maxv_one, ADV, N, a, slot, s)
  }
}

cudaError_t launch_step_begin(int N, double cfl, double tmax, int frozen, DevScalars *sc,
                              double *dt_hist, cudaStream_t s) {
  step_begin_kernel<<<1, 32, 0, s>>>(N, cfl, tmax, frozen, sc, dt_hist);
  return cudaGetLastError();
}

cudaError_t launch_tau(int K, double tau_scale, const int *vmapF, const double *maxv,
                       double *tau, cudaStream_t s) {
  const long n = 4L * K;
  tau_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(K, tau_scale, vmapF, maxv, tau);
  return cudaGetLastError();
}

cudaError_t launch_finite_check(const double *u, long vs, long n, int nvar, DevScalars *sc,
                                cudaStream_t s) {
  finite_check_kernel<<<148 * 8, 256, 0, s>>>(u, vs, n, nvar, sc);
  return cudaGetLastError();
}

cudaError_t launch_step_end(DevScalars *sc, cudaStream_t s) {
  step_end_kernel<<<1, 32, 0, s>>>(sc);
  return cudaGetLastError();
}

}  // namespace dglm
