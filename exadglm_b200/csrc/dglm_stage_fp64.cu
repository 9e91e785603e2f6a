// Fused FP64 LSERK stage: one kernel per Runge-Kutta stage.
//
// The reference runs each stage as five launches that round-trip every
// intermediate through HBM (euler_nopad_time.cu:63-103): update_ub writes the
// trace average, calc_fluxLM the face flux, calc_fluxes three volume fluxes,
// four batched cuBLAS DGEMMs build utmp, lserk_stage updates k and u.  Here a
// CTA owns a tile of E elements and does all of it on chip:
//
//   0. the tile's state u (all variables), its metrics, face data and vmapP
//      are staged in shared memory with coalesced loads;
//   1. volume fluxes F, G, W at every node, combined with the element's affine
//      metrics into fluxR/S/T (calc_fluxes, euler_dglm.cpp:186-251), go to a
//      shared column buffer B, one column per (variable, element);
//   2. acc += [WDr WDs WDt] * [fluxR; fluxS; fluxT];
//   3. the trace average ub = (u- + u+)/2 (update_ub, euler_dglm.cpp:87-107)
//      with u+ gathered through vmapP, and the face flux
//      (n.F(ub) - tau (ub - u-)) Fscale (calc_fluxLM, :110-183) replace B;
//   4. acc -= LIFT * fluxLM (update_rhs, :254-302);
//   5. epilogue: k = a k + dt rhs, u_out = u_in + b k (lserk_stage,
//      euler_time.cpp:15-38) with coalesced stores; on the fifth stage the
//      per-face wave speed of the new state (calc_maxv, euler_dglm.cpp:6-50)
//      and a device-wide max of maxv*Fscale for the next dt are fused in.
//
// Two contraction engines share this skeleton:
//   SIMT  register-tiled DFMA, R rows x CPT columns per thread, operators in
//         a k-major stacked copy read through L1;
//   DMMA  FP64 tensor-core mma.sync.m8n8k4, operators pre-swizzled into A
//         fragments (one coalesced 256-byte load per fragment), B fragments
//         from shared memory, 8x8 accumulators in registers.
//
// u is ping-ponged between two buffers (u_in -> u_out) because neighbouring
// tiles read u_in's face values while this tile writes its update.
//
// Shared layouts put the element index fastest ([..][e], row stride E+1)
// so that every phase's per-lane accesses are consecutive or odd-strided.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <type_traits>
#include <vector>

#include "dglm_common.cuh"

namespace dglm {

enum { ADV = 0, EUL = 1 };

// Euler flux with one reciprocal per node: v = m / rho, p = (gamma-1)(E -
// m.v/2), H = E + p.  The reference's per-term divisions
// (euler_dglm.cpp:152-168) agree with it to rounding.
__device__ __forceinline__ void euler_flux_fast(double g, const double q[5], double F[5],
                                                double G[5], double W[5]) {
  const double ir = 1.0 / q[0];
  const double vx = q[1] * ir, vy = q[2] * ir, vz = q[3] * ir;
  const double p = (g - 1) * (q[4] - 0.5 * (q[1] * vx + q[2] * vy + q[3] * vz));
  const double H = q[4] + p;
  F[0] = q[1]; F[1] = q[1] * vx + p; F[2] = q[2] * vx; F[3] = q[3] * vx; F[4] = H * vx;
  G[0] = q[2]; G[1] = q[1] * vy; G[2] = q[2] * vy + p; G[3] = q[3] * vy; G[4] = H * vy;
  W[0] = q[3]; W[1] = q[1] * vz; W[2] = q[2] * vz; W[3] = q[3] * vz + p; W[4] = H * vz;
}

// Centring of split-precision operands.  A flux that is constant over an
// element has zero DG right-hand side (the weak volume term equals the
// surface term on straight-sided tetrahedra), so subtracting each element's
// node-0 flux from all its flux values leaves the contraction's result
// unchanged, while the split parts carry only the within-element variation
// (smaller, and with it their rounding).  node0_fluxes writes F, G, W of the
// node-0 state of elements e = t, t + nt, ... < E to cen[e * 15 + (0..4,
// 5..9, 10..14)], reading variable v of element e at u[e * estride + v * vstride];
// centre_sub subtracts them from a node's flux.
constexpr int kCen = 15;
__device__ __forceinline__ void node0_fluxes(double g, const double *u, int estride,
                                             int vstride, int E, int t, int nt, double *cen) {
  for (int e = t; e < E; e += nt) {
    double q[5], F[5], G[5], W[5];
#pragma unroll
    for (int v = 0; v < 5; v++) q[v] = u[e * estride + v * vstride];
    euler_flux_fast(g, q, F, G, W);
#pragma unroll
    for (int v = 0; v < 5; v++) {
      cen[e * kCen + v] = F[v];
      cen[e * kCen + 5 + v] = G[v];
      cen[e * kCen + 10 + v] = W[v];
    }
  }
}
__device__ __forceinline__ void centre_sub(const double *c, double F[5], double G[5],
                                           double W[5]) {
#pragma unroll
  for (int v = 0; v < 5; v++) {
    F[v] -= c[v];
    G[v] -= c[5 + v];
    W[v] -= c[10 + v];
  }
}

// ---------------------------------------------------------------------------
// configuration
// ---------------------------------------------------------------------------

template <int PHYS, int N, int MODE, int E_, int R_, int CPT_, int WM_, int PR_ = 0>
struct Cfg {
  static constexpr int NV = PHYS == EUL ? 5 : 1;
  static constexpr int Np = np_of(N), Nfp = nfp_of(N), NFF = 4 * Nfp;
  static constexpr int E = E_, EP = E_ + 1;
  static constexpr int NCOL = NV * E;
  // SIMT tiling: R rows x CPT columns per thread
  static constexpr int R = R_, CPT = CPT_;
  static constexpr int G = (Np + R - 1) / R;
  static constexpr int CG = NCOL / CPT;
  // DMMA tiling: MT m-tiles of 8 rows, NT n-tiles of 8 columns; each warp
  // owns WM m-tiles x WN n-tiles
  static constexpr int MT = (Np + 7) / 8, NT = NCOL / 8;
  static constexpr int WM = WM_ > MT ? MT : WM_;
  static constexpr int WN = CPT_;
  static constexpr int MGROUPS = (MT + WM - 1) / WM;
  static constexpr int WARPS_D = MODE == MODE_DMMA ? MGROUPS * (NT / WN) : 0;
  // MMA16: split-precision mma.sync, m16n8k8 (TF32, PR_ = 2) or m16n8k16
  // (BF16: two parts, PR_ = 1; three parts, PR_ = 3)
  static constexpr bool M16 = MODE == MODE_MMA16;
  static constexpr int KSTEP16 = PR_ == 2 ? 8 : 16;
  static constexpr int NPARTS16 = PR_ == 3 ? 3 : 2, NPROD16 = PR_ == 3 ? 6 : 3;
  static constexpr int MT16 = (Np + 15) / 16;
  static constexpr int WM16 = WM_ > MT16 ? MT16 : WM_;
  static constexpr int MG16 = (MT16 + WM16 - 1) / WM16;
  static constexpr int WARPS_16 = M16 ? MG16 * (NT / WN) : 0;
  static constexpr int THREADS =
      MODE == MODE_SIMT ? CG * G : 32 * (M16 ? WARPS_16 : WARPS_D);
  static constexpr int KPAD = M16 ? KSTEP16 : 4;
  static constexpr int KV = 3 * Np, KVP = (KV + KPAD - 1) / KPAD * KPAD;   // volume k (padded)
  static constexpr int KF = NFF, KFP = (KF + KPAD - 1) / KPAD * KPAD;
  static constexpr int KSV16 = KVP / KSTEP16, KSF16 = KFP / KSTEP16, KST16 = KSV16 + KSF16;
  static constexpr int SL16 = (KST16 + 7) / 8;   // k-steps per FP32 slice (8 slices)
  static constexpr int IP = MODE == MODE_SIMT ? G * R : 8 * MT;     // padded rows
  static constexpr int BLD = MODE == MODE_SIMT ? NCOL : NCOL + 4;   // B row stride
  static constexpr int BROWS = KVP > KFP ? KVP : KFP;
  // shared memory
  static constexpr int S_U = NV * Np * EP;
  static constexpr int S_B = BROWS * BLD;
  static constexpr int S_GEO = 9 * E;
  static constexpr int S_FACE = 5 * 4 * E;                     // nx ny nz fs tau
  static constexpr int S_CEN = (MODE == MODE_MMA16 && PHYS == EUL) ? kCen * E : 0;
  static constexpr int VMLD = NFF + 1;                         // vmapP row stride (ints)
  static constexpr size_t SMEM = sizeof(double) * (S_U + S_B + S_GEO + S_FACE + S_CEN) +
                                 sizeof(int) * ((size_t)E * VMLD + NFF);
  static_assert(NCOL % CPT_ == 0, "columns must split evenly");
  static_assert(S_B >= NV * Np * EP, "epilogue reuses B for the rhs");
  static_assert(MODE == MODE_SIMT || NCOL % 8 == 0, "DMMA needs whole n-tiles");
  static_assert(MODE == MODE_SIMT || NT % WN == 0, "DMMA n-tiles must split over warps");
  static_assert(THREADS <= 1024, "block too large");
  static_assert(SMEM <= 232448, "shared memory per CTA exceeds 227 KB");
};

// ---------------------------------------------------------------------------
// contraction engines: acc += A[:, k range] * B[rows of the range, :]
// ---------------------------------------------------------------------------

template <class C, int KL>
__device__ __forceinline__ void contract_simt(const double *__restrict__ AT, int kofs,
                                              const double *sB, double (&acc)[C::R][C::CPT],
                                              int tid) {
  const int cg = tid % C::CG, rg = tid / C::CG;
  const double *Ab = AT + (long)kofs * C::IP + rg * C::R;
#pragma unroll 3
  for (int k = 0; k < KL; k++) {
    double bv[C::CPT], av[C::R];
#pragma unroll
    for (int j = 0; j < C::CPT; j++) bv[j] = sB[k * C::BLD + cg + j * C::CG];
#pragma unroll
    for (int r = 0; r < C::R; r++) av[r] = __ldg(Ab + (long)k * C::IP + r);
#pragma unroll
    for (int r = 0; r < C::R; r++)
#pragma unroll
      for (int j = 0; j < C::CPT; j++) acc[r][j] = fma(av[r], bv[j], acc[r][j]);
  }
}

__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

// A fragments are stored [kstep][mtile][lane] in the lane order of the
// m8n8k4 A operand (row = lane/4, col = lane%4): one coalesced load each.
// B fragments (row = lane%4, col = lane/4) come from sB.
template <class C, int KSTEPS>
__device__ __forceinline__ void contract_dmma(const double *__restrict__ Afrag, int kstep0,
                                              const double *sB,
                                              double (&acc)[C::WM][C::WN][2], int warp,
                                              int lane) {
  const int mg = warp % C::MGROUPS, ng = warp / C::MGROUPS;
  const int m0 = mg * C::WM, n0 = ng * C::WN;
  const double *Ab = Afrag + ((long)kstep0 * C::MT + m0) * 32 + lane;
  const double *Bb = sB + (lane & 3) * C::BLD + n0 * 8 + (lane >> 2);
#pragma unroll 2
  for (int ks = 0; ks < KSTEPS; ks++) {
    double av[C::WM], bv[C::WN];
#pragma unroll
    for (int i = 0; i < C::WM; i++)
      av[i] = (m0 + i < C::MT) ? __ldg(Ab + ((long)ks * C::MT + i) * 32) : 0.0;
#pragma unroll
    for (int j = 0; j < C::WN; j++) bv[j] = Bb[ks * 4 * C::BLD + j * 8];
#pragma unroll
    for (int i = 0; i < C::WM; i++)
#pragma unroll
      for (int j = 0; j < C::WN; j++) dmma_8x8x4(acc[i][j], av[i], bv[j]);
  }
}

// Split-precision mma.sync (legacy tensor-core path, for orders whose tcgen05
// operand images do not fit in shared memory).  A = the operator, its parts
// pre-split on the host into fragments [kstep][mtile][part][lane] (4 x 32
// bits per lane, one coalesced 512-byte load); B = the FP64 fluxes in
// shared memory, split in registers; NPROD16 part products per k-step into
// FP32 accumulators that are folded into FP64 every SL16 k-steps.  Euler
// fluxes are centred (node0_fluxes, centre_sub) before they are stored for
// the split.
//   m16n8k8 TF32:  a0=A[g][t] a1=A[g+8][t] a2=A[g][t+4] a3=A[g+8][t+4],
//                  b0=B[t][g] b1=B[t+4][g]
//   m16n8k16 BF16: a0=A[g][2t..2t+1] a1=A[g+8][2t..] a2=A[g][2t+8..] a3=A[g+8][2t+8..],
//                  b0=B[2t..2t+1][g] b1=B[2t+8..2t+9][g]  (low half = lower k)
//   C: c0=C[g][2t] c1=C[g][2t+1] c2=C[g+8][2t] c3=C[g+8][2t+1]
// with g = lane/4, t = lane%4.
__device__ __forceinline__ void mma_tf32_16x8x8(float (&d)[4], const unsigned (&a)[4],
                                                const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ void mma_bf16_16x8x16(float (&d)[4], const unsigned (&a)[4],
                                                 const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// parts of an FP64 value: TF32 (hi, lo) or BF16 (2 or 3 parts) as raw bits
template <int PR>
__device__ __forceinline__ void split_parts(double x, unsigned (&p)[3]) {
  const float f = (float)x;
  if (PR == 2) {
    unsigned h, l;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(f));
    const float r = f - __uint_as_float(h);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(r));
    p[0] = h;
    p[1] = l;
    p[2] = 0;
  } else {
    float r = f;
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const unsigned short b = __bfloat16_as_ushort(__float2bfloat16_rn(r));
      p[q] = b;
      r -= __uint_as_float((unsigned)b << 16);
    }
  }
}

template <class C>
__device__ __forceinline__ void prod16(int q, int &pa, int &pb) {
  if (C::NPARTS16 == 2) {
    pa = q == 0 ? 1 : 0;
    pb = q == 1 ? 1 : 0;
  } else {
    constexpr int A6[6] = {2, 1, 0, 1, 0, 0}, B6[6] = {0, 1, 2, 0, 1, 0};
    pa = A6[q];
    pb = B6[q];
  }
}

template <class C, int PR>
__device__ __forceinline__ void contract_m16(const uint4 *__restrict__ A16, int ks0, int nks,
                                             const double *sB,
                                             float (&acc)[C::WM16][C::WN][4],
                                             double (&tot)[C::WM16][C::WN][4], int warp,
                                             int lane) {
  constexpr int NP = C::NPARTS16, BLD = C::BLD;
  const int mg = warp % C::MG16, ng = warp / C::MG16;
  const int m0 = mg * C::WM16, n0 = ng * C::WN;
  const int g = lane >> 2, t = lane & 3;
#pragma unroll 1
  for (int ks = 0; ks < nks; ks++) {
    const int kg = ks0 + ks;
    unsigned bp[C::WN][3][2];
#pragma unroll
    for (int j = 0; j < C::WN; j++) {
      const double *Bc = sB + (n0 + j) * 8 + g + ks * C::KSTEP16 * BLD;
      if (PR == 2) {
        unsigned p0[3], p1[3];
        split_parts<PR>(Bc[t * BLD], p0);
        split_parts<PR>(Bc[(t + 4) * BLD], p1);
#pragma unroll
        for (int q = 0; q < NP; q++) {
          bp[j][q][0] = p0[q];
          bp[j][q][1] = p1[q];
        }
      } else {
        unsigned x0[3], x1[3], x2[3], x3[3];
        split_parts<PR>(Bc[(2 * t) * BLD], x0);
        split_parts<PR>(Bc[(2 * t + 1) * BLD], x1);
        split_parts<PR>(Bc[(2 * t + 8) * BLD], x2);
        split_parts<PR>(Bc[(2 * t + 9) * BLD], x3);
#pragma unroll
        for (int q = 0; q < NP; q++) {
          bp[j][q][0] = x0[q] | (x1[q] << 16);
          bp[j][q][1] = x2[q] | (x3[q] << 16);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < C::WM16; i++) {
      if (m0 + i >= C::MT16) continue;
      unsigned ap[3][4];
#pragma unroll
      for (int q = 0; q < NP; q++) {
        const uint4 v = __ldg(A16 + (((long)kg * C::MT16 + m0 + i) * NP + q) * 32 + lane);
        ap[q][0] = v.x;
        ap[q][1] = v.y;
        ap[q][2] = v.z;
        ap[q][3] = v.w;
      }
#pragma unroll
      for (int j = 0; j < C::WN; j++)
#pragma unroll
        for (int q = 0; q < C::NPROD16; q++) {
          int pa, pb;
          prod16<C>(q, pa, pb);
          if (PR == 2)
            mma_tf32_16x8x8(acc[i][j], ap[pa], bp[j][pb]);
          else
            mma_bf16_16x8x16(acc[i][j], ap[pa], bp[j][pb]);
        }
    }
    if ((kg + 1) % C::SL16 == 0 || kg + 1 == C::KST16) {
#pragma unroll
      for (int i = 0; i < C::WM16; i++)
#pragma unroll
        for (int j = 0; j < C::WN; j++)
#pragma unroll
          for (int c = 0; c < 4; c++) {
            tot[i][j][c] += (double)acc[i][j][c];
            acc[i][j][c] = 0.f;
          }
    }
  }
}

// ---------------------------------------------------------------------------
// the stage kernel
// ---------------------------------------------------------------------------

template <int PHYS, int N, int MODE, int E_, int R_, int CPT_, int WM_, int PR_>
__global__ void __launch_bounds__(Cfg<PHYS, N, MODE, E_, R_, CPT_, WM_, PR_>::THREADS)
    stage_fp64_kernel(const StageArgs a) {
  using C = Cfg<PHYS, N, MODE, E_, R_, CPT_, WM_, PR_>;
  constexpr int NV = C::NV, Np = C::Np, Nfp = C::Nfp, NFF = C::NFF, E = C::E, EP = C::EP,
                BLD = C::BLD, T = C::THREADS;
  constexpr bool SIMT = MODE == MODE_SIMT, M16 = MODE == MODE_MMA16;
  constexpr int AR = SIMT ? C::R : 1, AC = SIMT ? C::CPT : 1;     // SIMT accumulators
  constexpr int DM = (SIMT || M16) ? 1 : C::WM, DN = (SIMT || M16) ? 1 : C::WN;   // DMMA
  constexpr int QM = M16 ? C::WM16 : 1, QN = M16 ? C::WN : 1;     // MMA16 accumulators
  extern __shared__ __align__(16) double smem[];
  double *sU = smem;                    // [v][i][EP]
  double *sB = sU + C::S_U;             // [k][BLD], col = v*E + e
  double *sGeo = sB + C::S_B;           // [9][E]
  double *sFace = sGeo + C::S_GEO;      // [5][4][E]: nx ny nz fs tau
  double *sCen = sFace + C::S_FACE;    // [E][15]: node-0 fluxes (split modes, Euler)
  int *sVm = reinterpret_cast<int *>(sCen + C::S_CEN);     // [E][VMLD]
  int *sFm = sVm + E * C::VMLD;         // [NFF]

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const long e0 = (long)blockIdx.x * E;
  const int ne = (int)min((long)E, (long)a.K - e0);
  const long vs = a.vs;

  // 0. staging
  for (int i = tid; i < NFF; i += T) sFm[i] = a.Fmask[i];
  for (int v = 0; v < NV; v++) {
    const double *src = a.u_in + v * vs + e0 * Np;
    for (int g = tid; g < E * Np; g += T) {
      const int e = g / Np, i = g - e * Np;
      sU[(v * Np + i) * EP + e] = (g < ne * Np) ? src[g] : (v == 0 ? 1.0 : 0.0);
    }
  }
  for (int g = tid; g < 9 * E; g += T) {
    const int m = g / E, e = g - m * E;
    sGeo[g] = e < ne ? __ldg(a.geo + (long)m * a.gstride + e0 + e) : 0.0;
  }
  for (int g = tid; g < 4 * E; g += T) {
    const int e = g >> 2, f = g & 3;      // consecutive g: consecutive faces in HBM
    const long gf = (e0 + e) * 4 + f;
    const bool ok = e < ne;
    sFace[(0 * 4 + f) * E + e] = ok ? __ldg(a.nrm + gf) : 0.0;
    sFace[(1 * 4 + f) * E + e] = ok ? __ldg(a.nrm + 4L * a.gstride + gf) : 0.0;
    sFace[(2 * 4 + f) * E + e] = ok ? __ldg(a.nrm + 8L * a.gstride + gf) : 0.0;
    sFace[(3 * 4 + f) * E + e] = ok ? __ldg(a.fscale + gf) : 0.0;
    sFace[(4 * 4 + f) * E + e] = ok ? __ldg(a.tau + gf) : 0.0;
  }
  for (int g = tid; g < E * NFF; g += T) {
    const int e = g / NFF, fj = g - e * NFF;
    sVm[e * C::VMLD + fj] = g < ne * NFF ? __ldg(a.vmapP + e0 * NFF + g) : 0;
  }
  __syncthreads();
  if constexpr (M16 && PHYS == EUL) {
    node0_fluxes(a.gamma, sU, 1, Np * EP, E, tid, T, sCen);
    __syncthreads();
  }

  // 1. volume fluxes -> B rows [0, 3Np)
  for (int it = tid; it < E * Np; it += T) {
    const int i = it / E, e = it - i * E;
    const double *g = sGeo + e;
    const double rx = g[0], ry = g[E], rz = g[2 * E], sx = g[3 * E], sy = g[4 * E],
                 sz = g[5 * E], tx = g[6 * E], ty = g[7 * E], tz = g[8 * E];
    if (PHYS == EUL) {
      double q[5], F[5], Gf[5], W[5];
#pragma unroll
      for (int v = 0; v < 5; v++) q[v] = sU[(v * Np + i) * EP + e];
      euler_flux_fast(a.gamma, q, F, Gf, W);
      if constexpr (M16) centre_sub(sCen + e * kCen, F, Gf, W);
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const int col = v * E + e;
        sB[(0 * Np + i) * BLD + col] = rx * F[v] + ry * Gf[v] + rz * W[v];
        sB[(1 * Np + i) * BLD + col] = sx * F[v] + sy * Gf[v] + sz * W[v];
        sB[(2 * Np + i) * BLD + col] = tx * F[v] + ty * Gf[v] + tz * W[v];
      }
    } else {
      const long n = (e < ne) ? (e0 + e) * Np + i : 0;
      const double uu = sU[i * EP + e];
      const double F = __ldg(a.vel + n) * uu, Gf = __ldg(a.vel + vs + n) * uu,
                   W = __ldg(a.vel + 2 * vs + n) * uu;
      sB[(0 * Np + i) * BLD + e] = rx * F + ry * Gf + rz * W;
      sB[(1 * Np + i) * BLD + e] = sx * F + sy * Gf + sz * W;
      sB[(2 * Np + i) * BLD + e] = tx * F + ty * Gf + tz * W;
    }
  }
  if (!SIMT) {   // zero the k padding rows of the volume block
    for (int g = tid; g < (C::KVP - C::KV) * BLD; g += T) sB[C::KV * BLD + g] = 0.0;
  }
  __syncthreads();

  // 2. volume contraction
  double accS[AR][AC];
  double accD[DM][DN][2];
#pragma unroll
  for (int r = 0; r < AR; r++)
#pragma unroll
    for (int j = 0; j < AC; j++) accS[r][j] = 0.0;
#pragma unroll
  for (int i = 0; i < DM; i++)
#pragma unroll
    for (int j = 0; j < DN; j++) accD[i][j][0] = accD[i][j][1] = 0.0;
  float acc16[QM][QN][4];
  double tot16[QM][QN][4];
#pragma unroll
  for (int i = 0; i < QM; i++)
#pragma unroll
    for (int j = 0; j < QN; j++)
#pragma unroll
      for (int c = 0; c < 4; c++) {
        acc16[i][j][c] = 0.f;
        tot16[i][j][c] = 0.0;
      }
  if constexpr (SIMT) {
    contract_simt<C, C::KV>(a.AT, 0, sB, accS, tid);
  } else if constexpr (M16) {
    contract_m16<C, PR_>(reinterpret_cast<const uint4 *>(a.AT), 0, C::KSV16, sB, acc16, tot16,
                         warp, lane);
  } else {
    if (warp < C::WARPS_D) contract_dmma<C, C::KVP / 4>(a.AT, 0, sB, accD, warp, lane);
  }
  __syncthreads();

  // 3. face traces and fluxes -> B rows [0, NFF)
  for (int it = tid; it < E * NFF; it += T) {
    const int fj = it / E, e = it - fj * E, f = fj / Nfp;
    const int nodeM = sFm[fj];
    if (e >= ne) {
#pragma unroll
      for (int v = 0; v < NV; v++) sB[fj * BLD + v * E + e] = 0.0;
      continue;
    }
    const long idxP = sVm[e * C::VMLD + fj];
    const double nx = sFace[(0 * 4 + f) * E + e], ny = sFace[(1 * 4 + f) * E + e],
                 nz = sFace[(2 * 4 + f) * E + e], fs = sFace[(3 * 4 + f) * E + e],
                 tau = sFace[(4 * 4 + f) * E + e];
    if (PHYS == EUL) {
      double qm[5], qb[5], F[5], Gf[5], W[5];
#pragma unroll
      for (int v = 0; v < 5; v++) {
        qm[v] = sU[(v * Np + nodeM) * EP + e];
        qb[v] = 0.5 * (qm[v] + __ldg(a.u_in + v * vs + idxP));
      }
      euler_flux_fast(a.gamma, qb, F, Gf, W);
      if constexpr (M16) centre_sub(sCen + e * kCen, F, Gf, W);
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const double nd = nx * F[v] + ny * Gf[v] + nz * W[v];
        sB[fj * BLD + v * E + e] = (nd - tau * (qb[v] - qm[v])) * fs;
      }
    } else {
      const double um = sU[nodeM * EP + e];
      const double ub = 0.5 * (um + __ldg(a.u_in + idxP));
      const long nM = (e0 + e) * Np + nodeM;
      const double F = __ldg(a.vel + nM) * ub, Gf = __ldg(a.vel + vs + nM) * ub,
                   W = __ldg(a.vel + 2 * vs + nM) * ub;
      const double nd = nx * F + ny * Gf + nz * W;
      sB[fj * BLD + e] = (nd - tau * (ub - um)) * fs;
    }
  }
  if (!SIMT) {
    for (int g = tid; g < (C::KFP - C::KF) * BLD; g += T) sB[C::KF * BLD + g] = 0.0;
  }
  __syncthreads();

  // 4. lift contraction (A columns [3Np, 3Np+NFF) hold -LIFT)
  if constexpr (SIMT) {
    contract_simt<C, C::KF>(a.AT, C::KV, sB, accS, tid);
  } else if constexpr (M16) {
    contract_m16<C, PR_>(reinterpret_cast<const uint4 *>(a.AT), C::KSV16, C::KSF16, sB, acc16,
                         tot16, warp, lane);
  } else {
    if (warp < C::WARPS_D) contract_dmma<C, C::KFP / 4>(a.AT, C::KVP / 4, sB, accD, warp, lane);
  }
  __syncthreads();

  // 5. epilogue through shared memory: rhs as [v][i][EP] in B
  double *sR = sB;
  if constexpr (SIMT) {
    const int cg = tid % C::CG, rg = tid / C::CG;
#pragma unroll
    for (int r = 0; r < AR; r++) {
      const int i = rg * C::R + r;
      if (i < Np) {
#pragma unroll
        for (int j = 0; j < AC; j++) {
          const int col = cg + j * C::CG, v = col / E, e = col - v * E;
          sR[(v * Np + i) * EP + e] = accS[r][j];
        }
      }
    }
  } else if constexpr (M16) {
    const int mg = warp % C::MG16, ng = warp / C::MG16;
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int ii = 0; ii < QM; ii++) {
      if (mg * C::WM16 + ii >= C::MT16) continue;
#pragma unroll
      for (int jj = 0; jj < QN; jj++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
          const int i = (mg * C::WM16 + ii) * 16 + g + (c >= 2 ? 8 : 0);
          const int col = (ng * C::WN + jj) * 8 + 2 * t + (c & 1);
          const int v = col / E, e = col - v * E;
          if (i < Np) sR[(v * Np + i) * EP + e] = tot16[ii][jj][c];
        }
    }
  } else {
    if (warp < C::WARPS_D) {
      const int mg = warp % C::MGROUPS, ng = warp / C::MGROUPS;
#pragma unroll
      for (int ii = 0; ii < DM; ii++) {
        const int i = (mg * C::WM + ii) * 8 + (lane >> 2);
        if (i < Np) {
#pragma unroll
          for (int jj = 0; jj < DN; jj++) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const int col = (ng * C::WN + jj) * 8 + (lane & 3) * 2 + h;
              const int v = col / E, e = col - v * E;
              sR[(v * Np + i) * EP + e] = accD[ii][jj][h];
            }
          }
        }
      }
    }
  }
  __syncthreads();

  const double dt = a.dt_override >= 0 ? a.dt_override : a.sc->dt;
  // one flat loop over (variable, node): independent updates in flight;
  // nep = ne * Np is a literal for full tiles (divisions by a constant)
  auto items = [&](const int nep) {
    for (int vg = tid; vg < NV * nep; vg += T) {
      const int v = vg / nep, g = vg - v * nep;
      const int e = g / Np, i = g - e * Np;
      const int s = (v * Np + i) * EP + e;
      const long gi = v * vs + e0 * Np + g;
      const double rhs = sR[s];
      if (a.rhs_only) {
        a.u_out[gi] = rhs;
      } else {
        const double kn = a.rka * a.kreg[gi] + dt * rhs;
        const double un = sU[s] + a.rkb * kn;
        a.kreg[gi] = kn;
        a.u_out[gi] = un;
        sU[s] = un;
      }
    }
  };
  if (ne == E)
    items(E * Np);
  else
    items(ne * Np);
  if (PHYS != EUL || !a.last_stage || a.rhs_only) return;
  __syncthreads();

  // fused calc_maxv on the new state (Euler): per face max |v|^2 and c^2
  __shared__ unsigned long long sMax[32];
  unsigned long long local = 0ull;
  for (int it = tid; it < 4 * E; it += T) {
    const int f = it / E, e = it - f * E;
    if (e >= ne) continue;
    double mv2 = 0.0, mc2 = 0.0;
    bool bad = false;
    for (int j = 0; j < Nfp; j++) {
      const int nd = sFm[f * Nfp + j];
      const double u1 = sU[(0 * Np + nd) * EP + e], u2 = sU[(1 * Np + nd) * EP + e],
                   u3 = sU[(2 * Np + nd) * EP + e], u4 = sU[(3 * Np + nd) * EP + e],
                   u5 = sU[(4 * Np + nd) * EP + e];
      double v2, c2;
      node_speeds(a.gamma, u1, u2, u3, u4, u5, v2, c2);   // as in face_maxv_kernel
      mv2 = v2 > mv2 ? v2 : mv2;
      mc2 = c2 > mc2 ? c2 : mc2;
      bad |= (v2 != v2) || (c2 != c2);
    }
    const long gf = (e0 + e) * 4 + f;
    double mv = sqrt(mv2) + sqrt(mc2);
    if (bad) mv = __longlong_as_double(0x7ff8000000000000LL);
    a.maxv[gf] = mv;
    const unsigned long long b = dbits(mv * sFace[(3 * 4 + f) * E + e]);
    local = b > local ? b : local;
  }
  local = warp_max_bits(local);
  if ((tid & 31) == 0) sMax[tid >> 5] = local;
  __syncthreads();
  if (tid < 32) {
    unsigned long long v = tid < (T + 31) / 32 ? sMax[tid] : 0ull;
    v = warp_max_bits(v);
    if (tid == 0) atomicMax(&a.sc->acc[a.sc->parity ^ 1], v);
  }
}

#include "dglm_stage_pipe.cuh"
#include "dglm_stage_mixed.cuh"
#include "dglm_stage_tc.cuh"
#include "dglm_stage_tcb.cuh"

// Standalone calc_maxv (initial state, advection velocity, and the end of a
// step for the stage kernels that do not fuse it): maxv per face and a
// device-wide max of maxv*Fscale into sc->acc[slot] (slot < 0: the slot the
// fused copy would use, acc[parity ^ 1]).  A block walks tiles of ET whole
// elements (ET Np <= 256 consecutive nodes of each variable): one thread per
// node loads the node's variables (coalesced) and writes its |v|^2 and c^2
// (node_speeds) to shared memory, then loads the next tile's values, which
// are in flight while one thread per (element, face) takes the face maxima
// through Fmask.  Max is exact, so the result does not depend on the order;
// one atomic per block.
constexpr int kMaxvBlocksPerSM = 6;
template <int PHYS, int N>
__global__ void __launch_bounds__(256, kMaxvBlocksPerSM)
    face_maxv_kernel(const StageArgs a, int slot) {
  constexpr int Np = np_of(N), Nfp = nfp_of(N), NFF = 4 * Nfp;
  constexpr int ET = 256 / Np, NQ = PHYS == EUL ? 5 : 3;
  static_assert(ET >= 1 && 4 * ET <= 256, "a tile of whole elements fits the block");
  __shared__ double sV[ET * Np], sC[ET * Np];
  __shared__ int sFm[NFF];
  __shared__ unsigned long long sMax[8];
  const int t = threadIdx.x;
  for (int i = t; i < NFF; i += blockDim.x) sFm[i] = a.Fmask[i];
  const double *src = PHYS == EUL ? a.u_in : a.vel;
  double q[NQ];
  auto fetch = [&](long e0) {
    const long n = (a.K - e0 < ET ? a.K - e0 : ET) * Np;   // nodes of the tile (<= 0: none)
#pragma unroll
    for (int v = 0; v < NQ; v++) q[v] = t < n ? src[v * a.vs + e0 * Np + t] : 1.0;
  };
  unsigned long long local = 0ull;
  const long stride = (long)gridDim.x * ET;
  fetch((long)blockIdx.x * ET);
  for (long e0 = (long)blockIdx.x * ET; e0 < a.K; e0 += stride) {
    const int ne = (int)(a.K - e0 < ET ? a.K - e0 : ET);
    if (t < ne * Np) {
      double v2, c2 = 0.0;
      if (PHYS == EUL)
        node_speeds(a.gamma, q[0], q[1], q[2], q[3], q[4], v2, c2);
      else
        v2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
      sV[t] = v2;
      sC[t] = c2;
    }
    fetch(e0 + stride);
    __syncthreads();
    if (t < 4 * ne) {
      const int e = t >> 2, f = t & 3;
      double v2 = 0.0, c2 = 0.0;
      int bad = 0;
#pragma unroll 5
      for (int j = 0; j < Nfp; j++) {
        const int nd = e * Np + sFm[f * Nfp + j];
        const double w2 = sV[nd], d2 = sC[nd];
        bad |= (w2 != w2) || (d2 != d2);
        v2 = w2 > v2 ? w2 : v2;
        c2 = d2 > c2 ? d2 : c2;
      }
      const long gf = (e0 + e) * 4 + f;
      double mv = (PHYS == EUL) ? sqrt(v2) + sqrt(c2) : sqrt(v2);
      if (bad) mv = __longlong_as_double(0x7ff8000000000000LL);
      a.maxv[gf] = mv;
      const unsigned long long b = dbits(mv * a.fscale[gf]);
      local = b > local ? b : local;
    }
    __syncthreads();
  }
  local = warp_max_bits(local);
  if ((t & 31) == 0) sMax[t >> 5] = local;
  __syncthreads();
  if (t < 32) {
    unsigned long long v = t < (int)(blockDim.x >> 5) ? sMax[t] : 0ull;
    v = warp_max_bits(v);
    if (t == 0) atomicMax(&a.sc->acc[slot >= 0 ? slot : a.sc->parity ^ 1], v);
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
// variants and dispatch
// ---------------------------------------------------------------------------

struct Variant {
  StageVariantInfo info;
  cudaError_t (*launch)(const StageArgs &, cudaStream_t);
};

template <int PHYS, int N, int MODE, int E, int R, int CPT, int WM, int PR = 0>
static cudaError_t launch_v(const StageArgs &a, cudaStream_t s) {
  using C = Cfg<PHYS, N, MODE, E, R, CPT, WM, PR>;
  auto k = stage_fp64_kernel<PHYS, N, MODE, E, R, CPT, WM, PR>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)C::SMEM);
  if (e != cudaSuccess) return e;
  const int blocks = (a.K + C::E - 1) / C::E;
  k<<<blocks, C::THREADS, C::SMEM, s>>>(a);
  return cudaGetLastError();
}

static int sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

template <int PHYS, int N, int E, int WN, int WM, bool AS, int NG, int PR, int NB, int PW,
          int KSP, bool FU, bool KG, int CPS>
static cudaError_t launch_pipe(const StageArgs &a, cudaStream_t s) {
  using C = PCfg<PHYS, N, E, WN, WM, AS, NG, PR, NB, PW, KSP, FU, KG, CPS>;
  auto k = stage_pipe_kernel<PHYS, N, E, WN, WM, AS, NG, PR, NB, PW, KSP, FU, KG, CPS>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)C::SMEM);
  if (e != cudaSuccess) return e;
  const int ntiles = (a.K + E - 1) / E;
  const int grid = ntiles < CPS * sm_count() ? ntiles : CPS * sm_count();
  k<<<grid, C::THREADS, C::SMEM, s>>>(a, ntiles);
  return cudaGetLastError();
}

template <int PHYS, int N, int E, int WN, int WM, bool AS, int NG = 1, int PR = 0, int NB = 2,
          int PW = 1, int KSP = 1, bool FU = false, bool KG = false, int CPS = 1>
static Variant make_pipe() {
  using C = PCfg<PHYS, N, E, WN, WM, AS, NG, PR, NB, PW, KSP, FU, KG, CPS>;
  StageVariantInfo i{};
  i.mode = PR ? MODE_MMA16 : MODE_PIPE;
  i.E = E;
  i.R = 8;
  i.CPT = WN;
  i.WM = PR ? C::WM16 : C::WM;
  i.IP = 8 * C::MT;
  i.MT = PR ? C::MT16 : C::MT;
  i.KVP = C::KVP;
  i.KFP = C::KFP;
  i.threads = C::THREADS;
  i.smem = C::SMEM;
  i.groups = NG;
  i.persistent = 1;
  i.ring = NB;
  i.producers = PW;
  i.ksplit = KSP;
  i.fused = FU ? 1 : 0;
  i.k_global = KG ? 1 : 0;
  i.op_global = AS ? 0 : 1;
  i.ctas_per_sm = CPS;
  if (PR) {
    i.prec = PR == 2 ? DGLM_PREC_TF32X3 : PR == 3 ? DGLM_PREC_BF16X6 : DGLM_PREC_BF16X3;
    i.kstep = C::KSTEP16;
  }
  return Variant{i, &launch_pipe<PHYS, N, E, WN, WM, AS, NG, PR, NB, PW, KSP, FU, KG, CPS>};
}

template <int PHYS, int N, int E, int PREC, int NWC, int PW>
static cudaError_t launch_mixed(const StageArgs &a, cudaStream_t s) {
  using C = MCfg<PHYS, N, E, PREC, NWC, PW>;
  auto k = stage_mixed_kernel<PHYS, N, E, PREC, NWC, PW>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)C::SMEM);
  if (e != cudaSuccess) return e;
  const int ntiles = (a.K + E - 1) / E;
  const int grid = ntiles < sm_count() ? ntiles : sm_count();
  k<<<grid, C::THREADS, C::SMEM, s>>>(a, ntiles);
  return cudaGetLastError();
}

template <int PHYS, int N, int E, int PREC, int NWC = 8, int PW = 1>
static Variant make_mixed() {
  using C = MCfg<PHYS, N, E, PREC, NWC, PW>;
  StageVariantInfo i{};
  i.mode = MODE_MIXED;
  i.E = E;
  i.threads = C::THREADS;
  i.smem = C::SMEM;
  i.prec = PREC == PREC_TF32 ? DGLM_PREC_TF32X3
           : PREC == PREC_BF16X6 ? DGLM_PREC_BF16X6
                                 : DGLM_PREC_BF16X3;
  i.npad = C::NPAD;
  i.kva = C::KVA;
  i.kfa = C::KFA;
  i.bimg = C::BIMG;
  i.producers = PW;
  return Variant{i, &launch_mixed<PHYS, N, E, PREC, NWC, PW>};
}

template <int PHYS, int N, int E, int NF, int NB, int NPL, bool DF>
static cudaError_t launch_tc(const StageArgs &a, cudaStream_t s) {
  using C = TCfg<PHYS, N, E, NF, NB, NPL, DF>;
  auto k = stage_tc_kernel<PHYS, N, E, NF, NB, NPL, DF>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)C::SMEM);
  if (e != cudaSuccess) return e;
  const int ntiles = (a.K + E - 1) / E;
  const int grid = ntiles < sm_count() ? ntiles : sm_count();
  k<<<grid, C::THREADS, C::SMEM, s>>>(a, ntiles);
  return cudaGetLastError();
}

template <int PHYS, int N, int E, int NF, int NB, bool DB, bool DF>
static cudaError_t launch_tcb(const StageArgs &a, cudaStream_t s) {
  using C = TBCfg<PHYS, N, E, NF, NB, DB, DF>;
  auto k = stage_tcb_kernel<PHYS, N, E, NF, NB, DB, DF>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)C::SMEM);
  if (e != cudaSuccess) return e;
  const int ntiles = (a.K + E - 1) / E;
  const int grid = ntiles < sm_count() ? ntiles : sm_count();
  k<<<grid, C::THREADS, C::SMEM, s>>>(a, ntiles);
  return cudaGetLastError();
}

template <int PHYS, int N, int E, int NF, int NB, bool DB, bool DF = false>
static Variant make_tcb() {
  using C = TBCfg<PHYS, N, E, NF, NB, DB, DF>;
  StageVariantInfo i{};
  i.mode = MODE_TCB;
  i.E = E;
  i.threads = C::THREADS;
  i.smem = C::SMEM;
  i.prec = DGLM_PREC_BF16X3;
  i.npad = DB ? 2 : 1;   // operand image sets and accumulators
  i.kva = C::KVA;
  i.kfa = C::KFA;
  i.bimg = 128 * C::KT * 4;
  i.ring = NB;
  i.producers = NF;      // compute warps
  i.persistent = 1;
  i.WM = DF ? 1 : 0;     // 1: difference-form FP32 volume flux
  return Variant{i, &launch_tcb<PHYS, N, E, NF, NB, DB, DF>};
}

template <int PHYS, int N, int E, int NF, int NB, int NPL = 1, bool DF = false>
static Variant make_tc() {
  using C = TCfg<PHYS, N, E, NF, NB, NPL, DF>;
  StageVariantInfo i{};
  i.mode = MODE_TC;
  i.E = E;
  i.R = NPL;          // nodes per lane in a flux task
  i.WM = DF ? 1 : 0;  // 1: difference-form FP32 volume flux
  i.threads = C::THREADS;
  i.smem = C::SMEM;
  i.prec = DGLM_PREC_TF32X3;
  i.npad = C::NPQ;
  i.kva = C::KVA;
  i.kfa = C::KFA;
  i.bimg = 128 * C::KT * 4;
  i.ring = NB;
  i.producers = NF;   // compute warps
  i.persistent = 1;
  return Variant{i, &launch_tc<PHYS, N, E, NF, NB, NPL, DF>};
}

template <int PHYS, int N, int MODE, int E, int R, int CPT, int WM, int PR = 0>
static Variant make_v() {
  using C = Cfg<PHYS, N, MODE, E, R, CPT, WM, PR>;
  StageVariantInfo i{};
  i.mode = MODE;
  i.E = E;
  i.R = MODE == MODE_SIMT ? R : 8;
  i.CPT = CPT;
  i.WM = MODE == MODE_MMA16 ? C::WM16 : C::WM;
  i.IP = C::IP;
  i.MT = MODE == MODE_MMA16 ? C::MT16 : C::MT;
  i.KVP = C::KVP;
  i.KFP = C::KFP;
  i.threads = C::THREADS;
  i.smem = C::SMEM;
  if (MODE == MODE_MMA16) {
    i.prec = PR == 2 ? DGLM_PREC_TF32X3 : PR == 3 ? DGLM_PREC_BF16X6 : DGLM_PREC_BF16X3;
    i.kstep = C::KSTEP16;
  }
  return Variant{i, &launch_v<PHYS, N, MODE, E, R, CPT, WM, PR>};
}

// Candidate tile shapes per (physics, N); entry 0 is the default, the others
// are alternatives the tuner may pick.  SIMT(E, R rows, CPT columns per
// thread); DMMA(E, WN n-tiles, WM m-tiles per warp).
template <int PHYS, int N>
static const std::vector<Variant> &variants();

#define V_SIMT(P, NN, E, R, C) make_v<P, NN, MODE_SIMT, E, R, C, 1>()
#define V_DMMA(P, NN, E, WN, WM) make_v<P, NN, MODE_DMMA, E, 1, WN, WM>()
#define V_PIPE(P, NN, E, WN, WM, AS) make_pipe<P, NN, E, WN, WM, AS>()
#define V_PIPE2(P, NN, E, WN, WM, AS) make_pipe<P, NN, E, WN, WM, AS, 2>()
// two consumer groups, a ring of NB buffers and PW producer warps
#define V_PIPE2R(P, NN, E, WN, WM, NB, PW) make_pipe<P, NN, E, WN, WM, false, 2, 0, NB, PW>()
// one consumer group, a ring of NB buffers and PW producer warps
#define V_PIPER(P, NN, E, WN, WM, AS, NB, PW) make_pipe<P, NN, E, WN, WM, AS, 1, 0, NB, PW>()
// one consumer group, all m-tiles per warp, KSP k-chunks, PW producer warps
#define V_PIPEK(P, NN, E, WN, AS, KSP, PW) make_pipe<P, NN, E, WN, 99, AS, 1, 0, 2, PW, KSP>()
// as V_PIPEK with the volume and lift contractions fused into one pass
#define V_PIPEF(P, NN, E, WN, AS, KSP, PW) \
  make_pipe<P, NN, E, WN, 99, AS, 1, 0, 2, PW, KSP, true>()
// separate volume and lift passes, KSP k-chunks, the RK register fetched by the update
#define V_PIPEG(P, NN, E, WN, AS, KSP, PW) \
  make_pipe<P, NN, E, WN, 99, AS, 1, 0, 2, PW, KSP, false, true>()
// as V_PIPEF / V_PIPEG with WM m-tiles per warp (m-groups x n-blocks x k-chunks)
#define V_PIPEFW(P, NN, E, WN, WM, AS, KSP, PW) \
  make_pipe<P, NN, E, WN, WM, AS, 1, 0, 2, PW, KSP, true>()
#define V_PIPEGW(P, NN, E, WN, WM, KSP, PW) \
  make_pipe<P, NN, E, WN, WM, false, 1, 0, 2, PW, KSP, false, true>()
// two persistent CTAs per SM: separate passes, RK register from global memory
#define V_PIPE2C(P, NN, E, WN, WM, KSP, PW) \
  make_pipe<P, NN, E, WN, WM, false, 1, 0, 2, PW, KSP, false, true, 2>()
// pipelined split-precision mma.sync engine with the RK register fetched by the update
#define V_PM16G(P, NN, E, WN, WM, PR, PW) \
  make_pipe<P, NN, E, WN, WM, false, 1, PR, 2, PW, 1, false, true>()
#define V_TF32(P, NN, E) make_mixed<P, NN, E, PREC_TF32>()
#define V_BF16(P, NN, E) make_mixed<P, NN, E, PREC_BF16>()
#define V_TF32W(P, NN, E, W) make_mixed<P, NN, E, PREC_TF32, W>()
#define V_BF16X6(P, NN, E, W) make_mixed<P, NN, E, PREC_BF16X6, W>()
// split-precision mma.sync (legacy tensor cores): E, WN n-tiles, WM m-tiles
#define V_M16(P, NN, E, WN, WM, PR) make_v<P, NN, MODE_MMA16, E, 1, WN, WM, PR>()
#define V_PM16(P, NN, E, WN, WM, PR) make_pipe<P, NN, E, WN, WM, false, 1, PR>()
#define V_BF16W(P, NN, E, W) make_mixed<P, NN, E, PREC_BF16, W>()
// tcgen05 variants with PW producer warps
#define V_MXP(P, NN, E, PREC, W, PW) make_mixed<P, NN, E, PREC, W, PW>()
// split-TF32 with the operator in tensor memory: E elements, NF compute warps, NB ring slots
#define V_TC(P, NN, E, NF, NB) make_tc<P, NN, E, NF, NB>()
// the same with two nodes per lane in each flux task
#define V_TC2(P, NN, E, NF, NB) make_tc<P, NN, E, NF, NB, 2>()
// the same with the centred volume flux in difference form in FP32
#define V_TCD(P, NN, E, NF, NB) make_tc<P, NN, E, NF, NB, 1, true>()
// split-BF16 with the operator in tensor memory: DB = double-buffered images and accumulators
#define V_TCB(P, NN, E, NF, NB, DB) make_tcb<P, NN, E, NF, NB, DB>()
// the same with the centred volume flux in difference form in FP32
#define V_TCBD(P, NN, E, NF, NB, DB) make_tcb<P, NN, E, NF, NB, DB, true>()
#define DGLM_VARIANTS(P, NN, ...)                        \
  template <>                                            \
  const std::vector<Variant> &variants<P, NN>() {        \
    static const std::vector<Variant> v = {__VA_ARGS__}; \
    return v;                                            \
  }

DGLM_VARIANTS(EUL, 1, V_SIMT(EUL, 1, 128, 4, 5), V_DMMA(EUL, 1, 64, 4, 1))
DGLM_VARIANTS(EUL, 2, V_SIMT(EUL, 2, 64, 5, 5), V_DMMA(EUL, 2, 32, 4, 2))
DGLM_VARIANTS(EUL, 3, V_DMMA(EUL, 3, 16, 2, 3), V_SIMT(EUL, 3, 32, 5, 5),
              V_PIPE(EUL, 3, 8, 1, 3, true), V_PIPE(EUL, 3, 16, 1, 3, true),
              V_PIPEF(EUL, 3, 8, 1, true, 3, 2), V_PIPEF(EUL, 3, 16, 2, true, 3, 2),
              V_TC(EUL, 3, 8, 14, 3))
DGLM_VARIANTS(EUL, 4, V_PIPE(EUL, 4, 8, 1, 2, true), V_DMMA(EUL, 4, 8, 1, 5),
              V_SIMT(EUL, 4, 16, 5, 5), V_SIMT(EUL, 4, 16, 3, 5), V_DMMA(EUL, 4, 16, 1, 5),
              V_DMMA(EUL, 4, 16, 2, 5), V_PIPE(EUL, 4, 8, 1, 5, true),
              V_PIPE(EUL, 4, 8, 1, 5, false), V_PIPE(EUL, 4, 8, 1, 3, true),
              V_PIPE2(EUL, 4, 8, 1, 5, true), V_PIPE2(EUL, 4, 8, 1, 3, true),
              V_TF32W(EUL, 4, 8, 16), V_BF16W(EUL, 4, 8, 16), V_BF16X6(EUL, 4, 8, 16),
              V_TF32(EUL, 4, 8), V_BF16(EUL, 4, 8), V_BF16X6(EUL, 4, 8, 8),
              V_MXP(EUL, 4, 8, PREC_BF16, 15, 2), V_MXP(EUL, 4, 8, PREC_BF16X6, 8, 2),
              V_M16(EUL, 4, 8, 1, 3, 2), V_M16(EUL, 4, 8, 1, 1, 1), V_M16(EUL, 4, 8, 1, 1, 3),
              V_PM16(EUL, 4, 8, 1, 3, 1), V_PIPER(EUL, 4, 8, 1, 2, true, 2, 2),
              V_PIPE2R(EUL, 4, 8, 1, 5, 3, 2), V_PIPEF(EUL, 4, 8, 1, true, 3, 2),
              V_PIPEF(EUL, 4, 8, 1, true, 3, 1), V_PIPE2C(EUL, 4, 8, 1, 5, 2, 1),
              V_PIPE2C(EUL, 4, 8, 5, 1, 2, 1), V_PIPE2C(EUL, 4, 8, 1, 5, 2, 2),
              V_TC(EUL, 4, 8, 14, 3), V_TCB(EUL, 4, 8, 14, 2, true),
              V_TC2(EUL, 4, 8, 13, 3), V_TCD(EUL, 4, 8, 14, 3))
DGLM_VARIANTS(EUL, 5, V_PIPE(EUL, 5, 8, 1, 7, false), V_DMMA(EUL, 5, 8, 1, 7),
              V_SIMT(EUL, 5, 8, 7, 5), V_M16(EUL, 5, 8, 1, 2, 2), V_M16(EUL, 5, 8, 1, 2, 1),
              V_M16(EUL, 5, 8, 1, 2, 3), V_PIPEF(EUL, 5, 8, 1, false, 3, 2),
              V_PM16G(EUL, 5, 8, 1, 2, 1, 2), V_PIPEFW(EUL, 5, 8, 5, 1, false, 1, 2),
              V_PIPEFW(EUL, 5, 8, 5, 1, false, 2, 2), V_PIPEFW(EUL, 5, 8, 5, 2, false, 3, 2),
              V_TCB(EUL, 5, 8, 14, 2, true), V_TCBD(EUL, 5, 8, 14, 2, true))
DGLM_VARIANTS(EUL, 6, V_DMMA(EUL, 6, 8, 1, 6), V_SIMT(EUL, 6, 8, 7, 5),
              V_PIPEG(EUL, 6, 8, 1, false, 2, 2), V_PIPEG(EUL, 6, 8, 1, false, 2, 1),
              V_PM16G(EUL, 6, 8, 1, 2, 1, 2), V_PM16G(EUL, 6, 8, 1, 2, 2, 2),
              V_PM16G(EUL, 6, 8, 1, 2, 3, 2),
              V_M16(EUL, 6, 8, 1, 2, 2), V_M16(EUL, 6, 8, 1, 2, 1), V_M16(EUL, 6, 8, 1, 2, 3),
              V_PIPEGW(EUL, 6, 8, 5, 1, 1, 2), V_PIPEGW(EUL, 6, 8, 5, 1, 2, 2),
              V_PIPEGW(EUL, 6, 8, 5, 2, 2, 2), V_PIPEGW(EUL, 6, 8, 5, 2, 3, 2),
              V_PIPEGW(EUL, 6, 8, 5, 3, 2, 2), V_PIPEGW(EUL, 6, 8, 5, 3, 3, 2),
              V_PIPEGW(EUL, 6, 8, 5, 2, 2, 1), V_TCB(EUL, 6, 8, 14, 2, false),
              V_TCBD(EUL, 6, 8, 14, 2, false))
DGLM_VARIANTS(EUL, 7, V_DMMA(EUL, 7, 8, 1, 5), V_SIMT(EUL, 7, 4, 8, 5))
// N=8 Euler: the DMMA layout needs 8 elements per tile (40 columns), 242 KB
DGLM_VARIANTS(EUL, 8, V_SIMT(EUL, 8, 4, 8, 5), V_SIMT(EUL, 8, 4, 6, 5))
DGLM_VARIANTS(ADV, 1, V_SIMT(ADV, 1, 256, 4, 4), V_DMMA(ADV, 1, 64, 2, 1))
DGLM_VARIANTS(ADV, 2, V_SIMT(ADV, 2, 128, 5, 4), V_DMMA(ADV, 2, 64, 2, 2))
DGLM_VARIANTS(ADV, 3, V_DMMA(ADV, 3, 64, 2, 3), V_SIMT(ADV, 3, 64, 5, 4),
              V_PIPE(ADV, 3, 32, 1, 3, true), V_TF32(ADV, 3, 32), V_BF16(ADV, 3, 32),
              V_BF16X6(ADV, 3, 32, 8), V_PIPEF(ADV, 3, 32, 1, true, 3, 2))
DGLM_VARIANTS(ADV, 4, V_SIMT(ADV, 4, 64, 5, 4), V_DMMA(ADV, 4, 64, 2, 5),
              V_PIPEF(ADV, 4, 32, 1, false, 3, 2))
DGLM_VARIANTS(ADV, 5, V_SIMT(ADV, 5, 32, 7, 4), V_DMMA(ADV, 5, 32, 1, 7),
              V_PIPEF(ADV, 5, 16, 1, false, 4, 2))
DGLM_VARIANTS(ADV, 6, V_SIMT(ADV, 6, 32, 7, 4), V_DMMA(ADV, 6, 32, 1, 6),
              V_PIPEF(ADV, 6, 8, 1, false, 8, 2), V_PIPEF(ADV, 6, 8, 1, false, 12, 2),
              V_M16(ADV, 6, 32, 1, 2, 2), V_M16(ADV, 6, 32, 1, 2, 1),
              V_M16(ADV, 6, 32, 1, 2, 3), V_PM16G(ADV, 6, 16, 1, 2, 1, 2),
              V_PM16G(ADV, 6, 16, 1, 2, 2, 2), V_PM16G(ADV, 6, 16, 1, 2, 3, 2))
DGLM_VARIANTS(ADV, 7, V_SIMT(ADV, 7, 16, 8, 4), V_DMMA(ADV, 7, 16, 1, 5),
              V_PIPEF(ADV, 7, 8, 1, false, 8, 2))
DGLM_VARIANTS(ADV, 8, V_SIMT(ADV, 8, 16, 8, 4), V_DMMA(ADV, 8, 16, 1, 7),
              V_PIPEF(ADV, 8, 8, 1, false, 6, 2))

static const std::vector<Variant> *variant_list(int physics, int N) {
#define CASE(P, NN) \
  case NN: return &variants<P, NN>();
  if (physics == DGLM_EULER) {
    switch (N) { CASE(EUL, 1) CASE(EUL, 2) CASE(EUL, 3) CASE(EUL, 4)
                 CASE(EUL, 5) CASE(EUL, 6) CASE(EUL, 7) CASE(EUL, 8) }
  } else if (physics == DGLM_ADVECTION) {
    switch (N) { CASE(ADV, 1) CASE(ADV, 2) CASE(ADV, 3) CASE(ADV, 4)
                 CASE(ADV, 5) CASE(ADV, 6) CASE(ADV, 7) CASE(ADV, 8) }
  }
#undef CASE
  return nullptr;
}

bool stage_fp64_supported(int physics, int N) { return variant_list(physics, N) != nullptr; }

int stage_variant_count(int physics, int N) {
  auto *v = variant_list(physics, N);
  return v ? (int)v->size() : 0;
}

bool stage_variant_info(int physics, int N, int idx, StageVariantInfo *out) {
  auto *v = variant_list(physics, N);
  if (!v || idx < 0 || idx >= (int)v->size()) return false;
  *out = (*v)[idx].info;
  return true;
}

cudaError_t launch_stage_fp64(int physics, int N, int variant, const StageArgs &a,
                              cudaStream_t s) {
  auto *v = variant_list(physics, N);
  if (!v || variant < 0 || variant >= (int)v->size()) return cudaErrorInvalidValue;
  return (*v)[variant].launch(a, s);
}

template <int PHYS, int N>
static cudaError_t launch_maxv_one(const StageArgs &a, int slot, cudaStream_t s) {
  // tiles of 256 / Np whole elements, walked by as many blocks as are
  // resident at once (kMaxvBlocksPerSM by the launch bounds; a larger grid
  // leaves a tail of late-starting blocks)
  constexpr int ET = 256 / np_of(N);
  long blocks = (a.K + ET - 1) / ET;
  if (blocks > (long)kMaxvBlocksPerSM * sm_count()) blocks = (long)kMaxvBlocksPerSM * sm_count();
  face_maxv_kernel<PHYS, N><<<(int)blocks, 256, 0, s>>>(a, slot);
  return cudaGetLastError();
}

cudaError_t launch_face_maxv(int physics, int N, const StageArgs &a, int slot,
                             cudaStream_t s) {
#define CASE(P, NN) \
  case NN: return launch_maxv_one<P, NN>(a, slot, s);
  if (physics == DGLM_EULER) {
    switch (N) { CASE(EUL, 1) CASE(EUL, 2) CASE(EUL, 3) CASE(EUL, 4)
                 CASE(EUL, 5) CASE(EUL, 6) CASE(EUL, 7) CASE(EUL, 8) }
  } else {
    switch (N) { CASE(ADV, 1) CASE(ADV, 2) CASE(ADV, 3) CASE(ADV, 4)
                 CASE(ADV, 5) CASE(ADV, 6) CASE(ADV, 7) CASE(ADV, 8) }
  }
#undef CASE
  return cudaErrorInvalidValue;
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
