// Internal declarations shared by the libdglm translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "dglm.h"

namespace dglm {

constexpr int kMaxOrder = 8;
constexpr int kHistory = 65536;          // dt history ring (steps)
// bound of each wait of the pipelined stage kernels, in SM clock cycles
// (~1 s at the B200 clock); on expiry a CTA sets flag bit 4 and leaves
constexpr long long kWaitCycles = 2000000000LL;

__host__ __device__ constexpr int np_of(int N) { return (N + 1) * (N + 2) * (N + 3) / 6; }
__host__ __device__ constexpr int nfp_of(int N) { return (N + 1) * (N + 2) / 2; }

// Per-handle scalars that live on the device so a step needs no host round
// trip: the CFL dt is computed from a device-wide max of the face wave
// speeds (reference: cublasIdamax + a blocking copy, euler_nopad_dglm.cu:79-96).
struct DevScalars {
  double t;                       // simulated time
  double dt;                      // dt of the step in flight / last step
  double dt_fixed;                // > 0: prescribed dt instead of the CFL dt
  unsigned long long acc[2];      // max over faces of maxv*Fscale, as bits
  int tstep;                      // steps taken
  int parity;                     // which acc[] the next step reads
  int active;                     // 1 while t < tmax for the step in flight
  int flags;                      // bit 0: non-finite dt / wave speed; bit 1: non-finite state
};

// Doubles per element of the element record: rx ry rz sx sy sz tx ty tz,
// nx[4], ny[4], nz[4], Fscale[4] (faces 0..3), one pad (16-byte multiple).
constexpr int kRecord = 26;

// Arguments of the fused stage kernels.  Field arrays are one allocation
// with `vs` doubles between variables.
struct StageArgs {
  const double *AT;      // stacked operators, k-major: (3Np+NFF) x IP
  const double *geo;     // rx,ry,rz,sx,sy,sz,tx,ty,tz, each K doubles
  const double *fscale;  // K*4
  const double *nrm;     // nx, ny, nz, each K*4
  const double *erec;    // per-element record [K][kRecord] or null (see kRecord)
  const double *tau;     // K*4
  const int *vmapP;      // K*4*Nfp
  // compact face maps (dglm_set_compact_face_maps) or null: per face (e, f)
  // the neighbour element and a one-byte code of its node list, with
  // vmapP[e][f][j] = etoe[4e+f] Np + ftab[fcode[4e+f] Nfp + j]
  const int *etoe;
  const unsigned char *fcode;
  const int *ftab;
  const int *Fmask;      // 4*Nfp
  const double *vel;     // advection: vx, vy, vz with stride vs
  const double *u_in;
  double *u_out;
  double *kreg;
  double *maxv;          // K*4 (written on the last stage)
  DevScalars *sc;
  long vs;
  long gstride;          // elements between the 9 metric arrays and the 3
                         // normal components (K rounded up to 64)
  int K;
  double gamma;
  double rka, rkb;
  int last_stage;        // 1: also compute maxv of the new state (Euler)
  int rhs_only;          // 1: write the right-hand side to u_out, no LSERK update
  double dt_override;    // >= 0: use this dt instead of sc->dt
  long long wait_cycles; // bound of the hand-off waits between the warps of the
                         // pipelined kernels (kWaitCycles unless a test shortens it);
                         // waits for copies or MMAs already in flight keep kWaitCycles
};

// Neighbour node index vmapP[e0 NFF + idx] of face point idx = e NFF + f Nfp + j
// of the tile that starts at element e0, from the compact face maps (20 bytes
// per element instead of 4 NFF).  Producers branch on a.etoe once per tile,
// outside their unrolled load loops, so the vmapP loop stays branch-free.
template <int Np, int Nfp>
__device__ __forceinline__ int compact_neighbour_node(const StageArgs &a, long e0, int idx) {
  const int e = idx / (4 * Nfp), fj = idx - e * 4 * Nfp, f = fj / Nfp, j = fj - f * Nfp;
  const long ge = (e0 + e) * 4 + f;
  return __ldg(a.etoe + ge) * Np + __ldg(a.ftab + (int)__ldg(a.fcode + ge) * Nfp + j);
}

// Reference Euler flux (F, G, W) of the state q, in the arithmetic order of
// euler_dglm.cpp:152-168 / euler_nopad_dglm.cu:181-198 (vb2 is |m|^2).
__device__ __forceinline__ void euler_flux(double g, const double q[5], double F[5],
                                           double G[5], double W[5]) {
  const double u1 = q[0], u2 = q[1], u3 = q[2], u4 = q[3], u5 = q[4];
  const double v2 = u2 * u2 + u3 * u3 + u4 * u4;
  const double p = (g - 1) * (u5 - 0.5 * v2 / u1);
  F[0] = u2;
  F[1] = (u2 * u2) / u1 + p;
  F[2] = (u2 * u3) / u1;
  F[3] = (u2 * u4) / u1;
  F[4] = (u5 + p) * (u2 / u1);
  G[0] = u3;
  G[1] = u2 * u3 / u1;
  G[2] = (u3 * u3) / u1 + p;
  G[3] = u3 * u4 / u1;
  G[4] = (u5 + p) * (u3 / u1);
  W[0] = u4;
  W[1] = u2 * u4 / u1;
  W[2] = u3 * u4 / u1;
  W[3] = (u4 * u4) / u1 + p;
  W[4] = (u5 + p) * (u4 / u1);
}

// Maxima of non-negative doubles are taken on their bit patterns: for
// sign-bit-clear doubles the unsigned order is the numeric order, and a NaN
// (exponent all ones, non-zero mantissa) orders above +Inf, so it propagates
// into dt where the step kernel flags it.
__device__ __forceinline__ unsigned long long dbits(double v) {
  return (unsigned long long)__double_as_longlong(v);
}
__device__ __forceinline__ unsigned long long warp_max_bits(unsigned long long b) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long x = __shfl_xor_sync(0xffffffffu, b, o);
    b = x > b ? x : b;
  }
  return b;
}

// |v|^2 and the squared sound speed of one node's state, for the wave-speed
// maxima of the solver's steps (the fused copies in the stage kernels and the
// standalone face_maxv_kernel share it, so dt does not depend on which kernel
// computed maxv and a restarted run repeats the original bit for bit).  One
// division by rho, as a reciprocal; the per-kernel calc_maxv entry points
// below keep the reference's three divisions.
__device__ __forceinline__ void node_speeds(double gamma, double u1, double u2, double u3,
                                            double u4, double u5, double &v2, double &c2) {
  const double ir = 1.0 / u1;
  const double vx = u2 * ir, vy = u3 * ir, vz = u4 * ir;
  v2 = vx * vx + vy * vy + vz * vz;
  const double pres = (gamma - 1) * (u5 - 0.5 * u1 * v2);
  c2 = fabs(gamma * pres * ir);
}

// calc_maxv of face fi of element e (euler_nopad_dglm.cu:7-76,
// advec_nopad_dglm.cu:7-62): the largest |v| over the face nodes plus, for
// Euler, the largest sound speed, with the reference's divisions by rho.
// U is any struct with a member array p[5] of per-variable field pointers.
// Shared by the per-kernel entry point and the no-allocation variant, whose
// results must agree bit for bit.
template <class U>
__device__ __forceinline__ double face_max_speed(int physics, int Np, int Nfp, double gamma,
                                                 const int *__restrict__ Fmask, const U &u,
                                                 const double *vx, const double *vy,
                                                 const double *vz, long e, int fi) {
  double mv2 = 0, mc2 = 0;
  for (int j = 0; j < Nfp; j++) {
    const long n = e * Np + Fmask[fi * Nfp + j];
    if (physics == DGLM_EULER) {
      const double u1 = u.p[0][n], u2 = u.p[1][n], u3 = u.p[2][n], u4 = u.p[3][n],
                   u5 = u.p[4][n];
      const double ax = u2 / u1, ay = u3 / u1, az = u4 / u1;
      const double v2 = ax * ax + ay * ay + az * az;
      if (v2 > mv2) mv2 = v2;
      const double pres = (gamma - 1) * (u5 - 0.5 * u1 * v2);
      const double c2 = fabs(gamma * pres / u1);
      if (c2 > mc2) mc2 = c2;
    } else {
      const double v2 = vx[n] * vx[n] + vy[n] * vy[n] + vz[n] * vz[n];
      if (v2 > mv2) mv2 = v2;
    }
  }
  return physics == DGLM_EULER ? sqrt(mv2) + sqrt(mc2) : sqrt(mv2);
}

// error plumbing (dglm_solver.cu)
dglm_status set_error(dglm_status s, const std::string &msg);
dglm_status cuda_check(cudaError_t e, const char *what);

// contraction engines of the fused stage kernel
enum { MODE_SIMT = 0, MODE_DMMA = 1, MODE_PIPE = 2, MODE_MIXED = 3, MODE_MMA16 = 4, MODE_TC = 5,
       MODE_TCB = 6 };

// One compiled tile shape of the fused stage kernel.
struct StageVariantInfo {
  int mode;      // MODE_SIMT, MODE_DMMA or MODE_PIPE (persistent, TMA-fed DMMA)
  int E;         // elements per CTA
  int R;         // SIMT rows per thread (8 = one m-tile for DMMA)
  int CPT;       // SIMT columns per thread / DMMA n-tiles per warp
  int WM;        // DMMA m-tiles per warp
  int IP;        // SIMT: padded rows of the k-major operator copy
  int MT;        // DMMA: m-tiles (8 rows each)
  int KVP, KFP;  // DMMA: volume / lift k extents padded to 4
  int threads;
  size_t smem;
  int prec;      // dglm_precision of the contraction (0 FP64, 1 TF32x3, 2 BF16x3)
  int npad;      // MIXED: MMA N (output nodes, padded); TC: output nodes per lane quarter
  int kva, kfa;  // MIXED, TC: volume / lift K extents of the operand images
  int bimg;      // MIXED: bytes of the operator image (hi then lo); TC, TCB: tensor-memory image
  int groups;    // PIPE: consumer groups taking alternate tiles (1 or 2)
  int kstep;     // MMA16: K per mma.sync (8 TF32, 16 BF16)
  int persistent;  // 1: one CTA per SM walking the tiles (TMA-fed pipeline)
  int ring;        // PIPE: tile buffers in the producer/consumer ring (2 to 4)
  int producers;   // PIPE: producer warps sharing the neighbour gathers (1 to 4)
  int ksplit;      // PIPE: k-chunks of the DMMA contraction summed in the epilogue
  int fused;       // PIPE: 1 = volume and lift contractions in one DMMA pass
  int k_global;    // PIPE: 1 = the RK register is fetched by the update, not staged
  int op_global;   // PIPE: 1 = operator fragments read through L1, not staged in shared memory
  int ctas_per_sm; // PIPE: persistent CTAs per SM (2: two independent pipelines per SM)
};

// fused FP64 stage launcher (dglm_stage_fp64.cu)
bool stage_fp64_supported(int physics, int N);
int stage_variant_count(int physics, int N);
bool stage_variant_info(int physics, int N, int idx, StageVariantInfo *out);
cudaError_t launch_stage_fp64(int physics, int N, int variant, const StageArgs &a,
                              cudaStream_t s);
cudaError_t launch_face_maxv(int physics, int N, const StageArgs &a, int parity_slot,
                             cudaStream_t s);
cudaError_t launch_step_begin(int N, double cfl, double tmax, int frozen, DevScalars *sc,
                              double *dt_hist, cudaStream_t s);
cudaError_t launch_tau(int K, double tau_scale, const int *vmapF, const double *maxv,
                       double *tau, cudaStream_t s);
cudaError_t launch_step_end(DevScalars *sc, cudaStream_t s);
cudaError_t launch_finite_check(const double *u, long vs, long n, int nvar, DevScalars *sc,
                                cudaStream_t s);

}  // namespace dglm
