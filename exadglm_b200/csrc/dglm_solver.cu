// Solver handle: owns the device arrays of one mesh partition and runs the
// LSERK time loop (the reference's DataDev, euler_nopad_data_dev.cu:9-266,
// and runRK, euler_nopad_time.cu:32-108) as a captured CUDA graph of
//   step_begin (dt on the device) -> tau -> 5 fused stages -> step_end
// with no host synchronisation inside a step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "dglm_common.cuh"
#include "dglm_handle.cuh"

namespace dglm {

static thread_local std::string g_last_error;

dglm_status set_error(dglm_status s, const std::string &msg) {
  g_last_error = msg;
  return s;
}

dglm_status cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return DGLM_OK;
  return set_error(DGLM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace dglm

using namespace dglm;

namespace {

void drop_graphs(dglm_handle *h) {
  for (auto &g : h->graph) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
}

bool all_finite(const double *a, size_t n) {
  for (size_t i = 0; i < n; i++)
    if (!std::isfinite(a[i])) return false;
  return true;
}

bool in_range(const int *a, size_t n, long lo, long hi) {
  for (size_t i = 0; i < n; i++)
    if (a[i] < lo || a[i] >= hi) return false;
  return true;
}

}  // namespace

StageArgs dglm::stage_args(dglm_handle *h, const double *u_in, double *u_out, int s) {
  StageArgs a{};
  a.AT = h->AT;
  a.geo = h->geo;
  a.fscale = h->fscale;
  a.nrm = h->nrm;
  a.erec = h->erec;
  a.tau = h->tau;
  a.vmapP = h->vmapP;
  a.etoe = h->compact ? h->etoe : nullptr;
  a.fcode = h->compact ? h->fcode : nullptr;
  a.ftab = h->compact ? h->ftab : nullptr;
  a.Fmask = h->Fmask;
  a.vel = h->vel;
  a.u_in = u_in;
  a.u_out = u_out;
  a.kreg = h->kreg;
  a.maxv = h->maxv;
  a.sc = h->sc;
  a.vs = h->vs;
  a.gstride = h->Kp;
  a.K = h->d.K;
  a.gamma = h->d.gamma;
  a.rka = s >= 0 ? RKA[s] : 0.0;
  a.rkb = s >= 0 ? RKB[s] : 0.0;
  a.last_stage = (s == 4);
  a.rhs_only = 0;
  a.dt_override = -1.0;
  a.wait_cycles = h->wait_cycles > 0 ? h->wait_cycles : kWaitCycles;
  return a;
}

namespace {

// Doubles of the device operator copy for a variant's layout.
size_t op_doubles(const StageVariantInfo &v, int Np, int NFF) {
  if (v.mode == MODE_SIMT) return (size_t)(3 * Np + NFF) * v.IP;
  if (v.mode == MODE_MIXED || v.mode == MODE_TC || v.mode == MODE_TCB)
    return ((size_t)v.bimg + 7) / 8;
  if (v.mode == MODE_MMA16) {
    const int parts = v.prec == DGLM_PREC_BF16X6 ? 3 : 2;
    return (size_t)(v.KVP / v.kstep + v.KFP / v.kstep) * v.MT * parts * 64;   // 512 B each
  }
  return (size_t)(v.KVP / 4 + v.KFP / 4) * v.MT * 32;
}

size_t max_op_doubles(int physics, int N, int Np, int NFF) {
  size_t m = 0;
  StageVariantInfo v{};
  for (int i = 0; i < stage_variant_count(physics, N); i++)
    if (stage_variant_info(physics, N, i, &v)) m = std::max(m, op_doubles(v, Np, NFF));
  return m;
}

// Round-to-nearest (ties away) of a float to TF32 (10 mantissa bits), as
// cvt.rna.tf32.f32 does on the device.
uint32_t tf32_rna(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
  return u;
}
float f32_of(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
// Round-to-nearest-even of a float to bfloat16.
uint16_t bf16_rne(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

// Operator image of a mixed-precision variant: B = A^T blocks (volume: the
// 3Np columns of [WDr WDs WDt], lift: the NFF columns of -LIFT), each
// npad rows x (kva | kfa) K, K-major in 8-row x 16-byte core matrices,
// split into parts (TF32 / BF16: hi, lo; BF16x6: three BF16 parts):
// [part 0 vol][part 0 lift][part 1 vol][part 1 lift]...  The split uses the
// exact FP64 residual at every level.
std::vector<unsigned char> mixed_image(const dglm_handle *h, const StageVariantInfo &v) {
  const int Np = h->Np, NFF = h->NFF, KA = 3 * Np + NFF, KV = 3 * Np;
  const bool tf = v.prec == DGLM_PREC_TF32X3;
  const int parts = v.prec == DGLM_PREC_BF16X6 ? 3 : 2;
  const int S = tf ? 4 : 2, T = 16 / S;
  const int bv = v.npad * v.kva * S, bf = v.npad * v.kfa * S;
  std::vector<unsigned char> img((size_t)v.bimg, 0);
  auto put = [&](size_t base, int sbo, int r, int k, double x) {
    const size_t off = base + (size_t)(r / 8) * sbo + (size_t)(k / T) * 128 + (r % 8) * 16 +
                       (k % T) * S;
    double rest = x;
    for (int p = 0; p < parts; p++) {
      const size_t o = off + (size_t)p * (bv + bf);
      if (tf) {
        const uint32_t q = tf32_rna((float)rest);
        std::memcpy(&img[o], &q, 4);
        rest -= (double)f32_of(q);
      } else {
        const uint16_t q = bf16_rne((float)rest);
        const uint32_t qb = (uint32_t)q << 16;
        std::memcpy(&img[o], &q, 2);
        rest -= (double)f32_of(qb);
      }
    }
  };
  for (int n = 0; n < Np; n++) {
    for (int k = 0; k < KV; k++) put(0, v.kva / T * 128, n, k, h->Ahost[(size_t)n * KA + k]);
    for (int k = 0; k < NFF; k++)
      put((size_t)bv, v.kfa / T * 128, n, k, h->Ahost[(size_t)n * KA + KV + k]);
  }
  return img;
}

// Builds the variant's device layout of A = [WDr WDs WDt -LIFT] (Np rows,
// 3Np + NFF columns) from the host copy and uploads it.
//   SIMT: k-major with padded rows, AT[k * IP + i] = A(i, k);
//   DMMA: m8n8k4 A fragments, [kstep][mtile][lane] with row = 8*mtile +
//         lane/4 and column 4*kstep + lane%4 inside the volume block
//         (ksteps [0, KVP/4)) or the lift block (ksteps [KVP/4, ...)).
// Fragments of the split-precision mma.sync engine: per (k-step, m-tile,
// part) 32 lanes x 4 32-bit registers in the m16n8k8 TF32 / m16n8k16 BF16 A
// layout (see contract_m16), parts split with the exact FP64 residual.
std::vector<uint32_t> m16_fragments(const dglm_handle *h, const StageVariantInfo &v) {
  const int Np = h->Np, NFF = h->NFF, KA = 3 * Np + NFF, KV = 3 * Np;
  const bool tf = v.prec == DGLM_PREC_TF32X3;
  const int parts = v.prec == DGLM_PREC_BF16X6 ? 3 : 2;
  const int ksv = v.KVP / v.kstep, ksf = v.KFP / v.kstep;
  std::vector<uint32_t> out((size_t)(ksv + ksf) * v.MT * parts * 128, 0u);
  // operator entry for row r and k-column kk of k-step ks (0 outside)
  auto A = [&](int r, int ks, int kk) -> double {
    if (r >= Np) return 0.0;
    if (ks < ksv) {
      const int k = ks * v.kstep + kk;
      return k < KV ? h->Ahost[(size_t)r * KA + k] : 0.0;
    }
    const int k = (ks - ksv) * v.kstep + kk;
    return k < NFF ? h->Ahost[(size_t)r * KA + KV + k] : 0.0;
  };
  auto parts_of = [&](double x, uint32_t *p) {
    double rest = x;
    for (int q = 0; q < parts; q++) {
      if (tf) {
        p[q] = tf32_rna((float)rest);
        rest -= (double)f32_of(p[q]);
      } else {
        const uint16_t b = bf16_rne((float)rest);
        p[q] = b;
        rest -= (double)f32_of((uint32_t)b << 16);
      }
    }
  };
  for (int ks = 0; ks < ksv + ksf; ks++)
    for (int mt = 0; mt < v.MT; mt++)
      for (int lane = 0; lane < 32; lane++) {
        const int g = lane >> 2, t = lane & 3, r0 = mt * 16 + g;
        uint32_t reg[4][3] = {};
        if (tf) {
          const int rr[4] = {r0, r0 + 8, r0, r0 + 8}, kk[4] = {t, t, t + 4, t + 4};
          for (int c = 0; c < 4; c++) parts_of(A(rr[c], ks, kk[c]), reg[c]);
        } else {
          const int rr[4] = {r0, r0 + 8, r0, r0 + 8}, kk[4] = {2 * t, 2 * t, 2 * t + 8, 2 * t + 8};
          for (int c = 0; c < 4; c++) {
            uint32_t lo[3], hi[3];
            parts_of(A(rr[c], ks, kk[c]), lo);
            parts_of(A(rr[c], ks, kk[c] + 1), hi);
            for (int q = 0; q < parts; q++) reg[c][q] = lo[q] | (hi[q] << 16);
          }
        }
        for (int q = 0; q < parts; q++)
          for (int c = 0; c < 4; c++)
            out[((((size_t)ks * v.MT + mt) * parts + q) * 32 + lane) * 4 + c] = reg[c][q];
      }
  return out;
}

// Tensor-memory operator image of the split-TF32 kernel (stage_tc_kernel):
// 128 lanes x KT columns of TF32 bit patterns.  Lane 32q + 2j + p holds part
// p (0: hi, 1: lo) of operator row i = npq q + j; column k is the kernel's K
// order: volume k = (i'/4)*12 + d*4 + i'%4 for direction d and node i', face
// k = kva + f*nfpp + j' (nfpp = kfa / 4).  Padding columns and unused lanes
// are zero.  hi = TF32 rounding of x, lo = TF32 rounding of the exact FP64
// residual.
std::vector<uint32_t> tc_image(const dglm_handle *h, const StageVariantInfo &v) {
  const int Np = h->Np, Nfp = h->Nfp, KA = 3 * Np + h->NFF;
  const int KT = v.kva + v.kfa, npq = v.npad, nfpp = v.kfa / 4, ng = (Np + 3) / 4;
  std::vector<uint32_t> img((size_t)128 * KT, 0u);
  for (int k = 0; k < KT; k++) {
    int col = -1;
    if (k < v.kva) {
      const int g = k / 12, d = (k % 12) / 4, i = g * 4 + k % 4;
      if (g < ng && i < Np) col = d * Np + i;
    } else {
      const int f = (k - v.kva) / nfpp, j = (k - v.kva) % nfpp;
      if (j < Nfp) col = 3 * Np + f * Nfp + j;
    }
    if (col < 0) continue;
    for (int q = 0; q < 4; q++)
      for (int j = 0; j < npq; j++) {
        const int i = npq * q + j;
        if (i >= Np) continue;
        const double x = h->Ahost[(size_t)i * KA + col];
        const uint32_t hi = tf32_rna((float)x);
        const uint32_t lo = tf32_rna((float)(x - (double)f32_of(hi)));
        img[(size_t)(32 * q + 2 * j) * KT + k] = hi;
        img[(size_t)(32 * q + 2 * j + 1) * KT + k] = lo;
      }
  }
  return img;
}

// Tensor-memory image of the split-BF16 operator (stage_tcb_kernel): 128
// lanes (lane i = operator row i) x KT 32-bit columns; columns [0, KT/2)
// hold the BF16 hi parts, [KT/2, KT) the lo parts, two K values per column
// (the lower K in the low half), K in the kernel's order (volume k = (i/4)*12
// + d*4 + i%4 over kva columns, then face f node j at kva + f*nfpp + j).
std::vector<uint32_t> tcb_image(const dglm_handle *h, const StageVariantInfo &v) {
  const int Np = h->Np, Nfp = h->Nfp, KA = 3 * Np + h->NFF;
  const int KT = v.kva + v.kfa, half = KT / 2, nfpp = v.kfa / 4, ng = (Np + 3) / 4;
  std::vector<uint32_t> img((size_t)128 * KT, 0u);
  for (int k = 0; k < KT; k++) {
    int col = -1;
    if (k < v.kva) {
      const int g = k / 12, d = (k % 12) / 4, i = g * 4 + k % 4;
      if (g < ng && i < Np) col = d * Np + i;
    } else {
      const int f = (k - v.kva) / nfpp, j = (k - v.kva) % nfpp;
      if (j < Nfp) col = 3 * Np + f * Nfp + j;
    }
    if (col < 0) continue;
    const int c = k / 2, sh = (k & 1) * 16;
    for (int i = 0; i < Np; i++) {
      const double x = h->Ahost[(size_t)i * KA + col];
      const uint16_t hi = bf16_rne((float)x);
      const uint16_t lo = bf16_rne((float)(x - (double)f32_of((uint32_t)hi << 16)));
      img[(size_t)i * KT + c] |= (uint32_t)hi << sh;
      img[(size_t)i * KT + half + c] |= (uint32_t)lo << sh;
    }
  }
  return img;
}

dglm_status upload_operator_layout(dglm_handle *h) {
  const int Np = h->Np, NFF = h->NFF, KA = 3 * Np + NFF, KV = 3 * Np;
  const StageVariantInfo &v = h->vinfo;
  if (v.mode == MODE_TC || v.mode == MODE_TCB) {
    std::vector<uint32_t> img = v.mode == MODE_TC ? tc_image(h, v) : tcb_image(h, v);
    return cuda_check(cudaMemcpy(h->AT, img.data(), img.size() * 4, cudaMemcpyHostToDevice),
                      "operator upload");
  }
  if (v.mode == MODE_MMA16) {
    std::vector<uint32_t> fr = m16_fragments(h, v);
    return cuda_check(cudaMemcpy(h->AT, fr.data(), fr.size() * 4, cudaMemcpyHostToDevice),
                      "operator upload");
  }
  if (v.mode == MODE_MIXED) {
    std::vector<unsigned char> img = mixed_image(h, v);
    return cuda_check(cudaMemcpy(h->AT, img.data(), img.size(), cudaMemcpyHostToDevice),
                      "operator upload");
  }
  std::vector<double> out(op_doubles(v, Np, NFF), 0.0);
  auto A = [&](int i, int k) { return h->Ahost[(size_t)i * KA + k]; };
  if (v.mode == MODE_SIMT) {
    for (int k = 0; k < KA; k++)
      for (int i = 0; i < Np; i++) out[(size_t)k * v.IP + i] = A(i, k);
  } else {
    const int kv4 = v.KVP / 4, kf4 = v.KFP / 4;
    for (int ks = 0; ks < kv4 + kf4; ks++)
      for (int mt = 0; mt < v.MT; mt++)
        for (int lane = 0; lane < 32; lane++) {
          const int row = mt * 8 + lane / 4;
          int k;
          bool ok;
          if (ks < kv4) {
            k = ks * 4 + lane % 4;
            ok = k < KV;
          } else {
            const int kk = (ks - kv4) * 4 + lane % 4;
            k = KV + kk;
            ok = kk < NFF;
          }
          if (ok && row < Np) out[((size_t)ks * v.MT + mt) * 32 + lane] = A(row, k);
        }
  }
  return cuda_check(cudaMemcpy(h->AT, out.data(), sizeof(double) * out.size(),
                               cudaMemcpyHostToDevice),
                    "operator upload");
}

// Whether the step's wave-speed maximum runs as its own kernel after the
// fifth stage (Euler): inside the persistent stage kernels it costs more than
// the standalone face_maxv_kernel, whose result is the same bit for bit.
bool separate_maxv(const dglm_handle *h) { return h->d.physics == DGLM_EULER; }

// Kernel launches of one step: step_begin, tau (Euler), five stages, the
// separate wave-speed maximum where it applies, step_end.
int step_launches(const dglm_handle *h) {
  return (h->d.physics == DGLM_ADVECTION ? 7 : 8) + (separate_maxv(h) ? 1 : 0);
}

}  // namespace

// One LSERK step whose stage k reads in[k] and writes out[k] (for the
// adjoint's recording of stage inputs); dt, tau and the wave-speed max as in
// a normal step.
dglm_status dglm::issue_step_ptrs(dglm_handle *h, const double *const *in, double *const *out,
                                  cudaStream_t s) {
  const int frozen = h->d.physics == DGLM_ADVECTION;
  cudaError_t e = launch_step_begin(h->d.N, h->d.cfl, h->d.tmax, frozen, h->sc, h->dt_hist, s);
  if (e == cudaSuccess && !frozen)
    e = launch_tau(h->d.K, h->d.tau_scale, h->vmapF, h->maxv, h->tau, s);
  const bool sep = separate_maxv(h);
  for (int st = 0; st < 5 && e == cudaSuccess; st++) {
    StageArgs a = stage_args(h, in[st], out[st], st);
    if (sep) a.last_stage = 0;
    e = launch_stage_fp64(h->d.physics, h->d.N, h->variant, a, s);
  }
  if (e == cudaSuccess && sep)
    e = launch_face_maxv(h->d.physics, h->d.N, stage_args(h, out[4], nullptr, -1), -1, s);
  if (e == cudaSuccess) e = launch_step_end(h->sc, s);
  return cuda_check(e, "step launch");
}

namespace {

// Issues one LSERK step starting from u[cur] (ends in u[cur^1]).
dglm_status issue_step(dglm_handle *h, int cur, cudaStream_t s) {
  const int frozen = h->d.physics == DGLM_ADVECTION;
  cudaError_t e = launch_step_begin(h->d.N, h->d.cfl, h->d.tmax, frozen, h->sc, h->dt_hist, s);
  if (e == cudaSuccess && !frozen)
    e = launch_tau(h->d.K, h->d.tau_scale, h->vmapF, h->maxv, h->tau, s);
  const bool sep = separate_maxv(h);
  for (int st = 0; st < 5 && e == cudaSuccess; st++) {
    const int in = (cur + st) & 1;
    StageArgs a = stage_args(h, h->u[in], h->u[in ^ 1], st);
    if (sep) a.last_stage = 0;
    e = launch_stage_fp64(h->d.physics, h->d.N, h->variant, a, s);
  }
  // after five stages the new state is in u[cur ^ 1]
  if (e == cudaSuccess && sep)
    e = launch_face_maxv(h->d.physics, h->d.N, stage_args(h, h->u[cur ^ 1], nullptr, -1), -1,
                         s);
  if (e == cudaSuccess) e = launch_step_end(h->sc, s);
  return cuda_check(e, "step launch");
}

}  // namespace

// Scratch of the one-off right-hand-side evaluations (dglm_rhs,
// dglm_adjoint_rhs), allocated on first use.
dglm_status dglm::ensure_rhs_scratch(dglm_handle *h) {
  if (h->rhs_in) return DGLM_OK;
  dglm_status st = dalloc(h, &h->rhs_in, (size_t)h->nvar * h->vs);
  if (st == DGLM_OK) st = dalloc(h, &h->rhs_out, (size_t)h->nvar * h->vs);
  if (st == DGLM_OK) st = dalloc(h, &h->maxv_s, (size_t)4 * h->Kp);
  if (st == DGLM_OK) st = dalloc(h, &h->tau_s, (size_t)4 * h->Kp);
  if (st == DGLM_OK) st = dalloc(h, &h->sc_s, 1);
  if (st != DGLM_OK) return st;
  // on the handle's stream, ordered before the copies that fill them
  cudaStream_t s = h->stream;
  cudaError_t e = cudaMemsetAsync(h->rhs_in, 0, sizeof(double) * h->nvar * h->vs, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->maxv_s, 0, sizeof(double) * 4 * h->Kp, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->tau_s, 0, sizeof(double) * 4 * h->Kp, s);
  return cuda_check(e, "rhs scratch");
}

extern "C" {

const char *dglm_last_error(void) { return g_last_error.c_str(); }
int dglm_abi_version(void) { return DGLM_ABI_VERSION; }
int dglm_order_supported(int N) { return N >= 1 && N <= kMaxOrder; }

dglm_status dglm_create(const dglm_desc *desc, dglm_handle **out) {
  if (!desc || !out) return set_error(DGLM_ERR_INVALID, "dglm_create: NULL argument");
  *out = nullptr;
  const dglm_desc &d = *desc;
  if (d.physics != DGLM_EULER && d.physics != DGLM_ADVECTION)
    return set_error(DGLM_ERR_INVALID, "dglm_create: unknown physics");
  if (!stage_fp64_supported(d.physics, d.N))
    return set_error(DGLM_ERR_UNSUPPORTED,
                     "dglm_create: order N=" + std::to_string(d.N) + " is not built (1..8)");
  if (d.K <= 0) return set_error(DGLM_ERR_INVALID, "dglm_create: K must be positive");
  // node indices (vmapP, the reference's int32 format) must fit in int32, and
  // so must the face-point indices K*4*Nfp of the adjoint's partner map (4*Nfp
  // > Np at every order); checked on K rounded up to whole 64-element tiles
  {
    const long long kp = ((long long)d.K + 63) / 64 * 64;
    if (kp * np_of(d.N) > 2147483647LL)
      return set_error(DGLM_ERR_UNSUPPORTED,
                       "dglm_create: K*Np exceeds the int32 node index range");
    if (kp * 4 * nfp_of(d.N) > 2147483647LL)
      return set_error(DGLM_ERR_UNSUPPORTED,
                       "dglm_create: K*4*Nfp exceeds the int32 face-point index range");
  }
  if (d.precision != DGLM_PREC_FP64 && d.precision != DGLM_PREC_TF32X3 &&
      d.precision != DGLM_PREC_BF16X3 && d.precision != DGLM_PREC_BF16X6)
    return set_error(DGLM_ERR_INVALID, "dglm_create: unknown precision");
  int first = -1;
  {
    StageVariantInfo v{};
    for (int i = 0; i < stage_variant_count(d.physics, d.N) && first < 0; i++)
      if (stage_variant_info(d.physics, d.N, i, &v) && v.prec == d.precision) first = i;
  }
  if (first < 0)
    return set_error(DGLM_ERR_UNSUPPORTED,
                     "dglm_create: precision mode not built for this physics and order");
  if (!(d.cfl > 0) || !(d.tau_scale >= 0) || !(d.tmax > 0) ||
      (d.physics == DGLM_EULER && !(d.gamma > 1)))
    return set_error(DGLM_ERR_INVALID, "dglm_create: cfl/gamma/tau_scale/tmax out of range");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_error(DGLM_ERR_CUDA, "dglm_create: no CUDA device");
  if (d.device >= ndev) return set_error(DGLM_ERR_INVALID, "dglm_create: device out of range");

  dglm_handle *h = new dglm_handle();
  h->d = d;
  if (d.device < 0) cudaGetDevice(&h->dev); else h->dev = d.device;
  DeviceGuard g(h->dev);
  h->nvar = d.physics == DGLM_EULER ? 5 : 1;
  h->Np = np_of(d.N);
  h->Nfp = nfp_of(d.N);
  h->NFF = 4 * h->Nfp;
  h->variant = first;
  stage_variant_info(d.physics, d.N, first, &h->vinfo);
  // per-element arrays are padded to whole 64-element tiles (zero-filled) so
  // that every tile copy of the pipelined kernel is in bounds and aligned
  h->Kp = ((long)d.K + 63) / 64 * 64;
  const long n = h->Kp * h->Np;
  h->vs = (n + 31) / 32 * 32;  // 256-byte aligned variable blocks
  dglm_status st = DGLM_OK;
  const long K = h->Kp;
  auto chk = [&](dglm_status s) {
    if (st == DGLM_OK) st = s;
  };
  chk(dalloc(h, &h->AT, max_op_doubles(d.physics, d.N, h->Np, h->NFF)));
  chk(dalloc(h, &h->geo, (size_t)9 * K));
  chk(dalloc(h, &h->fscale, (size_t)4 * K));
  chk(dalloc(h, &h->nrm, (size_t)12 * K));
  if (d.physics == DGLM_EULER &&
      (d.precision == DGLM_PREC_TF32X3 || d.precision == DGLM_PREC_BF16X3))
    chk(dalloc(h, &h->erec, (size_t)kRecord * K));
  chk(dalloc(h, &h->tau, (size_t)4 * K));
  chk(dalloc(h, &h->maxv, (size_t)4 * K));
  // padded to whole tiles: the tensor-core kernel bulk-copies vmapP per tile
  chk(dalloc(h, &h->vmapP, (size_t)K * h->NFF));
  chk(dalloc(h, &h->vmapF, (size_t)4 * K));
  chk(dalloc(h, &h->Fmask, (size_t)h->NFF));
  if (d.physics == DGLM_ADVECTION) chk(dalloc(h, &h->vel, (size_t)3 * h->vs));
  chk(dalloc(h, &h->u[0], (size_t)h->nvar * h->vs));
  chk(dalloc(h, &h->u[1], (size_t)h->nvar * h->vs));
  chk(dalloc(h, &h->kreg, (size_t)h->nvar * h->vs));
  chk(dalloc(h, &h->sc, 1));
  chk(dalloc(h, &h->dt_hist, (size_t)kHistory));
  if (st == DGLM_OK) {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
      st = set_error(DGLM_ERR_CUDA, "dglm_create: stream creation failed");
    else
      h->own_stream = true;
  }
  if (st != DGLM_OK) {
    std::string msg = g_last_error;
    dglm_destroy(h);
    return set_error(st, msg);
  }
  // zero-padded tails stay zero for the whole life of the handle
  for (void *p : {(void *)h->u[0], (void *)h->u[1], (void *)h->kreg})
    cudaMemset(p, 0, sizeof(double) * h->nvar * h->vs);
  cudaMemset(h->geo, 0, sizeof(double) * 9 * K);
  cudaMemset(h->vmapP, 0, sizeof(int) * K * h->NFF);
  cudaMemset(h->nrm, 0, sizeof(double) * 12 * K);
  for (double *p : {h->fscale, h->tau, h->maxv}) cudaMemset(p, 0, sizeof(double) * 4 * K);
  if (h->vel) cudaMemset(h->vel, 0, sizeof(double) * 3 * h->vs);
  *out = h;
  return cuda_check(cudaDeviceSynchronize(), "dglm_create");
}

dglm_status dglm_destroy(dglm_handle *h) {
  if (!h) return DGLM_OK;
  DeviceGuard g(h->dev);
  if (h->stream) cudaStreamSynchronize(h->stream);
  drop_graphs(h);
  free_tape(h);
  for (cudaStream_t cs : {h->ens_cin, h->ens_cout})
    if (cs) {
      cudaStreamSynchronize(cs);
      cudaStreamDestroy(cs);
    }
  for (cudaEvent_t ev : h->ens_ev)
    if (ev) cudaEventDestroy(ev);
  for (void *p : h->allocs) cudaFree(p);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return DGLM_OK;
}

dglm_status dglm_set_stream(dglm_handle *h, void *stream) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_set_stream: NULL handle");
  DeviceGuard g(h->dev);
  cudaStreamSynchronize(h->stream);
  drop_graphs(h);
  if (h->own_stream) cudaStreamDestroy(h->stream);
  h->own_stream = false;
  h->stream = (cudaStream_t)stream;
  return DGLM_OK;
}

dglm_status dglm_upload_mesh(dglm_handle *h, const dglm_mesh_arrays *m) {
  if (!h || !m) return set_error(DGLM_ERR_INVALID, "dglm_upload_mesh: NULL argument");
  const long K = h->d.K, Np = h->Np, NFF = h->NFF;
  const double *req_d[] = {m->WDr, m->WDs, m->WDt, m->LIFT, m->rx, m->ry, m->rz, m->sx,
                           m->sy,  m->sz,  m->tx,  m->ty,   m->tz, m->Fscale, m->nx, m->ny,
                           m->nz};
  for (const double *p : req_d)
    if (!p) return set_error(DGLM_ERR_INVALID, "dglm_upload_mesh: a real array is NULL");
  if (!m->vmapP || !m->vmapF || !m->Fmask)
    return set_error(DGLM_ERR_INVALID, "dglm_upload_mesh: an index array is NULL");
  if (m->matrix_order != 'c' && m->matrix_order != 'f')
    return set_error(DGLM_ERR_INVALID, "dglm_upload_mesh: matrix_order must be 'c' or 'f'");
  if (h->d.physics == DGLM_ADVECTION && (!m->vx || !m->vy || !m->vz))
    return set_error(DGLM_ERR_INVALID, "dglm_upload_mesh: advection needs vx, vy, vz");
  // host-side validation of every index array and every real array
  if (!in_range(m->vmapP, (size_t)K * NFF, 0, K * Np))
    return set_error(DGLM_ERR_INVALID, "dglm_upload_mesh: vmapP entry outside [0, K*Np)");
  // compact face maps of an earlier mesh no longer apply (rebuilt on request)
  h->compact = h->compact_built = false;
  if (!in_range(m->vmapF, (size_t)4 * K, 0, 4 * K))
    return set_error(DGLM_ERR_INVALID, "dglm_upload_mesh: vmapF entry outside [0, 4K)");
  if (!in_range(m->Fmask, (size_t)NFF, 0, Np))
    return set_error(DGLM_ERR_INVALID, "dglm_upload_mesh: Fmask entry outside [0, Np)");
  const size_t nop = (size_t)Np * Np, nl = (size_t)Np * NFF;
  if (!all_finite(m->WDr, nop) || !all_finite(m->WDs, nop) || !all_finite(m->WDt, nop) ||
      !all_finite(m->LIFT, nl))
    return set_error(DGLM_ERR_INVALID, "dglm_upload_mesh: non-finite operator entry");
  for (int i = 4; i < 13; i++)
    if (!all_finite(req_d[i], (size_t)K))
      return set_error(DGLM_ERR_INVALID, "dglm_upload_mesh: non-finite metric");
  for (int i = 13; i < 17; i++)
    if (!all_finite(req_d[i], (size_t)4 * K))
      return set_error(DGLM_ERR_INVALID, "dglm_upload_mesh: non-finite face array");
  if (h->d.physics == DGLM_ADVECTION) {
    for (const double *p : {m->vx, m->vy, m->vz})
      if (!all_finite(p, (size_t)K * Np))
        return set_error(DGLM_ERR_INVALID, "dglm_upload_mesh: non-finite velocity");
  }

  // stacked operator A = [WDr WDs WDt -LIFT], row-major
  const bool cm = m->matrix_order == 'f';
  const long KA = 3 * Np + NFF;
  h->Ahost.assign((size_t)Np * KA, 0.0);
  auto at = [&](const double *M, long i, long j, long cols) {
    return cm ? M[j * Np + i] : M[i * cols + j];
  };
  for (long i = 0; i < Np; i++) {
    for (long j = 0; j < Np; j++) {
      h->Ahost[i * KA + j] = at(m->WDr, i, j, Np);
      h->Ahost[i * KA + Np + j] = at(m->WDs, i, j, Np);
      h->Ahost[i * KA + 2 * Np + j] = at(m->WDt, i, j, Np);
    }
    for (long j = 0; j < NFF; j++) h->Ahost[i * KA + 3 * Np + j] = -at(m->LIFT, i, j, NFF);
  }
  const long Kp = h->Kp;
  std::vector<double> geo((size_t)9 * Kp, 0.0), nrm((size_t)12 * Kp, 0.0);
  const double *g9[9] = {m->rx, m->ry, m->rz, m->sx, m->sy, m->sz, m->tx, m->ty, m->tz};
  for (int q = 0; q < 9; q++) std::memcpy(&geo[(size_t)q * Kp], g9[q], sizeof(double) * K);
  std::memcpy(&nrm[0], m->nx, sizeof(double) * 4 * K);
  std::memcpy(&nrm[(size_t)4 * Kp], m->ny, sizeof(double) * 4 * K);
  std::memcpy(&nrm[(size_t)8 * Kp], m->nz, sizeof(double) * 4 * K);

  DeviceGuard g(h->dev);
  cudaStreamSynchronize(h->stream);
  free_tape(h);   // the adjoint's operators and face pairing belong to the old mesh
  const auto H2D = cudaMemcpyHostToDevice;
  dglm_status os = upload_operator_layout(h);
  if (os != DGLM_OK) return os;
  cudaError_t e = cudaMemcpy(h->geo, geo.data(), sizeof(double) * geo.size(), H2D);
  if (e == cudaSuccess) e = cudaMemcpy(h->nrm, nrm.data(), sizeof(double) * nrm.size(), H2D);
  if (e == cudaSuccess) e = cudaMemcpy(h->fscale, m->Fscale, sizeof(double) * 4 * K, H2D);
  if (e == cudaSuccess && h->erec) {
    std::vector<double> rec((size_t)kRecord * Kp, 0.0);
    for (long k = 0; k < K; k++) {
      double *r = &rec[(size_t)k * kRecord];
      for (int q = 0; q < 9; q++) r[q] = g9[q][k];
      for (int f = 0; f < 4; f++) {
        r[9 + f] = m->nx[4 * k + f];
        r[13 + f] = m->ny[4 * k + f];
        r[17 + f] = m->nz[4 * k + f];
        r[21 + f] = m->Fscale[4 * k + f];
      }
    }
    e = cudaMemcpy(h->erec, rec.data(), sizeof(double) * rec.size(), H2D);
  }
  if (e == cudaSuccess) e = cudaMemcpy(h->vmapP, m->vmapP, sizeof(int) * K * NFF, H2D);
  if (e == cudaSuccess) e = cudaMemcpy(h->vmapF, m->vmapF, sizeof(int) * 4 * K, H2D);
  if (e == cudaSuccess) e = cudaMemcpy(h->Fmask, m->Fmask, sizeof(int) * NFF, H2D);
  if (h->d.physics == DGLM_ADVECTION) {
    const double *v3[3] = {m->vx, m->vy, m->vz};
    for (int q = 0; q < 3 && e == cudaSuccess; q++)
      e = cudaMemcpy(h->vel + (size_t)q * h->vs, v3[q], sizeof(double) * K * Np, H2D);
  }
  if (e != cudaSuccess) return cuda_check(e, "dglm_upload_mesh");
  h->mesh_ready = true;
  h->state_ready = false;
  return DGLM_OK;
}

dglm_status dglm_set_state(dglm_handle *h, const double *const *u, int on_device) {
  if (!h || !u) return set_error(DGLM_ERR_INVALID, "dglm_set_state: NULL argument");
  if (!h->mesh_ready) return set_error(DGLM_ERR_STATE, "dglm_set_state: upload the mesh first");
  const long n = (long)h->d.K * h->Np;
  for (int v = 0; v < h->nvar; v++)
    if (!u[v]) return set_error(DGLM_ERR_INVALID, "dglm_set_state: NULL variable pointer");
  DeviceGuard g(h->dev);
  cudaStream_t s = h->stream;
  h->cur = 0;
  cudaError_t e = cudaSuccess;
  for (int v = 0; v < h->nvar && e == cudaSuccess; v++)
    e = cudaMemcpyAsync(h->u[0] + (size_t)v * h->vs, u[v], sizeof(double) * n,
                        on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->kreg, 0, sizeof(double) * h->nvar * h->vs, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->sc, 0, sizeof(DevScalars), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->dt_hist, 0, sizeof(double) * kHistory, s);
  if (e != cudaSuccess) return cuda_check(e, "dglm_set_state");
  e = launch_finite_check(h->u[0], h->vs, n, h->nvar, h->sc, s);
  StageArgs a = stage_args(h, h->u[0], h->u[1], -1);
  if (e == cudaSuccess) e = launch_face_maxv(h->d.physics, h->d.N, a, 0, s);
  if (e == cudaSuccess && h->d.physics == DGLM_ADVECTION)
    e = launch_tau(h->d.K, h->d.tau_scale, h->vmapF, h->maxv, h->tau, s);
  int flags = 0;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMemcpy(&flags, &h->sc->flags, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_check(e, "dglm_set_state");
  if (flags & 2) {
    h->state_ready = false;
    return set_error(DGLM_ERR_NONFINITE, "dglm_set_state: non-finite value in the state");
  }
  h->state_ready = true;
  return DGLM_OK;
}

dglm_status dglm_get_state(dglm_handle *h, double *const *u, int on_device) {
  if (!h || !u) return set_error(DGLM_ERR_INVALID, "dglm_get_state: NULL argument");
  if (!h->state_ready) return set_error(DGLM_ERR_STATE, "dglm_get_state: no state set");
  DeviceGuard g(h->dev);
  const long n = (long)h->d.K * h->Np;
  cudaError_t e = cudaSuccess;
  for (int v = 0; v < h->nvar && e == cudaSuccess; v++) {
    if (!u[v]) return set_error(DGLM_ERR_INVALID, "dglm_get_state: NULL variable pointer");
    e = cudaMemcpyAsync(u[v], h->u[h->cur] + (size_t)v * h->vs, sizeof(double) * n,
                        on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        h->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  return cuda_check(e, "dglm_get_state");
}

// Device-side part of dglm_set_state for a state already in h->u[0]: clear
// t, tstep, k, the flags and the dt history, check the state for NaN/Inf and
// compute its face wave speeds (and tau for advection).  Asynchronous.
static cudaError_t reset_for_state(dglm_handle *h, cudaStream_t s) {
  h->cur = 0;
  cudaError_t e = cudaMemsetAsync(h->kreg, 0, sizeof(double) * h->nvar * h->vs, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->sc, 0, sizeof(DevScalars), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->dt_hist, 0, sizeof(double) * kHistory, s);
  if (e == cudaSuccess)
    e = launch_finite_check(h->u[0], h->vs, (long)h->d.K * h->Np, h->nvar, h->sc, s);
  StageArgs a = stage_args(h, h->u[0], h->u[1], -1);
  if (e == cudaSuccess) e = launch_face_maxv(h->d.physics, h->d.N, a, 0, s);
  if (e == cudaSuccess && h->d.physics == DGLM_ADVECTION)
    e = launch_tau(h->d.K, h->d.tau_scale, h->vmapF, h->maxv, h->tau, s);
  return e;
}

static dglm_status ensure_ensemble(dglm_handle *h, int count) {
  if (!h->ens_cin) {
    for (int b = 0; b < 2; b++) {
      dglm_status st = dalloc(h, &h->ens_in[b], (size_t)h->nvar * h->vs);
      if (st == DGLM_OK) st = dalloc(h, &h->ens_out[b], (size_t)h->nvar * h->vs);
      if (st != DGLM_OK) return st;
      // the tails past K*Np stay zero: whole buffers are copied into the state
      cudaError_t e = cudaMemset(h->ens_in[b], 0, sizeof(double) * h->nvar * h->vs);
      if (e != cudaSuccess) return cuda_check(e, "dglm_run_ensemble");
    }
    cudaError_t e = cudaStreamCreateWithFlags(&h->ens_cin, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->ens_cout, cudaStreamNonBlocking);
    for (int i = 0; i < 8 && e == cudaSuccess; i++)
      e = cudaEventCreateWithFlags(&h->ens_ev[i], cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_check(e, "dglm_run_ensemble: streams/events");
  }
  if (count > h->ens_cap) {
    const int cap = count > 2 * h->ens_cap ? count : 2 * h->ens_cap;
    dglm_status st = dalloc(h, &h->ens_flags, (size_t)cap);
    if (st != DGLM_OK) return st;
    h->ens_cap = cap;
  }
  return DGLM_OK;
}

dglm_status dglm_run_ensemble(dglm_handle *h, int count, const double *const *const *in,
                              double *const *const *out, int nsteps, int *first_bad) {
  if (first_bad) *first_bad = -1;
  if (!h || !in || !out) return set_error(DGLM_ERR_INVALID, "dglm_run_ensemble: NULL argument");
  if (!h->mesh_ready) return set_error(DGLM_ERR_STATE, "dglm_run_ensemble: upload the mesh first");
  if (count < 0 || nsteps < 0)
    return set_error(DGLM_ERR_INVALID, "dglm_run_ensemble: negative count or step count");
  for (int i = 0; i < count; i++) {
    if (!in[i] || !out[i]) return set_error(DGLM_ERR_INVALID, "dglm_run_ensemble: NULL member");
    for (int v = 0; v < h->nvar; v++)
      if (!in[i][v] || !out[i][v])
        return set_error(DGLM_ERR_INVALID, "dglm_run_ensemble: NULL variable pointer");
  }
  if (count == 0) return DGLM_OK;
  DeviceGuard g(h->dev);
  dglm_status st = ensure_ensemble(h, count);
  if (st != DGLM_OK) return st;
  // everything queued earlier on the handle's stream comes first
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_check(e, "dglm_run_ensemble");
  cudaEvent_t *in_ready = h->ens_ev, *in_free = h->ens_ev + 2, *out_ready = h->ens_ev + 4,
              *out_free = h->ens_ev + 6;
  const cudaStream_t S = h->stream, CI = h->ens_cin, CO = h->ens_cout;
  const size_t n = (size_t)h->d.K * h->Np, whole = sizeof(double) * h->nvar * h->vs;
  const int extra = h->d.physics == DGLM_ADVECTION ? 3 : 2;   // finite check, maxv, tau
  long launches = 0;
  h->launches = 0;
  h->state_ready = true;   // run_steps checks it; each member sets its state first
  // Every event is recorded (in host order) before any stream waits on that
  // recording: member i's copy-in, compute, copy-out are enqueued in turn.
  for (int i = 0; i < count && e == cudaSuccess; i++) {
    const int b = i & 1;
    // copy-in: waits until member i-2 has moved its input out of ens_in[b]
    e = cudaStreamWaitEvent(CI, in_free[b], 0);
    for (int v = 0; v < h->nvar && e == cudaSuccess; v++)
      e = cudaMemcpyAsync(h->ens_in[b] + (size_t)v * h->vs, in[i][v], sizeof(double) * n,
                          cudaMemcpyHostToDevice, CI);
    if (e == cudaSuccess) e = cudaEventRecord(in_ready[b], CI);
    // compute
    if (e == cudaSuccess) e = cudaStreamWaitEvent(S, in_ready[b], 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->u[0], h->ens_in[b], whole, cudaMemcpyDeviceToDevice, S);
    if (e == cudaSuccess) e = cudaEventRecord(in_free[b], S);
    if (e == cudaSuccess) e = reset_for_state(h, S);
    if (e != cudaSuccess) break;
    st = run_steps(h, nsteps);
    if (st != DGLM_OK) {
      cudaStreamSynchronize(CI);
      cudaStreamSynchronize(CO);
      cudaStreamSynchronize(S);
      return st;
    }
    launches += extra + h->launches;
    h->launches = 0;
    e = cudaStreamWaitEvent(S, out_free[b], 0);   // member i-2's copy-out is done
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h->ens_out[b], h->u[h->cur], whole, cudaMemcpyDeviceToDevice, S);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h->ens_flags + i, &h->sc->flags, sizeof(int), cudaMemcpyDeviceToDevice, S);
    if (e == cudaSuccess) e = cudaEventRecord(out_ready[b], S);
    // copy-out
    if (e == cudaSuccess) e = cudaStreamWaitEvent(CO, out_ready[b], 0);
    for (int v = 0; v < h->nvar && e == cudaSuccess; v++)
      e = cudaMemcpyAsync(out[i][v], h->ens_out[b] + (size_t)v * h->vs, sizeof(double) * n,
                          cudaMemcpyDeviceToHost, CO);
    if (e == cudaSuccess) e = cudaEventRecord(out_free[b], CO);
  }
  cudaError_t e2 = cudaStreamSynchronize(CI);
  cudaError_t e3 = cudaStreamSynchronize(S);
  cudaError_t e4 = cudaStreamSynchronize(CO);
  if (e == cudaSuccess) e = e2 != cudaSuccess ? e2 : (e3 != cudaSuccess ? e3 : e4);
  if (e != cudaSuccess) return cuda_check(e, "dglm_run_ensemble");
  h->launches = launches;
  std::vector<int> flags(count);
  e = cudaMemcpy(flags.data(), h->ens_flags, sizeof(int) * count, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_check(e, "dglm_run_ensemble");
  for (int i = 0; i < count; i++) {
    if (!(flags[i] & 7)) continue;
    if (first_bad) *first_bad = i;
    if (flags[i] & 4)
      return set_error(DGLM_ERR_CUDA, "dglm_run_ensemble: a bounded wait in a pipelined "
                                      "stage kernel expired; results are invalid");
    return set_error(DGLM_ERR_NONFINITE,
                     "dglm_run_ensemble: member " + std::to_string(i) +
                         " met a non-finite wave speed, dt or state");
  }
  return DGLM_OK;
}

}  // extern "C"

dglm_status dglm::run_steps(dglm_handle *h, int nsteps) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_step: NULL handle");
  if (!h->state_ready) return set_error(DGLM_ERR_STATE, "dglm_step: set a state first");
  if (nsteps < 0) return set_error(DGLM_ERR_INVALID, "dglm_step: negative step count");
  DeviceGuard g(h->dev);
  for (int i = 0; i < nsteps; i++) {
    const int c = h->cur;
    if (!h->graph[c]) {
      // capture one step from u[c]; fall back to direct launches on failure
      cudaGraph_t graph = nullptr;
      cudaStream_t cs = h->stream;
      bool ok = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      dglm_status st = ok ? issue_step(h, c, cs) : DGLM_OK;
      ok = (cudaStreamEndCapture(cs, &graph) == cudaSuccess) && ok && st == DGLM_OK;
      if (ok && cudaGraphInstantiate(&h->graph[c], graph, 0) != cudaSuccess) {
        h->graph[c] = nullptr;
        ok = false;
      }
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      if (!ok) {
        dglm_status s2 = issue_step(h, c, h->stream);
        if (s2 != DGLM_OK) return s2;
        h->launches += step_launches(h);
        h->cur ^= 1;
        continue;
      }
    }
    cudaError_t e = cudaGraphLaunch(h->graph[c], h->stream);
    if (e != cudaSuccess) return cuda_check(e, "dglm_step: graph launch");
    h->launches += step_launches(h);
    h->cur ^= 1;
  }
  return DGLM_OK;
}

extern "C" {

dglm_status dglm_step(dglm_handle *h, int nsteps) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_step: NULL handle");
  DeviceGuard g(h->dev);
  const double zero = 0.0;
  cudaError_t e = cudaMemcpyAsync(&h->sc->dt_fixed, &zero, sizeof(double),
                                  cudaMemcpyHostToDevice, h->stream);
  if (e != cudaSuccess) return cuda_check(e, "dglm_step");
  // the pageable source must stay alive until the copy is staged
  e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_check(e, "dglm_step");
  h->launches = 0;
  return run_steps(h, nsteps);
}

dglm_status dglm_step_fixed_dt(dglm_handle *h, int nsteps, double dt) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_step_fixed_dt: NULL handle");
  if (!(dt > 0) || !std::isfinite(dt))
    return set_error(DGLM_ERR_INVALID, "dglm_step_fixed_dt: dt must be positive and finite");
  DeviceGuard g(h->dev);
  cudaError_t e = cudaMemcpyAsync(&h->sc->dt_fixed, &dt, sizeof(double),
                                  cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_check(e, "dglm_step_fixed_dt");
  h->launches = 0;
  return run_steps(h, nsteps);
}

dglm_status dglm_stage(dglm_handle *h, int stage, double dt) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_stage: NULL handle");
  if (!h->state_ready) return set_error(DGLM_ERR_STATE, "dglm_stage: set a state first");
  if (stage < 0 || stage > 4 || !(dt >= 0) || !std::isfinite(dt))
    return set_error(DGLM_ERR_INVALID, "dglm_stage: stage must be 0..4 and dt >= 0");
  DeviceGuard g(h->dev);
  StageArgs a = stage_args(h, h->u[h->cur], h->u[h->cur ^ 1], stage);
  a.dt_override = dt;
  cudaError_t e = launch_stage_fp64(h->d.physics, h->d.N, h->variant, a, h->stream);
  if (e != cudaSuccess) return cuda_check(e, "dglm_stage");
  h->cur ^= 1;
  return DGLM_OK;
}

dglm_status dglm_sync(dglm_handle *h) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_sync: NULL handle");
  DeviceGuard g(h->dev);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_check(e, "dglm_sync");
  int flags = 0;
  e = cudaMemcpy(&flags, &h->sc->flags, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_check(e, "dglm_sync");
  if (flags & 4)
    return set_error(DGLM_ERR_CUDA,
                     "a bounded wait in a pipelined stage kernel expired; results are invalid");
  if (flags & 3)
    return set_error(DGLM_ERR_NONFINITE, "non-finite wave speed, dt or state met");
  return DGLM_OK;
}

dglm_status dglm_get_time(dglm_handle *h, double *t, double *dt, int *tstep) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_get_time: NULL handle");
  DeviceGuard g(h->dev);
  DevScalars s{};
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaMemcpy(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_check(e, "dglm_get_time");
  if (t) *t = s.t;
  if (dt) *dt = s.dt;
  if (tstep) *tstep = s.tstep;
  return DGLM_OK;
}

dglm_status dglm_set_time(dglm_handle *h, double t, int tstep) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_set_time: NULL handle");
  if (!(t >= 0) || tstep < 0) return set_error(DGLM_ERR_INVALID, "dglm_set_time: t < 0 or tstep < 0");
  if (!h->state_ready) return set_error(DGLM_ERR_STATE, "dglm_set_time: set the state first");
  DeviceGuard g(h->dev);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy(&h->sc->t, &t, sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(&h->sc->tstep, &tstep, sizeof(int), cudaMemcpyHostToDevice);
  return cuda_check(e, "dglm_set_time");
}

dglm_status dglm_get_dt_history(dglm_handle *h, int first, int count, double *dt_out) {
  if (!h || !dt_out || first < 0 || count < 0 || count > kHistory)
    return set_error(DGLM_ERR_INVALID, "dglm_get_dt_history: bad argument");
  DeviceGuard g(h->dev);
  std::vector<double> ring(kHistory);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy(ring.data(), h->dt_hist, sizeof(double) * kHistory, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_check(e, "dglm_get_dt_history");
  for (int i = 0; i < count; i++) dt_out[i] = ring[(first + i) % kHistory];
  return DGLM_OK;
}

dglm_status dglm_rhs(dglm_handle *h, const double *const *u, double *const *rhs) {
  if (!h || !u || !rhs) return set_error(DGLM_ERR_INVALID, "dglm_rhs: NULL argument");
  if (!h->mesh_ready) return set_error(DGLM_ERR_STATE, "dglm_rhs: upload the mesh first");
  DeviceGuard g(h->dev);
  dglm_status st = ensure_rhs_scratch(h);
  if (st != DGLM_OK) return st;
  cudaStream_t s = h->stream;
  const long n = (long)h->d.K * h->Np;
  cudaError_t e = cudaSuccess;
  for (int v = 0; v < h->nvar && e == cudaSuccess; v++)
    e = cudaMemcpyAsync(h->rhs_in + (size_t)v * h->vs, u[v], sizeof(double) * n,
                        cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->sc_s, 0, sizeof(DevScalars), s);
  StageArgs a = stage_args(h, h->rhs_in, h->rhs_out, -1);
  a.maxv = h->maxv_s;
  a.tau = h->tau_s;
  a.sc = h->sc_s;
  a.rhs_only = 1;
  if (e == cudaSuccess) e = launch_face_maxv(h->d.physics, h->d.N, a, 0, s);
  if (e == cudaSuccess) e = launch_tau(h->d.K, h->d.tau_scale, h->vmapF, h->maxv_s, h->tau_s, s);
  if (e == cudaSuccess) e = launch_stage_fp64(h->d.physics, h->d.N, h->variant, a, s);
  for (int v = 0; v < h->nvar && e == cudaSuccess; v++)
    e = cudaMemcpyAsync(rhs[v], h->rhs_out + (size_t)v * h->vs, sizeof(double) * n,
                        cudaMemcpyDeviceToDevice, s);
  int flags = 0;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMemcpy(&flags, &h->sc_s->flags, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_check(e, "dglm_rhs");
  if (flags & 4)
    return set_error(DGLM_ERR_CUDA,
                     "dglm_rhs: a bounded wait in a pipelined stage kernel expired");
  return DGLM_OK;
}

int dglm_variant_count(int physics, int N) { return stage_variant_count(physics, N); }

dglm_status dglm_variant_describe(int physics, int N, int variant, char *buf, size_t len) {
  StageVariantInfo v{};
  if (!buf || len == 0 || !stage_variant_info(physics, N, variant, &v))
    return set_error(DGLM_ERR_INVALID, "dglm_variant_describe: no such variant");
  if (v.mode == MODE_SIMT)
    snprintf(buf, len, "simt E=%d R=%d CPT=%d threads=%d smem=%zu", v.E, v.R, v.CPT, v.threads,
             v.smem);
  else if (v.mode == MODE_MMA16)
    snprintf(buf, len, "%smma16-%s E=%d WN=%d WM=%d threads=%d smem=%zu",
             v.persistent ? "pipe-" : "",
             v.prec == DGLM_PREC_TF32X3 ? "tf32x3" : v.prec == DGLM_PREC_BF16X6 ? "bf16x6"
                                                                                : "bf16x3",
             v.E, v.CPT, v.WM, v.threads, v.smem);
  else if (v.mode == MODE_TC)
    snprintf(buf, len, "tc-tmem-tf32x4 E=%d compute=%d threads=%d smem=%zu ring=%d%s%s", v.E,
             v.producers, v.threads, v.smem, v.ring, v.R == 2 ? " nodes/lane=2" : "",
             v.WM == 1 ? " vol=fp32-diff" : "");
  else if (v.mode == MODE_TCB)
    snprintf(buf, len, "tc-tmem-bf16x4 E=%d compute=%d threads=%d smem=%zu ring=%d buffers=%d%s",
             v.E, v.producers, v.threads, v.smem, v.ring, v.npad,
             v.WM == 1 ? " vol=fp32-diff" : "");
  else if (v.mode == MODE_MIXED) {
    const int n = snprintf(buf, len, "%s E=%d N=%d threads=%d smem=%zu",
                           v.prec == DGLM_PREC_TF32X3   ? "tcgen05-tf32x3"
                           : v.prec == DGLM_PREC_BF16X6 ? "tcgen05-bf16x6"
                                                        : "tcgen05-bf16x3",
                           v.E, v.npad, v.threads, v.smem);
    // producer warps are named only when there is more than one
    if (v.producers > 1 && n > 0 && (size_t)n < len)
      snprintf(buf + n, len - n, " prod=%d", v.producers);
  }
  else {
    const int n = snprintf(buf, len, "%s E=%d WN=%d WM=%d threads=%d smem=%zu%s",
                           v.mode == MODE_PIPE ? (v.groups == 2 ? "pipe2-dmma" : "pipe-dmma")
                                               : "dmma",
                           v.E, v.CPT, v.WM, v.threads, v.smem,
                           v.mode == MODE_PIPE && v.op_global ? " A=global" : "");
    // ring depth, producer warps and k-split are named only when they differ
    // from 2, 1 and 1; the fused pass and the global RK register always
    if (v.mode == MODE_PIPE &&
        (v.ring > 2 || v.producers > 1 || v.ksplit > 1 || v.fused || v.k_global ||
         v.ctas_per_sm > 1) && n > 0 &&
        (size_t)n < len) {
      int m = snprintf(buf + n, len - n, " ring=%d prod=%d", v.ring, v.producers);
      if (v.ksplit > 1 && m > 0 && (size_t)(n + m) < len)
        m += snprintf(buf + n + m, len - n - m, " ksplit=%d", v.ksplit);
      if (m > 0 && (size_t)(n + m) < len)
        m += snprintf(buf + n + m, len - n - m, "%s%s", v.fused ? " fused" : "",
                      v.k_global ? " k=global" : "");
      if (v.ctas_per_sm > 1 && m > 0 && (size_t)(n + m) < len)
        snprintf(buf + n + m, len - n - m, " ctas=%d", v.ctas_per_sm);
    }
  }
  return DGLM_OK;
}

dglm_status dglm_set_variant(dglm_handle *h, int variant) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_set_variant: NULL handle");
  StageVariantInfo v{};
  if (!stage_variant_info(h->d.physics, h->d.N, variant, &v))
    return set_error(DGLM_ERR_INVALID, "dglm_set_variant: no such variant");
  if (v.prec != h->d.precision)
    return set_error(DGLM_ERR_INVALID, "dglm_set_variant: variant is of another precision");
  DeviceGuard g(h->dev);
  cudaStreamSynchronize(h->stream);
  drop_graphs(h);
  h->variant = variant;
  h->vinfo = v;
  if (h->mesh_ready) return upload_operator_layout(h);
  return DGLM_OK;
}

int dglm_get_variant(dglm_handle *h) { return h ? h->variant : -1; }

dglm_status dglm_set_wait_limit(dglm_handle *h, long long cycles) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_set_wait_limit: NULL handle");
  if (cycles < 0) return set_error(DGLM_ERR_INVALID, "dglm_set_wait_limit: negative bound");
  DeviceGuard g(h->dev);
  cudaStreamSynchronize(h->stream);
  drop_graphs(h);   // the captured steps carry the bound in their arguments
  h->wait_cycles = cycles;
  return DGLM_OK;
}

dglm_status dglm_compact_face_maps(int K, int Np, int Nfp, const int *vmapP, int *etoe,
                                   unsigned char *code, int *lists, int max_lists,
                                   int *n_lists) {
  if (!vmapP || !etoe || !code || !n_lists || (max_lists > 0 && !lists))
    return set_error(DGLM_ERR_INVALID, "dglm_compact_face_maps: NULL argument");
  if (K < 1 || Np < 1 || Nfp < 1 || max_lists < 0 || max_lists > 256)
    return set_error(DGLM_ERR_INVALID, "dglm_compact_face_maps: bad sizes");
  // every face's trace must be one element's nodes; its local node list gets
  // a code (first seen, first numbered)
  std::map<std::vector<int>, int> seen;
  std::vector<int> loc(Nfp);
  for (size_t fc = 0; fc < (size_t)K * 4; fc++) {
    const int *p = vmapP + fc * Nfp;
    if (p[0] < 0 || (long long)p[0] >= (long long)K * Np)
      return set_error(DGLM_ERR_INVALID, "dglm_compact_face_maps: vmapP entry outside [0, K*Np)");
    const int n = p[0] / Np;
    for (int j = 0; j < Nfp; j++) {
      if (p[j] < 0 || p[j] / Np != n)
        return set_error(DGLM_ERR_UNSUPPORTED,
                         "dglm_compact_face_maps: a face's trace spans several elements");
      loc[j] = p[j] - n * Np;
    }
    auto it = seen.find(loc);
    if (it == seen.end()) {
      if ((int)seen.size() == max_lists)
        return set_error(DGLM_ERR_UNSUPPORTED,
                         "dglm_compact_face_maps: more distinct face node lists than max_lists");
      it = seen.emplace(loc, (int)seen.size()).first;
      std::copy(loc.begin(), loc.end(), lists + (size_t)it->second * Nfp);
    }
    etoe[fc] = n;
    code[fc] = (unsigned char)it->second;
  }
  *n_lists = (int)seen.size();
  return DGLM_OK;
}

dglm_status dglm_set_compact_face_maps(dglm_handle *h, int on) {
  if (!h) return set_error(DGLM_ERR_INVALID, "dglm_set_compact_face_maps: NULL handle");
  if (!h->mesh_ready)
    return set_error(DGLM_ERR_INVALID, "dglm_set_compact_face_maps: no mesh uploaded");
  DeviceGuard g(h->dev);
  cudaStreamSynchronize(h->stream);
  drop_graphs(h);   // the captured steps carry the map pointers in their arguments
  if (!on) {
    h->compact = false;
    return DGLM_OK;
  }
  if (!h->compact_built) {
    const int K = h->d.K, Np = h->Np, Nfp = h->Nfp, NFF = h->NFF;
    std::vector<int> vm((size_t)K * NFF), nb((size_t)K * 4), lists((size_t)256 * Nfp);
    std::vector<unsigned char> code((size_t)K * 4);
    cudaError_t e = cudaMemcpy(vm.data(), h->vmapP, sizeof(int) * vm.size(),
                               cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
      return set_error(DGLM_ERR_CUDA, std::string("dglm_set_compact_face_maps: ") +
                                          cudaGetErrorString(e));
    int nlists = 0;
    dglm_status st = dglm_compact_face_maps(K, Np, Nfp, vm.data(), nb.data(), code.data(),
                                            lists.data(), 256, &nlists);
    if (st != DGLM_OK) return st;
    if (!h->etoe) {
      st = dalloc(h, &h->etoe, (size_t)K * 4);
      if (st == DGLM_OK) st = dalloc(h, &h->fcode, (size_t)K * 4);
      if (st == DGLM_OK) st = dalloc(h, &h->ftab, (size_t)256 * Nfp);
      if (st != DGLM_OK) return st;
    }
    e = cudaMemcpy(h->etoe, nb.data(), sizeof(int) * nb.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(h->fcode, code.data(), code.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(h->ftab, lists.data(), sizeof(int) * nlists * Nfp, cudaMemcpyHostToDevice);
    if (e != cudaSuccess)
      return set_error(DGLM_ERR_CUDA, std::string("dglm_set_compact_face_maps: ") +
                                          cudaGetErrorString(e));
    h->ftab_lists = nlists;
    h->compact_built = true;
  }
  h->compact = true;
  return DGLM_OK;
}

int dglm_face_map_lists(dglm_handle *h) {
  return h && h->compact_built ? h->ftab_lists : 0;
}

long dglm_kernel_launches(dglm_handle *h) { return h ? h->launches : 0; }
size_t dglm_device_bytes(dglm_handle *h) { return h ? h->bytes : 0; }

}  // extern "C"
