// Batched advection: many independent meshes of uneven size and polynomial
// order advance together, one persistent launch per LSERK stage.
//
// The reference runs one mesh per process (advec_nopad_time.cu:32-108).
// Here a batch owns the concatenated per-element arrays of all its
// instances and a tile list: (instance, first element, count, order) with
// E_N elements per tile, E_N chosen per order so that tiles carry similar
// work (Np (3Np + NFF) multiply-adds per element).  Every CTA of the stage
// kernel walks the tile list with a static stride and runs the device
// function compiled for the tile's order -- one launch covers every order.
// The list is sorted by order, largest first, so each CTA gets a similar mix.
//
// Per tile (advection, one variable): stage u and the tile's metrics and
// face data in shared memory; volume fluxes v u combined with the metrics;
// contraction with [WDr WDs WDt] on the FP64 tensor cores (m8n8k4, the
// operator's A fragments per order, as the single-mesh DMMA path builds
// them); face traces through vmapP and the DGLM flux; contraction with
// -LIFT into the same accumulators; LSERK update with the instance's dt.
//
// Per instance: velocity v (constant, the per-node velocity the reference
// takes reduces to it), tau from the face wave speed |v| (update_tau,
// advec_dglm.cpp), the CFL dt from a per-instance max of |v| Fscale
// (calc_dt), clipped to tmax, and the simulated time.  Steps are captured as
// CUDA graphs.
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

struct BatchTile {
  int inst, e0, ne, N;
};

struct BatchInst {
  long node_off;   // first node of the instance in the field arrays
  long elem_off;   // first element in the per-element arrays
  long fp_off;     // first face point in vmapP
  int K, N;
  double vx, vy, vz, tau;
};

struct BatchScalars {
  double t, dt_cfl, dt;           // time, CFL dt, dt of the step in flight
  unsigned long long acc;         // max |v| Fscale over the instance's faces (bits)
  int tstep, active;
};

struct BatchArgs {
  const BatchTile *tiles;
  int ntiles;
  const BatchInst *inst;
  BatchScalars *sc;
  const double *ops[kMaxOrder + 1];   // A fragments per order
  const int *Fmask[kMaxOrder + 1];
  const double *geo;     // [9][gs]
  const double *nrm;     // [3][4 gs]
  const double *fscale;  // [4 gs]
  long gs;
  const int *vmapP;      // instance-local node ids
  const double *u_in;
  double *u_out, *kreg;
  double rka, rkb;
};

constexpr int kBatchThreads = 256;
constexpr int kBatchWarps = kBatchThreads / 32;

template <int N>
struct BT {
  static constexpr int Np = np_of(N), Nfp = nfp_of(N), NFF = 4 * Nfp;
  static constexpr int E = N <= 3 ? 64 : N == 4 ? 32 : 16;
  static constexpr int EP = E + 1;
  static constexpr int MT = (Np + 7) / 8, NT = E / 8;
  static constexpr int KV = 3 * Np, KVP = (KV + 3) / 4 * 4;
  static constexpr int KF = NFF, KFP = (KF + 3) / 4 * 4;
  static constexpr int BROWS = KVP > KFP ? KVP : KFP;
  static constexpr int BLD = E + 4;                 // conflict-free B fragments
  static constexpr int PAIRS = MT * NT, WP = (PAIRS + kBatchWarps - 1) / kBatchWarps;
  static constexpr int VMLD = NFF + 1;
  static constexpr int S_U = Np * EP, S_B = BROWS * BLD, S_GEO = 9 * E, S_FACE = 4 * 4 * E;
  static constexpr size_t SMEM =
      sizeof(double) * (S_U + S_B + S_GEO + S_FACE) + sizeof(int) * ((size_t)E * VMLD + NFF);
  static_assert(S_B >= Np * EP, "epilogue reuses B");
  static constexpr int KSTEPS = KVP / 4 + KFP / 4;   // A fragment k-steps
};

// 8- and 4-byte asynchronous global -> shared copies (all of a tile's staging
// is issued before one wait)
__device__ __forceinline__ void b_cp8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void b_cp4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void b_cp_wait() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

__device__ __forceinline__ void b_dmma(double (&d)[2], double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

template <int N>
__device__ __forceinline__ void batch_tile(const BatchArgs &a, const BatchTile &t,
                                           double *smem) {
  using C = BT<N>;
  constexpr int Np = C::Np, Nfp = C::Nfp, NFF = C::NFF, E = C::E, EP = C::EP, BLD = C::BLD,
                T = kBatchThreads;
  double *sU = smem;                 // [i][EP]
  double *sB = sU + C::S_U;          // [k][BLD]
  double *sGeo = sB + C::S_B;        // [9][E]
  double *sFace = sGeo + C::S_GEO;   // [4][4][E]: nx ny nz fs
  int *sVm = reinterpret_cast<int *>(sFace + C::S_FACE);
  int *sFm = sVm + E * C::VMLD;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const BatchInst I = a.inst[t.inst];
  const int ne = t.ne;
  const long eg0 = I.elem_off + t.e0;                 // global element of the tile
  const long nb = I.node_off + (long)t.e0 * Np;       // first node of the tile
  const double *Afrag = a.ops[N];
  const double dt = a.sc[t.inst].dt;

  // this thread's RK register values for the update, fetched now so their
  // latency overlaps the tile's work
  constexpr int KPT = (E * Np + T - 1) / T;
  double kr[KPT];
#pragma unroll
  for (int q = 0; q < KPT; q++) {
    const int g = tid + q * T;
    kr[q] = g < ne * Np ? a.kreg[nb + g] : 0.0;
  }
  // staging: every copy is issued before one wait; padding is zero-filled
  for (int i = tid; i < NFF; i += T) b_cp4(sFm + i, a.Fmask[N] + i);
  for (int g = tid; g < E * Np; g += T) {
    const int e = g / Np, i = g - e * Np;
    if (g < ne * Np)
      b_cp8(sU + i * EP + e, a.u_in + nb + g);
    else
      sU[i * EP + e] = 0.0;
  }
  for (int g = tid; g < 9 * E; g += T) {
    const int m = g / E, e = g - m * E;
    if (e < ne)
      b_cp8(sGeo + g, a.geo + (long)m * a.gs + eg0 + e);
    else
      sGeo[g] = 0.0;
  }
  for (int g = tid; g < 4 * E; g += T) {
    const int e = g >> 2, f = g & 3;
    const long gf = (eg0 + e) * 4 + f;
    if (e < ne) {
      b_cp8(sFace + (0 * 4 + f) * E + e, a.nrm + gf);
      b_cp8(sFace + (1 * 4 + f) * E + e, a.nrm + 4 * a.gs + gf);
      b_cp8(sFace + (2 * 4 + f) * E + e, a.nrm + 8 * a.gs + gf);
      b_cp8(sFace + (3 * 4 + f) * E + e, a.fscale + gf);
    } else {
      for (int q = 0; q < 4; q++) sFace[(q * 4 + f) * E + e] = 0.0;
    }
  }
  const long fp0 = I.fp_off + (long)t.e0 * NFF;
  for (int g = tid; g < E * NFF; g += T) {
    const int e = g / NFF, fj = g - e * NFF;
    if (g < ne * NFF)
      b_cp4(sVm + e * C::VMLD + fj, a.vmapP + fp0 + g);
    else
      sVm[e * C::VMLD + fj] = 0;
  }
  b_cp_wait();
  __syncthreads();

  // volume fluxes -> B rows [0, 3Np)
  for (int it = tid; it < E * Np; it += T) {
    const int i = it / E, e = it - i * E;
    const double *g = sGeo + e;
    const double uu = sU[i * EP + e];
    const double F = I.vx * uu, G = I.vy * uu, W = I.vz * uu;
    sB[(0 * Np + i) * BLD + e] = g[0] * F + g[E] * G + g[2 * E] * W;
    sB[(1 * Np + i) * BLD + e] = g[3 * E] * F + g[4 * E] * G + g[5 * E] * W;
    sB[(2 * Np + i) * BLD + e] = g[6 * E] * F + g[7 * E] * G + g[8 * E] * W;
  }
  for (int g = tid; g < (C::KVP - C::KV) * BLD; g += T) sB[C::KV * BLD + g] = 0.0;
  __syncthreads();

  double acc[C::WP][2];
#pragma unroll
  for (int j = 0; j < C::WP; j++) acc[j][0] = acc[j][1] = 0.0;
#pragma unroll
  for (int j = 0; j < C::WP; j++) {
    const int p = warp + kBatchWarps * j;
    if (p < C::PAIRS) {
      const int mt = p % C::MT, nt = p / C::MT;
      const double *Ab = Afrag + (long)mt * 32 + lane;
      const double *Bb = sB + (lane & 3) * BLD + nt * 8 + (lane >> 2);
#pragma unroll 4
      for (int ks = 0; ks < C::KVP / 4; ks++)
        b_dmma(acc[j], __ldg(Ab + (long)ks * C::MT * 32), Bb[ks * 4 * BLD]);
    }
  }
  __syncthreads();

  // face traces and fluxes -> B rows [0, NFF)
  for (int it = tid; it < E * NFF; it += T) {
    const int fj = it / E, e = it - fj * E, f = fj / Nfp;
    if (e >= ne) {
      sB[fj * BLD + e] = 0.0;
      continue;
    }
    const double um = sU[sFm[fj] * EP + e];
    const double ub = 0.5 * (um + a.u_in[I.node_off + sVm[e * C::VMLD + fj]]);
    const double F = I.vx * ub, G = I.vy * ub, W = I.vz * ub;
    const double nd = sFace[(0 * 4 + f) * E + e] * F + sFace[(1 * 4 + f) * E + e] * G +
                      sFace[(2 * 4 + f) * E + e] * W;
    sB[fj * BLD + e] = (nd - I.tau * (ub - um)) * sFace[(3 * 4 + f) * E + e];
  }
  for (int g = tid; g < (C::KFP - C::KF) * BLD; g += T) sB[C::KF * BLD + g] = 0.0;
  __syncthreads();

#pragma unroll
  for (int j = 0; j < C::WP; j++) {
    const int p = warp + kBatchWarps * j;
    if (p < C::PAIRS) {
      const int mt = p % C::MT, nt = p / C::MT;
      const double *Ab = Afrag + ((long)(C::KVP / 4) * C::MT + mt) * 32 + lane;
      const double *Bb = sB + (lane & 3) * BLD + nt * 8 + (lane >> 2);
#pragma unroll 4
      for (int ks = 0; ks < C::KFP / 4; ks++)
        b_dmma(acc[j], __ldg(Ab + (long)ks * C::MT * 32), Bb[ks * 4 * BLD]);
    }
  }
  __syncthreads();

  // rhs -> sB as [i][EP], then the LSERK update with coalesced stores
  double *sR = sB;
#pragma unroll
  for (int j = 0; j < C::WP; j++) {
    const int p = warp + kBatchWarps * j;
    if (p < C::PAIRS) {
      const int mt = p % C::MT, nt = p / C::MT;
      const int i = mt * 8 + (lane >> 2);
      if (i < Np) {
#pragma unroll
        for (int h = 0; h < 2; h++) sR[i * EP + nt * 8 + (lane & 3) * 2 + h] = acc[j][h];
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < KPT; q++) {
    const int g = tid + q * T;
    if (g >= ne * Np) continue;
    const int e = g / Np, i = g - e * Np;
    const double kn = a.rka * kr[q] + dt * sR[i * EP + e];
    a.kreg[nb + g] = kn;
    a.u_out[nb + g] = sU[i * EP + e] + a.rkb * kn;
  }
}

template <int N>
constexpr size_t bt_smem() {
  return BT<N>::SMEM;
}
constexpr size_t cmax(size_t a, size_t b) { return a > b ? a : b; }
constexpr size_t kBatchSmem =
    cmax(cmax(cmax(bt_smem<2>(), bt_smem<3>()), cmax(bt_smem<4>(), bt_smem<5>())), bt_smem<6>());

__global__ void __launch_bounds__(kBatchThreads, 3) batch_stage_kernel(const BatchArgs a) {
  extern __shared__ __align__(16) double smem[];
  for (int ti = blockIdx.x; ti < a.ntiles; ti += gridDim.x) {
    const BatchTile t = a.tiles[ti];
    switch (t.N) {
      case 2: batch_tile<2>(a, t, smem); break;
      case 3: batch_tile<3>(a, t, smem); break;
      case 4: batch_tile<4>(a, t, smem); break;
      case 5: batch_tile<5>(a, t, smem); break;
      case 6: batch_tile<6>(a, t, smem); break;
      default: break;
    }
    __syncthreads();
  }
}

// Per-instance max of |v| Fscale over its faces (calc_maxv + calc_dt of the
// reference with a frozen velocity), one block per instance.
__global__ void batch_wavespeed_kernel(const BatchInst *inst, const double *fscale,
                                       BatchScalars *sc) {
  const BatchInst I = inst[blockIdx.x];
  const double mv = sqrt(I.vx * I.vx + I.vy * I.vy + I.vz * I.vz);
  unsigned long long b = 0ull;
  for (long f = threadIdx.x; f < 4L * I.K; f += blockDim.x) {
    const unsigned long long x = dbits(mv * fscale[I.elem_off * 4 + f]);
    b = x > b ? x : b;
  }
  b = warp_max_bits(b);
  __shared__ unsigned long long s[32];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = b;
  __syncthreads();
  if (threadIdx.x < 32) {
    b = threadIdx.x < blockDim.x / 32 ? s[threadIdx.x] : 0ull;
    b = warp_max_bits(b);
    if (threadIdx.x == 0) sc[blockIdx.x].acc = b;
  }
}

// dt of every instance for the coming step: CFL dt (euler_time.cpp:49-57 /
// advec_time.cpp), clipped so the instance ends at tmax; 0 once it has.
__global__ void batch_step_begin_kernel(int n, const BatchInst *inst, double cfl, double tmax,
                                        BatchScalars *sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double m = __longlong_as_double((long long)sc[i].acc);
  double dt = (cfl / (2 * inst[i].N + 1)) * (1 / m);
  const int active = sc[i].t < tmax;
  if (active && sc[i].t + dt > tmax) dt = tmax - sc[i].t;
  if (!active) dt = 0.0;
  sc[i].dt_cfl = (cfl / (2 * inst[i].N + 1)) * (1 / m);
  sc[i].dt = dt;
  sc[i].active = active;
}

__global__ void batch_step_end_kernel(int n, BatchScalars *sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !sc[i].active) return;
  sc[i].t += sc[i].dt;
  sc[i].tstep += 1;
}

}  // namespace dglm

using namespace dglm;

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

struct BatchHostInst {
  int N, K;
  double v[3];
  std::vector<double> geo[9], nrm[3], fscale, u0;
  std::vector<int> vmapP;
};

struct dglm_batch {
  dglm_batch_desc d{};
  int dev = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<BatchHostInst> host;
  std::vector<double> Ahost[kMaxOrder + 1];   // stacked [WDr WDs WDt -LIFT] per order
  std::vector<int> Fm[kMaxOrder + 1];
  bool finalized = false;
  // device
  std::vector<void *> allocs;
  size_t bytes = 0;
  BatchArgs args{};
  BatchInst *inst = nullptr;
  BatchTile *tiles = nullptr;
  BatchScalars *sc = nullptr;
  double *u[2] = {nullptr, nullptr};
  int cur = 0, ntiles = 0, grid = 0;
  std::vector<BatchInst> hinst;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  long launches = 0;
};

namespace {



template <typename T>
dglm_status balloc(dglm_batch *b, T **p, size_t count) {
  void *q = nullptr;
  const size_t n = std::max<size_t>(count * sizeof(T), 16);
  cudaError_t e = cudaMalloc(&q, n);
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(DGLM_ERR_NOMEM, std::string("dglm_batch: cudaMalloc failed: ") +
                                         cudaGetErrorString(e));
  }
  b->allocs.push_back(q);
  b->bytes += n;
  *p = static_cast<T *>(q);
  return DGLM_OK;
}

// m8n8k4 A fragments of [WDr WDs WDt | -LIFT] (as the single-mesh DMMA
// layout): [kstep][mtile][lane], row 8*mtile + lane/4, column 4*kstep +
// lane%4 of the volume block, then of the lift block.
template <int N>
std::vector<double> batch_fragments(const std::vector<double> &A) {
  using C = BT<N>;
  const int Np = C::Np, NFF = C::NFF, KA = 3 * Np + NFF, KV = 3 * Np;
  const int kv4 = C::KVP / 4, kf4 = C::KFP / 4;
  std::vector<double> out((size_t)(kv4 + kf4) * C::MT * 32, 0.0);
  for (int ks = 0; ks < kv4 + kf4; ks++)
    for (int mt = 0; mt < C::MT; mt++)
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
        if (ok && row < Np) out[((size_t)ks * C::MT + mt) * 32 + lane] = A[(size_t)row * KA + k];
      }
  return out;
}

std::vector<double> fragments_for(int N, const std::vector<double> &A) {
  switch (N) {
    case 2: return batch_fragments<2>(A);
    case 3: return batch_fragments<3>(A);
    case 4: return batch_fragments<4>(A);
    case 5: return batch_fragments<5>(A);
    case 6: return batch_fragments<6>(A);
  }
  return {};
}

int tile_elems(int N) {
  switch (N) {
    case 2: return BT<2>::E;
    case 3: return BT<3>::E;
    case 4: return BT<4>::E;
    case 5: return BT<5>::E;
    case 6: return BT<6>::E;
  }
  return 0;
}

void drop_batch_graphs(dglm_batch *b) {
  for (auto &g : b->graph) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
}

cudaError_t issue_batch_step(dglm_batch *b, int cur, cudaStream_t s) {
  const int n = (int)b->hinst.size();
  const int tb = 128, nb = (n + tb - 1) / tb;
  batch_step_begin_kernel<<<nb, tb, 0, s>>>(n, b->inst, b->d.cfl, b->d.tmax, b->sc);
  cudaError_t e = cudaGetLastError();
  for (int st = 0; st < 5 && e == cudaSuccess; st++) {
    BatchArgs a = b->args;
    const int in = (cur + st) & 1;
    a.u_in = b->u[in];
    a.u_out = b->u[in ^ 1];
    a.rka = RKA[st];
    a.rkb = RKB[st];
    batch_stage_kernel<<<b->grid, kBatchThreads, kBatchSmem, s>>>(a);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    batch_step_end_kernel<<<nb, tb, 0, s>>>(n, b->sc);
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace

extern "C" {

dglm_status dglm_batch_create(const dglm_batch_desc *desc, dglm_batch **out) {
  if (!desc || !out) return set_error(DGLM_ERR_INVALID, "dglm_batch_create: NULL argument");
  *out = nullptr;
  if (desc->physics != DGLM_ADVECTION)
    return set_error(DGLM_ERR_UNSUPPORTED, "dglm_batch_create: batches are advection only");
  if (!(desc->cfl > 0) || !(desc->tau_scale >= 0) || !(desc->tmax > 0))
    return set_error(DGLM_ERR_INVALID, "dglm_batch_create: cfl/tau_scale/tmax out of range");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_error(DGLM_ERR_CUDA, "dglm_batch_create: no CUDA device");
  if (desc->device >= ndev)
    return set_error(DGLM_ERR_INVALID, "dglm_batch_create: device out of range");
  dglm_batch *b = new dglm_batch();
  b->d = *desc;
  if (desc->device < 0) cudaGetDevice(&b->dev); else b->dev = desc->device;
  DeviceGuard g(b->dev);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return set_error(DGLM_ERR_CUDA, "dglm_batch_create: stream creation failed");
  }
  b->own_stream = true;
  *out = b;
  return DGLM_OK;
}

dglm_status dglm_batch_add(dglm_batch *b, int N, int K, const dglm_mesh_arrays *m,
                           const double *u0, const double *velocity, int *index) {
  if (!b || !m || !u0 || !velocity)
    return set_error(DGLM_ERR_INVALID, "dglm_batch_add: NULL argument");
  if (b->finalized) return set_error(DGLM_ERR_STATE, "dglm_batch_add: batch already finalized");
  if (N < 2 || N > 6) return set_error(DGLM_ERR_UNSUPPORTED, "dglm_batch_add: orders 2..6");
  if (K <= 0) return set_error(DGLM_ERR_INVALID, "dglm_batch_add: K must be positive");
  const int Np = np_of(N), NFF = 4 * nfp_of(N);
  const double *req[] = {m->WDr, m->WDs, m->WDt, m->LIFT, m->rx, m->ry, m->rz, m->sx,
                         m->sy,  m->sz,  m->tx,  m->ty,   m->tz, m->Fscale, m->nx, m->ny, m->nz};
  for (const double *p : req)
    if (!p) return set_error(DGLM_ERR_INVALID, "dglm_batch_add: a real array is NULL");
  if (!m->vmapP || !m->Fmask) return set_error(DGLM_ERR_INVALID, "dglm_batch_add: index array is NULL");
  if (m->matrix_order != 'c' && m->matrix_order != 'f')
    return set_error(DGLM_ERR_INVALID, "dglm_batch_add: matrix_order must be 'c' or 'f'");
  for (long i = 0; i < (long)K * NFF; i++)
    if (m->vmapP[i] < 0 || m->vmapP[i] >= (long)K * Np)
      return set_error(DGLM_ERR_INVALID, "dglm_batch_add: vmapP entry outside [0, K*Np)");
  for (int i = 0; i < NFF; i++)
    if (m->Fmask[i] < 0 || m->Fmask[i] >= Np)
      return set_error(DGLM_ERR_INVALID, "dglm_batch_add: Fmask entry outside [0, Np)");
  for (long i = 0; i < (long)K * Np; i++)
    if (!std::isfinite(u0[i]))
      return set_error(DGLM_ERR_NONFINITE, "dglm_batch_add: non-finite initial state");
  for (int q = 0; q < 3; q++)
    if (!std::isfinite(velocity[q]))
      return set_error(DGLM_ERR_INVALID, "dglm_batch_add: non-finite velocity");
  // operators: one copy per order, the first instance of that order provides it
  const bool cm = m->matrix_order == 'f';
  const int KA = 3 * Np + NFF;
  std::vector<double> A((size_t)Np * KA);
  auto at = [&](const double *M, long i, long j, long cols) {
    return cm ? M[j * Np + i] : M[i * cols + j];
  };
  for (long i = 0; i < Np; i++) {
    for (long j = 0; j < Np; j++) {
      A[i * KA + j] = at(m->WDr, i, j, Np);
      A[i * KA + Np + j] = at(m->WDs, i, j, Np);
      A[i * KA + 2 * Np + j] = at(m->WDt, i, j, Np);
    }
    for (long j = 0; j < NFF; j++) A[i * KA + 3 * Np + j] = -at(m->LIFT, i, j, NFF);
  }
  std::vector<int> Fm(m->Fmask, m->Fmask + NFF);
  if (b->Ahost[N].empty()) {
    b->Ahost[N] = A;
    b->Fm[N] = Fm;
  } else if (b->Ahost[N] != A || b->Fm[N] != Fm) {
    return set_error(DGLM_ERR_INVALID,
                     "dglm_batch_add: operators differ from an earlier instance of this order");
  }
  BatchHostInst I;
  I.N = N;
  I.K = K;
  for (int q = 0; q < 3; q++) I.v[q] = velocity[q];
  const double *g9[9] = {m->rx, m->ry, m->rz, m->sx, m->sy, m->sz, m->tx, m->ty, m->tz};
  for (int q = 0; q < 9; q++) I.geo[q].assign(g9[q], g9[q] + K);
  I.nrm[0].assign(m->nx, m->nx + 4L * K);
  I.nrm[1].assign(m->ny, m->ny + 4L * K);
  I.nrm[2].assign(m->nz, m->nz + 4L * K);
  I.fscale.assign(m->Fscale, m->Fscale + 4L * K);
  I.vmapP.assign(m->vmapP, m->vmapP + (long)K * NFF);
  I.u0.assign(u0, u0 + (long)K * Np);
  b->host.push_back(std::move(I));
  if (index) *index = (int)b->host.size() - 1;
  return DGLM_OK;
}

dglm_status dglm_batch_finalize(dglm_batch *b) {
  if (!b) return set_error(DGLM_ERR_INVALID, "dglm_batch_finalize: NULL batch");
  if (b->finalized) return set_error(DGLM_ERR_STATE, "dglm_batch_finalize: already finalized");
  if (b->host.empty()) return set_error(DGLM_ERR_STATE, "dglm_batch_finalize: no instances");
  DeviceGuard g(b->dev);
  const int n = (int)b->host.size();
  long nodes = 0, elems = 0, fps = 0;
  b->hinst.resize(n);
  for (int i = 0; i < n; i++) {
    const BatchHostInst &H = b->host[i];
    const int Np = np_of(H.N), NFF = 4 * nfp_of(H.N);
    BatchInst &I = b->hinst[i];
    I.node_off = nodes;
    I.elem_off = elems;
    I.fp_off = fps;
    I.K = H.K;
    I.N = H.N;
    I.vx = H.v[0];
    I.vy = H.v[1];
    I.vz = H.v[2];
    // update_tau with maxv = |v| on both sides (advec_dglm.cpp)
    const double mv = std::sqrt(I.vx * I.vx + I.vy * I.vy + I.vz * I.vz);
    I.tau = 0.25 * (mv + mv) * b->d.tau_scale;
    nodes += ((long)H.K * Np + 31) / 32 * 32;
    elems += H.K;
    fps += (long)H.K * NFF;
  }
  const long gs = elems;
  // tiles, largest order first
  std::vector<BatchTile> tiles;
  for (int N = 6; N >= 2; N--)
    for (int i = 0; i < n; i++) {
      if (b->host[i].N != N) continue;
      const int E = tile_elems(N);
      for (int e0 = 0; e0 < b->host[i].K; e0 += E)
        tiles.push_back(BatchTile{i, e0, std::min(E, b->host[i].K - e0), N});
    }
  b->ntiles = (int)tiles.size();
  // host staging of the concatenated arrays
  std::vector<double> geo((size_t)9 * gs), nrm((size_t)12 * gs), fs((size_t)4 * gs),
      u0((size_t)nodes, 0.0);
  std::vector<int> vm((size_t)fps);
  for (int i = 0; i < n; i++) {
    const BatchHostInst &H = b->host[i];
    const BatchInst &I = b->hinst[i];
    for (int q = 0; q < 9; q++)
      std::copy(H.geo[q].begin(), H.geo[q].end(), geo.begin() + (size_t)q * gs + I.elem_off);
    for (int q = 0; q < 3; q++)
      std::copy(H.nrm[q].begin(), H.nrm[q].end(),
                nrm.begin() + (size_t)q * 4 * gs + 4 * I.elem_off);
    std::copy(H.fscale.begin(), H.fscale.end(), fs.begin() + 4 * I.elem_off);
    std::copy(H.vmapP.begin(), H.vmapP.end(), vm.begin() + I.fp_off);
    std::copy(H.u0.begin(), H.u0.end(), u0.begin() + I.node_off);
  }
  dglm_status st = DGLM_OK;
  auto chk = [&](dglm_status s) {
    if (st == DGLM_OK) st = s;
  };
  double *dgeo = nullptr, *dnrm = nullptr, *dfs = nullptr, *dk = nullptr;
  int *dvm = nullptr;
  chk(balloc(b, &b->inst, (size_t)n));
  chk(balloc(b, &b->sc, (size_t)n));
  chk(balloc(b, &b->tiles, tiles.size()));
  chk(balloc(b, &dgeo, geo.size()));
  chk(balloc(b, &dnrm, nrm.size()));
  chk(balloc(b, &dfs, fs.size()));
  chk(balloc(b, &dvm, vm.size()));
  chk(balloc(b, &b->u[0], (size_t)nodes));
  chk(balloc(b, &b->u[1], (size_t)nodes));
  chk(balloc(b, &dk, (size_t)nodes));
  if (st != DGLM_OK) return st;
  const auto H2D = cudaMemcpyHostToDevice;
  cudaError_t e = cudaMemcpy(b->inst, b->hinst.data(), sizeof(BatchInst) * n, H2D);
  if (e == cudaSuccess) e = cudaMemcpy(b->tiles, tiles.data(), sizeof(BatchTile) * tiles.size(), H2D);
  if (e == cudaSuccess) e = cudaMemcpy(dgeo, geo.data(), sizeof(double) * geo.size(), H2D);
  if (e == cudaSuccess) e = cudaMemcpy(dnrm, nrm.data(), sizeof(double) * nrm.size(), H2D);
  if (e == cudaSuccess) e = cudaMemcpy(dfs, fs.data(), sizeof(double) * fs.size(), H2D);
  if (e == cudaSuccess) e = cudaMemcpy(dvm, vm.data(), sizeof(int) * vm.size(), H2D);
  if (e == cudaSuccess) e = cudaMemcpy(b->u[0], u0.data(), sizeof(double) * nodes, H2D);
  if (e == cudaSuccess) e = cudaMemset(b->u[1], 0, sizeof(double) * nodes);
  if (e == cudaSuccess) e = cudaMemset(dk, 0, sizeof(double) * nodes);
  if (e == cudaSuccess) e = cudaMemset(b->sc, 0, sizeof(BatchScalars) * n);
  BatchArgs &a = b->args;
  a = BatchArgs{};
  for (int N = 2; N <= 6 && e == cudaSuccess; N++) {
    if (b->Ahost[N].empty()) continue;
    std::vector<double> fr = fragments_for(N, b->Ahost[N]);
    double *dops = nullptr;
    int *dfm = nullptr;
    if (balloc(b, &dops, fr.size()) != DGLM_OK || balloc(b, &dfm, b->Fm[N].size()) != DGLM_OK)
      return DGLM_ERR_NOMEM;
    e = cudaMemcpy(dops, fr.data(), sizeof(double) * fr.size(), H2D);
    if (e == cudaSuccess)
      e = cudaMemcpy(dfm, b->Fm[N].data(), sizeof(int) * b->Fm[N].size(), H2D);
    a.ops[N] = dops;
    a.Fmask[N] = dfm;
  }
  if (e != cudaSuccess) return cuda_check(e, "dglm_batch_finalize");
  a.tiles = b->tiles;
  a.ntiles = b->ntiles;
  a.inst = b->inst;
  a.sc = b->sc;
  a.geo = dgeo;
  a.nrm = dnrm;
  a.fscale = dfs;
  a.gs = gs;
  a.vmapP = dvm;
  a.kreg = dk;
  e = cudaFuncSetAttribute(batch_stage_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kBatchSmem);
  int per_sm = 0, sms = 0;
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_stage_kernel,
                                                      kBatchThreads, kBatchSmem);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->dev);
  if (e != cudaSuccess) return cuda_check(e, "dglm_batch_finalize");
  b->grid = std::max(1, std::min(b->ntiles, std::max(per_sm, 1) * sms));
  batch_wavespeed_kernel<<<n, 256, 0, b->stream>>>(b->inst, dfs, b->sc);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return cuda_check(e, "dglm_batch_finalize");
  b->host.clear();
  b->host.shrink_to_fit();
  b->cur = 0;
  b->finalized = true;
  return DGLM_OK;
}

dglm_status dglm_batch_step(dglm_batch *b, int nsteps) {
  if (!b) return set_error(DGLM_ERR_INVALID, "dglm_batch_step: NULL batch");
  if (!b->finalized) return set_error(DGLM_ERR_STATE, "dglm_batch_step: finalize first");
  if (nsteps < 0) return set_error(DGLM_ERR_INVALID, "dglm_batch_step: negative step count");
  DeviceGuard g(b->dev);
  b->launches = 0;
  for (int i = 0; i < nsteps; i++) {
    const int c = b->cur;
    if (!b->graph[c]) {
      cudaGraph_t graph = nullptr;
      cudaStream_t cs = b->stream;
      bool ok = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      cudaError_t le = ok ? issue_batch_step(b, c, cs) : cudaSuccess;
      ok = (cudaStreamEndCapture(cs, &graph) == cudaSuccess) && ok && le == cudaSuccess;
      if (ok && cudaGraphInstantiate(&b->graph[c], graph, 0) != cudaSuccess) {
        b->graph[c] = nullptr;
        ok = false;
      }
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      if (!ok) {
        cudaError_t e = issue_batch_step(b, c, b->stream);
        if (e != cudaSuccess) return cuda_check(e, "dglm_batch_step");
        b->launches += 7;
        b->cur ^= 1;
        continue;
      }
    }
    cudaError_t e = cudaGraphLaunch(b->graph[c], b->stream);
    if (e != cudaSuccess) return cuda_check(e, "dglm_batch_step: graph launch");
    b->launches += 7;
    b->cur ^= 1;
  }
  return DGLM_OK;
}

dglm_status dglm_batch_sync(dglm_batch *b) {
  if (!b) return set_error(DGLM_ERR_INVALID, "dglm_batch_sync: NULL batch");
  DeviceGuard g(b->dev);
  return cuda_check(cudaStreamSynchronize(b->stream), "dglm_batch_sync");
}

int dglm_batch_count(dglm_batch *b) {
  if (!b) return -1;
  return b->finalized ? (int)b->hinst.size() : (int)b->host.size();
}

dglm_status dglm_batch_get_state(dglm_batch *b, int index, double *u, int on_device) {
  if (!b || !u) return set_error(DGLM_ERR_INVALID, "dglm_batch_get_state: NULL argument");
  if (!b->finalized) return set_error(DGLM_ERR_STATE, "dglm_batch_get_state: finalize first");
  if (index < 0 || index >= (int)b->hinst.size())
    return set_error(DGLM_ERR_INVALID, "dglm_batch_get_state: no such instance");
  DeviceGuard g(b->dev);
  const BatchInst &I = b->hinst[index];
  cudaError_t e = cudaMemcpyAsync(u, b->u[b->cur] + I.node_off,
                                  sizeof(double) * (size_t)I.K * np_of(I.N),
                                  on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                  b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  return cuda_check(e, "dglm_batch_get_state");
}

dglm_status dglm_batch_get_time(dglm_batch *b, int index, double *t, double *dt, int *tstep) {
  if (!b) return set_error(DGLM_ERR_INVALID, "dglm_batch_get_time: NULL batch");
  if (!b->finalized) return set_error(DGLM_ERR_STATE, "dglm_batch_get_time: finalize first");
  if (index < 0 || index >= (int)b->hinst.size())
    return set_error(DGLM_ERR_INVALID, "dglm_batch_get_time: no such instance");
  DeviceGuard g(b->dev);
  BatchScalars s{};
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy(&s, b->sc + index, sizeof(BatchScalars), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_check(e, "dglm_batch_get_time");
  if (t) *t = s.t;
  if (dt) *dt = s.dt;
  if (tstep) *tstep = s.tstep;
  return DGLM_OK;
}

dglm_status dglm_batch_set_stream(dglm_batch *b, void *stream) {
  if (!b) return set_error(DGLM_ERR_INVALID, "dglm_batch_set_stream: NULL batch");
  DeviceGuard g(b->dev);
  cudaStreamSynchronize(b->stream);
  drop_batch_graphs(b);
  if (b->own_stream) cudaStreamDestroy(b->stream);
  b->own_stream = false;
  b->stream = (cudaStream_t)stream;
  return DGLM_OK;
}

long dglm_batch_kernel_launches(dglm_batch *b) { return b ? b->launches : -1; }

size_t dglm_batch_device_bytes(dglm_batch *b) { return b ? b->bytes : 0; }

dglm_status dglm_batch_destroy(dglm_batch *b) {
  if (!b) return DGLM_OK;
  DeviceGuard g(b->dev);
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_batch_graphs(b);
  for (void *p : b->allocs) cudaFree(p);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return DGLM_OK;
}

}  // extern "C"
