// Persistent, warp-specialised FP64 stage kernel (included by
// dglm_stage_fp64.cu, which defines EUL/ADV, euler_flux_fast and
// dmma_8x8x4).
//
// One CTA per SM (or two, CPS = 2) walks the element tiles t = blockIdx.x,
// +gridDim.x, ... with a ring of two to four shared-memory tile buffers:
//
//   producer warps  TMA bulk copies (cp.async.bulk, mbarrier complete_tx) of
//                   the next tile's state u, RK register k, metrics, face
//                   data (and advection velocity) -- all contiguous per tile
//                   -- plus cp.async gathers of the neighbour traces
//                   u[vmapP] straight into a [v][face node][e] layout;
//   consumer warps  volume flux -> DMMA volume contraction -> face flux ->
//                   DMMA lift contraction -> LSERK epilogue with coalesced
//                   stores; then release the buffer to the producer.
//
// The stacked operator's m8n8k4 A fragments are loaded into shared memory
// once per CTA (orders whose FP64 operators do not fit read them through L1).
// Every mbarrier wait is bounded by a clock limit; on expiry the CTA sets
// flag bit 2 in the device scalars and leaves after its copies settle.
// This header is included inside namespace dglm.
#pragma once

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *b, unsigned tx) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
               "r"(tx)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_test_wait(unsigned long long *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for the completion of the phase with the given parity.  With
// the default bound the thread suspends in try_wait between checks; a
// shortened bound (dglm_set_wait_limit) polls with the non-blocking
// test_wait, so that the bound and not try_wait's own suspension time decides
// when the wait gives up
__device__ __forceinline__ bool mbar_wait(unsigned long long *b, unsigned parity,
                                          long long limit = kWaitCycles) {
  if (limit < kWaitCycles) {
    const long long t0 = clock64();
    while (!mbar_test_wait(b, parity))
      if (clock64() - t0 > limit) return false;
    return true;
  }
  if (mbar_try_wait(b, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(b, parity))
    if (clock64() - t0 > limit) return false;
  return true;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes,
                                         unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_arrive_noinc(unsigned long long *b) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(b))
               : "memory");
}
__device__ __forceinline__ void consumer_sync(int nthreads) {
  asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}
// named barrier `id` over `nthreads` threads (consumer groups of the
// ping-pong variants use ids 1 + 2g and 2 + 2g)
__device__ __forceinline__ void group_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
__device__ __forceinline__ bool group_all(bool v, int id, int nthreads) {
  unsigned r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((unsigned)v), "r"(id), "r"(nthreads)
      : "memory");
  return r != 0;
}
// AND of a predicate over the consumer threads (named barrier 2)
__device__ __forceinline__ bool consumer_all(bool v, int nthreads) {
  unsigned r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, 2, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((unsigned)v), "r"(nthreads)
      : "memory");
  return r != 0;
}

template <int PHYS, int N, int E_, int WN_, int WM_, bool ASMEM, int NG_ = 1, int PR_ = 0,
          int NB_ = 2, int PW_ = 1, int KSP_ = 1, bool FU_ = false, bool KG_ = false,
          int CPS_ = 1>
struct PCfg {
  static constexpr int NV = PHYS == EUL ? 5 : 1;
  static constexpr int Np = np_of(N), Nfp = nfp_of(N), NFF = 4 * Nfp;
  static constexpr int E = E_, EP = E_ + 1, NCOL = NV * E;
  static constexpr int MT = (Np + 7) / 8, NT = NCOL / 8;
  static constexpr int WN = WN_, WM = WM_ > MT ? MT : WM_;
  static constexpr int MGROUPS = (MT + WM - 1) / WM;
  // PR_ != 0: split-precision mma.sync contraction (see contract_m16)
  static constexpr bool M16 = PR_ != 0;
  static constexpr int KSTEP16 = PR_ == 2 ? 8 : 16;
  static constexpr int NPARTS16 = PR_ == 3 ? 3 : 2, NPROD16 = PR_ == 3 ? 6 : 3;
  static constexpr int MT16 = (Np + 15) / 16;
  static constexpr int WM16 = WM_ > MT16 ? MT16 : WM_;
  static constexpr int MG16 = (MT16 + WM16 - 1) / WM16;
  static constexpr int NG = NG_;                        // consumer groups (ping-pong)
  static constexpr int NB = NB_;                        // tile buffers in the ring
  static constexpr int PW = PW_;                        // producer warps
  // KSP > 1: each DMMA warp takes its m-group x n-block over one of KSP
  // k-chunks of each contraction and stores a partial rhs; the epilogue sums
  // the KSP partials (with all m-tiles per warp: no padded m-tiles, fewer
  // operand loads per DMMA)
  static constexpr int KSP = KSP_;
  // FUSE: face-flux rows sit below the volume rows, both flux phases run
  // back to back and one DMMA pass covers the stacked k range
  static constexpr bool FUSE = FU_;
  // KG: the RK register is not staged; the update fetches it from global
  // memory (orders whose staged tiles would not fit twice otherwise)
  static constexpr bool KG = KG_;
  // CPS: persistent CTAs per SM.  Two independent pipelines on one SM let
  // one CTA's DMMA pass run while the other computes fluxes or updates
  static constexpr int CPS = CPS_;
  static constexpr int NWC = (M16 ? MG16 : MGROUPS) * (NT / WN) * KSP;   // consumer warps per group
  static constexpr int TC = 32 * NWC;                   // consumer threads per group
  static constexpr int THREADS = NG * TC + 32 * PW;     // + producer warps
  static constexpr int KPAD = M16 ? KSTEP16 : 4;
  static constexpr int KV = 3 * Np, KVP = (KV + KPAD - 1) / KPAD * KPAD;
  static constexpr int KF = NFF, KFP = (KF + KPAD - 1) / KPAD * KPAD;
  static constexpr int KS = KVP / 4 + KFP / 4;
  static constexpr int KSV16 = KVP / KSTEP16, KSF16 = KFP / KSTEP16, KST16 = KSV16 + KSF16;
  static constexpr int SL16 = (KST16 + 7) / 8;
  // rows of the contraction operand: the DMMA path pads the row stride to
  // 8 (mod 16) doubles and flips column bit 2 on rows whose bit 1 is set
  // (bcol), so that stores of two neighbouring rows by a half-warp and the
  // m8n8k4 B-fragment loads (rows k0..k0+3) both hit 16 distinct bank pairs
  static constexpr bool SWZ = !M16;
  static constexpr int BLD = M16 ? NCOL + 4 : NCOL + (24 - NCOL % 16) % 16;
  static constexpr int BROWS = FUSE ? KVP + KFP : KVP > KFP ? KVP : KFP;
  static constexpr int FR0 = FUSE ? KVP : 0;             // first face-flux row
  // neighbour traces [v][e][UPS] with UPS = 4 (mod 8): the face-flux
  // threads take 4 elements x 4 face nodes per half-warp, whose trace reads
  // (e * UPS + fj), face-data reads (e * 4 + f) and stores to four
  // consecutive contraction rows all land on distinct bank pairs; the
  // gathers write consecutive words
  static constexpr int UPS = NFF % 8 == 4 ? NFF : NFF + 4;
  // shared memory segments, in doubles (operator A fragments when ASMEM)
  static constexpr int S_AF = !ASMEM ? 0 : M16 ? KST16 * MT16 * NPARTS16 * 64 : KS * MT * 32;
  static constexpr int S_U = NV * E * Np, S_K = KG ? 0 : NV * E * Np, S_UP = NV * E * UPS;
  static constexpr int S_GEO = 9 * E, S_FACE = 5 * 4 * E;
  static constexpr int S_VEL = PHYS == EUL ? 0 : 3 * E * Np;
  static constexpr int S_BUF = S_U + S_K + S_UP + S_GEO + S_FACE + S_VEL;
  // one rhs (partial) [v][e][IP], IP = 2 (mod 4): accumulator stores (4 rows
  // x 4 column pairs per half-warp) and the epilogue's node-contiguous reads
  // are free of bank conflicts
  static constexpr int IP = Np + (6 - Np % 4) % 4;
  static constexpr int S_R = NV * E * IP;
  static constexpr int S_B = BROWS * BLD > KSP * S_R ? BROWS * BLD : KSP * S_R;
  // barriers: full[NB], empty[NB], the operator-image barrier, padding
  static constexpr int NBAR = 2 * NB + 2 > 8 ? 2 * NB + 2 : 8;
  // node-0 fluxes of a tile's elements, per consumer group (split modes, Euler)
  static constexpr int S_CEN = (M16 && PHYS == EUL) ? kCen * E : 0;
  static constexpr int S_MISC = NBAR + NFF / 2 + 1 + 32 * NG + 8 + NG * S_CEN;  // barriers,
                                                          // Fmask, reduction, node-0 fluxes
  static constexpr size_t SMEM =
      sizeof(double) * ((size_t)S_AF + NB * S_BUF + NG * S_B + S_MISC);
  // bytes the producer's bulk copies deliver per tile
  static constexpr unsigned TX = 8u * (S_U + S_K + S_GEO + S_FACE + S_VEL);
  static_assert(NCOL % 8 == 0 && NT % WN == 0, "n-tiles must split over the warps");
  static_assert((E * Np * 8) % 16 == 0 && (E * 8) % 16 == 0, "bulk copies need 16-byte sizes");
  static_assert(SMEM <= 232448, "shared memory per CTA exceeds 227 KB");
  static_assert(CPS == 1 || (CPS == 2 && 2 * (SMEM + 1024) <= 233472 && THREADS <= 1024),
                "two CTAs per SM must share its 228 KB of shared memory");
  static_assert(NG == 1 || NG == 2, "one or two consumer groups");
  static_assert(NB >= 2 && NB <= 4 && PW >= 1 && PW <= 4, "ring of 2..4, 1..4 producers");
  static_assert(KSP == 1 || !M16, "the k-split is a DMMA path");
  static_assert(!(FUSE && M16), "the fused contraction is a DMMA path");
  static_assert(FR0 % 4 == 0, "face rows start on a k-step");
  static_assert(NWC <= 32, "per-warp wave-speed maxima fit one warp");
  static_assert(!(M16 && ASMEM), "mma.sync operator fragments are read from global memory");
  static_assert(PHYS != EUL || S_B >= 8 * E * Nfp, "wave-speed terms reuse the rhs buffer");
  static_assert(S_UP % 2 == 0, "segments after the traces stay 16-byte aligned");
  static_assert(E % 4 == 0 && NFF % 4 == 0, "face-flux threads in 4 x 4 blocks");
  __device__ static __forceinline__ int bcol(int row, int col) {
    return SWZ ? col ^ (((row >> 1) & 1) << 2) : col;
  }
};

// Producer warps of the pipelined kernels: optional one-off bulk load of an
// operator image into shared memory (abar), then per tile (ring of C::NB
// buffers) TMA bulk copies of the tile's u, k, metrics, face data (and
// advection velocity), issued by producer warp 0, and cp.async gathers of the
// neighbour traces, split over the C::PW producer warps.  full[b] completes
// once the bulk bytes have landed and all 32 * PW lanes' gathers are done.
// `limit` bounds the waits for a free buffer; the final waits for the
// producer's own copies keep kWaitCycles.
template <class C, int PHYS>
__device__ __forceinline__ void pipe_producer(const StageArgs &a, int ntiles, void *op_smem,
                                              double *sBuf0, unsigned long long *full,
                                              unsigned long long *empty,
                                              unsigned long long *abar, unsigned op_bytes,
                                              int pw, int lane, long long limit) {
  constexpr int NV = C::NV, Np = C::Np, NFF = C::NFF, E = C::E, NB = C::NB;
  const long vs = a.vs, gs = a.gstride;
  const bool lead = pw == 0 && lane == 0;
  if (op_bytes && lead) {
    mbar_arrive_expect_tx(abar, op_bytes);
    bulk_g2s(op_smem, a.AT, op_bytes, abar);
  }
  int it = 0;
  bool ok = true;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
    const int b = it % NB;
    if (it >= NB && !mbar_wait(&empty[b], ((it / NB) - 1) & 1, limit)) {
      ok = false;
      break;
    }
    const long e0 = (long)t * E;
    const int ne = (int)min((long)E, (long)a.K - e0);
    double *B = sBuf0 + b * C::S_BUF;
    double *bU = B, *bK = bU + C::S_U, *bUP = bK + C::S_K, *bG = bUP + C::S_UP;
    double *bF = bG + C::S_GEO, *bV = bF + C::S_FACE;
    if (lead) {
      mbar_arrive_expect_tx(&full[b], C::TX);
      for (int v = 0; v < NV; v++) {
        bulk_g2s(bU + v * E * Np, a.u_in + v * vs + e0 * Np, 8u * E * Np, &full[b]);
        if (C::S_K)   // configurations that fetch k in the update stage none
          bulk_g2s(bK + v * E * Np, a.kreg + v * vs + e0 * Np, 8u * E * Np, &full[b]);
      }
      for (int m = 0; m < 9; m++) bulk_g2s(bG + m * E, a.geo + m * gs + e0, 8u * E, &full[b]);
      for (int q = 0; q < 3; q++)
        bulk_g2s(bF + q * 4 * E, a.nrm + q * 4 * gs + 4 * e0, 32u * E, &full[b]);
      bulk_g2s(bF + 3 * 4 * E, a.fscale + 4 * e0, 32u * E, &full[b]);
      bulk_g2s(bF + 4 * 4 * E, a.tau + 4 * e0, 32u * E, &full[b]);
      if (PHYS != EUL)
        for (int q = 0; q < 3; q++)
          bulk_g2s(bV + q * E * Np, a.vel + q * vs + e0 * Np, 8u * E * Np, &full[b]);
    }
    // neighbour traces u+ = u[vmapP] into [v][e][UPS]: all of this lane's
    // vmapP loads (or compact face-map lookups) are issued first, so their
    // latency is paid once
    constexpr int PT = 32 * C::PW;
    constexpr int GPL = (E * NFF + PT - 1) / PT;
    int vmr[GPL];
    if (a.etoe) {
#pragma unroll
      for (int j = 0; j < GPL; j++) {
        const int idx = 32 * pw + lane + PT * j;
        vmr[j] = idx < ne * NFF ? compact_neighbour_node<Np, C::Nfp>(a, e0, idx) : -1;
      }
    } else {
#pragma unroll
      for (int j = 0; j < GPL; j++) {
        const int idx = 32 * pw + lane + PT * j;
        vmr[j] = idx < ne * NFF ? __ldg(a.vmapP + e0 * NFF + idx) : -1;
      }
    }
#pragma unroll
    for (int j = 0; j < GPL; j++) {
      const int idx = 32 * pw + lane + PT * j;
      if (vmr[j] >= 0) {
        const int e = idx / NFF, fj = idx - e * NFF;
#pragma unroll
        for (int v = 0; v < NV; v++)
          cp_async8(bUP + (v * E + e) * C::UPS + fj, a.u_in + v * vs + vmr[j]);
      }
    }
    cp_async_arrive_noinc(&full[b]);
  }
  if (!ok) atomicOr(&a.sc->flags, 4);
  // let the copies of the last NB tiles settle before this warp leaves
  for (int j = (it > NB ? it - NB : 0); j < it; j++) mbar_wait(&full[j % NB], (j / NB) & 1);
  if (op_bytes) mbar_wait(abar, 0);
  asm volatile("cp.async.wait_all;" ::: "memory");
}

template <int PHYS, int N, int E_, int WN_, int WM_, bool ASMEM, int NG_, int PR_, int NB_,
          int PW_, int KSP_, bool FU_, bool KG_, int CPS_>
__global__ void __launch_bounds__(
    PCfg<PHYS, N, E_, WN_, WM_, ASMEM, NG_, PR_, NB_, PW_, KSP_, FU_, KG_, CPS_>::THREADS, CPS_)
    stage_pipe_kernel(const StageArgs a, int ntiles) {
  using C = PCfg<PHYS, N, E_, WN_, WM_, ASMEM, NG_, PR_, NB_, PW_, KSP_, FU_, KG_, CPS_>;
  constexpr int NV = C::NV, Np = C::Np, Nfp = C::Nfp, NFF = C::NFF, E = C::E,
                BLD = C::BLD, TC = C::TC;
  extern __shared__ __align__(16) double smem[];
  double *sAF = smem;
  double *sBuf0 = sAF + C::S_AF;
  double *sB0 = sBuf0 + C::NB * C::S_BUF;   // one working buffer per consumer group
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(sB0 + C::NG * C::S_B);
  unsigned long long *full = bars, *empty = bars + C::NB, *abar = bars + 2 * C::NB;
  int *sFm = reinterpret_cast<int *>(bars + C::NBAR);
  unsigned long long *sMax = reinterpret_cast<unsigned long long *>(sFm + NFF + (NFF & 1));

  const int ttid = threadIdx.x, twarp = ttid >> 5, lane = ttid & 31;
  const long vs = a.vs;

  if (ttid == 0) {
    for (int b = 0; b < C::NB; b++) {
      mbar_init(&full[b], 1 + 32 * C::PW);
      mbar_init(&empty[b], C::NWC);
    }
    mbar_init(abar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = ttid; i < NFF; i += C::THREADS) sFm[i] = a.Fmask[i];
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();

  auto buf = [&](int b) { return sBuf0 + b * C::S_BUF; };

  // ------------------------------------------------------------- producer
  if (twarp >= C::NG * C::NWC) {
    pipe_producer<C, PHYS>(a, ntiles, sAF, sBuf0, full, empty, abar, 8u * C::S_AF,
                           twarp - C::NG * C::NWC, lane, a.wait_cycles);
    return;
  }

  // ------------------------------------------------------------ consumers
  // Group g takes the CTA's tiles it = g, g + NG, ... from buffer it % NB;
  // with two groups one group's tensor-core phase overlaps the other's flux
  // and epilogue phases, and a ring deeper than two lets the producers fill
  // the next tile while both groups hold theirs.
  const int grp = twarp / C::NWC;
  const int warp = twarp - grp * C::NWC, tid = ttid - grp * TC;
  const int bar_sync = 1 + 2 * grp, bar_and = 2 + 2 * grp;
  double *sB = sB0 + grp * C::S_B;
  double *sCen = reinterpret_cast<double *>(sMax + 32 * C::NG) + grp * C::S_CEN;
  auto consumer_sync = [&](int n) { group_sync(bar_sync, n); };
  auto consumer_all = [&](bool v, int n) { return group_all(v, bar_and, n); };
  double acc[C::M16 ? 1 : C::WM][C::M16 ? 1 : C::WN][2];
  constexpr int QM = C::M16 ? C::WM16 : 1, QN = C::M16 ? C::WN : 1;
  float acc16[QM][QN][4];
  double tot16[QM][QN][4];
  const double dt = a.dt_override >= 0 ? a.dt_override : a.sc->dt;
  unsigned long long vmax = 0ull;
  bool ok = true;
  if (ASMEM) ok = consumer_all(mbar_wait(abar, 0, a.wait_cycles), TC);
  const double *Afrag = ASMEM ? sAF : a.AT;
  // DMMA warp roles: m-group, n-block and k-chunk.  With WN = NT a warp
  // feeds each operator fragment it loads to all n-tiles of the tile (the
  // fragments come from global memory for the orders whose operator does
  // not fit in shared memory)
  constexpr int NBLK = C::NT / C::WN;
  const int mg = warp % C::MGROUPS;
  const int ng = (warp / C::MGROUPS) % NBLK;
  const int kc = warp / (C::MGROUPS * NBLK);
  const int m0 = mg * C::WM, n0 = ng * C::WN;
  // acc += A[:, k-steps of this warp's chunk of [0, nks)] x sB rows; the A
  // fragments of k-step ks start at Afrag + a_off + ks * MT * 32
  auto dmma_phase = [&](long a_off, int nks) {
    const int kchunk = (nks + C::KSP - 1) / C::KSP;
    const int kb = kc * kchunk, ke = min(kb + kchunk, nks);
    const double *Ab = Afrag + a_off + (long)m0 * 32 + lane;
    // row k0 + (lane & 3) with k0 % 4 == 0: the swizzle bit is lane bit 1
    const double *Bb = sB + (lane & 3) * BLD + n0 * 8 + C::bcol(lane & 3, lane >> 2);
#pragma unroll 2
    for (int ks = kb; ks < ke; ks++) {
      double av[C::WM], bv[C::WN];
#pragma unroll
      for (int i = 0; i < C::WM; i++)
        av[i] = (m0 + i < C::MT) ? Ab[((long)ks * C::MT + i) * 32] : 0.0;
#pragma unroll
      for (int j = 0; j < C::WN; j++) bv[j] = Bb[ks * 4 * BLD + j * 8];
#pragma unroll
      for (int i = 0; i < C::WM; i++)
        if (m0 + i < C::MT)   // warp-uniform: m-tiles past MT are skipped
#pragma unroll
          for (int j = 0; j < C::WN; j++) dmma_8x8x4(acc[i][j], av[i], bv[j]);
    }
  };
  // phase bodies shared by the tile orders below
  // volume fluxes of the tile in ring buffer B -> operand rows [0, 3Np)
  auto vol_flux = [&](double *B) {
    const double *bU = B, *bG = B + C::S_U + C::S_K + C::S_UP;
    const double *bV = bG + C::S_GEO + C::S_FACE;
    for (int itm = tid; itm < E * Np; itm += TC) {
      const int i = itm / E, e = itm - i * E;
      const double *g = bG + e;
      const double rx = g[0], ry = g[E], rz = g[2 * E], sx = g[3 * E], sy = g[4 * E],
                   sz = g[5 * E], tx = g[6 * E], ty = g[7 * E], tz = g[8 * E];
      if (PHYS == EUL) {
        double q[5], F[5], Gf[5], W[5];
#pragma unroll
        for (int v = 0; v < 5; v++) q[v] = bU[v * E * Np + e * Np + i];
        euler_flux_fast(a.gamma, q, F, Gf, W);
        if constexpr (C::M16) centre_sub(sCen + e * kCen, F, Gf, W);
#pragma unroll
        for (int v = 0; v < 5; v++) {
          const int col = v * E + e, r0 = i, r1 = Np + i, r2 = 2 * Np + i;
          sB[r0 * BLD + C::bcol(r0, col)] = rx * F[v] + ry * Gf[v] + rz * W[v];
          sB[r1 * BLD + C::bcol(r1, col)] = sx * F[v] + sy * Gf[v] + sz * W[v];
          sB[r2 * BLD + C::bcol(r2, col)] = tx * F[v] + ty * Gf[v] + tz * W[v];
        }
      } else {
        const double uu = bU[e * Np + i];
        const double F = bV[e * Np + i] * uu, Gf = bV[E * Np + e * Np + i] * uu,
                     W = bV[2 * E * Np + e * Np + i] * uu;
        const int r0 = i, r1 = Np + i, r2 = 2 * Np + i;
        sB[r0 * BLD + C::bcol(r0, e)] = rx * F + ry * Gf + rz * W;
        sB[r1 * BLD + C::bcol(r1, e)] = sx * F + sy * Gf + sz * W;
        sB[r2 * BLD + C::bcol(r2, e)] = tx * F + ty * Gf + tz * W;
      }
    }
    for (int g = tid; g < (C::KVP - C::KV) * BLD; g += TC) sB[C::KV * BLD + g] = 0.0;

  };
  // face fluxes of the tile in ring buffer B -> operand rows [FR0, FR0 + NFF)
  auto face_flux = [&](double *B) {
    const double *bU = B, *bUP = B + C::S_U + C::S_K, *bF = bUP + C::S_UP + C::S_GEO;
    const double *bV = bF + C::S_FACE;
    for (int itm = tid; itm < E * NFF; itm += TC) {
      // 4 x 4 blocks of (element, face node), element blocks fastest
      const int blk = itm >> 4, eb = blk % (E / 4), fb = blk / (E / 4);
      const int e = eb * 4 + (itm & 3), fj = fb * 4 + ((itm >> 2) & 3), f = fj / Nfp;
      const int nodeM = sFm[fj];
      // face arrays arrive in their global order: [array][e][f]
      const double nx = bF[0 * 4 * E + e * 4 + f], ny = bF[1 * 4 * E + e * 4 + f],
                   nz = bF[2 * 4 * E + e * 4 + f], fs = bF[3 * 4 * E + e * 4 + f],
                   tau = bF[4 * 4 * E + e * 4 + f];
      if (PHYS == EUL) {
        double qm[5], qb[5], F[5], Gf[5], W[5];
#pragma unroll
        for (int v = 0; v < 5; v++) {
          qm[v] = bU[v * E * Np + e * Np + nodeM];
          qb[v] = 0.5 * (qm[v] + bUP[(v * E + e) * C::UPS + fj]);
        }
        euler_flux_fast(a.gamma, qb, F, Gf, W);
        if constexpr (C::M16) centre_sub(sCen + e * kCen, F, Gf, W);
#pragma unroll
        for (int v = 0; v < 5; v++) {
          const double nd = nx * F[v] + ny * Gf[v] + nz * W[v];
          const int r = C::FR0 + fj;
          sB[r * BLD + C::bcol(r, v * E + e)] = (nd - tau * (qb[v] - qm[v])) * fs;
        }
      } else {
        const double um = bU[e * Np + nodeM];
        const double ub = 0.5 * (um + bUP[e * C::UPS + fj]);
        const double F = bV[e * Np + nodeM] * ub, Gf = bV[E * Np + e * Np + nodeM] * ub,
                     W = bV[2 * E * Np + e * Np + nodeM] * ub;
        const double nd = nx * F + ny * Gf + nz * W;
        const int r = C::FR0 + fj;
        sB[r * BLD + C::bcol(r, e)] = (nd - tau * (ub - um)) * fs;
      }
    }
    for (int g = tid; g < (C::KFP - C::KF) * BLD; g += TC)
      sB[(C::FR0 + C::KF) * BLD + g] = 0.0;
  };
  // this warp's accumulators -> partial sums at sRb ([kc][v][e][IP])
  auto store_partials = [&](double *sRb) {
    if constexpr (C::M16) {
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
            if (i < Np) sRb[(v * E + e) * C::IP + i] = tot16[ii][jj][c];
          }
      }
    } else {
      double *sR = sRb + kc * C::S_R;   // this warp's k-chunk partial
#pragma unroll
      for (int ii = 0; ii < C::WM; ii++) {
        const int i = (m0 + ii) * 8 + (lane >> 2);
        if (i < Np) {
#pragma unroll
          for (int jj = 0; jj < C::WN; jj++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const int col = (n0 + jj) * 8 + (lane & 3) * 2 + h;
              const int v = col / E, e = col - v * E;
              sR[(v * E + e) * C::IP + i] = acc[ii][jj][h];
            }
        }
      }
    }
  };
  // LSERK update of the tile in ring buffer B (elements e0.., ne of them)
  // from the partial sums at sRb, then the fused wave speed on the last
  // stage (scratch at sRb)
  auto update = [&](double *B, long e0, int ne, double *sRb) {
    double *bU = B;
    const double *bK = B + C::S_U, *bF = B + C::S_U + C::S_K + C::S_UP + C::S_GEO;
    // the new state goes back to shared memory only for the fused wave speed
    const bool keep_u = PHYS == EUL && a.last_stage && !a.rhs_only;
    // one flat loop over (variable, node): every thread has independent
    // updates in flight.  nep = ne * Np is passed as a literal for full tiles
    // (ne == E), so the index divisions become multiplications.
    auto item = [&](int vg, double kold, const int nep) {
      const int v = vg / nep, g = vg - v * nep;
      const int e = g / Np, i = g - e * Np;
      const long gi = v * vs + e0 * Np + g;
      const int ri = (v * E + e) * C::IP + i;
      double rhs = sRb[ri];
#pragma unroll
      for (int c = 1; c < C::KSP; c++) rhs += sRb[c * C::S_R + ri];
      if (a.rhs_only) {
        a.u_out[gi] = rhs;
      } else {
        const double kn = a.rka * kold + dt * rhs;
        const double un = bU[v * E * Np + g] + a.rkb * kn;
        a.kreg[gi] = kn;
        a.u_out[gi] = un;
        if (keep_u) bU[v * E * Np + g] = un;
      }
    };
    auto items = [&](const int nep) {
      const int tot = NV * nep;
      if constexpr (C::KG) {
        // every k of this thread is requested before the first is used
        constexpr int IPT = (NV * E * Np + TC - 1) / TC;
        double kr[IPT];
#pragma unroll
        for (int q = 0; q < IPT; q++) {
          const int vg = tid + q * TC;
          kr[q] = 0.0;
          if (vg < tot && !a.rhs_only) kr[q] = a.kreg[(vg / nep) * vs + e0 * Np + vg % nep];
        }
#pragma unroll
        for (int q = 0; q < IPT; q++)
          if (tid + q * TC < tot) item(tid + q * TC, kr[q], nep);
      } else {
        for (int vg = tid; vg < tot; vg += TC) {
          const int v = vg / nep, g = vg - v * nep;
          item(vg, C::S_K ? bK[v * E * Np + g] : 0.0, nep);
        }
      }
    };
    if (ne == E)
      items(E * Np);
    else
      items(ne * Np);
    if (PHYS == EUL && a.last_stage && !a.rhs_only) {
      consumer_sync(TC);
      // fused calc_maxv on the new state
      // |v|^2 and c^2 at every face node in parallel (into the rhs staging
      // buffer, free by now), then the per-face max
      double *sW = sRb;
      for (int it = tid; it < 4 * E * Nfp; it += TC) {
        const int fe = it / Nfp, j = it - fe * Nfp, f = fe / E, e = fe - f * E;
        double v2 = 0.0, c2 = 0.0;
        if (e < ne) {
          const int nd = e * Np + sFm[f * Nfp + j];
          const double u1 = bU[nd], u2 = bU[E * Np + nd], u3 = bU[2 * E * Np + nd],
                       u4 = bU[3 * E * Np + nd], u5 = bU[4 * E * Np + nd];
          // as in face_maxv_kernel, so dt does not depend on which kernel
          // computed maxv (a restarted run repeats the original bit for bit)
          node_speeds(a.gamma, u1, u2, u3, u4, u5, v2, c2);
        }
        sW[2 * it] = v2;
        sW[2 * it + 1] = c2;
      }
      consumer_sync(TC);
      for (int itm = tid; itm < 4 * E; itm += TC) {
        const int f = itm / E, e = itm - f * E;
        if (e >= ne) continue;
        double mv2 = 0.0, mc2 = 0.0;
        bool bad = false;
        for (int j = 0; j < Nfp; j++) {
          const double v2 = sW[2 * (itm * Nfp + j)], c2 = sW[2 * (itm * Nfp + j) + 1];
          mv2 = v2 > mv2 ? v2 : mv2;
          mc2 = c2 > mc2 ? c2 : mc2;
          bad |= (v2 != v2) || (c2 != c2);
        }
        double mv = sqrt(mv2) + sqrt(mc2);
        if (bad) mv = __longlong_as_double(0x7ff8000000000000LL);
        a.maxv[(e0 + e) * 4 + f] = mv;
        const unsigned long long bits = dbits(mv * bF[3 * 4 * E + e * 4 + f]);
        vmax = bits > vmax ? bits : vmax;
      }
    }
  };
  int it = grp;
  for (int t = blockIdx.x + grp * gridDim.x; ok && t < ntiles; t += C::NG * gridDim.x, it += C::NG) {
    const int b = it % C::NB;
    if (!consumer_all(mbar_wait(&full[b], (it / C::NB) & 1, a.wait_cycles), TC)) {
      ok = false;
      break;
    }
    const long e0 = (long)t * E;
    const int ne = (int)min((long)E, (long)a.K - e0);
    double *B = buf(b);
    if constexpr (C::M16 && PHYS == EUL) {
      // the previous tile's face fluxes, the last readers, are past a barrier
      node0_fluxes(a.gamma, B, Np, E * Np, E, tid, TC, sCen);
      consumer_sync(TC);
    }
    vol_flux(B);

    // 2. volume contraction (FUSE: part of the one pass after the face fluxes)
    if constexpr (!C::FUSE) consumer_sync(TC);
    if constexpr (C::FUSE) {
    } else if constexpr (C::M16) {
#pragma unroll
      for (int i = 0; i < QM; i++)
#pragma unroll
        for (int j = 0; j < QN; j++)
#pragma unroll
          for (int c = 0; c < 4; c++) {
            acc16[i][j][c] = 0.f;
            tot16[i][j][c] = 0.0;
          }
      contract_m16<C, PR_>(reinterpret_cast<const uint4 *>(a.AT), 0, C::KSV16, sB, acc16,
                           tot16, warp, lane);
    } else {
#pragma unroll
      for (int i = 0; i < C::WM; i++)
#pragma unroll
        for (int j = 0; j < C::WN; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
      dmma_phase(0, C::KVP / 4);
    }
    if constexpr (!C::FUSE) consumer_sync(TC);

    face_flux(B);
    consumer_sync(TC);

    // 4. lift contraction (FUSE: the whole stacked contraction)
    if constexpr (C::FUSE) {
#pragma unroll
      for (int i = 0; i < C::WM; i++)
#pragma unroll
        for (int j = 0; j < C::WN; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
      dmma_phase(0, C::KVP / 4 + C::KFP / 4);
    } else if constexpr (C::M16) {
      contract_m16<C, PR_>(reinterpret_cast<const uint4 *>(a.AT), C::KSV16, C::KSF16, sB,
                           acc16, tot16, warp, lane);
    } else {
      dmma_phase((long)(C::KVP / 4) * C::MT * 32, C::KFP / 4);
    }
    consumer_sync(TC);

    store_partials(sB);
    consumer_sync(TC);
    update(B, e0, ne, sB);
    // release the buffer (generic-proxy writes into it precede the next TMA)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[b]);
  }
  if (!ok && tid == 0) atomicOr(&a.sc->flags, 4);
  if (PHYS == EUL && a.last_stage && !a.rhs_only) {
    vmax = warp_max_bits(vmax);
    if (lane == 0) sMax[grp * 32 + warp] = vmax;
    consumer_sync(TC);
    if (tid < 32) {
      unsigned long long v = tid < C::NWC ? sMax[grp * 32 + tid] : 0ull;
      v = warp_max_bits(v);
      if (tid == 0) atomicMax(&a.sc->acc[a.sc->parity ^ 1], v);
    }
  }
}
