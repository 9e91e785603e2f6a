// Mixed-precision stage kernel on the 5th-generation tensor cores (included
// by dglm_stage_fp64.cu after dglm_stage_pipe.cuh, inside namespace dglm).
//
// Same persistent, TMA-fed pipeline as stage_pipe_kernel; only the two
// contractions change.  The volume block ([WDr WDs WDt] x [fluxR; fluxS;
// fluxT]) and the lift block (-LIFT x fluxLM) run as tcgen05.mma with
//   D[m][n] += A[m][k] * B[n][k],   m = (variable, element), n = output node,
// A = the tile's fluxes, B = the operator, both K-major in shared memory in
// the no-swizzle core-matrix layout (8 rows x 16 bytes), the accumulator D
// (FP32) in tensor memory.  Every FP64 operand x is split as x = hi + lo
// (hi = x rounded to TF32 or BF16, lo = the rounding error rounded again) and
// the product is taken in three passes, hi*hi + hi*lo + lo*hi, accumulating
// in FP32.  Fluxes, the LSERK state and update, metrics and face data stay
// FP64; only the contraction operands and its accumulator are reduced.
// Euler fluxes are centred before the split (each element's node-0 flux,
// formed once per tile by node0_fluxes, subtracted; the right-hand side is
// unchanged), so the split parts carry only the within-element variation.
//
// Per tile: flux phase writes the volume operand -> one thread issues the
// volume MMAs and commits to an mbarrier -> once they have read the operand
// the face phase overwrites it with the lift operand -> lift MMAs -> the
// accumulator is read back with tcgen05.ld into the FP64 epilogue.  The MMAs
// of a tile go round-robin to NACC tensor-memory accumulators, so
// consecutive MMAs do not wait on each other and each FP32 running sum
// covers only 1/NACC of the terms; the partials are added on read-back.
#pragma once

#include <cuda_bf16.h>

enum { PREC_BF16 = 1, PREC_TF32 = 2, PREC_BF16X6 = 3 };

// ---- tcgen05 / TMEM helpers ------------------------------------------------
__device__ __forceinline__ void tmem_alloc(unsigned *dst_smem, unsigned ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_commit(unsigned long long *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
template <int PREC>
__device__ __forceinline__ void tc_mma(unsigned dtmem, unsigned long long adesc,
                                       unsigned long long bdesc, unsigned idesc, int accum) {
  if (PREC == PREC_TF32)
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
  else
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
}
// 32 lanes x 8 columns of 32-bit accumulator per warp
__device__ __forceinline__ void tmem_ld8(unsigned taddr, float (&r)[8]) {
  unsigned v[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7])
      : "r"(taddr)
      : "memory");
  for (int i = 0; i < 8; i++) r[i] = __uint_as_float(v[i]);
}
__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// shared-memory matrix descriptor: K-major, no swizzle, core matrices of 8
// rows x 16 bytes; lbo = byte step between the two K core matrices of one
// MMA, sbo = byte step between 8-row groups; version field 1 (sm_100)
__device__ __forceinline__ unsigned long long smem_desc(unsigned saddr, unsigned lbo,
                                                        unsigned sbo) {
  return (unsigned long long)((saddr >> 4) & 0x3FFFu) |
         ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// x = hi + lo with hi, lo in the operand format (stored as raw bits).  The
// split runs on the FP32 value of x (one conversion from FP64): hi carries
// 11 (TF32) or 8 (BF16) significant bits and lo the next ones, so the FP32
// rounding of x (2^-24) is below what the pair keeps.
__device__ __forceinline__ void split_tf32(double x, unsigned &hi, unsigned &lo) {
  const float f = (float)x;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(f));
  const float r = f - __uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}
__device__ __forceinline__ void split_bf16(double x, unsigned short &hi, unsigned short &lo) {
  const float f = (float)x;
  const __nv_bfloat16 h = __float2bfloat16_rn(f);
  const __nv_bfloat16 l = __float2bfloat16_rn(f - __bfloat162float(h));
  hi = __bfloat16_as_ushort(h);
  lo = __bfloat16_as_ushort(l);
}

// x = b0 + b1 + b2 in BF16 (24 significant bits of the FP32 value of x)
__device__ __forceinline__ void split_bf16x3(double x, unsigned short (&p)[3]) {
  const float f = (float)x;
  const __nv_bfloat16 b0 = __float2bfloat16_rn(f);
  const float r1 = f - __bfloat162float(b0);
  const __nv_bfloat16 b1 = __float2bfloat16_rn(r1);
  const __nv_bfloat16 b2 = __float2bfloat16_rn(r1 - __bfloat162float(b1));
  p[0] = __bfloat16_as_ushort(b0);
  p[1] = __bfloat16_as_ushort(b1);
  p[2] = __bfloat16_as_ushort(b2);
}

template <int PHYS, int N, int E_, int PREC, int NWC_ = 8, int PW_ = 1>
struct MCfg {
  static constexpr int NV = PHYS == EUL ? 5 : 1;
  static constexpr int NB = 2, PW = PW_;   // tile ring and producer warps (pipe_producer)
  static constexpr int Np = np_of(N), Nfp = nfp_of(N), NFF = 4 * Nfp;
  static constexpr int E = E_, EP = E_ + 1, NCOL = NV * E;
  static constexpr int M = NCOL <= 64 ? 64 : 128;            // MMA rows
  // rows stored per operand image: the MMA reads M rows, but rows past NCOL
  // only feed accumulator rows that are never read back, so an image keeps
  // its NCOL rows (in 8-row groups) and the MMA's reads of the rest land in
  // the next image or the FP64 buffers behind it (any bit pattern will do)
  static constexpr int MA = (NCOL + 7) / 8 * 8;
  static constexpr int NPAD = M == 64 ? (Np + 7) / 8 * 8 : (Np + 15) / 16 * 16;   // MMA N
  // NACC accumulators, each summing the terms of a slice of K in FP32; the
  // slices are added in FP64 when the tile is read back
  static constexpr int S = PREC == PREC_TF32 ? 4 : 2;         // operand bytes
  // operands split into NPARTS parts; NPROD part products per k-step:
  // two parts -> a1 b0 + a0 b1 + a0 b0; three parts -> the six products
  // with part indices summing to at most 2
  static constexpr int NPARTS = PREC == PREC_BF16X6 ? 3 : 2;
  static constexpr int NPROD = PREC == PREC_BF16X6 ? 6 : 3;
  static constexpr int T = 16 / S;                              // elements per core row
  static constexpr int KSTEP = 32 / S;                          // K per MMA
  static constexpr int KV = 3 * Np, KVA = (KV + KSTEP - 1) / KSTEP * KSTEP;
  static constexpr int KF = NFF, KFA = (KF + KSTEP - 1) / KSTEP * KSTEP;
  static constexpr int KAM = KVA > KFA ? KVA : KFA;
  static constexpr int KSV = KVA / KSTEP, KSF = KFA / KSTEP, KST = KSV + KSF;   // k-steps
  // every accumulator receives at least one k-step, and they fit in 512 columns
  static constexpr int NACC0 = NPAD * 8 <= 512 ? 8 : NPAD * 4 <= 512 ? 4 : 2;
  static constexpr int NACC = NACC0 < KST ? NACC0 : KST;
  // MMA issuers: lane 0 of warps 0..NISS-1, issuer w owns accumulators j with
  // j % NISS == w (one thread's tcgen05.mma issue rate bounds tiny MMAs)
  static constexpr int NISS = NACC % 4 == 0 ? 4 : NACC % 2 == 0 ? 2 : 1;
  static constexpr int TCOLS = NACC * NPAD <= 32 ? 32 : NACC * NPAD <= 64 ? 64
                               : NACC * NPAD <= 128 ? 128 : NACC * NPAD <= 256 ? 256 : 512;
  static constexpr int SBO_A = KAM / T * 128, SBO_BV = KVA / T * 128, SBO_BF = KFA / T * 128;
  // byte sizes
  static constexpr int BV_BYTES = NPAD * KVA * S, BF_BYTES = NPAD * KFA * S;
  static constexpr int BIMG = NPARTS * (BV_BYTES + BF_BYTES);   // part 0, part 1, ...
  static constexpr int NWC = NWC_, TC = 32 * NWC, THREADS = TC + 32 * PW;
  // FP64 pipeline buffers (as in PCfg)
  // neighbour traces [v][e][UPS], written by pipe_producer (conflict-free
  // gathers and face-flux reads)
  static constexpr int UPS = E >= 16 ? NFF + 1 : NFF + 2;
  static constexpr int S_U = NV * E * Np, S_K = NV * E * Np, S_UP = NV * E * UPS;
  static constexpr int S_GEO = 9 * E, S_FACE = 5 * 4 * E;
  static constexpr int S_VEL = PHYS == EUL ? 0 : 3 * E * Np;
  static constexpr int S_BUF = S_U + S_K + S_UP + S_GEO + S_FACE + S_VEL;
  static constexpr int S_R = NV * Np * EP;
  // + barriers, tensor-memory address, Fmask, maxima, node-0 fluxes [E][15] (Euler)
  static constexpr int S_CEN = PHYS == EUL ? kCen * E : 0;
  static constexpr size_t FP64_BYTES =
      sizeof(double) * (2 * (size_t)S_BUF + S_R + S_CEN) + 1024;
  // separate volume and lift operands let the face phase overlap the volume
  // MMAs; used where they fit next to the rest
  static constexpr bool SEPL =
      (size_t)BIMG + (size_t)NPARTS * MA * (KVA + KFA) * S + FP64_BYTES <= 232448;
  static constexpr int AV_BYTES = MA * (SEPL ? KVA : KAM) * S;  // one part, volume (or shared)
  static constexpr int AF_BYTES = SEPL ? MA * KFA * S : 0;      // one part, lift
  static constexpr int SBO_AV = (SEPL ? KVA : KAM) / T * 128, SBO_AF = (SEPL ? KFA : KAM) / T * 128;
  static constexpr int A_BYTES = AV_BYTES + AF_BYTES;           // one part
  static constexpr size_t SMEM = (size_t)BIMG + (size_t)NPARTS * A_BYTES + FP64_BYTES;
  static constexpr unsigned TX = 8u * (S_U + S_K + S_GEO + S_FACE + S_VEL);
  // instruction descriptor: F32 accumulate, A/B format, K-major A and B, N, M
  static constexpr unsigned IDESC = (1u << 4) | ((PREC == PREC_TF32 ? 2u : 1u) << 7) |
                                    ((PREC == PREC_TF32 ? 2u : 1u) << 10) |
                                    ((unsigned)(NPAD >> 3) << 17) | ((unsigned)(M >> 4) << 24);
  static_assert(NCOL <= 128, "one MMA tile covers at most 128 columns");
  static_assert(BIMG % 16 == 0 && AV_BYTES % 16 == 0 && AF_BYTES % 16 == 0,
                "16-byte operand images");
  static_assert(SMEM <= 232448, "shared memory per CTA exceeds 227 KB");
  static_assert(NPAD <= 256, "MMA N limit");
  static_assert(NACC * NPAD <= 512, "tensor memory has 512 columns");
  static_assert(NWC >= NISS && NACC % NISS == 0, "issuers split the accumulators evenly");
  static_assert(PHYS != EUL || S_R >= 8 * E * Nfp, "wave-speed terms reuse the rhs buffer");
  static_assert(SMEM < (1u << 18), "descriptor start addresses must fit 14 bits (>> 4)");
  // the MMA's reads of rows [MA, M) of the last image stay inside the CTA's
  // shared memory (the FP64 buffers follow the operand images)
  static_assert((size_t)(M - MA) / 8 * (KAM > KVA ? KAM : KVA) / T * 128 <= FP64_BYTES,
                "reads past the last operand image stay in shared memory");
};

// byte offset of element (r, k) in a K-major core-matrix image with 8-row
// group stride sbo
template <class C>
__device__ __forceinline__ int core_off(int r, int k, int sbo) {
  return (r >> 3) * sbo + (k / C::T) * 128 + (r & 7) * 16 + (k % C::T) * C::S;
}

// operand element (r, k) split into its parts; part p of the image starts
// at A + p * C::A_BYTES, the row-group stride is sbo
template <class C, int PREC>
__device__ __forceinline__ void put_split(unsigned char *A, int r, int k, int sbo, double x) {
  const int off = core_off<C>(r, k, sbo);
  if (PREC == PREC_TF32) {
    unsigned h, l;
    split_tf32(x, h, l);
    *reinterpret_cast<unsigned *>(A + off) = h;
    *reinterpret_cast<unsigned *>(A + C::A_BYTES + off) = l;
  } else if (PREC == PREC_BF16) {
    unsigned short h, l;
    split_bf16(x, h, l);
    *reinterpret_cast<unsigned short *>(A + off) = h;
    *reinterpret_cast<unsigned short *>(A + C::A_BYTES + off) = l;
  } else {
    unsigned short p[3];
    split_bf16x3(x, p);
#pragma unroll
    for (int q = 0; q < 3; q++)
      *reinterpret_cast<unsigned short *>(A + q * C::A_BYTES + off) = p[q];
  }
}

// part indices (a, b) of product q of a k-step
template <class C>
__device__ __forceinline__ void prod_parts(int q, int &pa, int &pb) {
  if (C::NPARTS == 2) {
    pa = q == 0 ? 1 : 0;
    pb = q == 1 ? 1 : 0;
  } else {
    constexpr int A6[6] = {2, 1, 0, 1, 0, 0}, B6[6] = {0, 1, 2, 0, 1, 0};
    pa = A6[q];
    pb = B6[q];
  }
}

template <int PHYS, int N, int E_, int PREC, int NWC_, int PW_>
__global__ void __launch_bounds__(MCfg<PHYS, N, E_, PREC, NWC_, PW_>::THREADS, 1)
    stage_mixed_kernel(const StageArgs a, int ntiles) {
  using C = MCfg<PHYS, N, E_, PREC, NWC_, PW_>;
  constexpr int NV = C::NV, Np = C::Np, Nfp = C::Nfp, NFF = C::NFF, E = C::E, EP = C::EP,
                TC = C::TC;
  extern __shared__ __align__(16) double smem[];
  // [operator parts][operand parts: volume (or shared) + lift][FP64 buffers]
  unsigned char *sBimg = reinterpret_cast<unsigned char *>(smem);
  unsigned char *sA = sBimg + C::BIMG;                       // part p at p * A_BYTES
  double *sBuf0 = reinterpret_cast<double *>(sA + C::NPARTS * C::A_BYTES);
  double *sR = sBuf0 + 2 * C::S_BUF;
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(sR + C::S_R);
  unsigned long long *full = bars, *empty = bars + 2, *abar = bars + 4, *mbar = bars + 5;
  unsigned *sTmem = reinterpret_cast<unsigned *>(bars + 6);
  int *sFm = reinterpret_cast<int *>(bars + 8);
  unsigned long long *sMax = reinterpret_cast<unsigned long long *>(sFm + NFF + (NFF & 1));
  double *sCen = reinterpret_cast<double *>(sMax + 32);   // [E][15] node-0 fluxes

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long vs = a.vs;

  if (tid == 0) {
    mbar_init(&full[0], 1 + 32 * C::PW);
    mbar_init(&full[1], 1 + 32 * C::PW);
    mbar_init(&empty[0], C::NWC);
    mbar_init(&empty[1], C::NWC);
    mbar_init(abar, 1);
    mbar_init(mbar, C::NISS);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < NFF; i += C::THREADS) sFm[i] = a.Fmask[i];
  // zero every operand part once: its K padding columns stay zero (rows past
  // NCOL are not stored, see MCfg::MA)
  for (int i = tid; i < C::NPARTS * C::A_BYTES / 16; i += C::THREADS)
    reinterpret_cast<uint4 *>(sA)[i] = make_uint4(0, 0, 0, 0);
  if (warp == 0) tmem_alloc(sTmem, C::TCOLS);
  tc_fence_before();
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *sTmem;

  if (warp >= C::NWC) {
    pipe_producer<C, PHYS>(a, ntiles, sBimg, sBuf0, full, empty, abar, C::BIMG, warp - C::NWC,
                           lane, kWaitCycles);
    return;
  }

  const double dt = a.dt_override >= 0 ? a.dt_override : a.sc->dt;
  unsigned char *sAV = sA, *sAF = sA + C::AV_BYTES * (C::SEPL ? 1 : 0);
  const unsigned aV = smem_u32(sAV), aF = smem_u32(sAF);
  const unsigned opV = smem_u32(sBimg), opF = opV + C::BV_BYTES;
  constexpr unsigned BPART = C::BV_BYTES + C::BF_BYTES;       // operator part stride
  unsigned long long vmax = 0ull;
  bool ok = consumer_all(mbar_wait(abar, 0), TC);
  int it = 0, mma_phase = 0;
  bool mma_pending = false;   // a commit issued whose phase has not been observed

  // MMAs of one operand block (volume: k-steps [0, KSV), lift: [KSV, KST)),
  // issued by lane 0 of warps 0..NISS-1; MMA g of the tile (product q of
  // k-step ks) goes to accumulator g % NACC, the first NACC initialise them
  auto issue = [&](unsigned abase, int sbo_a, unsigned bbase, int sbo_b, int ks0, int nks) {
    if (lane == 0 && warp < C::NISS) {
      tc_fence_after();
      unsigned long long ad[C::NPARTS], bd[C::NPARTS];
#pragma unroll
      for (int q = 0; q < C::NPARTS; q++) {
        ad[q] = smem_desc(abase + q * C::A_BYTES, 128, sbo_a);
        bd[q] = smem_desc(bbase + q * BPART, 128, sbo_b);
      }
#pragma unroll 1
      for (int ks = 0; ks < nks; ks++) {
#pragma unroll
        for (int q = 0; q < C::NPROD; q++) {
          const int g = C::NPROD * (ks0 + ks) + q, j = g % C::NACC;
          if (j % C::NISS != warp) continue;
          int pa, pb;
          prod_parts<C>(q, pa, pb);
          // a k-step advances the start address by 256 bytes (16 in the field)
          tc_mma<PREC>(tmem + j * C::NPAD, ad[pa] + 16ull * ks, bd[pb] + 16ull * ks, C::IDESC,
                       g >= C::NACC);
        }
      }
      tc_commit(mbar);
    }
  };

  for (int t = blockIdx.x; ok && t < ntiles; t += gridDim.x, it++) {
    const int b = it & 1;
    if (!consumer_all(mbar_wait(&full[b], (it >> 1) & 1), TC)) {
      ok = false;
      break;
    }
    const long e0 = (long)t * E;
    const int ne = (int)min((long)E, (long)a.K - e0);
    double *B = sBuf0 + b * C::S_BUF;
    double *bU = B, *bK = bU + C::S_U, *bUP = bK + C::S_K, *bG = bUP + C::S_UP;
    double *bF = bG + C::S_GEO, *bV = bF + C::S_FACE;
    if (PHYS == EUL) {
      // the previous tile's face fluxes, the last readers, are past a barrier
      node0_fluxes(a.gamma, bU, Np, E * Np, E, tid, TC, sCen);
      consumer_sync(TC);
    }

    // 1. volume fluxes -> operand rows m = v*E + e, k = d*Np + i
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
        centre_sub(sCen + e * kCen, F, Gf, W);
#pragma unroll
        for (int v = 0; v < 5; v++) {
          const int m = v * E + e;
          put_split<C, PREC>(sAV, m, i, C::SBO_AV, rx * F[v] + ry * Gf[v] + rz * W[v]);
          put_split<C, PREC>(sAV, m, Np + i, C::SBO_AV, sx * F[v] + sy * Gf[v] + sz * W[v]);
          put_split<C, PREC>(sAV, m, 2 * Np + i, C::SBO_AV, tx * F[v] + ty * Gf[v] + tz * W[v]);
        }
      } else {
        const double uu = bU[e * Np + i];
        const double F = bV[e * Np + i] * uu, Gf = bV[E * Np + e * Np + i] * uu,
                     W = bV[2 * E * Np + e * Np + i] * uu;
        put_split<C, PREC>(sAV, e, i, C::SBO_AV, rx * F + ry * Gf + rz * W);
        put_split<C, PREC>(sAV, e, Np + i, C::SBO_AV, sx * F + sy * Gf + sz * W);
        put_split<C, PREC>(sAV, e, 2 * Np + i, C::SBO_AV, tx * F + ty * Gf + tz * W);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    consumer_sync(TC);
    issue(aV, C::SBO_AV, opV, C::SBO_BV, 0, C::KSV);
    mma_pending = true;
    if (!C::SEPL) {
      // the volume MMAs must have read the shared operand before it is reused
      if (!consumer_all(mbar_wait(mbar, mma_phase), TC)) {
        ok = false;
        break;
      }
      mma_phase ^= 1;
      mma_pending = false;
      tc_fence_after();
    }

    // 3. face fluxes -> lift operand rows m, k = fj (overlaps the volume MMAs
    //    when the lift operand has its own buffer)
    for (int itm = tid; itm < E * NFF; itm += TC) {
      const int fj = itm / E, e = itm - fj * E, f = fj / Nfp;
      const int nodeM = sFm[fj];
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
        centre_sub(sCen + e * kCen, F, Gf, W);
#pragma unroll
        for (int v = 0; v < 5; v++) {
          const double nd = nx * F[v] + ny * Gf[v] + nz * W[v];
          put_split<C, PREC>(sAF, v * E + e, fj, C::SBO_AF, (nd - tau * (qb[v] - qm[v])) * fs);
        }
      } else {
        const double um = bU[e * Np + nodeM];
        const double ub = 0.5 * (um + bUP[e * C::UPS + fj]);
        const double F = bV[e * Np + nodeM] * ub, Gf = bV[E * Np + e * Np + nodeM] * ub,
                     W = bV[2 * E * Np + e * Np + nodeM] * ub;
        const double nd = nx * F + ny * Gf + nz * W;
        put_split<C, PREC>(sAF, e, fj, C::SBO_AF, (nd - tau * (ub - um)) * fs);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    consumer_sync(TC);
    if (C::SEPL) {
      // the volume commits' phase is waited for before the next commit: a
      // parity wait cannot tell a phase from the one two phases later, so
      // two phases of this barrier must never complete unobserved
      if (!consumer_all(mbar_wait(mbar, mma_phase), TC)) {
        ok = false;
        break;
      }
      mma_phase ^= 1;
      mma_pending = false;
      tc_fence_after();
    }
    issue(aF, C::SBO_AF, opF, C::SBO_BF, C::KSV, C::KSF);
    mma_pending = true;
    // a commit arrives once all earlier MMAs of its thread are done
    if (!consumer_all(mbar_wait(mbar, mma_phase), TC)) {
      ok = false;
      break;
    }
    mma_phase ^= 1;
    mma_pending = false;
    tc_fence_after();

    // 5. accumulator -> sR as [v][i][EP] (row m lives in TMEM lane
    //    (m % 16) + 32 (m / 16) for M = 64, lane m for M = 128)
    {
      // warp w reads lane quarter w % 4 (the quarter a warp may access) and
      // every (NWC / 4)-th group of 8 columns
      const int q = warp & 3, cstart = 8 * (warp >> 2), cstep = 8 * (C::NWC / 4);
      const int m = C::M == 64 ? 16 * q + lane : 32 * q + lane;
      const bool valid = (C::M == 64 ? lane < 16 : true) && m < C::NCOL;
      const int v = m / E, e = m - (m / E) * E;
#pragma unroll 1
      for (int c0 = cstart; c0 < C::NPAD; c0 += cstep) {
        // the partial sums are added in FP32 (the error of each partial, a
        // slice of the K terms, dominates) and converted once
        float r[C::NACC][8];
#pragma unroll
        for (int j = 0; j < C::NACC; j++)
          tmem_ld8(tmem + ((unsigned)(32 * q) << 16) + j * C::NPAD + c0, r[j]);
        tmem_ld_wait();
        if (valid) {
#pragma unroll
          for (int c = 0; c < 8; c++) {
            float sum = r[0][c];
#pragma unroll
            for (int j = 1; j < C::NACC; j++) sum += r[j][c];
            if (c0 + c < Np) sR[(v * Np + c0 + c) * EP + e] = (double)sum;
          }
        }
      }
    }
    tc_fence_before();
    consumer_sync(TC);
    // 6. LSERK update with coalesced stores; the new state goes back to
    //    shared memory only when the fused wave-speed pass reads it
    const bool keep_u = PHYS == EUL && a.last_stage && !a.rhs_only;
    // one flat loop over (variable, node): every thread has independent
    // updates in flight.  nep = ne * Np is a literal for full tiles, so the
    // index divisions become multiplications.
    auto items = [&](const int nep) {
      for (int vg = tid; vg < NV * nep; vg += TC) {
        const int v = vg / nep, g = vg - v * nep;
        const int e = g / Np, i = g - e * Np;
        const long gi = v * vs + e0 * Np + g;
        const double rhs = sR[(v * Np + i) * EP + e];
        if (a.rhs_only) {
          a.u_out[gi] = rhs;
        } else {
          const double kn = a.rka * bK[v * E * Np + g] + dt * rhs;
          const double un = bU[v * E * Np + g] + a.rkb * kn;
          a.kreg[gi] = kn;
          a.u_out[gi] = un;
          if (keep_u) bU[v * E * Np + g] = un;
        }
      }
    };
    if (ne == E)
      items(E * Np);
    else
      items(ne * Np);
    if (PHYS == EUL && a.last_stage && !a.rhs_only) {
      consumer_sync(TC);
      // |v|^2 and c^2 at every face node in parallel (into the rhs staging
      // buffer, free by now), then the per-face max
      double *sW = sR;
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
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[b]);
  }
  if (!ok && tid == 0) atomicOr(&a.sc->flags, 4);
  // MMAs still in flight finish before the tensor memory is released
  if (!ok && mma_pending) mbar_wait(mbar, mma_phase);
  if (PHYS == EUL && a.last_stage && !a.rhs_only) {
    vmax = warp_max_bits(vmax);
    if (lane == 0) sMax[warp] = vmax;
    consumer_sync(TC);
    if (tid < 32) {
      unsigned long long v = tid < C::NWC ? sMax[tid] : 0ull;
      v = warp_max_bits(v);
      if (tid == 0) atomicMax(&a.sc->acc[a.sc->parity ^ 1], v);
    }
  }
  // release tensor memory (warp 0 allocated it)
  tc_fence_before();
  consumer_sync(TC);
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, C::TCOLS);
  }
}
