// Split-BF16 stage kernel with the operator resident in tensor memory, for
// the orders whose split-TF32 operator does not fit there (included by
// dglm_stage_fp64.cu after dglm_stage_tc.cuh, inside namespace dglm).
//
// The same pipeline as stage_tc_kernel (producer warp, MMA warp, compute
// warps; node-0 centring; bounded mbarrier hand-offs), with the contraction
// as tcgen05.mma kind::f16 on BF16 parts:
//   A = the stacked operator [WDr WDs WDt -LIFT] in TENSOR MEMORY, lane i =
//       operator row (output node) i; part p (0: BF16 hi, 1: BF16 lo of the
//       FP64 entry) in columns [A_COL + p KT/2, A_COL + (p+1) KT/2), two K
//       values per 32-bit column (the lower K in the low half);
//   B = the tile's centred fluxes, split hi/lo in BF16 and stacked along N
//       (row n = p NCOL + v E + e) in K-major 8-row x 16-byte core matrices;
//   D = FP32 accumulators in tensor memory, lane i, column n.
// Per k-step (K = 16) two MMAs, A_hi x B and A_lo x B, accumulate into the
// same D, so D[i][c] + D[i][NCOL + c] is the sum of all four part products.
// Each operand keeps 16 significant bits (~2^-17 relative); with the fluxes
// centred on each element's node-0 flux the split parts carry only the
// within-element variation.
//
// Tensor memory: KT columns of operator (both parts) plus the accumulator;
// at N = 6 (KT = 368) one accumulator and one operand image set fit
// (DBUF = false): the flux tasks of tile t+1 then wait for MMA(t) to have
// read the image, and MMA(t+1) for the epilogue to have read D.  At N = 5
// (KT = 272) both are double-buffered (DBUF = true) as in stage_tc_kernel.
// K order as in stage_tc_kernel: volume k = (i/4)*12 + d*4 + i%4, faces at
// KVA + f NFPP + j; KVA and KFA are multiples of 16 (one MMA's K).
#pragma once

template <int PHYS, int N, int E_, int NC_, int NB_, bool DBUF_, bool DF_ = false>
struct TBCfg {
  static constexpr int NV = PHYS == EUL ? 5 : 1;
  static constexpr int Np = np_of(N), Nfp = nfp_of(N), NFF = 4 * Nfp;
  static constexpr int E = E_, NC = NC_, NB = NB_;
  static constexpr bool DBUF = DBUF_;
  static constexpr int NBUF = DBUF ? 2 : 1;              // operand image sets = accumulators
  static constexpr int NCOL = NV * E;
  static constexpr int MN = (2 * NCOL + 15) / 16 * 16;   // MMA N: both parts, padded to 16
  static constexpr int NG = (Np + 3) / 4;                // volume node groups of 4
  static constexpr int KV = 12 * NG, KVA = (KV + 15) / 16 * 16;
  static constexpr int NFPP = (Nfp + 3) / 4 * 4;
  static constexpr int KFA = 4 * NFPP;                   // a multiple of 16
  static constexpr int KT = KVA + KFA, KSV = KVA / 16, KSF = KFA / 16;
  static constexpr int SBO_V = KVA / 8 * 128, SBO_F = KFA / 8 * 128;
  static constexpr int BV_BYTES = MN / 8 * SBO_V, BF_BYTES = MN / 8 * SBO_F;
  static constexpr int B_BYTES = BV_BYTES + BF_BYTES;
  // tensor memory: the accumulators, then the operator (KT 32-bit columns:
  // KT/2 per part, two BF16 per column)
  static constexpr int D_COLS = MN, A_COL = NBUF * MN, A_PART = KT / 2;
  static constexpr int TMEM_COLS = 512;
  static constexpr int NQ = (Np + 31) / 32;              // lane quarters holding output nodes
  static constexpr int UPS = NFF % 8 == 4 ? NFF : NFF + 4;
  static constexpr int S_U = NV * E * Np, S_UP = NV * E * UPS;
  static constexpr int S_REC = kRecord * E, S_TAU = 4 * E;
  static constexpr int S_BUF = S_U + S_UP + S_REC + S_TAU;
  static constexpr unsigned TX = 8u * (S_U + S_REC + S_TAU);
  static constexpr int NCOPY = NV + 2;
  static constexpr int NCEN = 7, S_C = E * NV * NCEN;
  static constexpr int S_R = NV * E * Np;   // rhs (and new state) staging [v][e][i], doubles
  static constexpr int NEB = E / 8, NJB = NFPP / 4;
  static constexpr int VOL_WT = NEB * NG, FACE_WT = NEB * 4 * NJB;
  static constexpr int NTASK = VOL_WT + FACE_WT;
  static constexpr int PROD_WARP = NC, MMA_WARP = NC + 1, NWARPS = NC + 2;
  static constexpr int THREADS = 32 * NWARPS, TC = 32 * NC;
  static constexpr int KPT = (NV * E * Np + TC - 1) / TC;
  static constexpr int GPL = (E * NFF + 31) / 32;
  static constexpr size_t OFF_RING = NBUF * (size_t)B_BYTES;
  static constexpr size_t OFF_R = OFF_RING + 8 * (size_t)NB * S_BUF;
  static constexpr size_t OFF_C = OFF_R + 8 * (size_t)S_R;
  // DF: the centred volume flux in difference form in FP32, as in
  // stage_tc_kernel's vol_task_df; FP32 metrics and node-0 state [slot][e][NDF]
  static constexpr bool DF = DF_;
  static constexpr int NDF = 17, S_DF = DF ? 2 * E * NDF : 0;
  static constexpr size_t OFF_DF = OFF_C + 8 * 2 * (size_t)S_C;
  static constexpr size_t OFF_BAR = OFF_DF + (4 * (size_t)S_DF + 15) / 16 * 16;
  // barriers: full[NB], empty[NB], flux_done[2], mma_done[2], d_free[2],
  // cen[2], vol_done[2] (index 0 only for the single-buffered ones)
  static constexpr int NBARS = 2 * NB + 10;
  static constexpr size_t SMEM = OFF_BAR + 8 * (NBARS + 1) + 4 * NFF + 8 * 32 + 64;
  // instruction descriptor: F32 accumulate, BF16 A and B, both K-major, N, M = 128
  static constexpr unsigned IDESC =
      (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(MN >> 3) << 17) | ((128u >> 4) << 24);
  static_assert(PHYS == EUL, "the tensor-memory operator kernel is built for Euler");
  static_assert(E % 8 == 0 && MN <= 256, "MMA N for M = 128");
  static_assert(Np <= 128, "one output node per tensor-memory lane");
  static_assert(NBUF * D_COLS + KT <= TMEM_COLS, "accumulators and operator fit tensor memory");
  static_assert(KT % 16 == 0 && A_PART % 8 == 0, "whole MMAs and 8-column operator loads");
  static_assert(NC >= 4, "compute warps NC-4 .. NC-1 cover the four tensor-memory lane quarters");
  static_assert(NCOPY <= 32 && 4 * E <= 32, "producer and MMA warp lane assignments");
  static_assert(NB >= 2 && NB <= 4, "ring of 2..4 tile buffers");
  static_assert((E * Np * 8) % 16 == 0, "16-byte bulk copies");
  static_assert(THREADS <= 1024 && NWARPS <= 32, "block size");
  static_assert(SMEM <= 232448, "shared memory per CTA exceeds 227 KB");
  static_assert(SMEM < (1u << 18), "descriptor start addresses fit 14 bits (>> 4)");
};

// tcgen05.mma with A from tensor memory, B from shared memory (kind::f16, BF16)
__device__ __forceinline__ void tc_mma_ts_bf16(unsigned dtmem, unsigned atmem,
                                               unsigned long long bdesc, unsigned idesc,
                                               int accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(dtmem),
      "r"(atmem), "l"(bdesc), "r"(idesc), "r"(accum)
      : "memory");
}
// x = hi + lo in BF16 (raw bits) from the FP32 value of x
__device__ __forceinline__ void split_bf16_pair(double x, unsigned short &hi,
                                                unsigned short &lo) {
  const float f = __double2float_rn(x);
  const __nv_bfloat16 h = __float2bfloat16_rn(f);
  hi = __bfloat16_as_ushort(h);
  lo = __bfloat16_as_ushort(__float2bfloat16_rn(f - __bfloat162float(h)));
}

template <int PHYS, int N, int E_, int NC_, int NB_, bool DBUF_, bool DF_ = false>
__global__ void __launch_bounds__(TBCfg<PHYS, N, E_, NC_, NB_, DBUF_, DF_>::THREADS, 1)
    stage_tcb_kernel(const StageArgs a, int ntiles) {
  using C = TBCfg<PHYS, N, E_, NC_, NB_, DBUF_, DF_>;
  constexpr int NV = C::NV, Np = C::Np, Nfp = C::Nfp, NFF = C::NFF, E = C::E, NB = C::NB,
                NC = C::NC, TC = C::TC, NCOL = C::NCOL, NBUF = C::NBUF;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  double *sRing = reinterpret_cast<double *>(smem_raw + C::OFF_RING);
  double *sR = reinterpret_cast<double *>(smem_raw + C::OFF_R);
  double *sC0 = reinterpret_cast<double *>(smem_raw + C::OFF_C);
  float *sDF = reinterpret_cast<float *>(smem_raw + C::OFF_DF);
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem_raw + C::OFF_BAR);
  unsigned long long *full = bars, *empty = bars + NB, *flux_done = bars + 2 * NB,
                     *mma_done = flux_done + 2, *d_free = flux_done + 4, *cen = flux_done + 6,
                     *vol_done = flux_done + 8;
  unsigned *sTmem = reinterpret_cast<unsigned *>(bars + C::NBARS);
  int *sFm = reinterpret_cast<int *>(bars + C::NBARS + 1);
  unsigned long long *sMax = reinterpret_cast<unsigned long long *>(sFm + NFF + (NFF & 1));

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long vs = a.vs;
  const long long lim = a.wait_cycles;
  const int my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  auto ring = [&](int it) { return sRing + (it % NB) * C::S_BUF; };
  auto tile_e0 = [&](int it) { return ((long)blockIdx.x + (long)it * gridDim.x) * E; };
  // operand image set / accumulator of tile t, and the barrier phase of its
  // use of that buffer
  auto bsel = [&](int t) { return DBUF_ ? (t & 1) : 0; };
  auto bphase = [&](int t) { return DBUF_ ? ((t >> 1) & 1) : (t & 1); };

  if (tid == 0) {
    for (int b = 0; b < NB; b++) {
      mbar_init(&full[b], 1 + 32);
      mbar_init(&empty[b], NC);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&flux_done[b], NC);
      mbar_init(&vol_done[b], NC);
      mbar_init(&mma_done[b], 1);
      mbar_init(&d_free[b], C::NQ);
      mbar_init(&cen[b], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < NFF; i += C::THREADS) sFm[i] = a.Fmask[i];
  for (int i = tid; i < (int)(C::OFF_RING / 16); i += C::THREADS)
    reinterpret_cast<uint4 *>(smem_raw)[i] = make_uint4(0, 0, 0, 0);
  if (warp == 0) tmem_alloc(sTmem, C::TMEM_COLS);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *sTmem;
  // the operator image (128 lanes x KT columns) into tensor memory
  if (warp < 4) {
    const unsigned *img =
        reinterpret_cast<const unsigned *>(a.AT) + (size_t)(32 * warp + lane) * C::KT;
#pragma unroll 1
    for (int c = 0; c < C::KT; c += 8) {
      unsigned r[8];
#pragma unroll
      for (int i = 0; i < 8; i++) r[i] = __ldg(img + c + i);
      tmem_st8(tmem + ((unsigned)(32 * warp) << 16) + C::A_COL + c, r);
    }
    tmem_st_wait();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  const double dt = a.dt_override >= 0 ? a.dt_override : a.sc->dt;
  const double gam = a.gamma;
  const bool keep_u = PHYS == EUL && a.last_stage && !a.rhs_only;
  unsigned long long vmax = 0ull;
  bool ok = true;

  if (warp < NC) {
    // ------------------------------------------------------- compute warps
    // byte offset of operand element (row n, k) in an image of SBO bytes per
    // 8-row group: 8-row x 16-byte core matrices, K-major
    auto boff = [](int n, int k, int sbo) {
      return (n >> 3) * sbo + (k >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2;
    };
    auto vol_task = [&](int it, int wt, int ne, unsigned char *sBv) {
      const int eb = wt / C::NG, g = wt - eb * C::NG;
      const int e = eb * 8 + (lane & 7), i = 4 * g + (lane >> 3);
      const bool okn = e < ne && i < Np;
      const double *bU = ring(it), *bR = bU + C::S_U + C::S_UP + e * kRecord;
      unsigned short hv[5][3], lv[5][3];
      if (okn) {
        const double *cn = sC0 + (it & 1) * C::S_C + e * NV * C::NCEN;
        double q[5], F[5], G[5], W[5];
#pragma unroll
        for (int v = 0; v < 5; v++) q[v] = bU[v * E * Np + e * Np + i];
        euler_flux_fast(gam, q, F, G, W);
        double m[9];
#pragma unroll
        for (int x = 0; x < 9; x++) m[x] = bR[x];
#pragma unroll
        for (int v = 0; v < 5; v++)
#pragma unroll
          for (int d = 0; d < 3; d++)
            split_bf16_pair(fma(m[3 * d + 2], W[v],
                                fma(m[3 * d + 1], G[v], fma(m[3 * d], F[v],
                                                            -cn[v * C::NCEN + d]))),
                            hv[v][d], lv[v][d]);
      } else {
#pragma unroll
        for (int v = 0; v < 5; v++)
#pragma unroll
          for (int d = 0; d < 3; d++) hv[v][d] = lv[v][d] = 0;
      }
#pragma unroll
      for (int v = 0; v < 5; v++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const int n = v * E + e, k = g * 12 + d * 4 + (lane >> 3);
          *reinterpret_cast<unsigned short *>(sBv + boff(n, k, C::SBO_V)) = hv[v][d];
          *reinterpret_cast<unsigned short *>(sBv + boff(n + NCOL, k, C::SBO_V)) = lv[v][d];
        }
    };
    // DF: the centred volume flux in difference form in FP32 (the algebra of
    // stage_tc_kernel's vol_task_df), split into BF16 parts
    auto vol_task_df = [&](int it, int wt, int ne, unsigned char *sBv) {
      const int eb = wt / C::NG, g = wt - eb * C::NG;
      const int e = eb * 8 + (lane & 7), i = 4 * g + (lane >> 3);
      const bool okn = e < ne && i < Np;
      const double *bU = ring(it);
      unsigned short hv[5][3], lv[5][3];
      if (okn) {
        const float *sd = sDF + (it & 1) * E * C::NDF + e * C::NDF;
        float du[5];
#pragma unroll
        for (int v = 0; v < 5; v++)
          du[v] = __double2float_rn(bU[v * E * Np + e * Np + i] - bU[v * E * Np + e * Np]);
        const float v0[3] = {sd[10], sd[11], sd[12]}, m0[3] = {sd[13], sd[14], sd[15]};
        const float dr = du[0], dE = du[4], ir1 = 1.0f / (sd[9] + dr);
        float dv[3], m1[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          dv[c] = (du[1 + c] - v0[c] * dr) * ir1;
          m1[c] = m0[c] + du[1 + c];
        }
        float dmv[3][3];
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
          for (int b = 0; b < 3; b++) dmv[c][b] = fmaf(du[1 + c], v0[b], m1[c] * dv[b]);
        const float dp = (float)(gam - 1.0) * (dE - 0.5f * (dmv[0][0] + dmv[1][1] + dmv[2][2]));
        const float dH = dE + dp, H1 = sd[16] + dH;
        float Fd[3][5];
#pragma unroll
        for (int b = 0; b < 3; b++) {
          Fd[b][0] = du[1 + b];
          Fd[b][1] = dmv[0][b];
          Fd[b][2] = dmv[1][b];
          Fd[b][3] = dmv[2][b];
          Fd[b][4] = fmaf(dH, v0[b], H1 * dv[b]);
          Fd[b][1 + b] += dp;
        }
#pragma unroll
        for (int v = 0; v < 5; v++)
#pragma unroll
          for (int d = 0; d < 3; d++) {
            const float X =
                fmaf(sd[3 * d + 2], Fd[2][v], fmaf(sd[3 * d + 1], Fd[1][v], sd[3 * d] * Fd[0][v]));
            const __nv_bfloat16 h = __float2bfloat16_rn(X);
            hv[v][d] = __bfloat16_as_ushort(h);
            lv[v][d] = __bfloat16_as_ushort(__float2bfloat16_rn(X - __bfloat162float(h)));
          }
      } else {
#pragma unroll
        for (int v = 0; v < 5; v++)
#pragma unroll
          for (int d = 0; d < 3; d++) hv[v][d] = lv[v][d] = 0;
      }
#pragma unroll
      for (int v = 0; v < 5; v++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const int n = v * E + e, k = g * 12 + d * 4 + (lane >> 3);
          *reinterpret_cast<unsigned short *>(sBv + boff(n, k, C::SBO_V)) = hv[v][d];
          *reinterpret_cast<unsigned short *>(sBv + boff(n + NCOL, k, C::SBO_V)) = lv[v][d];
        }
    };
    auto face_task = [&](int it, int wt, int ne, unsigned char *sBf) {
      const int eb = wt / (4 * C::NJB), f = (wt / C::NJB) & 3, jb = wt % C::NJB;
      const int e = eb * 8 + (lane & 7), j = jb * 4 + (lane >> 3);
      const bool okn = e < ne && j < Nfp;
      const double *bU = ring(it), *bUP = bU + C::S_U;
      const double *bR = bUP + C::S_UP + e * kRecord, *bT = bUP + C::S_UP + C::S_REC;
      unsigned short hv[5], lv[5];
      if (okn) {
        const int fj = f * Nfp + j, nodeM = sFm[fj];
        const double nx = bR[9 + f], ny = bR[13 + f], nz = bR[17 + f], fs = bR[21 + f],
                     tau = bT[e * 4 + f];
        const double *cn = sC0 + (it & 1) * C::S_C + e * NV * C::NCEN + 3 + f;
        double qm[5], qb[5], F[5], G[5], W[5];
#pragma unroll
        for (int v = 0; v < 5; v++) {
          qm[v] = bU[v * E * Np + e * Np + nodeM];
          qb[v] = 0.5 * (qm[v] + bUP[(v * E + e) * C::UPS + fj]);
        }
        euler_flux_fast(gam, qb, F, G, W);
#pragma unroll
        for (int v = 0; v < 5; v++) {
          const double nd = fma(nz, W[v], fma(ny, G[v], nx * F[v]));
          split_bf16_pair(fma(nd - tau * (qb[v] - qm[v]), fs, -cn[v * C::NCEN]), hv[v], lv[v]);
        }
      } else {
#pragma unroll
        for (int v = 0; v < 5; v++) hv[v] = lv[v] = 0;
      }
      const int k = f * C::NFPP + j;
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const int n = v * E + e;
        *reinterpret_cast<unsigned short *>(sBf + boff(n, k, C::SBO_F)) = hv[v];
        *reinterpret_cast<unsigned short *>(sBf + boff(n + NCOL, k, C::SBO_F)) = lv[v];
      }
    };

    // D of ring iteration `it` (its MMAs complete) into the rhs staging:
    // warps NC-4 .. NC-1 read lane quarter warp % 4 (node 32 q + lane) and
    // add the two parts; the accumulator is then free for the next MMAs
    auto read_d = [&](int it) {
      const int q = warp & 3;
      if (warp < NC - 4 || q >= C::NQ) return;
      const int db = bsel(it), node = 32 * q + lane;
      float r[2 * NCOL];
      const unsigned row = tmem + ((unsigned)(32 * q) << 16) + db * C::D_COLS;
#pragma unroll
      for (int c = 0; c < 2 * NCOL; c += 4) tmem_ld4(row + c, r + c);
      tmem_ld_wait();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&d_free[db]);
      if (node < Np)
#pragma unroll
        for (int c = 0; c < NCOL; c++) sR[c * Np + node] = (double)(r[c] + r[NCOL + c]);
    };
    // this thread's RK register and state values of ring iteration `it` (the
    // ring slot is released once the flux tasks are done, so the update reads
    // u from global memory, an L2 hit); the element count is a literal for
    // full tiles, so the index divisions become multiplications
    double kr[C::KPT], ur[C::KPT];
    auto load_ku = [&](int it) {
      const long e0 = tile_e0(it);
      const int ne = (int)min((long)E, (long)a.K - e0);
      auto body = [&](auto nepc) {
        const int nep = nepc;
#pragma unroll
        for (int r = 0; r < C::KPT; r++) {
          const int x = tid + r * TC;
          kr[r] = ur[r] = 0.0;
          if (!a.rhs_only && x < NV * nep) {
            const int v = x / nep, g = x - v * nep;
            kr[r] = a.kreg[v * vs + e0 * Np + g];
            ur[r] = a.u_in[v * vs + e0 * Np + g];
          }
        }
      };
      if (ne == E)
        body(std::integral_constant<int, E * Np>{});
      else
        body(ne * Np);
    };
    // LSERK update of ring iteration `it` from the staged rhs (complete:
    // after a barrier behind read_d); on the last stage the new state goes
    // to the staging for the fused wave speed
    auto update = [&](int it) {
      const long e0 = tile_e0(it);
      const int ne = (int)min((long)E, (long)a.K - e0);
      auto body = [&](auto nepc) {
        const int nep = nepc;
#pragma unroll
        for (int r = 0; r < C::KPT; r++) {
          const int x = tid + r * TC;
          if (x < NV * nep) {
            const int v = x / nep, g = x - v * nep;
            const int si = v * E * Np + g;
            const long gi = v * vs + e0 * Np + g;
            const double rhs = sR[si];
            if (a.rhs_only) {
              a.u_out[gi] = rhs;
            } else {
              const double kn = a.rka * kr[r] + dt * rhs;
              const double un = ur[r] + a.rkb * kn;
              a.kreg[gi] = kn;
              a.u_out[gi] = un;
              if (keep_u) sR[si] = un;
            }
          }
        }
      };
      if (ne == E)
        body(std::integral_constant<int, E * Np>{});
      else
        body(ne * Np);
      if (keep_u) {
        // fused calc_maxv on the new state (node_speeds, as in face_maxv_kernel);
        // metrics and Fscale from the element records in global memory
        consumer_sync(TC);
        // one lane per face node, LPF lanes per face, maxima by shuffles
        constexpr int LPF = Nfp <= 16 ? 16 : 32, FPW = 32 / LPF;
        const int jn = lane % LPF;
        for (int f0 = warp * FPW; f0 < 4 * E; f0 += NC * FPW) {
          const int fx = f0 + lane / LPF, f = fx / E, e = fx - f * E;
          const bool on = fx < 4 * E && e < ne;
          double v2 = 0.0, c2 = 0.0;
          int bad = 0;
          if (on && jn < Nfp) {
            const int nd = e * Np + sFm[f * Nfp + jn];
            const double u1 = sR[nd], u2 = sR[E * Np + nd], u3 = sR[2 * E * Np + nd],
                         u4 = sR[3 * E * Np + nd], u5 = sR[4 * E * Np + nd];
            node_speeds(gam, u1, u2, u3, u4, u5, v2, c2);
            bad = (v2 != v2) || (c2 != c2);
          }
#pragma unroll
          for (int o = LPF / 2; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, v2, o);
            const double oc = __shfl_xor_sync(0xffffffffu, c2, o);
            v2 = ov > v2 ? ov : v2;
            c2 = oc > c2 ? oc : c2;
            bad |= __shfl_xor_sync(0xffffffffu, bad, o);
          }
          if (on && jn == 0) {
            double mv = sqrt(v2) + sqrt(c2);
            if (bad) mv = __longlong_as_double(0x7ff8000000000000LL);
            a.maxv[(e0 + e) * 4 + f] = mv;
            const unsigned long long bits = dbits(mv * __ldg(a.erec + (e0 + e) * kRecord + 21 + f));
            vmax = bits > vmax ? bits : vmax;
          }
        }
      }
    };

    for (int it = 0; ok && it < my_tiles; it++) {
      const int ne = (int)min((long)E, (long)a.K - tile_e0(it));
      // the tile's data and node-0 terms; with one image set and accumulator
      // also MMA(it - 1) done, whose D is read back before the tasks so the
      // MMAs of this tile can start as soon as its operand is written (with
      // two, the set's last reader MMA(it - 2) was seen done in iteration it - 1)
      bool w = mbar_wait(&full[it % NB], (it / NB) & 1, lim) &&
               mbar_wait(&cen[it & 1], (it >> 1) & 1, lim);
      if (!DBUF_ && it > 0) w = w && mbar_wait(&mma_done[0], (it - 1) & 1, lim);
      if (!consumer_all(w, TC)) {
        ok = false;
        break;
      }
      tc_fence_after();
      if (!DBUF_ && it > 0) read_d(it - 1);
      unsigned char *sBv = smem_raw + bsel(it) * C::B_BYTES, *sBf = sBv + C::BV_BYTES;
      // one image set: vol_done once this warp's last volume task is written,
      // so the volume MMAs (on the critical path then) start while the face
      // tasks run
      auto vol_signal = [&]() {
        if constexpr (!DBUF_) {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0) mbar_arrive(&vol_done[0]);
        }
      };
      if (warp >= C::VOL_WT) vol_signal();
      for (int wt = warp; wt < C::NTASK; wt += NC) {
        if (wt < C::VOL_WT) {
          if constexpr (C::DF)
            vol_task_df(it, wt, ne, sBv);
          else
            vol_task(it, wt, ne, sBv);
          if (wt + NC >= C::VOL_WT) vol_signal();
        } else {
          face_task(it, wt - C::VOL_WT, ne, sBf);
        }
      }
      // operand written; the ring slot is no longer read by this warp
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&flux_done[bsel(it)]);
        mbar_arrive(&empty[it % NB]);
      }
      if (it > 0) {
        // two accumulators: the reader warps (which carry fewer flux tasks)
        // read D(it - 1) right after their own tasks; the barrier then also
        // carries the wait status
        bool w2 = true;
        if (DBUF_) {
          w2 = mbar_wait(&mma_done[bsel(it - 1)], bphase(it - 1), lim);
          if (w2) {
            tc_fence_after();
            read_d(it - 1);
          }
        }
        load_ku(it - 1);
        if (!consumer_all(w2, TC)) {
          ok = false;
          break;
        }
        update(it - 1);
      }
    }
    if (ok && my_tiles > 0) {
      const int last = my_tiles - 1;
      load_ku(last);
      ok = consumer_all(mbar_wait(&mma_done[bsel(last)], bphase(last), lim), TC);
      if (ok) {
        tc_fence_after();
        read_d(last);
        consumer_sync(TC);
        update(last);
      }
    }
  } else if (warp == C::PROD_WARP) {
    // ------------------------------------------------------ producer warp
    int it = 0;
    for (; it < my_tiles; it++) {
      const int b = it % NB;
      if (it >= NB && !mbar_wait(&empty[b], ((it / NB) - 1) & 1, lim)) {
        ok = false;
        break;
      }
      const long e0 = tile_e0(it);
      const int ne = (int)min((long)E, (long)a.K - e0);
      double *bU = ring(it), *bUP = bU + C::S_U, *bR = bUP + C::S_UP, *bT = bR + C::S_REC;
      if (lane == 0) mbar_arrive_expect_tx(&full[b], C::TX);
      __syncwarp();
      if (lane < NV)
        bulk_g2s(bU + lane * E * Np, a.u_in + lane * vs + e0 * Np, 8u * E * Np, &full[b]);
      else if (lane == NV)
        bulk_g2s(bR, a.erec + e0 * kRecord, 8u * C::S_REC, &full[b]);
      else if (lane == NV + 1)
        bulk_g2s(bT, a.tau + 4 * e0, 8u * C::S_TAU, &full[b]);
      int vmr[C::GPL];
      if (a.etoe) {
#pragma unroll
        for (int g = 0; g < C::GPL; g++) {
          const int idx = lane + 32 * g;
          vmr[g] = idx < ne * NFF ? compact_neighbour_node<Np, Nfp>(a, e0, idx) : -1;
        }
      } else {
#pragma unroll
        for (int g = 0; g < C::GPL; g++) {
          const int idx = lane + 32 * g;
          vmr[g] = idx < ne * NFF ? __ldg(a.vmapP + e0 * NFF + idx) : -1;
        }
      }
#pragma unroll
      for (int g = 0; g < C::GPL; g++) {
        const int idx = lane + 32 * g;
        if (vmr[g] >= 0) {
          const int e = idx / NFF, fj = idx - e * NFF;
#pragma unroll
          for (int v = 0; v < NV; v++)
            cp_async8(bUP + (v * E + e) * C::UPS + fj, a.u_in + v * vs + vmr[g]);
        }
      }
      cp_async_arrive_noinc(&full[b]);
    }
    for (int j = (it > NB ? it - NB : 0); j < it; j++) mbar_wait(&full[j % NB], (j / NB) & 1);
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else {
    // ----------------------------------------------------------- MMA warp
    auto centers = [&](int t) {
      const int e = lane >> 2, r = lane & 3;
      const int ne = (int)min((long)E, (long)a.K - tile_e0(t));
      const double *bU = ring(t), *bR = bU + C::S_U + C::S_UP + e * kRecord;
      double *c = sC0 + (t & 1) * C::S_C + e * NV * C::NCEN;
      if (e >= ne) {
        if (r == 0)
#pragma unroll
          for (int x = 0; x < NV * C::NCEN; x++) c[x] = 0.0;
        return;
      }
      double q[5], F[5], G[5], W[5];
#pragma unroll
      for (int v = 0; v < 5; v++) q[v] = bU[v * E * Np + e * Np];
      euler_flux_fast(gam, q, F, G, W);
      if (r == 0) {
        if constexpr (C::DF) {
          // FP32 metrics and node-0 state of the difference-form volume flux
          float *sd = sDF + (t & 1) * E * C::NDF + e * C::NDF;
#pragma unroll
          for (int x = 0; x < 9; x++) sd[x] = __double2float_rn(bR[x]);
          const float r0 = __double2float_rn(q[0]), E0 = __double2float_rn(q[4]);
          const float m0[3] = {__double2float_rn(q[1]), __double2float_rn(q[2]),
                               __double2float_rn(q[3])};
          const float ir0 = 1.0f / r0;
          const float v0[3] = {m0[0] * ir0, m0[1] * ir0, m0[2] * ir0};
          const float p0 =
              (float)(gam - 1.0) * (E0 - 0.5f * (m0[0] * v0[0] + m0[1] * v0[1] + m0[2] * v0[2]));
          sd[9] = r0;
#pragma unroll
          for (int c2 = 0; c2 < 3; c2++) {
            sd[10 + c2] = v0[c2];
            sd[13 + c2] = m0[c2];
          }
          sd[16] = E0 + p0;
        } else {
#pragma unroll
          for (int d = 0; d < 3; d++) {
            const double mx = bR[3 * d], my = bR[3 * d + 1], mz = bR[3 * d + 2];
#pragma unroll
            for (int v = 0; v < 5; v++) c[v * C::NCEN + d] = mx * F[v] + my * G[v] + mz * W[v];
          }
        }
      } else {
        const int nf = r == 3 ? 2 : 1;   // r = 1: face 0, r = 2: face 1, r = 3: faces 2, 3
#pragma unroll
        for (int h = 0; h < nf; h++) {
          const int f = r - 1 + h;
          const double nx = bR[9 + f], ny = bR[13 + f], nz = bR[17 + f], fs = bR[21 + f];
#pragma unroll
          for (int v = 0; v < 5; v++)
            c[v * C::NCEN + 3 + f] = (nx * F[v] + ny * G[v] + nz * W[v]) * fs;
        }
      }
    };
    auto centers_of = [&](int t) -> bool {
      const bool w = mbar_wait(&full[t % NB], (t / NB) & 1, lim);
      if (w) centers(t);
      __syncwarp();
      if (lane == 0 && w) mbar_arrive(&cen[t & 1]);
      return __all_sync(0xffffffffu, w);
    };
    int nm = 0;
    if (my_tiles > 0 && !centers_of(0)) ok = false;
    for (int it = 0; ok && it < my_tiles; it++) {
      const int b = bsel(it);
      // the volume operand (with two image sets: the whole operand), and the
      // accumulator (read back by read_d(it - NBUF))
      bool w = DBUF_ ? mbar_wait(&flux_done[b], bphase(it), lim)
                     : mbar_wait(&vol_done[0], bphase(it), lim);
      if (w && it >= NBUF) w = mbar_wait(&d_free[b], bphase(it - NBUF), lim);
      if (!__all_sync(0xffffffffu, w)) {
        ok = false;
        break;
      }
      const unsigned d = tmem + b * C::D_COLS;
      const unsigned bv = smem_u32(smem_raw + b * C::B_BYTES), bf = bv + C::BV_BYTES;
      if (lane == 0) {
        tc_fence_after();
#pragma unroll 1
        for (int ks = 0; ks < C::KSV; ks++) {
          const unsigned long long bd = smem_desc(bv + ks * 256, 128, C::SBO_V);
          tc_mma_ts_bf16(d, tmem + C::A_COL + ks * 8, bd, C::IDESC, ks > 0);
          tc_mma_ts_bf16(d, tmem + C::A_COL + C::A_PART + ks * 8, bd, C::IDESC, 1);
        }
      }
      __syncwarp();
      // the face operand; on expiry the volume MMAs are still committed, so
      // their completion can be waited for before the CTA leaves
      if (!DBUF_) w = mbar_wait(&flux_done[b], bphase(it), lim);
      const bool fw = __all_sync(0xffffffffu, w);
      if (lane == 0) {
        tc_fence_after();
#pragma unroll 1
        for (int ks = 0; fw && ks < C::KSF; ks++) {
          const unsigned long long bd = smem_desc(bf + ks * 256, 128, C::SBO_F);
          const int kc = C::KVA / 2 + ks * 8;
          tc_mma_ts_bf16(d, tmem + C::A_COL + kc, bd, C::IDESC, 1);
          tc_mma_ts_bf16(d, tmem + C::A_COL + C::A_PART + kc, bd, C::IDESC, 1);
        }
        tc_commit(&mma_done[b]);
      }
      __syncwarp();
      nm++;
      if (!fw) {
        ok = false;
        break;
      }
      // the next tile's node-0 terms while the tensor cores work
      if (it + 1 < my_tiles && !centers_of(it + 1)) {
        ok = false;
        break;
      }
    }
    // the MMAs issued (and their barrier arrivals) are complete before
    // tensor and shared memory are released, on expiry too
    if (lane == 0)
      for (int t = (nm > NBUF ? nm - NBUF : 0); t < nm; t++)
        mbar_wait(&mma_done[bsel(t)], bphase(t));
  }
  if (!ok) atomicOr(&a.sc->flags, 4);
  if (keep_u) {
    vmax = warp_max_bits(vmax);
    if (lane == 0) sMax[warp] = vmax;
  }
  tc_fence_before();
  __syncthreads();
  if (keep_u && tid < 32) {
    unsigned long long v = tid < C::NWARPS ? sMax[tid] : 0ull;
    v = warp_max_bits(v);
    if (tid == 0) atomicMax(&a.sc->acc[a.sc->parity ^ 1], v);
  }
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, C::TMEM_COLS);
  }
}
