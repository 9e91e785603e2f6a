// Split-TF32 stage kernel with the operator resident in tensor memory
// (included by dglm_stage_fp64.cu after dglm_stage_mixed.cuh, inside
// namespace dglm).
//
// The contraction rhs = [WDr WDs WDt -LIFT] x [fluxR; fluxS; fluxT; fluxLM]
// of a tile of E elements runs as tcgen05.mma (kind::tf32) with
//   D[m][n] += A[m][k] * B[n][k],
//   A = the stacked operator in TENSOR MEMORY (M = 128 lanes, loaded once per
//       CTA): lane 32q + 2j + p holds part p (0: TF32 hi, 1: TF32 lo) of
//       operator row i = NPQ q + j, so both parts of an output node sit in
//       neighbouring lanes of one warp's lane quarter;
//   B = the tile's fluxes in shared memory, split x = hi + lo; row
//       n = p NCOL + v E + e holds part p of (variable v, element e), so one
//       MMA per k-step multiplies both parts (rows past 2 NCOL stay zero);
//       two image sets, so that the fluxes of tile t+1 are written while the
//       MMAs of tile t read theirs;
//   D = FP32 accumulators in tensor memory, double-buffered across tiles:
//       column n of lane (i, p') holds A_p' . B_p of column n mod NCOL.
// The right-hand side of (v, e) at node i is the sum of the four part
// products D[(i,0)][c] + D[(i,0)][NCOL + c] + D[(i,1)][c] + D[(i,1)][NCOL + c].
//
// Centring.  Before the split every flux value of an element has that
// element's flux at node 0 subtracted: fluxR/S/T = metric . (F(u_i) - F(u_0))
// and fluxLM = Fscale_f (n_f . (F(u*) - F(u_0)) - tau (u* - u-)).  A constant
// flux has zero DG right-hand side (the weak volume term equals the surface
// term for constant data on straight-sided tetrahedra, to FP64 rounding), so
// the contraction of the centred fluxes IS the right-hand side, while the
// values that reach the tensor cores are the within-element variations: an
// order of magnitude smaller than the fluxes for resolved solutions, and with
// them the TF32 representation and FP32 accumulation errors.  The node-0
// terms metric_d . F(u_0) and Fscale_f n_f . F(u_0) of a tile are formed once
// per element (by the MMA warp, one tile ahead) and subtracted in the first
// FMA of each flux value.
//
// K order.  Volume columns are node-group major, k = (i/4)*12 + d*4 + i%4
// (d = r, s, t); face columns follow at KVA + f NFPP + j.  A warp task covers
// 8 elements x 4 consecutive nodes, so each store of the task fills one
// 8-row x 16-byte core matrix.
//
// Warps: NC compute warps, one producer warp, one MMA warp.
//   producer    per tile, into a ring of NB buffers: bulk copies of u (one
//               per variable), of the element records (metrics, normals,
//               Fscale) and of tau, one copy per lane; cp.async gathers of
//               the neighbour traces u[vmapP].
//   MMA         once the compute warps have written operand image set t%2
//               (flux_done[t%2]): all lanes form the node-0 terms of tile t+1
//               (cen[(t+1)%2]); then lane 0, once accumulator D[t%2] is free
//               (d_free[t%2]), issues the volume and face MMAs of tile t,
//               committed to mma_done[t%2].
//   compute     per tile t: loads of tile t-1's RK register values, the
//               volume and face flux tasks of t into image set t%2, then the
//               epilogue of t-1: the wait for MMA(t-1); warps NC-4 .. NC-1
//               (at Euler N=4 with one node per lane, 25 tasks over 14
//               warps, three of them carry one flux task, not two; with two
//               nodes per lane, NPL = 2, 13 tasks, every warp at most one)
//               read D[(t-1)%2]
//               (lane quarter warp % 4) and add the parts into the rhs
//               staging; all compute warps do the LSERK update with
//               coalesced stores.
// The tensor cores work on tile t while the compute warps finish t-1 and
// start t+1.  Every wait is bounded; on expiry a warp sets flag bit 2, waits
// (with the default bound) for the MMAs and copies it issued, and leaves.
//
// Variants: NPL = 2 gives each lane two nodes of a flux task (13 tasks per
// tile at N=4); DF forms the centred volume flux in difference form in FP32
// (vol_task_df: no cancelling term, ~1e-7 of each value, the split's own
// precision) from each element's FP32 metrics and node-0 state, which the
// MMA warp writes with the node-0 terms.  The face flux stays FP64 in all.
#pragma once

template <int PHYS, int N, int E_, int NC_, int NB_, int NPL_ = 1, bool DF_ = false>
struct TCfg {
  static constexpr int NV = PHYS == EUL ? 5 : 1;
  static constexpr int Np = np_of(N), Nfp = nfp_of(N), NFF = 4 * Nfp;
  static constexpr int E = E_, NC = NC_, NB = NB_;
  static constexpr int NCOL = NV * E;                    // (variable, element) columns
  static constexpr int MN = (2 * NCOL + 15) / 16 * 16;   // MMA N: both parts, padded to 16
  static constexpr int NPQ = (Np + 3) / 4;               // output nodes per lane quarter
  static constexpr int NG = (Np + 3) / 4;                // volume node groups of 4
  static constexpr int KV = 12 * NG, KVA = (KV + 7) / 8 * 8;
  static constexpr int NFPP = (Nfp + 3) / 4 * 4;
  static constexpr int KFA = 4 * NFPP;
  static constexpr int KT = KVA + KFA, KSV = KVA / 8, KSF = KFA / 8;
  static constexpr int SBO_V = KVA / 4 * 128, SBO_F = KFA / 4 * 128;
  static constexpr int BV_BYTES = MN / 8 * SBO_V, BF_BYTES = MN / 8 * SBO_F;
  static constexpr int B_BYTES = BV_BYTES + BF_BYTES;    // one operand image set
  // tensor memory: D0, D1, then the operator
  static constexpr int D_COLS = MN, A_COL = 2 * MN;
  static constexpr int TMEM_COLS = 512;
  // tile ring buffer (doubles): u [v][e][i], neighbour traces [v][e][UPS],
  // element records [e][kRecord], tau [e][f]
  static constexpr int UPS = NFF % 8 == 4 ? NFF : NFF + 4;
  static constexpr int S_U = NV * E * Np, S_UP = NV * E * UPS;
  static constexpr int S_REC = kRecord * E, S_TAU = 4 * E;
  static constexpr int S_BUF = S_U + S_UP + S_REC + S_TAU;
  static constexpr unsigned TX = 8u * (S_U + S_REC + S_TAU);
  static constexpr int NCOPY = NV + 2;                   // bulk copies per tile
  // node-0 terms [e][v][NCEN] (3 volume directions, 4 faces), two slots
  static constexpr int NCEN = 7, S_C = E * NV * NCEN;
  // rhs staging [v][e][i] (FP32: the sum of the four part products)
  static constexpr int S_R = NV * E * Np;
  // warp tasks per tile: volume (8 elements x one node group of 4), face
  // (8 elements x 4 nodes of one face)
  // (8 elements x 8 nodes with NPL = 2 nodes per lane: pairs of groups)
  static constexpr int NPL = NPL_;
  // DF: the centred volume flux F(u_i) - F(u_0) in difference form in FP32
  // (vol_task_df), from each element's FP32 metrics and node-0 state, which
  // the MMA warp writes one tile ahead: [slot][e][NDF] floats
  static constexpr bool DF = DF_;
  static constexpr int NDF = 17;
  static constexpr int NEB = E / 8, NJB = NFPP / 4;
  static constexpr int NGP = (NG + 1) / 2, NJP = (NJB + 1) / 2;
  static constexpr int VOL_WT = NEB * (NPL == 2 ? NGP : NG);
  static constexpr int FACE_WT = NEB * 4 * (NPL == 2 ? NJP : NJB);
  static constexpr int NTASK = VOL_WT + FACE_WT;
  static constexpr int PROD_WARP = NC, MMA_WARP = NC + 1, NWARPS = NC + 2;
  static constexpr int THREADS = 32 * NWARPS, TC = 32 * NC;
  static constexpr int KPT = (NV * E * Np + TC - 1) / TC;   // update values per compute thread
  static constexpr int GPL = (E * NFF + 31) / 32;        // gathers per producer lane
  static constexpr size_t OFF_RING = 2 * (size_t)B_BYTES;
  static constexpr size_t OFF_R = OFF_RING + 8 * (size_t)NB * S_BUF;
  static constexpr size_t OFF_C = OFF_R + (4 * (size_t)S_R + 15) / 16 * 16;
  static constexpr int S_DF = DF ? 2 * E * NDF : 0;
  static constexpr size_t OFF_DF = OFF_C + 8 * 2 * (size_t)S_C;
  static constexpr size_t OFF_BAR = OFF_DF + (4 * (size_t)S_DF + 15) / 16 * 16;
  // barriers: full[NB], empty[NB], flux_done[2], mma_done[2], d_free[2],
  // cen[2]; then the tensor-memory address, Fmask, maxima
  static constexpr int NBARS = 2 * NB + 8;
  static constexpr size_t SMEM = OFF_BAR + 8 * (NBARS + 1) + 4 * NFF + 8 * 32 + 64;
  // instruction descriptor: F32 accumulate, TF32 A and B, both K-major, N, M = 128
  static constexpr unsigned IDESC =
      (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(MN >> 3) << 17) | ((128u >> 4) << 24);
  static_assert(PHYS == EUL, "the tensor-memory operator kernel is built for Euler");
  static_assert(E % 8 == 0 && MN <= 256, "MMA N for M = 128");
  static_assert(2 * NPQ <= 32, "both operator parts of a quarter's nodes fit its 32 lanes");
  static_assert(2 * D_COLS + KT <= TMEM_COLS, "accumulators and operator fit tensor memory");
  static_assert(NC >= 4, "compute warps NC-4 .. NC-1 cover the four tensor-memory lane quarters");
  static_assert(NCOPY <= 32, "one producer lane per bulk copy");
  static_assert(4 * E <= 32, "the MMA warp forms node-0 terms with 4 lanes per element");
  static_assert(NCOL <= 64 && NCOL % 2 == 0,
                "an epilogue lane holds both parts of its row's columns, split in halves");
  static_assert(NB >= 2 && NB <= 4, "ring of 2..4 tile buffers");
  static_assert(NPL == 1 || NPL == 2, "one or two nodes per lane in a flux task");
  static_assert(!DF || NPL == 1, "the difference-form volume flux has one node per lane");
  static_assert((E * Np * 8) % 16 == 0, "16-byte bulk copies");
  static_assert(THREADS <= 1024 && NWARPS <= 32, "block size");
  static_assert(SMEM <= 232448, "shared memory per CTA exceeds 227 KB");
  static_assert(SMEM < (1u << 18), "descriptor start addresses fit 14 bits (>> 4)");
};

// tcgen05.mma with A from tensor memory, B from shared memory (kind::tf32)
__device__ __forceinline__ void tc_mma_ts(unsigned dtmem, unsigned atmem,
                                          unsigned long long bdesc, unsigned idesc, int accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(dtmem),
      "r"(atmem), "l"(bdesc), "r"(idesc), "r"(accum)
      : "memory");
}
__device__ __forceinline__ void tmem_st8(unsigned taddr, const unsigned (&r)[8]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
      : "memory");
}
__device__ __forceinline__ void tmem_st_wait() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_ld4(unsigned taddr, float *r) {
  unsigned v[4];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "r"(taddr)
               : "memory");
#pragma unroll
  for (int i = 0; i < 4; i++) r[i] = __uint_as_float(v[i]);
}
// x = hi + lo as TF32 bit patterns (FP32 containers) of the FP32 value of x:
// hi keeps the top 11 significant bits of FP32(x) (truncated), lo the exact
// FP32 remainder, of which the MMA reads the top 11 bits
__device__ __forceinline__ void split_tf32_pair(double x, unsigned &hi, unsigned &lo) {
  const float f = __double2float_rn(x);
  hi = __float_as_uint(f) & 0xffffe000u;
  lo = __float_as_uint(f - __uint_as_float(hi));
}

template <int PHYS, int N, int E_, int NC_, int NB_, int NPL_ = 1, bool DF_ = false>
__global__ void __launch_bounds__(TCfg<PHYS, N, E_, NC_, NB_, NPL_, DF_>::THREADS, 1)
    stage_tc_kernel(const StageArgs a, int ntiles) {
  using C = TCfg<PHYS, N, E_, NC_, NB_, NPL_, DF_>;
  constexpr int NV = C::NV, Np = C::Np, Nfp = C::Nfp, NFF = C::NFF, E = C::E, NB = C::NB,
                NC = C::NC, TC = C::TC, NCOL = C::NCOL;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  double *sRing = reinterpret_cast<double *>(smem_raw + C::OFF_RING);
  float *sR = reinterpret_cast<float *>(smem_raw + C::OFF_R);
  double *sC0 = reinterpret_cast<double *>(smem_raw + C::OFF_C);
  float *sDF = reinterpret_cast<float *>(smem_raw + C::OFF_DF);
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem_raw + C::OFF_BAR);
  unsigned long long *full = bars, *empty = bars + NB, *flux_done = bars + 2 * NB,
                     *mma_done = flux_done + 2, *d_free = flux_done + 4, *cen = flux_done + 6;
  unsigned *sTmem = reinterpret_cast<unsigned *>(bars + C::NBARS);
  int *sFm = reinterpret_cast<int *>(bars + C::NBARS + 1);
  unsigned long long *sMax = reinterpret_cast<unsigned long long *>(sFm + NFF + (NFF & 1));

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long vs = a.vs;
  const long long lim = a.wait_cycles;
  const int my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  auto ring = [&](int it) { return sRing + (it % NB) * C::S_BUF; };
  auto tile_e0 = [&](int it) { return ((long)blockIdx.x + (long)it * gridDim.x) * E; };

  if (tid == 0) {
    for (int b = 0; b < NB; b++) {
      mbar_init(&full[b], 1 + 32);   // the byte-count arrive + each producer lane's gathers
      mbar_init(&empty[b], NC);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&flux_done[b], NC);
      mbar_init(&mma_done[b], 1);
      mbar_init(&d_free[b], 4);
      mbar_init(&cen[b], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < NFF; i += C::THREADS) sFm[i] = a.Fmask[i];
  // the operand images start zeroed: the volume K padding [KV, KVA) and the
  // rows past 2 NCOL are never written
  for (int i = tid; i < (int)(C::OFF_RING / 16); i += C::THREADS)
    reinterpret_cast<uint4 *>(smem_raw)[i] = make_uint4(0, 0, 0, 0);
  if (warp == 0) tmem_alloc(sTmem, C::TMEM_COLS);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *sTmem;
  // the operator image (128 lanes x KT TF32 columns) into tensor memory:
  // warp q < 4 writes lanes 32q .. 32q + 31
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
    // volume fluxes of ring iteration `it`, task wt: 8 elements x nodes
    // 4g .. 4g+3, centred and split into operand image sBv
    auto vol_task = [&](int it, int wt, int ne, unsigned char *sBv) {
      const int eb = wt / C::NG, g = wt - eb * C::NG;
      const int e = eb * 8 + (lane & 7), i = 4 * g + (lane >> 3);
      const bool okn = e < ne && i < Np;
      const double *bU = ring(it), *bR = bU + C::S_U + C::S_UP + e * kRecord;
      unsigned hv[5][3], lv[5][3];
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
            // the node-0 term enters the first FMA of the metric combination
            split_tf32_pair(fma(m[3 * d + 2], W[v],
                                fma(m[3 * d + 1], G[v], fma(m[3 * d], F[v],
                                                            -cn[v * C::NCEN + d]))),
                            hv[v][d], lv[v][d]);
      } else {
#pragma unroll
        for (int v = 0; v < 5; v++)
#pragma unroll
          for (int d = 0; d < 3; d++) hv[v][d] = lv[v][d] = 0u;
      }
#pragma unroll
      for (int v = 0; v < 5; v++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const int n = v * E + e, k = g * 12 + d * 4 + (lane >> 3);
          const int off = (k >> 2) * 128 + (n & 7) * 16 + (k & 3) * 4;
          *reinterpret_cast<unsigned *>(sBv + (n >> 3) * C::SBO_V + off) = hv[v][d];
          *reinterpret_cast<unsigned *>(sBv + ((n + NCOL) >> 3) * C::SBO_V + off) = lv[v][d];
        }
    };

    // face fluxes of ring iteration `it`, task wt: each lane one face node
    // of 8 elements x 4 nodes of one face, neighbour traces staged; image sBf
    auto face_task = [&](int it, int wt, int ne, unsigned char *sBf) {
      const int eb = wt / (4 * C::NJB), f = (wt / C::NJB) & 3, jb = wt % C::NJB;
      const int e = eb * 8 + (lane & 7), j = jb * 4 + (lane >> 3);
      const bool okn = e < ne && j < Nfp;
      const double *bU = ring(it), *bUP = bU + C::S_U;
      const double *bR = bUP + C::S_UP + e * kRecord, *bT = bUP + C::S_UP + C::S_REC;
      unsigned hv[5], lv[5];
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
          split_tf32_pair(fma(nd - tau * (qb[v] - qm[v]), fs, -cn[v * C::NCEN]), hv[v], lv[v]);
        }
      } else {
#pragma unroll
        for (int v = 0; v < 5; v++) hv[v] = lv[v] = 0u;
      }
      const int k = f * C::NFPP + j;
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const int n = v * E + e;
        const int off = (k >> 2) * 128 + (n & 7) * 16 + (k & 3) * 4;
        *reinterpret_cast<unsigned *>(sBf + (n >> 3) * C::SBO_F + off) = hv[v];
        *reinterpret_cast<unsigned *>(sBf + ((n + NCOL) >> 3) * C::SBO_F + off) = lv[v];
      }
    };

    // DF: the same volume task with the centred flux F(u_i) - F(u_0) formed
    // in difference form in FP32.  With du = u_i - u_0 (an FP64 subtraction,
    // rounded once) and the node-0 state (rho0, m0, v0 = m0/rho0, H0):
    //   dv_a = (dm_a - v0_a drho) / rho_i,  d(m_a v_b) = dm_a v0_b + m_a,i dv_b,
    //   dp = (gamma-1) (dE - d(m.v)/2),  d(H v_a) = dH v0_a + H_i dv_a,
    // so no term cancels and FP32 carries each value to ~1e-7 of its size,
    // the precision of the TF32 split that follows; the metric combination
    // and the split run in FP32 too.
    auto vol_task_df = [&](int it, int wt, int ne, unsigned char *sBv) {
      const int eb = wt / C::NG, g = wt - eb * C::NG;
      const int e = eb * 8 + (lane & 7), i = 4 * g + (lane >> 3);
      const bool okn = e < ne && i < Np;
      const double *bU = ring(it);
      unsigned hv[5][3], lv[5][3];
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
        // direction b: (dm_b, d(m_x v_b), d(m_y v_b), d(m_z v_b), d(H v_b)) + dp on 1 + b
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
            hv[v][d] = __float_as_uint(X) & 0xffffe000u;
            lv[v][d] = __float_as_uint(X - __uint_as_float(hv[v][d]));
          }
      } else {
#pragma unroll
        for (int v = 0; v < 5; v++)
#pragma unroll
          for (int d = 0; d < 3; d++) hv[v][d] = lv[v][d] = 0u;
      }
#pragma unroll
      for (int v = 0; v < 5; v++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const int n = v * E + e, k = g * 12 + d * 4 + (lane >> 3);
          const int off = (k >> 2) * 128 + (n & 7) * 16 + (k & 3) * 4;
          *reinterpret_cast<unsigned *>(sBv + (n >> 3) * C::SBO_V + off) = hv[v][d];
          *reinterpret_cast<unsigned *>(sBv + ((n + NCOL) >> 3) * C::SBO_V + off) = lv[v][d];
        }
    };

    // NPL = 2: task wt of the volume covers 8 elements x node groups 2gp and
    // 2gp + 1; lane (e = lane % 8, h = bit 3, group = bit 4) takes nodes
    // 4g + 2h and 4g + 2h + 1, two independent flux chains whose columns
    // are neighbours in one core-matrix row (one 8-byte store per part), and
    // the element's metrics and node-0 terms serve both.  Node indices past
    // the element are clamped for the loads and their values written as 0.
    auto vol_task2 = [&](int it, int wt, int ne, unsigned char *sBv) {
      const int eb = wt / C::NGP, g = 2 * (wt - eb * C::NGP) + (lane >> 4);
      if (g >= C::NG) return;   // the empty half of an odd group count
      const int h = (lane >> 3) & 1, e = eb * 8 + (lane & 7), i0 = 4 * g + 2 * h;
      const double *bU = ring(it), *bR = bU + C::S_U + C::S_UP + e * kRecord;
      const double *cn = sC0 + (it & 1) * C::S_C + e * NV * C::NCEN;
      const bool on0 = e < ne && i0 < Np, on1 = e < ne && i0 + 1 < Np;
      double F[2][5], G[2][5], W[2][5];
#pragma unroll
      for (int s = 0; s < 2; s++) {
        const int i = min(i0 + s, Np - 1);
        double q[5];
#pragma unroll
        for (int v = 0; v < 5; v++) q[v] = bU[v * E * Np + e * Np + i];
        euler_flux_fast(gam, q, F[s], G[s], W[s]);
      }
      double m[9];
#pragma unroll
      for (int x = 0; x < 9; x++) m[x] = bR[x];
#pragma unroll
      for (int v = 0; v < 5; v++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const double c = -cn[v * C::NCEN + d];
          unsigned hi0, lo0, hi1, lo1;
          split_tf32_pair(fma(m[3 * d + 2], W[0][v], fma(m[3 * d + 1], G[0][v],
                                                         fma(m[3 * d], F[0][v], c))),
                          hi0, lo0);
          split_tf32_pair(fma(m[3 * d + 2], W[1][v], fma(m[3 * d + 1], G[1][v],
                                                         fma(m[3 * d], F[1][v], c))),
                          hi1, lo1);
          const int n = v * E + e, k = g * 12 + d * 4 + 2 * h;
          const int off = (k >> 2) * 128 + (n & 7) * 16 + (k & 3) * 4;
          *reinterpret_cast<uint2 *>(sBv + (n >> 3) * C::SBO_V + off) =
              make_uint2(on0 ? hi0 : 0u, on1 ? hi1 : 0u);
          *reinterpret_cast<uint2 *>(sBv + ((n + NCOL) >> 3) * C::SBO_V + off) =
              make_uint2(on0 ? lo0 : 0u, on1 ? lo1 : 0u);
        }
    };

    // NPL = 2: face task wt covers 8 elements x face nodes 8jp .. 8jp + 7 of
    // one face, lane (e, h, bit 4) face nodes j0 = 4jb + 2h and j0 + 1
    auto face_task2 = [&](int it, int wt, int ne, unsigned char *sBf) {
      const int eb = wt / (4 * C::NJP), f = (wt / C::NJP) & 3;
      const int jb = 2 * (wt % C::NJP) + (lane >> 4);
      if (jb >= C::NJB) return;
      const int h = (lane >> 3) & 1, e = eb * 8 + (lane & 7), j0 = 4 * jb + 2 * h;
      const double *bU = ring(it), *bUP = bU + C::S_U;
      const double *bR = bUP + C::S_UP + e * kRecord, *bT = bUP + C::S_UP + C::S_REC;
      const double nx = bR[9 + f], ny = bR[13 + f], nz = bR[17 + f], fs = bR[21 + f],
                   tau = bT[e * 4 + f];
      const double *cn = sC0 + (it & 1) * C::S_C + e * NV * C::NCEN + 3 + f;
      const bool on0 = e < ne && j0 < Nfp, on1 = e < ne && j0 + 1 < Nfp;
      unsigned hv[2][5], lv[2][5];
#pragma unroll
      for (int s = 0; s < 2; s++) {
        const int fj = f * Nfp + min(j0 + s, Nfp - 1), nodeM = sFm[fj];
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
          split_tf32_pair(fma(nd - tau * (qb[v] - qm[v]), fs, -cn[v * C::NCEN]), hv[s][v],
                          lv[s][v]);
        }
      }
      const int k = f * C::NFPP + j0;
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const int n = v * E + e;
        const int off = (k >> 2) * 128 + (n & 7) * 16 + (k & 3) * 4;
        *reinterpret_cast<uint2 *>(sBf + (n >> 3) * C::SBO_F + off) =
            make_uint2(on0 ? hv[0][v] : 0u, on1 ? hv[1][v] : 0u);
        *reinterpret_cast<uint2 *>(sBf + ((n + NCOL) >> 3) * C::SBO_F + off) =
            make_uint2(on0 ? lv[0][v] : 0u, on1 ? lv[1][v] : 0u);
      }
    };

    // this thread's RK register values of ring iteration `it` (update order:
    // x = tid + r TC over (variable, element node)); the element count is a
    // literal for full tiles, so the index divisions are multiplications
    double kr[C::KPT];
    auto load_k = [&](int it) {
      const long e0 = tile_e0(it);
      const int ne = (int)min((long)E, (long)a.K - e0);
      auto body = [&](auto nepc) {
        const int nep = nepc;
#pragma unroll
        for (int r = 0; r < C::KPT; r++) {
          const int x = tid + r * TC;
          kr[r] = 0.0;
          if (!a.rhs_only && x < NV * nep) {
            const int v = x / nep, g = x - v * nep;
            kr[r] = a.kreg[v * vs + e0 * Np + g];
          }
        }
      };
      if (ne == E)
        body(std::integral_constant<int, E * Np>{});
      else
        body(ne * Np);
    };

    // epilogue of ring iteration `it` from accumulator buffer it % 2, with
    // its RK register values in kr; false when the wait for its MMAs expired
    // (on every compute warp alike)
    // D of ring iteration `it` into the rhs staging, by warps NC-4 .. NC-1
    // (lane quarter warp % 4; where the tasks do not divide evenly they carry
    // the fewer, so they read while the others finish): waits for
    // MMA(it) itself; false when that wait expired.  Lane 2j + p of quarter q
    // holds row (node NPQ q + j, operator part p).
    auto read_d = [&](int it) -> bool {
      const int db = it & 1;
      // every compute warp sees MMA(it) complete before it rewrites that
      // tile's operand image set (the non-readers' wait is short: by then
      // the MMAs are usually done)
      if (!mbar_wait(&mma_done[db], (it >> 1) & 1, lim)) return false;
      if (warp < NC - 4) return true;
      tc_fence_after();
      const int q = warp & 3, p = lane & 1, j = lane >> 1, node = C::NPQ * q + j;
      const bool on = j < C::NPQ && node < Np;
      float r[2 * NCOL];
      const unsigned row = tmem + ((unsigned)(32 * q) << 16) + db * C::D_COLS;
#pragma unroll
      for (int c = 0; c < 2 * NCOL; c += 4) tmem_ld4(row + c, r + c);
      tmem_ld_wait();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&d_free[db]);   // the accumulator is free for tile it + 2
      // part products of this row, then the partner's half: lane p takes
      // columns [p H, (p+1) H) (register indices stay compile-time)
      constexpr int H = NCOL / 2;
#pragma unroll
      for (int c = 0; c < H; c++) {
        const float lo_half = r[c] + r[NCOL + c], hi_half = r[H + c] + r[NCOL + H + c];
        const float other = __shfl_xor_sync(0xffffffffu, p ? lo_half : hi_half, 1);
        if (on) sR[(p * H + c) * Np + node] = (p ? hi_half : lo_half) + other;
      }
      return true;
    };

    // epilogue of ring iteration `it`: read_d(it) by the reader warps, then
    // (after a barrier that also carries their wait status) the update;
    // false when a wait expired (on every compute warp alike)
    auto epilogue = [&](int it) -> bool {
      const long e0 = tile_e0(it);
      const int ne = (int)min((long)E, (long)a.K - e0);
      double *bU = ring(it);
      // the staged rhs of tile it is complete (and the previous update's
      // reads of the staging happened before the readers began: the
      // iteration's first barrier separates them)
      if (!consumer_all(read_d(it), TC)) return false;
      // LSERK update over (variable, element node): staged rhs, u and the
      // RK register values, coalesced stores
      auto update = [&](auto nepc) {
        const int nep = nepc;
#pragma unroll
        for (int r = 0; r < C::KPT; r++) {
          const int x = tid + r * TC;
          if (x < NV * nep) {
            const int v = x / nep, g = x - v * nep;
            const int si = v * E * Np + g;
            const long gi = v * vs + e0 * Np + g;
            const double rhs = (double)sR[si];
            if (a.rhs_only) {
              a.u_out[gi] = rhs;
            } else {
              const double kn = a.rka * kr[r] + dt * rhs;
              const double un = bU[si] + a.rkb * kn;
              a.kreg[gi] = kn;
              a.u_out[gi] = un;
              if (keep_u) bU[si] = un;
            }
          }
        }
      };
      if (ne == E)
        update(std::integral_constant<int, E * Np>{});
      else
        update(ne * Np);
      if (keep_u) {
        // fused calc_maxv on the new state: per face, max |v|^2 and c^2 over
        // its nodes (node_speeds, as in face_maxv_kernel, so dt does not
        // depend on which kernel computed maxv)
        consumer_sync(TC);
        const double *bR = bU + C::S_U + C::S_UP;
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
            const double u1 = bU[nd], u2 = bU[E * Np + nd], u3 = bU[2 * E * Np + nd],
                         u4 = bU[3 * E * Np + nd], u5 = bU[4 * E * Np + nd];
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
            const unsigned long long bits = dbits(mv * bR[e * kRecord + 21 + f]);
            vmax = bits > vmax ? bits : vmax;
          }
        }
      }
      // this warp is done with the ring slot (generic-proxy writes precede
      // the producer's next bulk copies into it)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[it % NB]);
      return true;
    };

    for (int it = 0; ok && it < my_tiles; it++) {
      const int ne = (int)min((long)E, (long)a.K - tile_e0(it));
      // the tile's data and its node-0 terms; image set it % 2 was last read
      // by MMA(it - 2), whose completion every compute warp saw in
      // epilogue(it - 2)
      const bool w = mbar_wait(&full[it % NB], (it / NB) & 1, lim) &&
                     mbar_wait(&cen[it & 1], (it >> 1) & 1, lim);
      if (!consumer_all(w, TC)) {
        ok = false;
        break;
      }
      // the previous tile's RK register values, in flight during the tasks
      if (it > 0) load_k(it - 1);
      unsigned char *sBv = smem_raw + (it & 1) * C::B_BYTES, *sBf = sBv + C::BV_BYTES;
      for (int wt = warp; wt < C::NTASK; wt += NC) {
        if constexpr (C::NPL == 2) {
          if (wt < C::VOL_WT)
            vol_task2(it, wt, ne, sBv);
          else
            face_task2(it, wt - C::VOL_WT, ne, sBf);
        } else if constexpr (C::DF) {
          if (wt < C::VOL_WT)
            vol_task_df(it, wt, ne, sBv);
          else
            face_task(it, wt - C::VOL_WT, ne, sBf);
        } else {
          if (wt < C::VOL_WT)
            vol_task(it, wt, ne, sBv);
          else
            face_task(it, wt - C::VOL_WT, ne, sBf);
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&flux_done[it & 1]);
      if (it > 0 && !epilogue(it - 1)) {
        ok = false;
        break;
      }
    }
    if (ok && my_tiles > 0) {
      load_k(my_tiles - 1);
      if (!epilogue(my_tiles - 1)) ok = false;
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
      // bulk copies, one per lane, after lane 0 has posted the byte count
      if (lane == 0) mbar_arrive_expect_tx(&full[b], C::TX);
      __syncwarp();
      if (lane < NV)
        bulk_g2s(bU + lane * E * Np, a.u_in + lane * vs + e0 * Np, 8u * E * Np, &full[b]);
      else if (lane == NV)
        bulk_g2s(bR, a.erec + e0 * kRecord, 8u * C::S_REC, &full[b]);
      else if (lane == NV + 1)
        bulk_g2s(bT, a.tau + 4 * e0, 8u * C::S_TAU, &full[b]);
      // neighbour traces u+ = u[vmapP] into [v][e][UPS]: this lane's vmapP
      // entries are loaded before its gathers are issued
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
    // the copies of the last NB tiles land before this warp leaves
    for (int j = (it > NB ? it - NB : 0); j < it; j++) mbar_wait(&full[j % NB], (j / NB) & 1);
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else {
    // ----------------------------------------------------------- MMA warp
    // node-0 terms of ring iteration t into centre slot t & 1: lane
    // 4e + r evaluates F(u_0) of element e, then r = 0 the three volume
    // terms, r = 1..3 the face terms of faces r - 1 and (r = 3) 3
    auto centers = [&](int t) {
      const int e = lane >> 2, r = lane & 3;
      const int ne = (int)min((long)E, (long)a.K - tile_e0(t));
      const double *bU = ring(t), *bR = bU + C::S_U + C::S_UP + e * kRecord;
      double *c = sC0 + (t & 1) * C::S_C + e * NV * C::NCEN;
      if (e >= E) return;
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
    // the terms of tile t once its data has landed; false on expiry
    auto centers_of = [&](int t) -> bool {
      const bool w = mbar_wait(&full[t % NB], (t / NB) & 1, lim);
      if (w) centers(t);
      __syncwarp();
      if (lane == 0 && w) mbar_arrive(&cen[t & 1]);
      return __all_sync(0xffffffffu, w);
    };
    int nm = 0;   // tiles whose MMAs were issued and committed
    if (my_tiles > 0 && !centers_of(0)) ok = false;
    for (int it = 0; ok && it < my_tiles; it++) {
      const int b = it & 1;
      bool w = mbar_wait(&flux_done[b], (it >> 1) & 1, lim);
      // the next tile's node-0 terms while the tensor cores are idle
      if (__all_sync(0xffffffffu, w) && it + 1 < my_tiles) w = centers_of(it + 1);
      if (w && it >= 2) w = mbar_wait(&d_free[b], ((it >> 1) - 1) & 1, lim);
      if (!__all_sync(0xffffffffu, w)) {
        ok = false;
        break;
      }
      if (lane == 0) {
        tc_fence_after();
        const unsigned d = tmem + b * C::D_COLS;
        const unsigned bv = smem_u32(smem_raw + b * C::B_BYTES), bf = bv + C::BV_BYTES;
#pragma unroll 1
        for (int ks = 0; ks < C::KSV; ks++)
          tc_mma_ts(d, tmem + C::A_COL + ks * 8, smem_desc(bv + ks * 256, 128, C::SBO_V),
                    C::IDESC, ks > 0);
#pragma unroll 1
        for (int ks = 0; ks < C::KSF; ks++)
          tc_mma_ts(d, tmem + C::A_COL + C::KVA + ks * 8,
                    smem_desc(bf + ks * 256, 128, C::SBO_F), C::IDESC, 1);
        tc_commit(&mma_done[b]);
      }
      __syncwarp();
      nm++;
    }
    // the MMAs issued (and their barrier arrivals) are complete before
    // tensor and shared memory are released, on expiry too
    if (lane == 0)
      for (int t = (nm > 2 ? nm - 2 : 0); t < nm; t++) mbar_wait(&mma_done[t & 1], (t >> 1) & 1);
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
