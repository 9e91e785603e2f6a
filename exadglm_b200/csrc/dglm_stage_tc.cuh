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
//   B = the tile's fluxes in shared memory, one row per (variable, element),
//       n = v E + e, split x = hi + lo into two K-major images;
//   D = FP32 accumulators in tensor memory, double-buffered across tiles.
// Per k-step two MMAs (B hi, B lo) accumulate into the same D, so D holds
// (A_hi + A_lo)(B_hi + B_lo): all four part products.
//
// Centring.  Before the split every flux value of an element has that
// element's flux at node 0 subtracted: fluxR/S/T - metric . F(u_0) and
// fluxLM - Fscale_f n_f . F(u_0).  A constant flux has zero DG right-hand
// side (the weak volume term equals the surface term for constant data on
// straight-sided tetrahedra, to FP64 rounding), so the contraction of the
// centred fluxes IS the right-hand side, while the values that reach the
// tensor cores are the within-element variations: an order of magnitude
// smaller than the fluxes for resolved solutions, and with them the TF32
// representation and FP32 accumulation errors.
//
// K order.  Volume columns are node-group major, k = (i/4)*12 + d*4 + i%4
// (d = r, s, t), so a thread that computes nodes i, i+1 stores 8 contiguous
// bytes per (variable, direction); face columns follow at KVA + f NFPP + j.
//
// NW warps, no producer warp: thread 0 issues each tile's bulk copies (u,
// metrics, face data, vmapP) into a ring of NB buffers, and an L2 prefetch
// of its RK register, when the tile NB places earlier has released the slot
// (16 warps then keep 128 registers each).  The warps run, for tile t:
//   volume fluxes of t (and the node-0 fluxes of t+1) -> MMA volume(t)
//   wait MMA face(t-1) -> read D(t-1) from tensor memory -> LSERK update of
//   t-1 (RK register from global memory, coalesced stores)
//   face fluxes of t (neighbour traces gathered from L2) -> MMA face(t)
// so the tensor cores work on tile t while the CUDA cores finish t-1 and
// start t+1.  Every wait is bounded; on expiry the CTA sets flag bit 2,
// waits (bounded) for its MMAs and copies in flight and leaves.
#pragma once

template <int PHYS, int N, int E_, int NW_, int NB_>
struct TCfg {
  static constexpr int NV = PHYS == EUL ? 5 : 1;
  static constexpr int Np = np_of(N), Nfp = nfp_of(N), NFF = 4 * Nfp;
  static constexpr int E = E_, NW = NW_, NB = NB_;
  static constexpr int NCOL = NV * E;                    // MMA N
  static constexpr int NPQ = (Np + 3) / 4;               // output nodes per lane quarter
  static constexpr int NG = (Np + 3) / 4;                // volume node groups of 4
  static constexpr int NPAIR = 2 * NG;                   // volume node pairs
  static constexpr int KV = 12 * NG, KVA = (KV + 7) / 8 * 8;
  static constexpr int NFPP = (Nfp + 3) / 4 * 4, NFPAIR = NFPP / 2;
  static constexpr int KFA = 4 * NFPP;
  static constexpr int KT = KVA + KFA, KSV = KVA / 8, KSF = KFA / 8;
  static constexpr int SBO_V = KVA / 4 * 128, SBO_F = KFA / 4 * 128;
  static constexpr int BV_PART = NCOL / 8 * SBO_V, BF_PART = NCOL / 8 * SBO_F;
  // tensor memory: D0, D1, then the operator
  static constexpr int D_COLS = NCOL, A_COL = 2 * NCOL;
  static constexpr int TMEM_COLS = 512;
  // tile ring buffer (doubles): u [v][e][i], metrics [9][e], face data
  // [nx ny nz fs tau][e][f], vmapP [e][NFF] (ints)
  static constexpr int S_U = NV * E * Np, S_GEO = 9 * E, S_FACE = 20 * E;
  static constexpr int S_VM = (E * NFF + 1) / 2;
  static constexpr int S_BUF = S_U + S_GEO + S_FACE + S_VM;
  static constexpr unsigned TX = 8u * (S_U + S_GEO + S_FACE) + 4u * E * NFF;
  // node-0 flux terms per element: 3 volume directions + 4 faces, per variable
  static constexpr int NCEN = 7;
  static constexpr int S_C = E * NV * NCEN;
  static constexpr int IP = Np;                          // rhs staging row stride
  // warp tasks: 8 elements x 4 node pairs (volume) or 4 face-node pairs (face)
  static constexpr int NEB = E / 8, NHB = (NPAIR + 3) / 4, NJB = (NFPAIR + 3) / 4;
  static constexpr int VOL_WT = NEB * NHB, FACE_WT = NEB * 4 * NJB;
  static constexpr int THREADS = 32 * NW;
  static constexpr size_t OFF_BV = 0, OFF_BF = 2 * (size_t)BV_PART;
  static constexpr size_t OFF_RING = OFF_BF + 2 * (size_t)BF_PART;
  static constexpr size_t OFF_C = OFF_RING + 8 * (size_t)NB * S_BUF;
  static constexpr size_t OFF_BAR = OFF_C + 8 * 2 * (size_t)S_C;
  static constexpr size_t SMEM = OFF_BAR + 8 * (NB + 4) + 4 * NFF + 8 * 32 + 64;
  // instruction descriptor: F32 accumulate, TF32 A and B, both K-major, N, M = 128
  static constexpr unsigned IDESC =
      (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(NCOL >> 3) << 17) | ((128u >> 4) << 24);
  static_assert(PHYS == EUL, "the tensor-memory operator kernel is built for Euler");
  static_assert(E % 8 == 0 && NCOL % 16 == 0 && NCOL <= 256, "MMA N for M = 128");
  static_assert(2 * NPQ <= 32, "both operator parts of a quarter's nodes fit its 32 lanes");
  static_assert(2 * D_COLS + KT <= TMEM_COLS, "accumulators and operator fit tensor memory");
  static_assert(NW % 4 == 0 && NCOL % (2 * (NW / 4)) == 0, "epilogue warps split the columns");
  static_assert(E <= 32, "one lane per element computes the node-0 fluxes");
  // NB >= 3: the slot of tile t+1 is refilled by the epilogue of tile t+1-NB,
  // which runs before the node-0 fluxes of t+1 are computed
  static_assert(NB >= 3 && NB <= 4, "ring of 3..4 tile buffers");
  static_assert(2 * (size_t)BF_PART >= 8 * (size_t)NCOL * IP &&
                    2 * (size_t)BF_PART >= 8 * 8 * (size_t)E * Nfp,
                "rhs staging and wave-speed scratch fit the face operand images");
  static_assert((E * Np * 8) % 16 == 0 && (E * NFF * 4) % 16 == 0, "16-byte bulk copies");
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
  for (int i = 0; i < 4; i++) r[i] = __uint_as_float(v[i]);
}
__device__ __forceinline__ void l2_prefetch(const void *p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
// x = hi + lo as TF32 bit patterns (FP32 containers) of the FP32 value of x
__device__ __forceinline__ void split_tf32_pair(double x, unsigned &hi, unsigned &lo) {
  const float f = __double2float_rn(x);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(f));
  const float r = f - __uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

template <int PHYS, int N, int E_, int NW_, int NB_>
__global__ void __launch_bounds__(TCfg<PHYS, N, E_, NW_, NB_>::THREADS, 1)
    stage_tc_kernel(const StageArgs a, int ntiles) {
  using C = TCfg<PHYS, N, E_, NW_, NB_>;
  constexpr int NV = C::NV, Np = C::Np, Nfp = C::Nfp, NFF = C::NFF, E = C::E, NB = C::NB,
                NW = C::NW, TC = 32 * C::NW;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *sBv = smem_raw + C::OFF_BV;             // [hi image][lo image]
  unsigned char *sBf = smem_raw + C::OFF_BF;
  double *sRing = reinterpret_cast<double *>(smem_raw + C::OFF_RING);
  double *sC0 = reinterpret_cast<double *>(smem_raw + C::OFF_C);
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem_raw + C::OFF_BAR);
  unsigned long long *full = bars, *bar_v = bars + NB, *bar_f = bars + NB + 1;
  unsigned *sTmem = reinterpret_cast<unsigned *>(bars + NB + 2);
  int *sFm = reinterpret_cast<int *>(bars + NB + 4);
  unsigned long long *sMax = reinterpret_cast<unsigned long long *>(sFm + NFF + (NFF & 1));
  double *sR = reinterpret_cast<double *>(sBf);           // rhs staging, aliases the face images

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long vs = a.vs;

  if (tid == 0) {
    for (int b = 0; b < NB; b++) mbar_init(&full[b], 1);
    mbar_init(bar_v, 1);
    mbar_init(bar_f, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < NFF; i += C::THREADS) sFm[i] = a.Fmask[i];
  // the operand images start zeroed: the volume K padding [KV, KVA) is never written
  for (int i = tid; i < (int)(C::OFF_RING / 16); i += C::THREADS)
    reinterpret_cast<uint4 *>(smem_raw)[i] = make_uint4(0, 0, 0, 0);
  if (warp == 0) tmem_alloc(sTmem, C::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *sTmem;

  auto ring = [&](int it) { return sRing + (it % NB) * C::S_BUF; };

  // bulk copies of ring iteration `it` (tile blockIdx.x + it * gridDim.x)
  // into slot it % NB, completing full[it % NB]; thread 0 only
  auto load_tile = [&](int it) {
    const long t = blockIdx.x + (long)it * gridDim.x;
    const int b = it % NB;
    const long e0 = t * E;
    double *B = ring(it);
    double *bU = B, *bG = bU + C::S_U, *bF = bG + C::S_GEO, *bVm = bF + C::S_FACE;
    mbar_arrive_expect_tx(&full[b], C::TX);
    for (int v = 0; v < NV; v++)
      bulk_g2s(bU + v * E * Np, a.u_in + v * vs + e0 * Np, 8u * E * Np, &full[b]);
    for (int m = 0; m < 9; m++) bulk_g2s(bG + m * E, a.geo + m * a.gstride + e0, 8u * E, &full[b]);
    for (int q = 0; q < 3; q++)
      bulk_g2s(bF + q * 4 * E, a.nrm + q * 4 * a.gstride + 4 * e0, 32u * E, &full[b]);
    bulk_g2s(bF + 3 * 4 * E, a.fscale + 4 * e0, 32u * E, &full[b]);
    bulk_g2s(bF + 4 * 4 * E, a.tau + 4 * e0, 32u * E, &full[b]);
    bulk_g2s(bVm, a.vmapP + e0 * NFF, 4u * E * NFF, &full[b]);
    if (!a.rhs_only)
      for (int v = 0; v < NV; v++) l2_prefetch(a.kreg + v * vs + e0 * Np, 8u * E * Np);
  };
  const int my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  int loaded = 0;   // ring iterations whose copies thread 0 has issued
  if (tid == 0)
    for (; loaded < NB && loaded < my_tiles; loaded++) load_tile(loaded);

  // the operator image (128 lanes x KT TF32 columns) into tensor memory:
  // warp q < 4 writes lanes 32q .. 32q + 31
  if (warp < 4) {
    const unsigned *img = reinterpret_cast<const unsigned *>(a.AT) + (size_t)(32 * warp + lane) * C::KT;
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
  consumer_sync(TC);
  tc_fence_after();

  const double dt = a.dt_override >= 0 ? a.dt_override : a.sc->dt;
  const double gam = a.gamma;
  const bool keep_u = PHYS == EUL && a.last_stage && !a.rhs_only;
  unsigned long long vmax = 0ull;
  int nv_issued = 0, nf_issued = 0, nv_done = 0, nf_done = 0;

  // node-0 fluxes of the tile in ring slot `it` (lane e < E): the volume
  // terms metric_d . F(u_0) and the face terms Fscale_f n_f . F(u_0)
  auto centers = [&](int it, long e0) -> bool {
    const bool ok = mbar_wait(&full[it % NB], (it / NB) & 1, a.wait_cycles);
    const int e = lane;
    if (ok && e < E) {
      const int ne = (int)min((long)E, (long)a.K - e0);
      const double *bU = ring(it), *bG = bU + C::S_U, *bF = bG + C::S_GEO;
      double *c = sC0 + (it & 1) * C::S_C + e * NV * C::NCEN;
      if (e < ne) {
        double q[5], F[5], G[5], W[5];
#pragma unroll
        for (int v = 0; v < 5; v++) q[v] = bU[v * E * Np + e * Np];
        euler_flux_fast(gam, q, F, G, W);
        double m[9];
#pragma unroll
        for (int i = 0; i < 9; i++) m[i] = bG[i * E + e];
        double nf[4][4];
#pragma unroll
        for (int f = 0; f < 4; f++)
#pragma unroll
          for (int x = 0; x < 4; x++) nf[f][x] = bF[x * 4 * E + e * 4 + f];
#pragma unroll
        for (int v = 0; v < 5; v++) {
#pragma unroll
          for (int d = 0; d < 3; d++)
            c[v * C::NCEN + d] = m[3 * d] * F[v] + m[3 * d + 1] * G[v] + m[3 * d + 2] * W[v];
#pragma unroll
          for (int f = 0; f < 4; f++)
            c[v * C::NCEN + 3 + f] =
                (nf[f][0] * F[v] + nf[f][1] * G[v] + nf[f][2] * W[v]) * nf[f][3];
        }
      } else {
#pragma unroll
        for (int x = 0; x < NV * C::NCEN; x++) c[x] = 0.0;
      }
    }
    return ok;
  };

  // volume fluxes of the tile in ring slot `it`, warp task wt: 8 elements x
  // 4 node pairs, centred and split into the two volume images
  auto vol_task = [&](int it, int wt, int ne) {
    const int eb = wt / C::NHB, hb = wt - eb * C::NHB;
    const int e = eb * 8 + (lane & 7), h = hb * 4 + (lane >> 3);
    if (h >= C::NPAIR) return;
    const bool live = e < ne;
    const double *bU = ring(it), *bG = bU + C::S_U;
    const double *cen = sC0 + (it & 1) * C::S_C + e * NV * C::NCEN;
    double m[9];
#pragma unroll
    for (int i = 0; i < 9; i++) m[i] = bG[i * E + e];
    unsigned h0[5][3], l0[5][3];
#pragma unroll
    for (int r = 0; r < 2; r++) {
      const int i = 2 * h + r;
      const bool ok = live && i < Np;
      double F[5], G[5], W[5];
      if (ok) {
        double q[5];
#pragma unroll
        for (int v = 0; v < 5; v++) q[v] = bU[v * E * Np + e * Np + i];
        euler_flux_fast(gam, q, F, G, W);
      }
#pragma unroll
      for (int v = 0; v < 5; v++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
          unsigned hi = 0u, lo = 0u;
          if (ok)
            split_tf32_pair(m[3 * d] * F[v] + m[3 * d + 1] * G[v] + m[3 * d + 2] * W[v] -
                                cen[v * C::NCEN + d],
                            hi, lo);
          if (r == 0) {
            h0[v][d] = hi;
            l0[v][d] = lo;
          } else {
            const int n = v * E + e, k0 = (h >> 1) * 12 + d * 4 + (h & 1) * 2;
            const int off = (n >> 3) * C::SBO_V + (k0 >> 2) * 128 + (n & 7) * 16 + (k0 & 3) * 4;
            *reinterpret_cast<uint2 *>(sBv + off) = make_uint2(h0[v][d], hi);
            *reinterpret_cast<uint2 *>(sBv + C::BV_PART + off) = make_uint2(l0[v][d], lo);
          }
        }
    }
  };

  // face fluxes of the tile in ring slot `it`, warp task wt: 8 elements x 4
  // face-node pairs of one face; neighbour traces gathered from global memory
  auto face_task = [&](int it, int wt, int ne) {
    const int eb = wt / (4 * C::NJB), f = (wt / C::NJB) & 3, jb = wt % C::NJB;
    const int e = eb * 8 + (lane & 7), jp = jb * 4 + (lane >> 3);
    if (jp >= C::NFPAIR) return;
    const bool live = e < ne;
    const double *bU = ring(it), *bF = bU + C::S_U + C::S_GEO;
    const int *bVm = reinterpret_cast<const int *>(bF + C::S_FACE);
    const double *cen = sC0 + (it & 1) * C::S_C + e * NV * C::NCEN + 3 + f;
    const double nx = bF[0 * 4 * E + e * 4 + f], ny = bF[1 * 4 * E + e * 4 + f],
                 nz = bF[2 * 4 * E + e * 4 + f], fs = bF[3 * 4 * E + e * 4 + f],
                 tau = bF[4 * 4 * E + e * 4 + f];
    // both nodes' neighbour values are requested before either is used
    double qp[2][5];
    int nodeM[2];
    bool ok[2];
#pragma unroll
    for (int r = 0; r < 2; r++) {
      const int j = 2 * jp + r;
      ok[r] = live && j < Nfp;
      const int fj = f * Nfp + (ok[r] ? j : 0);
      nodeM[r] = sFm[fj];
      const long idxP = ok[r] ? bVm[e * NFF + fj] : 0;
#pragma unroll
      for (int v = 0; v < 5; v++) qp[r][v] = ok[r] ? __ldg(a.u_in + v * vs + idxP) : 0.0;
    }
    unsigned hv[2][5], lv[2][5];
#pragma unroll
    for (int r = 0; r < 2; r++) {
      double qm[5], qb[5], F[5], G[5], W[5];
#pragma unroll
      for (int v = 0; v < 5; v++) {
        qm[v] = ok[r] ? bU[v * E * Np + e * Np + nodeM[r]] : 1.0;
        qb[v] = 0.5 * (qm[v] + (ok[r] ? qp[r][v] : 1.0));
      }
      euler_flux_fast(gam, qb, F, G, W);
#pragma unroll
      for (int v = 0; v < 5; v++) {
        hv[r][v] = lv[r][v] = 0u;
        if (ok[r]) {
          const double nd = nx * F[v] + ny * G[v] + nz * W[v];
          split_tf32_pair((nd - tau * (qb[v] - qm[v])) * fs - cen[v * C::NCEN], hv[r][v],
                          lv[r][v]);
        }
      }
    }
    const int k0 = f * C::NFPP + 2 * jp;
#pragma unroll
    for (int v = 0; v < 5; v++) {
      const int n = v * E + e;
      const int off = (n >> 3) * C::SBO_F + (k0 >> 2) * 128 + (n & 7) * 16 + (k0 & 3) * 4;
      *reinterpret_cast<uint2 *>(sBf + off) = make_uint2(hv[0][v], hv[1][v]);
      *reinterpret_cast<uint2 *>(sBf + C::BF_PART + off) = make_uint2(lv[0][v], lv[1][v]);
    }
  };

  // MMAs of one region into accumulator buffer `db`, issued by thread 0
  auto issue = [&](bool vol, int db) {
    if (tid != 0) return;
    tc_fence_after();
    const unsigned d = tmem + db * C::D_COLS;
    const unsigned base = smem_u32(vol ? sBv : sBf);
    const int nks = vol ? C::KSV : C::KSF, sbo = vol ? C::SBO_V : C::SBO_F;
    const unsigned part = vol ? C::BV_PART : C::BF_PART;
    const unsigned acol = tmem + C::A_COL + (vol ? 0 : C::KVA);
#pragma unroll 1
    for (int ks = 0; ks < nks; ks++) {
      const unsigned long long bh = smem_desc(base + ks * 256, 128, sbo);
      const unsigned long long bl = smem_desc(base + part + ks * 256, 128, sbo);
      tc_mma_ts(d, acol + ks * 8, bh, C::IDESC, (vol && ks == 0) ? 0 : 1);
      tc_mma_ts(d, acol + ks * 8, bl, C::IDESC, 1);
    }
    tc_commit(vol ? bar_v : bar_f);
  };

  // epilogue of the tile in ring slot `it` (elements e0.., ne of them) from
  // accumulator buffer `db`: tensor memory -> rhs staging -> LSERK update
  auto epilogue = [&](int it, long e0, int ne, int db) {
    // 1. warp w reads lane quarter w % 4, columns [s CPS, (s+1) CPS) with
    //    s = w / 4; lane 2j + p holds part p of node NPQ (w % 4) + j
    constexpr int NSL = NW / 4, CPS = C::NCOL / NSL, HALF = CPS / 2;
    const int q = warp & 3, s = warp >> 2;
    float r[CPS];
#pragma unroll
    for (int c = 0; c < CPS; c += 4)
      tmem_ld4(tmem + ((unsigned)(32 * q) << 16) + db * C::D_COLS + s * CPS + c, r + c);
    tmem_ld_wait();
    tc_fence_before();
    const int p = lane & 1, j = lane >> 1, node = C::NPQ * q + j;
    const bool on = j < C::NPQ && node < Np;
#pragma unroll
    for (int c = 0; c < HALF; c++) {
      const float mine = p ? r[c + HALF] : r[c];
      const float other = __shfl_xor_sync(0xffffffffu, p ? r[c] : r[c + HALF], 1);
      const int col = s * CPS + c + p * HALF;
      if (on) sR[col * C::IP + node] = (double)(mine + other);
    }
    consumer_sync(TC);
    // 2. LSERK update, one flat loop over (variable, element, node)
    double *bU = ring(it);
    auto items = [&](const int nep) {
      constexpr int IPT = (NV * E * Np + TC - 1) / TC;
      double kr[IPT];
#pragma unroll
      for (int u = 0; u < IPT; u++) {
        const int vg = tid + u * TC;
        kr[u] = 0.0;
        if (vg < NV * nep && !a.rhs_only) {
          const int v = vg / nep, g = vg - v * nep;
          kr[u] = a.kreg[v * vs + e0 * Np + g];
        }
      }
#pragma unroll
      for (int u = 0; u < IPT; u++) {
        const int vg = tid + u * TC;
        if (vg >= NV * nep) continue;
        const int v = vg / nep, g = vg - v * nep;
        const int e = g / Np, i = g - e * Np;
        const long gi = v * vs + e0 * Np + g;
        const double rhs = sR[(v * E + e) * C::IP + i];
        if (a.rhs_only) {
          a.u_out[gi] = rhs;
        } else {
          const double kn = a.rka * kr[u] + dt * rhs;
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
    if (keep_u) {
      // fused calc_maxv on the new state: |v|^2 and c^2 at every face node
      // (scratch over the rhs staging), then the per-face max
      consumer_sync(TC);
      const double *bF = bU + C::S_U + C::S_GEO;
      double *sW = sR;
      for (int x = tid; x < 4 * E * Nfp; x += TC) {
        const int fe = x / Nfp, jj = x - fe * Nfp, f = fe / E, e = fe - f * E;
        double v2 = 0.0, c2 = 0.0;
        if (e < ne) {
          const int nd = e * Np + sFm[f * Nfp + jj];
          const double u1 = bU[nd], u2 = bU[E * Np + nd], u3 = bU[2 * E * Np + nd],
                       u4 = bU[3 * E * Np + nd], u5 = bU[4 * E * Np + nd];
          // divisions as in face_maxv_kernel, so dt does not depend on which
          // kernel computed maxv
          const double vx = u2 / u1, vy = u3 / u1, vz = u4 / u1;
          v2 = vx * vx + vy * vy + vz * vz;
          const double pres = (gam - 1) * (u5 - 0.5 * u1 * v2);
          c2 = fabs(gam * pres / u1);
        }
        sW[2 * x] = v2;
        sW[2 * x + 1] = c2;
      }
      consumer_sync(TC);
      for (int x = tid; x < 4 * E; x += TC) {
        const int f = x / E, e = x - f * E;
        if (e >= ne) continue;
        double mv2 = 0.0, mc2 = 0.0;
        bool bad = false;
        for (int jj = 0; jj < Nfp; jj++) {
          const double v2 = sW[2 * (x * Nfp + jj)], c2 = sW[2 * (x * Nfp + jj) + 1];
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
    // the ring slot is free: its generic-proxy writes precede the bulk copies
    // of the tile NB iterations on, which thread 0 issues into it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    consumer_sync(TC);   // the staging (face images) is free for the next face phase
    if (tid == 0 && it + NB < my_tiles) {
      load_tile(it + NB);
      loaded = it + NB + 1;
    }
  };

  bool ok = true;
  const int t0 = blockIdx.x;
  if (t0 < ntiles) ok = consumer_all(warp != 0 || centers(0, (long)t0 * E), TC);
  int it = 0;
  long pe0 = 0;
  int pne = 0;
  for (int t = t0; ok && t < ntiles; t += gridDim.x, it++) {
    const long e0 = (long)t * E;
    const int ne = (int)min((long)E, (long)a.K - e0);
    // tile data landed; MMA volume(t-1) has read the volume images
    bool w = mbar_wait(&full[it % NB], (it / NB) & 1, a.wait_cycles);
    if (it > 0) w = w && mbar_wait(bar_v, (it - 1) & 1, a.wait_cycles);
    if (!consumer_all(w, TC)) {
      ok = false;
      break;
    }
    if (it > 0) nv_done++;
    // volume fluxes of t; one more warp task computes the node-0 fluxes of t+1
    const bool more = t + (int)gridDim.x < ntiles;
    bool cok = true;
    for (int wt = warp; wt < C::VOL_WT + 1; wt += NW) {
      if (wt < C::VOL_WT)
        vol_task(it, wt, ne);
      else if (more)
        cok = centers(it + 1, e0 + (long)gridDim.x * E);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    if (!consumer_all(cok, TC)) {
      ok = false;
      break;
    }
    issue(true, it & 1);
    nv_issued++;
    if (it > 0) {
      // MMA face(t-1) complete: accumulator (it-1)&1 is final, face images free
      if (!consumer_all(mbar_wait(bar_f, (it - 1) & 1, a.wait_cycles), TC)) {
        ok = false;
        break;
      }
      nf_done++;
      tc_fence_after();
      epilogue(it - 1, pe0, pne, (it - 1) & 1);
    }
    for (int wt = warp; wt < C::FACE_WT; wt += NW) face_task(it, wt, ne);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    consumer_sync(TC);
    issue(false, it & 1);
    nf_issued++;
    pe0 = e0;
    pne = ne;
  }
  if (ok && it > 0) {
    if (consumer_all(mbar_wait(bar_f, (it - 1) & 1, a.wait_cycles), TC)) {
      nf_done++;
      nv_done = nv_issued;
      tc_fence_after();
      epilogue(it - 1, pe0, pne, (it - 1) & 1);
    } else {
      ok = false;
    }
  }
  if (!ok && tid == 0) {
    atomicOr(&a.sc->flags, 4);
    // MMAs and bulk copies still in flight finish before the CTA releases
    // its tensor memory and shared memory
    if (nf_issued > nf_done) mbar_wait(bar_f, (nf_issued - 1) & 1);
    if (nv_issued > nv_done) mbar_wait(bar_v, (nv_issued - 1) & 1);
    for (int j = (loaded > NB ? loaded - NB : 0); j < loaded; j++)
      mbar_wait(&full[j % NB], (j / NB) & 1);
  }
  if (keep_u) {
    vmax = warp_max_bits(vmax);
    if (lane == 0) sMax[warp] = vmax;
    consumer_sync(TC);
    if (tid < 32) {
      unsigned long long v = tid < NW ? sMax[tid] : 0ull;
      v = warp_max_bits(v);
      if (tid == 0) atomicMax(&a.sc->acc[a.sc->parity ^ 1], v);
    }
  }
  tc_fence_before();
  consumer_sync(TC);
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, C::TMEM_COLS);
  }
}
