// dglm_calc_maxv_dt_static: calc_maxv (euler_nopad_dglm.cu:7-76 /
// advec_nopad_dglm.cu:7-62) and calc_dt (:79-96) in two launches that need
// no caller-owned intermediate.  The reference, like dglm_calc_maxv +
// dglm_calc_dt, passes the per-face array maxv*Fscale between the two steps;
// here each block of the first launch reduces its faces to one partial
// maximum, kept in a file-scope device array, and a one-block second launch
// reduces the partials to dt.
//
// Scratch: g_maxv_partials, kStaticPartials doubles' worth of bit patterns
// (512 KiB), one per block of kFacesPerBlock faces, so at most
// kStaticPartials * kFacesPerBlock / 4 = 4,194,304 elements per call.  Every
// slot the second launch reads is written by the first launch of the same
// call, so nothing in the scratch has to start at zero.  Calls that overlap
// on one device (different streams or host threads) share the scratch and
// race; callers serialise them.
//
// The device address of the scratch is looked up once per device, with that
// device current, by the first call on it (cudaGetSymbolAddress, which may
// load the module); make that first call before any stream capture.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "dglm_common.cuh"

namespace dglm {
namespace {

constexpr int kStaticPartials = 65536;
constexpr int kFacesPerBlock = 256;
constexpr long kStaticMaxElements = (long)kStaticPartials * kFacesPerBlock / 4;
static_assert(kStaticMaxElements == DGLM_MAXV_DT_STATIC_MAX_ELEMENTS,
              "header limit and scratch size disagree");

static __device__ __align__(256) unsigned long long g_maxv_partials[kStaticPartials];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned long long *g_partials_ptr[kMaxDevices] = {};

struct U5 {
  const double *p[5];
};

// One thread per face: maxv as calc_maxv computes it, and the block's max of
// maxv*Fscale (as bits: non-negative doubles order like their bit patterns,
// and a NaN sorts above every finite value) into partials[blockIdx.x].
__global__ void __launch_bounds__(kFacesPerBlock)
    maxv_partials_kernel(int physics, int Np, int Nfp, long nfaces, double gamma,
                         const int *__restrict__ Fmask, const double *__restrict__ Fscale, U5 u,
                         const double *vx, const double *vy, const double *vz, double *maxv,
                         unsigned long long *partials) {
  __shared__ unsigned long long s[kFacesPerBlock / 32];
  const long f = blockIdx.x * (long)kFacesPerBlock + threadIdx.x;
  unsigned long long b = 0ull;
  if (f < nfaces) {
    const long e = f / 4;
    const int fi = (int)(f % 4);
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
    const double mv = physics == DGLM_EULER ? sqrt(mv2) + sqrt(mc2) : sqrt(mv2);
    maxv[f] = mv;
    b = dbits(mv * Fscale[f]);
  }
  b = warp_max_bits(b);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = b;
  __syncthreads();
  if (threadIdx.x < 32) {
    b = threadIdx.x < kFacesPerBlock / 32 ? s[threadIdx.x] : 0ull;
    b = warp_max_bits(b);
    if (threadIdx.x == 0) partials[blockIdx.x] = b;
  }
}

// dt = cfl/(2N+1) / max(partials[0..nparts)), as calc_dt forms it.
__global__ void __launch_bounds__(1024)
    dt_from_partials_kernel(int N, int nparts, double cfl,
                            const unsigned long long *__restrict__ partials, double *dt) {
  __shared__ unsigned long long s[32];
  unsigned long long b = 0ull;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    const unsigned long long x = partials[i];
    b = x > b ? x : b;
  }
  b = warp_max_bits(b);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = b;
  __syncthreads();
  if (threadIdx.x < 32) {
    b = threadIdx.x < blockDim.x / 32 ? s[threadIdx.x] : 0ull;
    b = warp_max_bits(b);
    if (threadIdx.x == 0) {
      const double m = __longlong_as_double((long long)b);
      *dt = (cfl / (2 * N + 1)) * (1 / m);
    }
  }
}

// Device address of the scratch on the current device (looked up once).
dglm_status partials_address(unsigned long long **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_check(e, "dglm_calc_maxv_dt_static: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(DGLM_ERR_UNSUPPORTED, "dglm_calc_maxv_dt_static: device index above 63");
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_partials_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_maxv_partials);
    if (e != cudaSuccess)
      return cuda_check(e, "dglm_calc_maxv_dt_static: cudaGetSymbolAddress of the scratch");
    g_partials_ptr[dev] = static_cast<unsigned long long *>(p);
  }
  *out = g_partials_ptr[dev];
  return DGLM_OK;
}

}  // namespace
}  // namespace dglm

using namespace dglm;

extern "C" dglm_status dglm_calc_maxv_dt_static(int physics, int N, int nelem, double gamma,
                                                double cfl, const int *Fmask,
                                                const double *Fscale, const double *const *u,
                                                const double *vx, const double *vy,
                                                const double *vz, double *maxv, double *dt_dev,
                                                void *stream) {
  if (N < 1 || N > kMaxOrder || nelem <= 0 || !Fmask || !Fscale || !maxv || !dt_dev ||
      (physics != DGLM_EULER && physics != DGLM_ADVECTION))
    return set_error(DGLM_ERR_INVALID, "dglm_calc_maxv_dt_static: bad argument");
  if (nelem > kStaticMaxElements)
    return set_error(DGLM_ERR_INVALID,
                     "dglm_calc_maxv_dt_static: nelem " + std::to_string(nelem) +
                         " is above the static scratch limit of " +
                         std::to_string(kStaticMaxElements) +
                         " elements; use dglm_calc_maxv + dglm_calc_dt");
  U5 up{};
  if (physics == DGLM_EULER) {
    if (!u) return set_error(DGLM_ERR_INVALID, "dglm_calc_maxv_dt_static: u is NULL");
    for (int v = 0; v < 5; v++) {
      if (!u[v]) return set_error(DGLM_ERR_INVALID, "dglm_calc_maxv_dt_static: u[v] is NULL");
      up.p[v] = u[v];
    }
  } else if (!vx || !vy || !vz) {
    return set_error(DGLM_ERR_INVALID, "dglm_calc_maxv_dt_static: velocity is NULL");
  }
  unsigned long long *partials = nullptr;
  dglm_status st = partials_address(&partials);
  if (st != DGLM_OK) return st;
  const long nf = 4L * nelem;
  const int nblocks = (int)((nf + kFacesPerBlock - 1) / kFacesPerBlock);
  cudaStream_t s = (cudaStream_t)stream;
  maxv_partials_kernel<<<nblocks, kFacesPerBlock, 0, s>>>(
      physics, np_of(N), nfp_of(N), nf, gamma, Fmask, Fscale, up, vx, vy, vz, maxv, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_check(e, "dglm_calc_maxv_dt_static");
  dt_from_partials_kernel<<<1, 1024, 0, s>>>(N, nblocks, cfl, partials, dt_dev);
  return cuda_check(cudaGetLastError(), "dglm_calc_maxv_dt_static");
}
