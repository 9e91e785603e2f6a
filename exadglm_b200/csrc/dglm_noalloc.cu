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
// The device address of the scratch is looked up once per device context,
// with that device current, by the first call in it (cudaGetSymbolAddress,
// which may load the module); make that first call before any stream
// capture.  The lookup is keyed on the context's unique id, so after a
// cudaDeviceReset (a new primary context, the module loaded anew) the next
// call looks the address up again instead of using the old one.
#include <cuda.h>
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
unsigned long long g_partials_ctx[kMaxDevices] = {};   // context id the address belongs to

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
    const double mv = face_max_speed(physics, Np, Nfp, gamma, Fmask, u, vx, vy, vz, f / 4,
                                     (int)(f % 4));
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

// Unique id of the current context (driver entry points looked up through
// the runtime, so the library needs no link against libcuda).
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

// false when the queries are unavailable or no context is current yet
bool current_context_id(unsigned long long *id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult q1{}, q2{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
        !f1 || !f2)
      return false;
    get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
    get_id = reinterpret_cast<CtxGetIdFn>(f2);
  }
  CUcontext ctx = nullptr;
  return get_current(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, id) == CUDA_SUCCESS;
}

// Device address of the scratch in the current context (looked up once per
// device context).
dglm_status partials_address(unsigned long long **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_check(e, "dglm_calc_maxv_dt_static: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(DGLM_ERR_UNSUPPORTED, "dglm_calc_maxv_dt_static: device index above 63");
  std::lock_guard<std::mutex> lock(g_setup_mu);
  unsigned long long ctx = 0;
  const bool have = current_context_id(&ctx);
  if (!have || !g_partials_ptr[dev] || g_partials_ctx[dev] != ctx) {
    // also makes the device's primary context current if none was yet
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_maxv_partials);
    if (e != cudaSuccess)
      return cuda_check(e, "dglm_calc_maxv_dt_static: cudaGetSymbolAddress of the scratch");
    if (!current_context_id(&ctx))
      return set_error(DGLM_ERR_CUDA, "dglm_calc_maxv_dt_static: no current CUDA context");
    g_partials_ptr[dev] = static_cast<unsigned long long *>(p);
    g_partials_ctx[dev] = ctx;
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
