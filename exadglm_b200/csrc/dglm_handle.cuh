// Internal: the solver handle and the helpers shared by the translation
// units that operate on it (dglm_solver.cu, dglm_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "dglm_common.cuh"

struct AdjointTape;

struct dglm_handle {
  dglm_desc d{};
  int nvar = 0, Np = 0, Nfp = 0, NFF = 0;
  int variant = 0;
  dglm::StageVariantInfo vinfo{};
  std::vector<double> Ahost;      // stacked [WDr WDs WDt -LIFT], Np x (3Np+NFF) row-major
  long vs = 0;                    // doubles between variables of a field
  long Kp = 0;                    // K rounded up to a multiple of 64 (tile padding)
  int dev = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // mesh, operators
  double *AT = nullptr, *geo = nullptr, *fscale = nullptr, *nrm = nullptr;
  double *tau = nullptr, *maxv = nullptr, *vel = nullptr;
  int *vmapP = nullptr, *vmapF = nullptr, *Fmask = nullptr;
  // per-element record [Kp][kRecord] (TF32x3 and BF16x3 Euler handles): the 9 metrics,
  // nx, ny, nz and Fscale of the 4 faces, one pad double; one bulk copy per
  // tile in the tensor-memory kernel
  double *erec = nullptr;
  // compact face maps (dglm_set_compact_face_maps), built from vmapP on first
  // use: per face the neighbour element and a code of its node list
  int *etoe = nullptr, *ftab = nullptr;
  unsigned char *fcode = nullptr;
  int ftab_lists = 0;
  bool compact_built = false, compact = false;
  // state
  double *u[2] = {nullptr, nullptr};
  double *kreg = nullptr;
  int cur = 0;
  dglm::DevScalars *sc = nullptr;
  double *dt_hist = nullptr;
  // one-off right-hand side evaluation
  double *rhs_in = nullptr, *rhs_out = nullptr, *maxv_s = nullptr, *tau_s = nullptr;
  dglm::DevScalars *sc_s = nullptr;
  bool mesh_ready = false, state_ready = false;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  long launches = 0;
  size_t bytes = 0;
  std::vector<void *> allocs;
  long long wait_cycles = 0;     // > 0: shortened hand-off wait bound (dglm_set_wait_limit)
  AdjointTape *tape = nullptr;   // discrete adjoint (dglm_adjoint.cu)
  int adj_variant = 0;           // adjoint tile shape
  // dglm_run_ensemble: double-buffered device copies of the members' input
  // and output states, a copy-in and a copy-out stream, and their events
  // (in_ready[2], in_free[2], out_ready[2], out_free[2])
  double *ens_in[2] = {nullptr, nullptr}, *ens_out[2] = {nullptr, nullptr};
  int *ens_flags = nullptr;
  int ens_cap = 0;
  cudaStream_t ens_cin = nullptr, ens_cout = nullptr;
  cudaEvent_t ens_ev[8] = {};
};


namespace dglm {

// Carpenter & Kennedy 5-stage 4th-order 2N-storage coefficients
// (euler_data.cpp:41-60).
constexpr double RKA[5] = {0.0, -567301805773.0 / 1357537059087.0,
                       -2404267990393.0 / 2016746695238.0, -3550918686646.0 / 2091501179385.0,
                       -1275806237668.0 / 842570457699.0};
constexpr double RKB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                       1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                       2277821191437.0 / 14882151754819.0};

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (dev >= 0 && dev != prev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

template <typename T>
inline dglm_status dalloc(dglm_handle *h, T **p, size_t count) {
  void *q = nullptr;
  const size_t n = count * sizeof(T);
  cudaError_t e = cudaMalloc(&q, n ? n : 16);
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(DGLM_ERR_NOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
  }
  h->allocs.push_back(q);
  h->bytes += n;
  *p = static_cast<T *>(q);
  return DGLM_OK;
}

StageArgs stage_args(dglm_handle *h, const double *u_in, double *u_out, int s);
void free_tape(dglm_handle *h);
dglm_status run_steps(dglm_handle *h, int nsteps);
dglm_status issue_step_ptrs(dglm_handle *h, const double *const *in, double *const *out,
                            cudaStream_t s);
dglm_status ensure_rhs_scratch(dglm_handle *h);

}  // namespace dglm
