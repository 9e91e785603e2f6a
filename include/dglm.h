/*
 * dglm.h -- C ABI of the B200 (sm_100a) explicit DGLM solver library
 * (libdglm.so): the right-hand side and 5-stage low-storage Runge-Kutta
 * step of ExaDGLM for linear advection (nvar = 1) and compressible Euler
 * (nvar = 5) on one tetrahedral mesh partition.
 *
 * The reference has no library interface: its single-GPU solver is a main()
 * that reads the .bin files of datain/, loops runRK() and writes dataout/ snapshots
 * (dim3/src/cuda/euler_nopad_main.cu:4-20), with kernels that take raw
 * device pointers (dim3/src/cuda/euler_nopad_dglm.cu, euler_nopad_time.cu).
 * This header is the boundary that replaces it:
 *
 *   - a solver handle (dglm_create ... dglm_destroy) that owns the device
 *     arrays the reference's DataDev owns (euler_nopad_data_dev.cu:9-266)
 *     and runs its runRK (euler_nopad_time.cu:32-108) as fused kernels;
 *   - one entry point per reference kernel (calc_maxv, calc_dt, update_tau,
 *     update_ub, calc_fluxLM, calc_fluxes, update_rhs, lserk_stage) with the
 *     reference's argument meaning, on caller-owned device arrays.
 *
 * Conventions
 *   - All pointers are plain C pointers; "device" pointers are CUDA device
 *     addresses of the current device, "host" pointers are CPU memory.
 *   - Field arrays keep the reference layout: one array per conserved
 *     variable ("per-variable pointer tables", the reference's p_u), each of
 *     K*Np doubles with node i of element e at e*Np + i.  Trace arrays (ub,
 *     fluxLM) hold K*4*Nfp doubles at (e*4 + f)*Nfp + j.
 *   - Operators WDr/WDs/WDt (Np x Np) and LIFT (Np x 4Nfp) are given with a
 *     matrix_order flag: 'c' row-major (the CPU datain) or 'f' column-major
 *     (the GPU datain, dglm_3d_launcher.py:144-147).
 *   - stream may be NULL (the legacy default stream).
 *   - Every function returns a dglm_status; dglm_last_error() gives the
 *     message of the calling thread's last failure.  Nothing prints.
 */
#ifndef DGLM_H
#define DGLM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DGLM_ABI_VERSION 1

typedef enum {
    DGLM_OK = 0,
    DGLM_ERR_INVALID = 1,      /* bad argument, size or index array */
    DGLM_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    DGLM_ERR_NONFINITE = 3,    /* NaN/Inf met in the state or in dt */
    DGLM_ERR_UNSUPPORTED = 4,  /* order / physics / precision not built */
    DGLM_ERR_STATE = 5,        /* call out of order (e.g. step before mesh) */
    DGLM_ERR_NOMEM = 6,        /* device allocation failed */
    DGLM_ERR_IO = 7            /* file read/write failed */
} dglm_status;

typedef enum { DGLM_ADVECTION = 0, DGLM_EULER = 1 } dglm_physics;

/* Arithmetic of the four operator contractions.  The state, the LSERK
 * registers, the geometric factors and the face fluxes stay FP64 in every
 * mode. */
typedef enum {
    DGLM_PREC_FP64 = 0,        /* plain method: FP64 throughout */
    DGLM_PREC_TF32X3 = 1,      /* split TF32 (2 parts) on tcgen05, FP32 accumulate; the
                                  operator-in-tensor-memory kernel forms all 4 products */
    DGLM_PREC_BF16X3 = 2,      /* split BF16 (2 parts), 3 products (4 with the
                                  operator in tensor memory), FP32 accumulate */
    DGLM_PREC_BF16X6 = 3       /* split-BF16, 3 parts (24 bits), 6 products, FP32 accumulate */
} dglm_precision;
/* In every mixed mode the Euler fluxes are centred on each element's node-0
 * flux before the split (the right-hand side is unchanged); the LSERK state,
 * the face fluxes, the metrics and the update stay FP64.  The volume fluxes
 * are FP64 too, except in the TF32 tensor-memory variant "vol=fp32-diff"
 * (the tuned pick for Euler N=4 TF32X3), which forms the centred volume
 * flux F(u_i) - F(u_0) in difference form in FP32 from u_i - u_0 (an FP64
 * subtraction), where no term cancels, to about the precision of the split. */

/* Solver description: the reference's compile-time common.h parameters
 * (dglm_3d_launcher.py:152-205) as run-time values. */
typedef struct {
    int N;             /* polynomial order (NP, NFP follow) */
    int physics;       /* dglm_physics; NVAR = 1 or 5 */
    int K;             /* number of elements (datain dim.bin) */
    int precision;     /* dglm_precision */
    double cfl;        /* CFL */
    double gamma;      /* GAMMA (Euler) */
    double tau_scale;  /* TAU_SCALE */
    double tmax;       /* TMAX: the last step is clipped to end at tmax */
    int device;        /* CUDA device ordinal (DEVID); -1 keeps the current */
} dglm_desc;

/* Mesh and operator arrays (the .bin files of datain/), all HOST pointers. */
typedef struct {
    const double *WDr, *WDs, *WDt;        /* Np x Np */
    const double *LIFT;                   /* Np x 4Nfp */
    char matrix_order;                    /* 'c' or 'f' */
    const double *rx, *ry, *rz, *sx, *sy, *sz, *tx, *ty, *tz;   /* K */
    const double *Fscale, *nx, *ny, *nz;  /* K*4 */
    const int *EtoB, *vmapF;              /* K*4 */
    const int *vmapP;                     /* K*4*Nfp */
    const int *Fmask;                     /* 4*Nfp */
    const double *vx, *vy, *vz;           /* K*Np, advection only (NULL for Euler) */
} dglm_mesh_arrays;

typedef struct dglm_handle dglm_handle;

const char *dglm_last_error(void);
int dglm_abi_version(void);
/* 1 when the library was built with kernels for order N, else 0. */
int dglm_order_supported(int N);

/* --- solver handle (replaces DataHost/DataDev + runRK + main) ------------ */
dglm_status dglm_create(const dglm_desc *desc, dglm_handle **out);
dglm_status dglm_destroy(dglm_handle *h);
dglm_status dglm_set_stream(dglm_handle *h, void *cuda_stream);
/* Validates every index array on the host (0 <= vmapP < K*Np, 0 <= vmapF <
 * 4K, 0 <= Fmask < Np) and all real arrays for NaN/Inf, then uploads. */
dglm_status dglm_upload_mesh(dglm_handle *h, const dglm_mesh_arrays *mesh);
/* u: nvar pointers to K*Np doubles (host or device per on_device).  Resets
 * t, tstep and the RK register k to zero and computes the face wave speeds
 * of the new state.  The uploaded state is checked for NaN/Inf on the
 * device (DGLM_ERR_NONFINITE).  Synchronises the handle's stream. */
dglm_status dglm_set_state(dglm_handle *h, const double *const *u, int on_device);
dglm_status dglm_get_state(dglm_handle *h, double *const *u, int on_device);
/* Advances nsteps LSERK steps (runRK) on the handle's stream without host
 * synchronisation; dt is computed on the device from the CFL condition and
 * clipped at tmax; steps requested after t reaches tmax change nothing. */
dglm_status dglm_step(dglm_handle *h, int nsteps);
/* Same with a prescribed dt (dt > 0) instead of the CFL dt. */
dglm_status dglm_step_fixed_dt(dglm_handle *h, int nsteps, double dt);
/* One LSERK stage (0..4) of the current state with a prescribed dt and the
 * handle's current tau, without the per-step dt/tau work (for timing the
 * stage kernel on its own).  Asynchronous. */
dglm_status dglm_stage(dglm_handle *h, int stage, double dt);
/* Synchronises the stream and reports device-side flags: DGLM_ERR_NONFINITE
 * for a non-finite wave speed, dt or state, DGLM_ERR_CUDA when a bounded
 * wait inside a pipelined stage kernel expired (the step's results are then
 * invalid).  The flags are cleared by dglm_set_state. */
dglm_status dglm_sync(dglm_handle *h);
/* Time, last dt and step counter (synchronises). */
dglm_status dglm_get_time(dglm_handle *h, double *t, double *dt, int *tstep);
/* Sets the simulated time and step counter after dglm_set_state, so that a
 * run restarted from a saved state continues where it stopped (t clipped at
 * tmax as usual, step numbering and dt history continuing from tstep).
 * No counterpart in the reference, which has no restart; t >= 0 and
 * tstep >= 0, else DGLM_ERR_INVALID.  Synchronises the handle's stream. */
dglm_status dglm_set_time(dglm_handle *h, double t, int tstep);
/* Runs `count` independent initial states through the handle, each for
 * nsteps CFL steps from t = 0: per member the work of dglm_set_state,
 * dglm_step and dglm_get_state, without their host synchronisations.  in[i]
 * and out[i] are HOST arrays of nvar pointers to K*Np doubles in host
 * memory.  Member i+1's host->device copy and member i-1's device->host copy
 * run on their own streams while member i computes (double-buffered device
 * copies of the states), so with page-locked host memory the transfers
 * overlap the compute and each other; no in[] buffer may overlap an out[]
 * buffer (the copies of different members run concurrently).  Returns when
 * every result is in out[]; the handle then holds the last member's state
 * and time.
 * DGLM_ERR_NONFINITE when a member's input or steps met a non-finite value,
 * with *first_bad (may be NULL) the first such member, else -1.  Holds
 * 4 state-sized device buffers from the first call on.  No counterpart in
 * the reference (one initial state per run of its executable). */
dglm_status dglm_run_ensemble(dglm_handle *h, int count, const double *const *const *in,
                              double *const *const *out, int nsteps, int *first_bad);
/* dt of steps [first, first+count) taken since dglm_set_state (synchronises);
 * the history keeps the most recent 65536 steps. */
dglm_status dglm_get_dt_history(dglm_handle *h, int first, int count, double *dt_out);
/* One right-hand side on device state u (nvar device pointers) into rhs
 * (nvar device pointers), with maxv/tau taken from u as runRK does at the
 * start of a step. */
dglm_status dglm_rhs(dglm_handle *h, const double *const *u, double *const *rhs);
/* Tile shapes ("variants") of the fused stage kernel compiled for (physics,
 * N); variant 0 is the default.  dglm_variant_describe writes a one-line
 * description such as "dmma E=16 WN=2 WM=5 threads=160 smem=104000". */
int dglm_variant_count(int physics, int N);
dglm_status dglm_variant_describe(int physics, int N, int variant, char *buf, size_t len);
/* Selects the variant used by the handle (rebuilds the operator layout). */
dglm_status dglm_set_variant(dglm_handle *h, int variant);
int dglm_get_variant(dglm_handle *h);
/* Bound, in SM clock cycles, of each hand-off wait between the warps of the
 * pipelined stage kernels (a tile's copies landing, a buffer or an MMA
 * result becoming free); 0 restores the default (2e9, about one second).
 * When a wait runs out, the CTA sets an error flag, waits (with the default
 * bound) for its own copies and MMAs in flight and leaves; dglm_sync and
 * dglm_rhs then return DGLM_ERR_CUDA and the handle's state is invalid until
 * the next dglm_set_state.  A short bound makes waits expire on purpose:
 * this is how the expiry path is tested.  No counterpart in the reference,
 * whose kernels have no waits between warps. */
dglm_status dglm_set_wait_limit(dglm_handle *h, long long cycles);
/* Compact face maps.  on = 1 builds, from the uploaded vmapP (once per mesh),
 * per face (e, f) the neighbour element and a one-byte code of the
 * neighbour's local node list (a table of at most 256 lists of Nfp node
 * indices; a conforming tetrahedral mesh has at most 24), 5 bytes per face
 * instead of 4 Nfp, and has the producer warps of the persistent stage
 * kernels (FP64 pipelined, tensor-memory TF32 and BF16) form each neighbour
 * node index from it instead of reading vmapP; the other kernels keep
 * reading vmapP.  Results are bit for bit those of vmapP.  on = 0 returns
 * to vmapP.  DGLM_ERR_UNSUPPORTED when a face's trace is not made of one
 * element's nodes or the mesh needs more than 256 node lists.  The
 * reference builds vmapP from the compact EtoE/EtoF connectivity
 * (mesh_3d_core.cpp:309-356) and its kernels read vmapP
 * (euler_nopad_dglm.cu:115-135). */
dglm_status dglm_set_compact_face_maps(dglm_handle *h, int on);
/* Distinct face node lists of the handle's compact face maps (0 before they
 * are built). */
int dglm_face_map_lists(dglm_handle *h);
/* Host only: the compact form of a vmapP (K x 4 x Nfp ints) that
 * dglm_set_compact_face_maps builds.  etoe[4e+f] is the neighbour element,
 * code[4e+f] the index of its local node list in lists (room for max_lists
 * <= 256 lists of Nfp ints), so that vmapP[e][f][j] = etoe[4e+f] Np +
 * lists[code[4e+f] Nfp + j]; *n_lists receives the number of lists.
 * DGLM_ERR_UNSUPPORTED when a face's trace spans several elements or needs
 * more than max_lists lists.  The reference derives vmapP from its EtoE/EtoF
 * tables (mesh_3d_core.cpp:309-356) and keeps no compact form. */
dglm_status dglm_compact_face_maps(int K, int Np, int Nfp, const int *vmapP, int *etoe,
                                   unsigned char *code, int *lists, int max_lists,
                                   int *n_lists);
/* Number of kernels the last dglm_step call launched (for accounting). */
long dglm_kernel_launches(dglm_handle *h);
/* Device bytes held by the handle. */
size_t dglm_device_bytes(dglm_handle *h);

/* --- per-kernel entry points (reference kernels, caller-owned device arrays)
 * Shapes as in the reference; nvar pointer tables are HOST arrays of device
 * pointers.  N selects NP/NFP.  Each launches on `stream`. */

/* euler_nopad_dglm.cu:7-76 / advec_nopad_dglm.cu:7-62.  u: nvar device
 * pointers (Euler) or NULL with vx,vy,vz (advection). */
dglm_status dglm_calc_maxv(int physics, int N, int nelem, double gamma, const int *Fmask,
                           const double *Fscale, const double *const *u, const double *vx,
                           const double *vy, const double *vz, double *maxv, double *maxv_fs,
                           void *stream);
/* euler_nopad_dglm.cu:79-96, on the device: dt = cfl/(2N+1)/max(maxv_fs),
 * written to *dt_dev (device) -- no host round trip. */
dglm_status dglm_calc_dt(int N, int nelem, double cfl, const double *maxv_fs, double *dt_dev,
                         void *stream);
/* euler_nopad_dglm.cu:99-112 */
dglm_status dglm_update_tau(int nelem, double tau_scale, const int *vmapF, const double *maxv,
                            double *tau, void *stream);
/* euler_nopad_dglm.cu:115-135 */
dglm_status dglm_update_ub(int N, int nvar, int nelem, const int *Fmask, const int *vmapP,
                           const double *const *u, double *const *ub, void *stream);
/* euler_nopad_dglm.cu:138-210 / advec_nopad_dglm.cu:120-165 */
dglm_status dglm_calc_fluxLM(int physics, int N, int nelem, double gamma, const int *Fmask,
                             const double *nx, const double *ny, const double *nz,
                             const double *tau, const double *Fscale, const double *vx,
                             const double *vy, const double *vz, const double *const *ub,
                             const double *const *u, double *const *fluxLM, void *stream);
/* euler_nopad_dglm.cu:213-266 / advec_nopad_dglm.cu:168-189.  geo: 9 device
 * pointers rx, ry, rz, sx, sy, sz, tx, ty, tz. */
dglm_status dglm_calc_fluxes(int physics, int N, int nelem, double gamma,
                             const double *const *geo, const double *vx, const double *vy,
                             const double *vz, const double *const *u, double *const *fluxR,
                             double *const *fluxS, double *const *fluxT, void *stream);
/* euler_nopad_dglm.cu:269-300 (the four cuBLAS GEMMs) as one kernel:
 * utmp = WDr fluxR + WDs fluxS + WDt fluxT - LIFT fluxLM per variable. */
dglm_status dglm_update_rhs(int N, int nvar, int nelem, const double *WDr, const double *WDs,
                            const double *WDt, const double *LIFT, char matrix_order,
                            const double *const *fluxR, const double *const *fluxS,
                            const double *const *fluxT, const double *const *fluxLM,
                            double *const *utmp, void *stream);
/* euler_nopad_time.cu:15-29 */
dglm_status dglm_lserk_stage(int N, int nvar, int nelem, double dt, double rka, double rkb,
                             const double *const *utmp, double *const *k, double *const *u,
                             void *stream);

/* No counterpart in the reference.  calc_maxv followed by calc_dt (as
 * dglm_calc_maxv + dglm_calc_dt) without the caller-owned maxv_fs array:
 * writes maxv (4*nelem doubles) and dt (*dt_dev, device).  Allocates
 * nothing: per-block partial maxima live in a 512 KiB file-scope device
 * array, so nelem is limited to DGLM_MAXV_DT_STATIC_MAX_ELEMENTS (larger
 * meshes: DGLM_ERR_INVALID).  For callers whose device memory is owned by
 * another allocator (a framework's caching pool holding the HBM) or whose
 * time loop must not call cudaMalloc/cudaFree (cudaFree synchronises the
 * device and stalls work queued on other streams), and so cannot provide
 * the 4*nelem-double intermediate.  Nothing in the scratch needs to start at
 * zero.  The first call on a device looks the scratch up (and may load the
 * module): make it before any stream capture.  Calls that overlap on one
 * device (other streams, other host threads) share the scratch and race:
 * serialise them. */
#define DGLM_MAXV_DT_STATIC_MAX_ELEMENTS 4194304
dglm_status dglm_calc_maxv_dt_static(int physics, int N, int nelem, double gamma, double cfl,
                                     const int *Fmask, const double *Fscale,
                                     const double *const *u, const double *vx,
                                     const double *vy, const double *vz, double *maxv,
                                     double *dt_dev, void *stream);

/* ---- discrete adjoint ----------------------------------------------------
 * No counterpart in the reference (it has no adjoint).  Gradients of an
 * objective of the final state with respect to the initial state, for FP64
 * handles, with dt and the face penalty tau frozen at the values of the
 * recorded forward run (both are non-smooth maxima of the state).
 *
 * dglm_adjoint_record: nsteps CFL steps (as dglm_step) from the current
 * state, storing the state every checkpoint_every steps and each step's dt
 * and tau on the device.  The state afterwards is the final state, as after
 * dglm_step.  Device memory: (ceil(nsteps/every) + 5 min(every, nsteps))
 * states plus nsteps x 4K doubles of tau (Euler).
 * dglm_adjoint_backward: lam_0 = (du_T/du_0)^T lam_T for the recorded run.
 * Each checkpoint segment is recomputed once (its 5 stage inputs per step
 * kept), then swept in reverse: one launch per stage.  nvar pointers each,
 * host or device (on_device).
 * dglm_adjoint_replay: the recorded run again from the current state with
 * the recorded dt and tau (for finite-difference checks); the simulated time
 * is not advanced.
 * dglm_adjoint_rhs: out = R'(u)^T mu on device fields, tau computed from u
 * as dglm_rhs does.  Errors: DGLM_ERR_UNSUPPORTED for mixed precision, for
 * N > 6, or for a mesh whose face points do not pair one to one. */
dglm_status dglm_adjoint_record(dglm_handle *h, int nsteps, int checkpoint_every);
dglm_status dglm_adjoint_backward(dglm_handle *h, const double *const *lam_T,
                                  double *const *lam_0, int on_device);
dglm_status dglm_adjoint_replay(dglm_handle *h);
dglm_status dglm_adjoint_rhs(dglm_handle *h, const double *const *u, const double *const *mu,
                             double *const *out);
dglm_status dglm_adjoint_tape_bytes(dglm_handle *h, size_t *bytes);
/* dglm_adjoint_record_capped: as dglm_adjoint_record, with the tape held
 * under max_bytes of device memory (the whole tape, as dglm_adjoint_tape_bytes
 * reports it) by binomial checkpointing (revolve, Griewank and Walther 2000):
 * the run is cut into chunks of `leaf` steps, `slots` state checkpoints are
 * kept, and the backward pass recomputes each chunk's stage inputs once plus
 * the fewest forward steps the slots allow.  The recording picks leaf and
 * slots for the least recomputation under the cap and places the first
 * checkpoints of the schedule while it runs.  The gradient equals that of a
 * dglm_adjoint_record recording (tau is recomputed from the recomputed
 * states, bit for bit as the forward run computed it).  DGLM_ERR_NOMEM when
 * max_bytes is below the minimum (one checkpoint and one step's stage
 * inputs); dglm_adjoint_replay is not available for capped recordings.
 * dglm_adjoint_tape_plan: leaf, slots and the forward steps the next
 * backward pass recomputes (fixed-interval recordings: checkpoint_every,
 * segments, 0).
 * dglm_adjoint_schedule: the schedule itself, for nsteps, leaf and slots
 * (host only, no device): spine[q] = chunk whose start state slot q holds
 * after the recording (slot 0: chunk 0); actions as 5 ints each, (0, src,
 * chunk, count, dst) = advance count chunks from the state of `chunk` in
 * slot src into slot dst (-1: a scratch state), (1, src, chunk, 1, -1) =
 * reverse `chunk` from its start state in slot src; prestored: whether the
 * spine checkpoints are in place (the first backward pass after a
 * recording). */
dglm_status dglm_adjoint_record_capped(dglm_handle *h, int nsteps, size_t max_bytes);
dglm_status dglm_adjoint_tape_plan(dglm_handle *h, int *leaf, int *slots,
                                   long long *advance_steps);
dglm_status dglm_adjoint_schedule(int nsteps, int leaf, int slots, int prestored, int *spine,
                                  int max_spine, int *n_spine, int *actions, int max_actions,
                                  int *n_actions, long long *advance_steps);
/* Tile shapes of the adjoint stage kernel for (physics, N); selecting one
 * drops the tape (record again). */
int dglm_adjoint_variant_count(int physics, int N);
dglm_status dglm_adjoint_variant_describe(int physics, int N, int variant, char *buf,
                                          size_t len);
dglm_status dglm_adjoint_set_variant(dglm_handle *h, int variant);

/* ---- batches of independent meshes -------------------------------------
 * No counterpart in the reference (one mesh per process there).  Linear
 * advection on many meshes of different size and order (2..6) advanced
 * together: one persistent kernel launch per LSERK stage covers every
 * instance, steps run as CUDA graphs, each instance has its own CFL dt
 * (clipped to tmax) and time.  The velocity of an instance is constant.
 * Use: dglm_batch_create, dglm_batch_add per instance (host arrays in the
 * layouts of dglm_upload_mesh; u0 has K*Np values), dglm_batch_finalize
 * (uploads, builds the tile list, computes the per-instance dt), then
 * dglm_batch_step / dglm_batch_get_state / dglm_batch_get_time. */
typedef struct dglm_batch dglm_batch;
typedef struct {
    int physics;        /* DGLM_ADVECTION */
    double cfl, tau_scale, tmax;
    int device;         /* CUDA device; -1 = current */
} dglm_batch_desc;
dglm_status dglm_batch_create(const dglm_batch_desc *desc, dglm_batch **out);
dglm_status dglm_batch_add(dglm_batch *b, int N, int K, const dglm_mesh_arrays *m,
                           const double *u0, const double *velocity, int *index);
dglm_status dglm_batch_finalize(dglm_batch *b);
dglm_status dglm_batch_step(dglm_batch *b, int nsteps);
dglm_status dglm_batch_sync(dglm_batch *b);
int dglm_batch_count(dglm_batch *b);
dglm_status dglm_batch_get_state(dglm_batch *b, int index, double *u, int on_device);
dglm_status dglm_batch_get_time(dglm_batch *b, int index, double *t, double *dt, int *tstep);
dglm_status dglm_batch_set_stream(dglm_batch *b, void *stream);
long dglm_batch_kernel_launches(dglm_batch *b);
size_t dglm_batch_device_bytes(dglm_batch *b);
dglm_status dglm_batch_destroy(dglm_batch *b);

#ifdef __cplusplus
}
#endif
#endif /* DGLM_H */
