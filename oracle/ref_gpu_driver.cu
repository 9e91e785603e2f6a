// Fixed-step C driver around the reference GPU solver (test and benchmark
// infrastructure: the second baseline, the reference's own CUDA + cuBLAS
// path on the same GPU).
//
// Compiled by oracle/build_ref.py together with the reference's own
// dim3/src/cuda/euler_nopad_{data_host,data_dev,dglm,time}.cu through a
// generated common.h (the launcher's macros, dglm_3d_launcher.py:410-456);
// nothing from the reference is copied here.  The reference's main()
// (euler_nopad_main.cu:4-20) loops runRK until TMAX and writes snapshots;
// this driver exposes runRK (euler_nopad_time.cu:32-108) for a given number of
// steps, with the initial state set by the caller instead of init_u
// (euler_nopad_init.cu, a separately linked unit in the reference).
#include "common.h"

std::string ref_datain, ref_dataout;

static DataHost *g_host = nullptr;
static DataDev *g_dev = nullptr;

extern "C" {

int ref_gpu_order() { return N; }
int ref_gpu_np() { return NP; }
int ref_gpu_nvar() { return NVAR; }
double ref_gpu_cfl() { return CFL; }
double ref_gpu_gamma() { return GAMMA; }
double ref_gpu_tau_scale() { return TAU_SCALE; }

// Reads datain/*.bin ('f' matrix order) through the reference's DataHost and
// uploads it with its DataDev; returns nelem.
int ref_gpu_open(const char *datain) {
    ref_datain = datain;
    if (!ref_datain.empty() && ref_datain.back() != '/') ref_datain += '/';
    ref_dataout = ref_datain;
    delete g_dev;
    delete g_host;
    g_host = new DataHost();
    g_dev = new DataDev(*g_host);
    return g_host->nelem;
}

void ref_gpu_close() {
    delete g_dev;
    delete g_host;
    g_dev = nullptr;
    g_host = nullptr;
}

// u: NVAR host blocks of nelem*NP doubles; k, t and tstep are reset.
int ref_gpu_set_state(const double *u) {
    DataHost &host = *g_host;
    DataDev &dev = *g_dev;
    const size_t n = (size_t)host.nelem * NP;
    for (int v = 0; v < NVAR; v++) {
        cudaMemcpy(dev.p_u[v], u + v * n, n * sizeof(REAL), cudaMemcpyHostToDevice);
        cudaMemset(dev.p_k[v], 0, n * sizeof(REAL));
    }
    host.t = 0;
    host.tstep = 0;
    host.last_tstep = false;
    return (int)cudaDeviceSynchronize();
}

int ref_gpu_get_state(double *u) {
    DataHost &host = *g_host;
    DataDev &dev = *g_dev;
    const size_t n = (size_t)host.nelem * NP;
    for (int v = 0; v < NVAR; v++)
        cudaMemcpy(u + v * n, dev.p_u[v], n * sizeof(REAL), cudaMemcpyDeviceToHost);
    return (int)cudaDeviceSynchronize();
}

// Runs nsteps of runRK (stops early once t reaches TMAX) and waits for the
// device; returns the steps done, or -1 on a CUDA error.
int ref_gpu_run(int nsteps) {
    DataHost &host = *g_host;
    DataDev &dev = *g_dev;
    int done = 0;
    for (; done < nsteps && host.t < TMAX; done++) runRK(host, dev);
    if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) return -1;
    return done;
}

double ref_gpu_time() { return g_host->t; }
double ref_gpu_last_dt() { return g_host->dt; }
int ref_gpu_tstep() { return g_host->tstep; }

}  // extern "C"
