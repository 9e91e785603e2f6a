// Fixed-step C driver around the reference CPU solver (test infrastructure).
//
// Compiled by oracle/build_ref.py together with the reference's own
// dim3/src/cpp/{euler,advec}_{data,dglm,time}.cpp through a generated
// common.h; nothing from the reference is copied here.  The reference's
// main() (euler_main.cpp:4-16) loops runRK until TMAX; this driver instead
// exposes runRK (euler_time.cpp:41-107 / advec_time.cpp:224-292) for a given
// number of steps and the per-kernel calls of one right-hand side, so tests
// and the CPU-baseline leg of the benchmark can call the reference directly.
// The initial state is set by the caller, which is the reference's own
// mechanism (init.cpp is a separately linked unit).
#include "common.h"

double ref_cfl = 0.8, ref_gamma = 1.4, ref_tau_scale = 1.2, ref_tmax = 1000.0;
std::string ref_datain, ref_dataout;

static DataHost *g_host = nullptr;

#ifdef REF_EULER
static inline REAL *field(std::vector<std::vector<REAL>> &f, int v) { return f[v].data(); }
#define STATE host.p_u
#define KREG host.p_k
#define UTMP host.p_utmp
#define UB host.p_ub
#define FLR host.p_fluxR
#define FLS host.p_fluxS
#define FLT host.p_fluxT
#define FLM host.p_fluxLM
#else
static inline REAL *field(std::vector<REAL> &f, int) { return f.data(); }
#define STATE host.u
#define KREG host.k
#define UTMP host.utmp
#define UB host.ub
#define FLR host.fluxR
#define FLS host.fluxS
#define FLT host.fluxT
#define FLM host.fluxLM
#endif

extern "C" {

int ref_order() { return N; }
int ref_np() { return NP; }
int ref_nfp() { return NFP; }
int ref_nvar() { return NVAR; }

// Reads datain/*.bin through the reference's DataHost; returns nelem.
int ref_open(const char *datain, double cfl, double gamma, double tau_scale, double tmax) {
    ref_datain = datain;
    if (!ref_datain.empty() && ref_datain.back() != '/') ref_datain += '/';
    ref_dataout = ref_datain;
    ref_cfl = cfl; ref_gamma = gamma; ref_tau_scale = tau_scale; ref_tmax = tmax;
    delete g_host;
    g_host = new DataHost();
    return g_host->nelem;
}

void ref_close() { delete g_host; g_host = nullptr; }

// u: NVAR blocks of nelem*NP doubles; k is reset to zero, t and tstep too.
void ref_set_state(const double *u) {
    DataHost &host = *g_host;
    size_t n = (size_t)host.nelem * NP;
    for (int v = 0; v < NVAR; v++) {
        REAL *dst = field(STATE, v), *kk = field(KREG, v);
        for (size_t i = 0; i < n; i++) { dst[i] = u[v * n + i]; kk[i] = 0; }
    }
    host.t = 0; host.tstep = 0; host.last_tstep = false;
}

void ref_get_state(double *u) {
    DataHost &host = *g_host;
    size_t n = (size_t)host.nelem * NP;
    for (int v = 0; v < NVAR; v++) {
        const REAL *src = field(STATE, v);
        for (size_t i = 0; i < n; i++) u[v * n + i] = src[i];
    }
}

// Advection only: per-node velocity, 3 blocks (vx, vy, vz) of nelem*NP.
void ref_set_velocity(const double *vel) {
#ifdef REF_ADVEC
    DataHost &host = *g_host;
    size_t n = (size_t)host.nelem * NP;
    for (size_t i = 0; i < n; i++) {
        host.vx[i] = vel[i]; host.vy[i] = vel[n + i]; host.vz[i] = vel[2 * n + i];
    }
#else
    (void)vel;
#endif
}

// Runs nsteps of runRK (stops early once t reaches TMAX); returns steps done.
int ref_run(int nsteps) {
    DataHost &host = *g_host;
    int done = 0;
    for (; done < nsteps && host.t < TMAX; done++) runRK(host);
    return done;
}

double ref_time() { return g_host->t; }
double ref_last_dt() { return g_host->dt; }
int ref_tstep() { return g_host->tstep; }

// One right-hand side on the current state with the per-step quantities
// (maxv, dt, tau) taken from that state, in the reference's kernel order.
double ref_rhs() {
    DataHost &host = *g_host;
#ifdef REF_EULER
    calc_maxv(host.nelem, host.Fmask.data(), host.Fscale.data(), host.p_u.data(),
              host.maxv.data(), host.maxv_fs.data());
#else
    calc_maxv(host.nelem, host.Fmask.data(), host.Fscale.data(), host.vx.data(), host.vy.data(),
              host.vz.data(), host.maxv.data(), host.maxv_fs.data());
#endif
    REAL dt = calc_dt(host.nelem, host.maxv_fs.data());
    update_tau(host.nelem, host.vmapF.data(), host.maxv.data(), host.tau.data());
#ifdef REF_EULER
    update_ub(host.nelem, host.Fmask.data(), host.vmapP.data(), host.p_u.data(), host.p_ub.data());
    calc_fluxLM(host.nelem, host.t, host.Fmask.data(), host.EtoB.data(), host.nx.data(),
                host.ny.data(), host.nz.data(), host.px.data(), host.py.data(), host.pz.data(),
                host.tau.data(), host.Fscale.data(), host.p_ub.data(), host.p_u.data(),
                host.p_fluxLM.data());
    calc_fluxes(host.nelem, host.rx.data(), host.ry.data(), host.rz.data(), host.sx.data(),
                host.sy.data(), host.sz.data(), host.tx.data(), host.ty.data(), host.tz.data(),
                host.p_u.data(), host.p_fluxR.data(), host.p_fluxS.data(), host.p_fluxT.data());
    update_rhs(host.nelem, host.WDr.data(), host.WDs.data(), host.WDt.data(), host.LIFT.data(),
               host.p_fluxR.data(), host.p_fluxS.data(), host.p_fluxT.data(),
               host.p_fluxLM.data(), host.p_utmp.data());
#else
    update_ub(host.nelem, host.Fmask.data(), host.vmapP.data(), host.u.data(), host.ub.data());
    calc_fluxLM(host.nelem, host.t, host.Fmask.data(), host.EtoB.data(), host.nx.data(),
                host.ny.data(), host.nz.data(), host.px.data(), host.py.data(), host.pz.data(),
                host.vx.data(), host.vy.data(), host.vz.data(), host.tau.data(),
                host.Fscale.data(), host.ub.data(), host.u.data(), host.fluxLM.data());
    calc_fluxes(host.nelem, host.rx.data(), host.ry.data(), host.rz.data(), host.sx.data(),
                host.sy.data(), host.sz.data(), host.tx.data(), host.ty.data(), host.tz.data(),
                host.vx.data(), host.vy.data(), host.vz.data(), host.u.data(), host.fluxR.data(),
                host.fluxS.data(), host.fluxT.data());
    update_rhs(host.nelem, host.WDr.data(), host.WDs.data(), host.WDt.data(), host.LIFT.data(),
               host.fluxR.data(), host.fluxS.data(), host.fluxT.data(), host.fluxLM.data(),
               host.utmp.data());
#endif
    return dt;
}

// Copies an internal array after ref_rhs(): name is one of maxv, maxv_fs,
// tau, ub, fluxLM, fluxR, fluxS, fluxT, utmp.  Returns doubles written.
long ref_fetch(const char *name, double *out) {
    DataHost &host = *g_host;
    std::string s(name);
    auto put1 = [&](const std::vector<REAL> &a) {
        for (size_t i = 0; i < a.size(); i++) out[i] = a[i];
        return (long)a.size();
    };
    if (s == "maxv") return put1(host.maxv);
    if (s == "maxv_fs") return put1(host.maxv_fs);
    if (s == "tau") return put1(host.tau);
    size_t nv = (s == "ub" || s == "fluxLM") ? (size_t)host.nelem * NFACE * NFP
                                            : (size_t)host.nelem * NP;
    for (int v = 0; v < NVAR; v++) {
        const REAL *src = nullptr;
        if (s == "ub") src = field(UB, v);
        else if (s == "fluxLM") src = field(FLM, v);
        else if (s == "fluxR") src = field(FLR, v);
        else if (s == "fluxS") src = field(FLS, v);
        else if (s == "fluxT") src = field(FLT, v);
        else if (s == "utmp") src = field(UTMP, v);
        else return -1;
        for (size_t i = 0; i < nv; i++) out[v * nv + i] = src[i];
    }
    return (long)(NVAR * nv);
}

}  // extern "C"
