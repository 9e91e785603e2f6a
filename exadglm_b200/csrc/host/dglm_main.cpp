// dglm_main: the drop-in executable for the reference's single-GPU solver
// (dim3/src/cuda/{euler,advec}_nopad_main.cu:4-20 with its init.cu and
// DataHost/DataDev).  It reads the same datain/*.bin, runs to TMAX through
// libdglm.so, writes the same dataout/u_NNNNNNN.bin (advection) or
// u1_NNNNNNN.bin (Euler density) snapshots and prints the same line
//   tstep=%d, dt=%.8f, t=%.5f
// every print_tstep steps and at the last step, so the launcher's stdout
// parser (dglm_3d_launcher.py:316-325) reads it unchanged.
//
// The compile-time common.h parameters of the reference become flags:
//   --datain DIR --dataout DIR --physics euler|advection --tmax T
//   [--cfl 0.8] [--gamma 1.4] [--tau-scale 1.2] [--device 0]
//   [--matrix-order f|c] [--precision fp64|tf32x3|bf16x3|bf16x6] [--variant V]
// Full state and restart (not in the reference, which writes only u1):
//   --full-state            every snapshot also writes the other fields
//                           (u2..u5_NNNNNNN.bin for Euler) and t_NNNNNNN.bin
//                           (three doubles: t, the step number and the print
//                           interval, 0 before the first step)
//   --restart-dir DIR --restart-step S
//                           start from DIR's full-state snapshot of step S
//                           and continue the step numbering from there
// The initial state is datain/u0.bin (nvar x K x Np doubles) when present,
// otherwise the reference's own init_u (euler_init.cpp:5-35,
// advec_init.cpp:5-25); the advection velocity is datain/v{x,y,z}.bin when
// present, otherwise (1, 1, 1) as in advec_init.cpp.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "dglm.h"

namespace {

const double kPi = 3.14159265358979323846;

template <typename T>
bool read_bin(const std::string &path, std::vector<T> &v, size_t count, bool required = true,
              bool exact = false) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) {
    if (required) std::fprintf(stderr, "dglm_main: cannot read %s\n", path.c_str());
    return false;
  }
  const size_t bytes = (size_t)f.tellg();
  if (count == 0) count = bytes / sizeof(T);
  if (bytes < count * sizeof(T) || (exact && bytes != count * sizeof(T))) {
    std::fprintf(stderr, "dglm_main: %s holds %zu bytes, expected %zu\n", path.c_str(), bytes,
                 count * sizeof(T));
    return false;
  }
  v.resize(count);
  f.seekg(0);
  f.read(reinterpret_cast<char *>(v.data()), (std::streamsize)(count * sizeof(T)));
  return (bool)f;
}

bool write_bin(const std::string &path, const double *p, size_t n) {
  std::ofstream f(path, std::ios::binary);
  if (!f) return false;
  f.write(reinterpret_cast<const char *>(p), (std::streamsize)(n * sizeof(double)));
  return (bool)f;
}

// print interval of the reference (euler_time.cpp:4-12): the leading digit
// of (tmax/dt)/30 times its power of ten
int find_print_tstep(double tmax, double dt, int base) {
  const long interval = (long)(tmax / dt) / base;
  const std::string s = std::to_string(interval);
  const int head = s[0] - '0';
  long p = 1;
  for (size_t i = 1; i < s.size(); i++) p *= 10;
  const long r = head * p;
  return r > 0 ? (int)r : 1;
}

// name of field v (0-based) of a snapshot: u_ (advection), u1_..u5_ (Euler)
std::string field_name(int v, int tstep, bool euler) {
  const std::string s = std::to_string(tstep);
  return std::string(euler ? "u" + std::to_string(v + 1) + "_" : "u_") +
         std::string(7 - s.size(), '0') + s + ".bin";
}
std::string time_name(int tstep) {
  const std::string s = std::to_string(tstep);
  return "t_" + std::string(7 - s.size(), '0') + s + ".bin";
}

std::string snap_name(int tstep, bool euler) {
  std::string s = std::to_string(tstep);
  return std::string(euler ? "u1_" : "u_") + std::string(7 - s.size(), '0') + s + ".bin";
}

int order_from_np(long Np) {
  for (int N = 0; N < 64; N++)
    if ((long)(N + 1) * (N + 2) * (N + 3) / 6 == Np) return N;
  return -1;
}

int fail(const char *what) {
  std::fprintf(stderr, "dglm_main: %s: %s\n", what, dglm_last_error());
  return 1;
}

}  // namespace

int main(int argc, char **argv) {
  std::string datain, dataout, physics = "euler", order = "f", precision = "fp64";
  std::string restart_dir;
  double cfl = 0.8, gamma = 1.4, tau_scale = 1.2, tmax = -1;
  int device = 0, variant = -1, restart_step = -1;
  bool full_state = false;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "dglm_main: %s needs a value\n", a.c_str());
        std::exit(2);
      }
      return argv[++i];
    };
    if (a == "--datain") datain = next();
    else if (a == "--dataout") dataout = next();
    else if (a == "--physics") physics = next();
    else if (a == "--cfl") cfl = std::atof(next().c_str());
    else if (a == "--gamma") gamma = std::atof(next().c_str());
    else if (a == "--tau-scale") tau_scale = std::atof(next().c_str());
    else if (a == "--tmax") tmax = std::atof(next().c_str());
    else if (a == "--device") device = std::atoi(next().c_str());
    else if (a == "--matrix-order") order = next();
    else if (a == "--precision") precision = next();
    else if (a == "--variant") variant = std::atoi(next().c_str());
    else if (a == "--full-state") full_state = true;
    else if (a == "--restart-dir") restart_dir = next();
    else if (a == "--restart-step") restart_step = std::atoi(next().c_str());
    else {
      std::fprintf(stderr, "dglm_main: unknown argument %s\n", a.c_str());
      return 2;
    }
  }
  if (datain.empty() || dataout.empty() || tmax <= 0) {
    std::fprintf(stderr, "usage: dglm_main --datain DIR --dataout DIR --physics euler|advection "
                         "--tmax T [--cfl C] [--gamma G] [--tau-scale S] [--device D] "
                         "[--matrix-order f|c] [--precision fp64|tf32x3|bf16x3|bf16x6]\n");
    return 2;
  }
  if (physics != "euler" && physics != "advection") {
    std::fprintf(stderr, "dglm_main: unknown physics %s (euler, advection)\n", physics.c_str());
    return 2;
  }
  if (order != "c" && order != "f") {
    std::fprintf(stderr, "dglm_main: unknown matrix order %s (c, f)\n", order.c_str());
    return 2;
  }
  if (precision != "fp64" && precision != "tf32x3" && precision != "bf16x3" &&
      precision != "bf16x6") {
    std::fprintf(stderr, "dglm_main: unknown precision %s (fp64, tf32x3, bf16x3, bf16x6)\n",
                 precision.c_str());
    return 2;
  }
  if (!restart_dir.empty() && restart_step < 0) {
    std::fprintf(stderr, "dglm_main: --restart-dir needs --restart-step\n");
    return 2;
  }
  if (datain.back() != '/') datain += '/';
  if (dataout.back() != '/') dataout += '/';
  if (!restart_dir.empty() && restart_dir.back() != '/') restart_dir += '/';
  const bool euler = physics == "euler";
  const int nvar = euler ? 5 : 1;

  std::vector<int> dim;
  if (!read_bin(datain + "dim.bin", dim, 1)) return 1;
  const long K = dim[0];
  std::vector<double> WDr;
  if (!read_bin(datain + "WDr.bin", WDr, 0)) return 1;
  const long Np = (long)std::llround(std::sqrt((double)WDr.size()));
  const int N = order_from_np(Np);
  if (N < 1 || Np * Np != (long)WDr.size()) {
    std::fprintf(stderr, "dglm_main: WDr.bin is not an Np x Np operator\n");
    return 1;
  }
  const long Nfp = (long)(N + 1) * (N + 2) / 2, NF = 4 * Nfp;
  std::vector<double> WDs, WDt, LIFT, g[9], Fs, nx, ny, nz, px, py, pz;
  std::vector<int> EtoB, vmapF, vmapP, Fmask;
  const char *gn[9] = {"rx", "ry", "rz", "sx", "sy", "sz", "tx", "ty", "tz"};
  bool ok = read_bin(datain + "WDs.bin", WDs, Np * Np) && read_bin(datain + "WDt.bin", WDt, Np * Np) &&
            read_bin(datain + "LIFT.bin", LIFT, Np * NF) &&
            read_bin(datain + "Fscale.bin", Fs, 4 * K) && read_bin(datain + "nx.bin", nx, 4 * K) &&
            read_bin(datain + "ny.bin", ny, 4 * K) && read_bin(datain + "nz.bin", nz, 4 * K) &&
            read_bin(datain + "px.bin", px, K * Np) && read_bin(datain + "py.bin", py, K * Np) &&
            read_bin(datain + "pz.bin", pz, K * Np) && read_bin(datain + "EtoB.bin", EtoB, 4 * K) &&
            read_bin(datain + "vmapF.bin", vmapF, 4 * K) &&
            read_bin(datain + "vmapP.bin", vmapP, K * NF) && read_bin(datain + "Fmask.bin", Fmask, NF);
  for (int q = 0; q < 9 && ok; q++) ok = read_bin(datain + gn[q] + ".bin", g[q], K);
  if (!ok) return 1;

  // initial state and velocity
  const size_t n = (size_t)K * Np;
  std::vector<double> u0;
  std::vector<double> vel[3];
  double t0 = 0;
  int tstep0 = 0, print_tstep = 0;
  if (!restart_dir.empty()) {   // a full-state snapshot: every field and t
    u0.assign(nvar * n, 0.0);
    for (int v = 0; v < nvar; v++) {
      std::vector<double> f;
      if (!read_bin(restart_dir + field_name(v, restart_step, euler), f, n, true, true))
        return 1;
      std::copy(f.begin(), f.end(), u0.begin() + v * n);
    }
    std::vector<double> tt;
    if (!read_bin(restart_dir + time_name(restart_step), tt, 3, true, true)) return 1;
    t0 = tt[0];
    tstep0 = (int)std::llround(tt[1]);
    if (tstep0 != restart_step || !(t0 >= 0)) {
      std::fprintf(stderr, "dglm_main: %s holds step %d at t=%g, not step %d\n",
                   time_name(restart_step).c_str(), tstep0, t0, restart_step);
      return 1;
    }
    // the original run's print interval: a non-negative whole number of steps
    if (!(tt[2] >= 0) || tt[2] != std::floor(tt[2]) || tt[2] > 2147483647.0) {
      std::fprintf(stderr, "dglm_main: %s holds print interval %g, not a step count >= 0\n",
                   time_name(restart_step).c_str(), tt[2]);
      return 1;
    }
    print_tstep = (int)tt[2];   // keeps the original run's interval
  } else if (!read_bin(datain + "u0.bin", u0, nvar * n, false)) {
    u0.assign(nvar * n, 0.0);
    for (size_t i = 0; i < n; i++) {
      const double x = px[i], y = py[i], z = pz[i];
      if (euler) {   // euler_init.cpp:5-35
        const double vx = 1., vy = -0.5, vz = 1., p = 1.;
        const double r = 1 + 0.2 * std::sin(2 * kPi * (x + y + z));
        u0[i] = r;
        u0[n + i] = r * vx;
        u0[2 * n + i] = r * vy;
        u0[3 * n + i] = r * vz;
        u0[4 * n + i] = p / (gamma - 1) + 0.5 * r * (vx * vx + vy * vy + vz * vz);
      } else {       // advec_init.cpp:5-25
        u0[i] = std::sin(2 * kPi * x) * std::sin(2 * kPi * y) * std::sin(2 * kPi * z);
      }
    }
  }
  if (!euler) {
    const char *vn[3] = {"vx", "vy", "vz"};
    for (int q = 0; q < 3; q++)
      if (!read_bin(datain + vn[q] + ".bin", vel[q], n, false)) vel[q].assign(n, 1.0);
  }

  dglm_desc d{};
  d.N = N;
  d.physics = euler ? DGLM_EULER : DGLM_ADVECTION;
  d.K = (int)K;
  d.precision = precision == "tf32x3"   ? DGLM_PREC_TF32X3
                : precision == "bf16x3" ? DGLM_PREC_BF16X3
                : precision == "bf16x6" ? DGLM_PREC_BF16X6
                                        : DGLM_PREC_FP64;
  d.cfl = cfl;
  d.gamma = gamma;
  d.tau_scale = tau_scale;
  d.tmax = tmax;
  d.device = device;
  dglm_handle *h = nullptr;
  if (dglm_create(&d, &h) != DGLM_OK) return fail("create");
  if (variant >= 0 && dglm_set_variant(h, variant) != DGLM_OK) return fail("set_variant");
  dglm_mesh_arrays m{};
  m.WDr = WDr.data(); m.WDs = WDs.data(); m.WDt = WDt.data(); m.LIFT = LIFT.data();
  m.matrix_order = order == "c" ? 'c' : 'f';
  m.rx = g[0].data(); m.ry = g[1].data(); m.rz = g[2].data();
  m.sx = g[3].data(); m.sy = g[4].data(); m.sz = g[5].data();
  m.tx = g[6].data(); m.ty = g[7].data(); m.tz = g[8].data();
  m.Fscale = Fs.data(); m.nx = nx.data(); m.ny = ny.data(); m.nz = nz.data();
  m.EtoB = EtoB.data(); m.vmapF = vmapF.data(); m.vmapP = vmapP.data(); m.Fmask = Fmask.data();
  if (!euler) { m.vx = vel[0].data(); m.vy = vel[1].data(); m.vz = vel[2].data(); }
  if (dglm_upload_mesh(h, &m) != DGLM_OK) return fail("upload_mesh");
  std::vector<const double *> up(nvar);
  for (int v = 0; v < nvar; v++) up[v] = u0.data() + v * n;
  if (dglm_set_state(h, up.data(), 0) != DGLM_OK) return fail("set_state");
  if (!restart_dir.empty() && dglm_set_time(h, t0, tstep0) != DGLM_OK) return fail("set_time");

  std::vector<double> out(nvar * n);
  std::vector<double *> op(nvar);
  for (int v = 0; v < nvar; v++) op[v] = out.data() + v * n;
  // the reference's snapshot (u_ or u1_); with --full-state every field and t
  auto write_snapshot = [&](const double *u, int tstep, double t) -> bool {
    if (!write_bin(dataout + snap_name(tstep, euler), u, n)) return false;
    if (!full_state) return true;
    for (int v = 1; v < nvar; v++)
      if (!write_bin(dataout + field_name(v, tstep, euler), u + v * n, n)) return false;
    const double tt[3] = {t, (double)tstep, (double)print_tstep};
    return write_bin(dataout + time_name(tstep), tt, 3);
  };
  auto snapshot = [&](int tstep, double t) -> bool {
    if (dglm_get_state(h, op.data(), 0) != DGLM_OK) return false;
    return write_snapshot(out.data(), tstep, t);
  };
  if (restart_dir.empty() && !write_snapshot(u0.data(), 0, 0.0)) {
    std::fprintf(stderr, "dglm_main: cannot write to %s\n", dataout.c_str());
    return 1;
  }

  double t = t0, dt = 0;
  int tstep = tstep0;
  while (t < tmax) {
    const int chunk = print_tstep ? print_tstep - tstep % print_tstep : 1;
    if (dglm_step(h, chunk) != DGLM_OK) return fail("step");
    if (dglm_sync(h) != DGLM_OK) return fail("step");
    if (dglm_get_time(h, &t, &dt, &tstep) != DGLM_OK) return fail("time");
    if (tstep == tstep0) break;
    double last_dt = 0;
    if (dglm_get_dt_history(h, tstep - 1, 1, &last_dt) != DGLM_OK) return fail("time");
    if (print_tstep == 0) {
      double dt0 = 0;
      dglm_get_dt_history(h, tstep0, 1, &dt0);
      print_tstep = find_print_tstep(tmax, dt0, 30);
    }
    const bool last = !(t < tmax);
    if (tstep % print_tstep == 0 || last) {
      std::printf("tstep=%d, dt=%.8f, t=%.5f\n", tstep, last_dt, t);
      std::fflush(stdout);
      if (!snapshot(tstep, t)) return fail("snapshot");
    }
  }
  dglm_destroy(h);
  return 0;
}
