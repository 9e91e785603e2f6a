#!/usr/bin/env python
"""Benchmark: Euler N=4 DOF-stage updates per second on a B200.

Workload (the headline configuration): compressible Euler, gamma 1.4,
periodic unit cube of 32^3 hexahedra x 6 = 196,608 tetrahedra, N=4 (Np=35),
5 conserved variables, rho = 1 + 0.2 sin(2 pi (x+y+z)), v = (1, 0.5, 0.25),
p = 1, CFL 0.4, FP64.  Synthetic: the mesh and state are generated here.

A bench "step" is one LSERK time step (5 stages) over the whole mesh.
DOF-stages per step = K * Np * 5 variables * 5 stages.

Arms:
  default            libdglm.so: state resident in HBM, steps as captured
                     CUDA graphs (value); e2e through the C ABI with the state
                     copied host->device and back every step, the copies of
                     neighbouring steps overlapped with the compute
                     (dglm_run_ensemble; e2e), and the same as separate
                     set-state / step / get-state calls (e2e.serial).
  --impl reference   the reference's own CPU solver (oracle/_ref, compiled
                     from its sources) on this machine's cores; falls back to
                     the oracle's C restatement when oracle/_ref is absent.

Multi-GPU (torchrun): every rank advances its own replica of the workload
("replicas only": the single-partition path has no exchange step); value is
the sum over ranks of DOF-stages divided by the max over ranks of the time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Euler N=4 DOF-stage/s (FP64)"
UNIT = "DOF-stage/s"
NOMINAL_FP64_TFLOPS = 40.0     # B200 datasheet FP64 (vector and tensor)
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=32, help="hexahedra per axis (K = 6 n^3)")
    ap.add_argument("--order", type=int, default=4)
    ap.add_argument("--precision", default="fp64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only", choices=["fp64", "mixed", "face_maps", "adjoint", "batch",
                                       "precision",
                                       "gpu_baseline"],
                    default=None,
                    help="run one section alone (profiling); prints that section's object")
    ap.add_argument("--accuracy-steps", type=int, default=200,
                    help="steps of the mixed-vs-FP64 relative L2 comparison")
    ap.add_argument("--adjoint-n", type=int, default=16,
                    help="hexahedra per axis of the adjoint workload (K = 6 n^3)")
    ap.add_argument("--adjoint-steps", type=int, default=500)
    ap.add_argument("--adjoint-every", type=int, default=50, help="checkpoint spacing")
    ap.add_argument("--adjoint-caps-gib", default="2,8",
                    help="tape caps (GiB) of the capped (binomial checkpointing) adjoint runs")
    ap.add_argument("--adjoint-large-cap-gib", type=float, default=16.0,
                    help="tape cap of the capped adjoint at the headline size (0: skip)")
    ap.add_argument("--batch-count", type=int, default=256, help="instances of the batch workload")
    ap.add_argument("--precision-n", type=int, default=48,
                    help="hexahedra per axis of the N=6 precision study (K = 6 n^3)")
    ap.add_argument("--batch-steps", type=int, default=100)
    ap.add_argument("--batch-sequential", type=int, default=256,
                    help="instances also run one by one through single-mesh handles")
    return ap.parse_args()


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return FALLBACK_PEAKS, "fallback"


def bytes_per_element_stage(nvar, Np, Nfp, advection=False):
    """Algorithmic HBM bytes per element-stage of the fused design: read u,
    write u', read k, write k; 9 metrics + 4 Fscale + 12 normals + 4 tau;
    vmapP (int32); advection adds the per-node velocity."""
    b = 4 * nvar * Np * 8 + 29 * 8 + 4 * 4 * Nfp
    if advection:
        b += 3 * Np * 8
    return b


def flops_per_element_stage(nvar, Np, Nfp):
    """FMA = 2 flops; the three volume and the LIFT contractions only."""
    return nvar * (6 * Np * Np + 2 * Np * 4 * Nfp)


def variant_shape(desc):
    """A variant description without its smem=<bytes> field (the shared-memory
    size moves with layout changes that leave the tile shape alone)."""
    return " ".join(w for w in desc.split() if not w.startswith("smem="))


def read_traffic(desc, K):
    """Per-launch DRAM bytes of the stage kernel variant `desc` on a K-element
    mesh, from the committed ncu summaries (profiles/stage_traffic.txt: lines
    '<K> <bytes_per_launch> <variant shape>').  A capture on a smaller mesh of
    the same variant is scaled by K (these kernels stream each element's data
    once per launch, so their DRAM traffic grows in proportion to K).  None
    when the variant has no capture."""
    path = os.path.join(ROOT, "profiles", "stage_traffic.txt")
    if not os.path.exists(path):
        return None
    want = variant_shape(desc)
    scaled = None
    with open(path) as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            parts = line.split(None, 2)
            if len(parts) != 3 or parts[2].strip() != want:
                continue
            try:
                k0, b0 = int(parts[0]), float(parts[1])
            except ValueError:
                continue
            if k0 == K:
                return b0
            scaled = b0 * K / k0
    return scaled


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_problem(a):
    from exadglm_b200 import problem as P
    return P.euler_sine(n=a.n, N=a.order, cfl=0.4)


def workload_config(a, p, world):
    """The `config` object of both arms' JSON lines."""
    return {"workload": f"euler_sine N={p.N} K={p.K} (n={a.n}^3 x 6) CFL 0.4, "
                        f"{a.precision}, one replica per GPU",
            "K": p.K, "N": p.N, "Np": p.Np, "nvar": p.nvar, "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (state 3 x 275 MB)"}


def dof_stages_per_step(p):
    return p.K * p.Np * p.nvar * 5


def cpu_reference_rate(p, steps, threads=None):
    """Time `steps` LSERK steps of the reference CPU solver (or the oracle
    port) on this host.  Returns (rate, kind, cores, seconds)."""
    import oracle
    threads = threads or os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    if oracle.ref_available(p.physics, p.N):
        r = oracle.RefSolver(p)
        r.run(1)                                  # warm the caches / page in
        r.set_state(p.u0)
        t0 = time.perf_counter()
        done = r.run(steps)
        dt = time.perf_counter() - t0
        r.close()
        kind = "reference"
    else:
        o = oracle.Oracle(p)
        o.run(1)
        t0 = time.perf_counter()
        _, _, clk, _ = o.run(steps)
        dt = time.perf_counter() - t0
        done = clk.tstep
        kind = "port"
    return dof_stages_per_step(p) * done / dt, kind, threads, dt


def run_reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    p = build_problem(a)
    import oracle
    threads = os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    have_ref = oracle.ref_available(p.physics, p.N)
    solver = oracle.RefSolver(p) if have_ref else oracle.Oracle(p)
    kind = "reference" if have_ref else "port"

    def one_step():
        if have_ref:
            solver.run(1)
        else:
            solver_state["u"], solver_state["k"], _, _ = solver.run(
                1, u=solver_state["u"], k=solver_state["k"])

    solver_state = {"u": p.u0.copy(), "k": None}
    for _ in range(a.warmup):
        one_step()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        one_step()
    el = time.perf_counter() - t0
    rate = dof_stages_per_step(p) * a.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT,
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * el / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(a, p, a.gpus),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{a.steps} full LSERK steps of the K={p.K} mesh",
                         "compile": "g++ -O3 -std=c++11 -fopenmp -march="
                                    + oracle.ref_march(p.physics, p.N)},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if have_ref:
        solver.close()
    print(json.dumps(line), flush=True)
    return 0


def reduce_max(x, dist=None):
    """Max of a per-rank scalar over the process group (identity without
    one); the tensor lives where the backend wants it (CUDA for NCCL, CPU
    for gloo)."""
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world, units_per_step, steps, ms_max):
    """Whole-job rate of `world` replicas: all ranks' units over the slowest
    rank's time."""
    return world * units_per_step * steps / (ms_max * 1e-3)


def _events(stream):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    return e0, e1


def face_maps_section(a, p, stream):
    """A/B of the neighbour-node source on the same handle: vmapP (4 Nfp ints
    per face) against the compact face maps (neighbour element and a one-byte
    node-list code per face), alternated twice, FP64 and TF32x3."""
    import numpy as np
    from exadglm_b200.capi import Solver, variants
    out = {"bytes_per_element": {"vmapP": 4 * 4 * p.Nfp, "compact": 4 * 5}}
    for prec in ("fp64", "tf32x3"):
        s = Solver(p, precision=prec)
        s.set_stream(stream.cuda_stream)
        ms = {False: [], True: []}
        for on in (False, True, False, True):
            s.set_compact_face_maps(on)
            s.step(a.warmup)
            s.sync()
            e0, e1 = _events(stream)
            e0.record(stream)
            s.step(a.steps)
            e1.record(stream)
            e1.synchronize()
            s.sync()
            ms[on].append(e0.elapsed_time(e1) / a.steps)
        out[prec] = {"kernel": variants(p.physics, p.N)[s.variant()],
                     "vmapP_ms_per_step": float(np.min(ms[False])),
                     "compact_ms_per_step": float(np.min(ms[True])),
                     "node_lists": s.face_map_lists()}
        s.close()
    return out


def mixed_section(a, p, stream, fp64_ms_per_step):
    """Mixed-precision stage kernels on the same workload: throughput, speed-up
    over the FP64 path and relative L2 against FP64 after --accuracy-steps."""
    import numpy as np
    import torch
    from exadglm_b200.capi import Solver, variants
    S = a.accuracy_steps
    ref = Solver(p, precision="fp64")
    ref.set_stream(stream.cuda_stream)
    ref.step(S)
    ref.sync()
    u64 = ref.get_state()
    ref.close()
    per_step = dof_stages_per_step(p)
    out = {"accuracy_steps": S}
    for prec in ("tf32x3", "bf16x3"):
        try:
            s = Solver(p, precision=prec)
        except Exception as exc:        # precision not built for this order
            out[prec] = {"unavailable": str(exc)}
            continue
        s.set_stream(stream.cuda_stream)
        s.step(a.warmup)
        s.sync()
        e0, e1 = _events(stream)
        e0.record(stream)
        s.step(a.steps)
        e1.record(stream)
        e1.synchronize()
        s.sync()
        ms = e0.elapsed_time(e1) / a.steps
        stage_ms = stage_alone_ms(s, stream)
        s.set_state(p.u0)
        clocks = ClockSampler(torch.cuda.current_device())
        clocks.start()
        s.step(S)
        s.sync()
        clk = clocks.stop()
        um = s.get_state()
        per_field = [float(np.linalg.norm(um[v] - u64[v]) / np.linalg.norm(u64[v]))
                     for v in range(p.nvar)]
        out[prec] = {
            "value": per_step / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
            # null when the FP64 path was not timed in this run (--only mixed)
            "speedup_vs_fp64": (fp64_ms_per_step / ms if fp64_ms_per_step is not None
                                else None),
            "rel_l2_vs_fp64": float(np.linalg.norm(um - u64) / np.linalg.norm(u64)),
            "rel_l2_per_field": per_field,
            "kernel": variants("euler", p.N)[s.variant()],
            "roofline": hbm_roofline(p, stage_ms, variants("euler", p.N)[s.variant()]),
            "clocks_during_accuracy_run": clk,
        }
        s.close()
    return out


def stage_alone_ms(s, stream, reps=25):
    """Mean time of one stage-kernel launch (CUDA events on the solver's
    stream, after warm-up launches), for the roofline."""
    import torch
    _, dt, _ = s.time()
    for i in range(5):
        s.stage(i % 5, dt)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream.synchronize()
    e0.record(stream)
    for i in range(reps):
        s.stage(i % 5, dt)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def hbm_roofline(p, stage_ms, desc):
    """Achieved algorithmic HBM bandwidth of one stage launch against the
    measured copy peak (the bound of the mixed-precision path)."""
    peaks, kind = load_peaks()
    B = bytes_per_element_stage(p.nvar, p.Np, p.Nfp) * p.K
    g = B / (stage_ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": g, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": g / peaks["hbm_gbs"], "launch_ms": stage_ms,
            "algorithmic_bytes_per_launch": B, "traffic": read_traffic(desc, p.K),
            "peak_source": f"{kind} hbm_gbs"}


def gpu_baseline_section(a, p, rank):
    """The reference's own GPU path (its CUDA kernels and cuBLAS batched
    DGEMMs, compiled for sm_100a from its sources into oracle/_ref) on the
    same workload and GPU: steps timed with the host clock around its runRK
    loop, which synchronises every step (calc_dt's blocking copy)."""
    import oracle
    if not oracle.gpu_ref_available(p.N):
        return {"unavailable": "oracle/_ref holds no reference GPU build"}
    ref = oracle.RefGpuSolver(p)
    ref.run(a.warmup)
    ref.set_state(p.u0)
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    t0 = time.perf_counter()
    done = ref.run(a.steps)
    el = time.perf_counter() - t0
    clk = clocks.stop()
    ref.close()
    return {"value": dof_stages_per_step(p) * done / el, "unit": UNIT,
            "ms_per_step": 1e3 * el / done, "steps": done, "clocks": clk,
            "what": "reference euler_nopad_*.cu (CUDA kernels + cuBLAS DgemmBatched), "
                    "nvcc -O3 -arch sm_100a, same mesh and state, one process"}


def adjoint_section(a, stream):
    """Discrete adjoint on the gradient-check workload: Euler N=4, K = 6 n^3,
    J = 1/2 ||rho(T) - rho_target||^2 after --adjoint-steps steps, checkpoint
    every --adjoint-every steps, dt and tau frozen.  The ratio is backward
    (recomputation included) over a plain forward run, both per step, timed
    with CUDA events on the solver's stream."""
    import numpy as np
    import torch
    from exadglm_b200 import problem as P
    from exadglm_b200.capi import Solver
    pa = P.euler_sine(n=a.adjoint_n, N=4, noise=1e-3, seed=5)
    pt = P.euler_sine(n=a.adjoint_n, N=4, v=(1.05, 0.45, 0.3), noise=1e-3, seed=5,
                      mesh=pa.mesh)
    T = a.adjoint_steps
    s = Solver(pa)
    s.set_stream(stream.cuda_stream)
    s.set_state(pt.u0)
    s.step(T)
    s.sync()
    rho_target = s.get_state()[0]
    nv, n = pa.nvar, pa.K * pa.Np
    s.set_state(pa.u0)
    s.step(max(a.warmup, 3))
    s.sync()

    def timed(fn):
        e0, e1 = _events(stream)
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    s.set_state(pa.u0)
    fwd = timed(lambda: s.step(T))
    lam = torch.zeros((nv, n), dtype=torch.float64, device="cuda")
    grad = torch.empty_like(lam)
    lp = [lam[v].data_ptr() for v in range(nv)]
    gp = [grad[v].data_ptr() for v in range(nv)]
    # warm-up pass (sizes the tape), then the timed record + reverse sweep
    s.set_state(pa.u0)
    s.adjoint_record(T, a.adjoint_every)
    torch.cuda.synchronize()
    s.adjoint_backward_device(lp, gp)
    s.set_state(pa.u0)
    rec = timed(lambda: s.adjoint_record(T, a.adjoint_every))
    uT = s.get_state()
    lam[0] = torch.from_numpy(uT[0] - rho_target).cuda()
    torch.cuda.synchronize()                      # lam is written on torch's stream
    bwd = timed(lambda: s.adjoint_backward_device(lp, gp))
    out = {
        "workload": f"euler_sine N=4 K={pa.K} (n={a.adjoint_n}) + 1e-3 noise, "
                    f"J = 1/2||rho(T)-rho_target||^2, T = {T} steps, checkpoint every "
                    f"{a.adjoint_every}, dt and tau frozen",
        "fwd_ms_per_step": fwd / T, "record_ms_per_step": rec / T, "bwd_ms_per_step": bwd / T,
        "ratio_bwd_over_fwd": bwd / fwd, "ratio_bwd_over_record": bwd / rec,
        "J": float(0.5 * np.dot(uT[0] - rho_target, uT[0] - rho_target)),
        "grad_norm": float(torch.linalg.norm(grad).item()),
        "tape_bytes": s.adjoint_tape_bytes(),
    }
    # binomial checkpointing under a cap: same gradient, fewer bytes, the
    # recomputed forward steps on top of the backward pass
    g_fixed = grad.clone()
    capped = []
    for cap_gib in [float(c) for c in a.adjoint_caps_gib.split(",") if c.strip()]:
        cap = int(cap_gib * 2**30)
        s.set_state(pa.u0)
        rec_c = timed(lambda: s.adjoint_record_capped(T, cap))
        leaf, slots, adv = s.adjoint_tape_plan()
        bwd_c = timed(lambda: s.adjoint_backward_device(lp, gp))
        capped.append({
            "cap_bytes": cap, "tape_bytes": s.adjoint_tape_bytes(), "leaf_steps": leaf,
            "slots": slots, "advance_steps": adv, "record_ms_per_step": rec_c / T,
            "bwd_ms_per_step": bwd_c / T, "ratio_bwd_over_fwd": bwd_c / fwd,
            "grad_rel_l2_vs_fixed": float(torch.linalg.norm(grad - g_fixed) /
                                          torch.linalg.norm(g_fixed))})
    out["capped"] = capped
    s.close()
    if a.adjoint_large_cap_gib > 0:
        out["capped_headline_size"] = adjoint_large(a, stream, timed)
    return out


def adjoint_large(a, stream, timed):
    """Capped adjoint at the headline size: Euler N=4, K = 6 n^3 (--n), 200
    steps, J = 1/2 ||rho(T)||^2, tape capped at --adjoint-large-cap-gib."""
    import torch
    from exadglm_b200 import problem as P
    from exadglm_b200.capi import Solver
    p = P.euler_sine(n=a.n, N=4, cfl=0.4)
    T, cap = 200, int(a.adjoint_large_cap_gib * 2**30)
    s = Solver(p)
    s.set_stream(stream.cuda_stream)
    s.step(3)
    s.sync()
    s.set_state(p.u0)
    fwd = timed(lambda: s.step(T))
    s.set_state(p.u0)
    rec = timed(lambda: s.adjoint_record_capped(T, cap))
    leaf, slots, adv = s.adjoint_tape_plan()
    nv, n = p.nvar, p.K * p.Np
    uT = s.get_state()
    lam = torch.zeros((nv, n), dtype=torch.float64, device="cuda")
    lam[0] = torch.from_numpy(uT[0]).cuda()
    grad = torch.empty_like(lam)
    torch.cuda.synchronize()
    bwd = timed(lambda: s.adjoint_backward_device([lam[v].data_ptr() for v in range(nv)],
                                                  [grad[v].data_ptr() for v in range(nv)]))
    out = {"workload": f"euler_sine N=4 K={p.K} (n={a.n}) CFL 0.4, J = 1/2||rho(T)||^2, "
                       f"T = {T} steps", "cap_bytes": cap,
           "tape_bytes": s.adjoint_tape_bytes(), "leaf_steps": leaf, "slots": slots,
           "advance_steps": adv, "fwd_ms_per_step": fwd / T, "record_ms_per_step": rec / T,
           "bwd_ms_per_step": bwd / T, "ratio_bwd_over_fwd": bwd / fwd,
           "grad_norm": float(torch.linalg.norm(grad).item())}
    s.close()
    return out


def batch_section(a, stream):
    """Many independent advection meshes (n in 4..24, N in 2..6, seeded):
    one launch per stage for the whole batch, against the same instances run
    one after another through single-mesh handles.  Both timed with CUDA
    events around the stepping only."""
    import torch
    from exadglm_b200 import problem as P
    from exadglm_b200.capi import BatchSolver, Solver
    t0 = time.perf_counter()
    probs = P.batch_instances(count=a.batch_count, seed=0)
    setup_s = time.perf_counter() - t0
    S = a.batch_steps
    dofs = sum(p.K * p.Np for p in probs) * 5          # DOF-stages per step

    def timed(fn):
        e0, e1 = _events(stream)
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    b = BatchSolver(probs)
    b.set_stream(stream.cuda_stream)
    b.step(3)
    b.sync()
    ms = timed(lambda: b.step(S))
    launches = b.kernel_launches()
    b.close()
    out = {
        "workload": f"{len(probs)} advection instances, n~U{{4..24}}, N~U{{2..6}}, seed 0, "
                    f"{S} steps, CFL 0.5",
        "K_total": int(sum(p.K for p in probs)),
        "dof_stages_per_step": dofs, "steps": S, "ms": ms,
        "value": dofs * S / (ms * 1e-3), "unit": UNIT, "gpu_launches": launches,
        "instances_by_order": {str(N): sum(1 for p in probs if p.N == N) for N in range(2, 7)},
        "host_setup_s": setup_s,
    }
    nseq = min(a.batch_sequential, len(probs))
    if nseq:
        seq_ms, seq_dofs = 0.0, 0
        for p in probs[:nseq]:
            s = Solver(p)
            s.set_stream(stream.cuda_stream)
            s.step(2)
            s.sync()
            seq_ms += timed(lambda: s.step(S))
            seq_dofs += p.K * p.Np * 5 * S
            s.close()
        out["sequential"] = {"instances": nseq, "ms": seq_ms,
                             "value": seq_dofs / (seq_ms * 1e-3),
                             "what": "the same instances one after another, one handle each"}
        out["speedup_vs_sequential"] = out["value"] / out["sequential"]["value"]
    return out


def precision_section(a, stream):
    """Precision study: Euler N=6 on n^3 x 6 tets (default 48 -> K = 663,552),
    the headline initial state, --accuracy-steps steps of the FP64 path and
    of each mixed mode from the same state; relative L2 against FP64 per field,
    and ms per step of each."""
    import numpy as np
    import torch
    from exadglm_b200 import problem as P
    from exadglm_b200.capi import Solver, variants
    p6 = P.euler_sine(n=a.precision_n, N=6, cfl=0.4)
    S = a.accuracy_steps
    out = {"workload": f"euler_sine N=6 K={p6.K} (n={a.precision_n}) CFL 0.4, {S} steps"}
    ref = None
    for prec in ("fp64", "tf32x3", "bf16x6", "bf16x3"):
        s = Solver(p6, precision=prec)
        s.set_stream(stream.cuda_stream)
        s.step(2)
        s.sync()
        s.set_state(p6.u0)
        e0, e1 = _events(stream)
        clocks = ClockSampler(torch.cuda.current_device())
        clocks.start()
        e0.record(stream)
        s.step(S)
        e1.record(stream)
        e1.synchronize()
        s.sync()
        clk = clocks.stop()
        u = s.get_state()
        ms = e0.elapsed_time(e1) / S
        row = {"ms_per_step": ms, "kernel": variants("euler", 6)[s.variant()],
               "value": dof_stages_per_step(p6) / (ms * 1e-3), "unit": UNIT, "clocks": clk}
        if ref is None:
            ref = u
        else:
            row["rel_l2_vs_fp64"] = float(np.linalg.norm(u - ref) / np.linalg.norm(ref))
            row["rel_l2_per_field"] = [float(np.linalg.norm(u[v] - ref[v]) / np.linalg.norm(ref[v]))
                                       for v in range(p6.nvar)]
            row["speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / ms
        out[prec] = row
        s.close()
    return out


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference_arm(a)

    import numpy as np
    import torch
    from exadglm_b200.capi import Solver, variants

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return reduce_max(x, dist)

    p = build_problem(a)
    stream = torch.cuda.Stream()
    if a.only in ("mixed", "face_maps", "adjoint", "batch", "precision", "gpu_baseline"):
        res = (mixed_section(a, p, stream, None) if a.only == "mixed"
               else face_maps_section(a, p, stream) if a.only == "face_maps"
               else adjoint_section(a, stream) if a.only == "adjoint"
               else precision_section(a, stream) if a.only == "precision"
               else gpu_baseline_section(a, p, rank) if a.only == "gpu_baseline"
               else batch_section(a, stream))
        if rank == 0:
            print(json.dumps({a.only: res}), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0
    s = Solver(p, precision=a.precision, device=local)
    s.set_stream(stream.cuda_stream)
    per_step = dof_stages_per_step(p)

    # ---- device-resident value -------------------------------------------
    s.step(a.warmup)
    s.sync()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    s.step(a.steps)
    ev1.record(stream)
    launches = s.kernel_launches()
    ev1.synchronize()
    s.sync()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    barrier()
    ms_max = max_over_ranks(ms)
    value = replica_rate(world, per_step, a.steps, ms_max)

    # ---- stage kernel alone, for the roofline -----------------------------
    stage_ms = stage_alone_ms(s, stream)
    peaks, peak_kind = load_peaks()
    B = bytes_per_element_stage(p.nvar, p.Np, p.Nfp) * p.K
    F = flops_per_element_stage(p.nvar, p.Np, p.Nfp) * p.K
    achieved_gbs = B / (stage_ms * 1e-3) / 1e9
    achieved_tf = F / (stage_ms * 1e-3) / 1e12
    vdesc = variants("euler", p.N)[s.variant()]
    roof = {
        "kernel": vdesc,
        "bound": "hbm", "achieved": achieved_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
        "frac": achieved_gbs / peaks["hbm_gbs"], "traffic": read_traffic(vdesc, p.K),
        "peak_source": f"{peak_kind} hbm_gbs (burst, kernel timed alone)",
        "algorithmic_bytes_per_launch": B, "launch_ms": stage_ms,
        "binding_roof": "fp64",
        "fp64": {"achieved_tflops": achieved_tf, "peak_tflops": NOMINAL_FP64_TFLOPS,
                 "peak_source": "nominal B200 FP64 (not measured on this pool)",
                 "frac": achieved_tf / NOMINAL_FP64_TFLOPS, "flops_per_launch": F},
    }

    # ---- end to end through the C ABI with host buffers --------------------
    # Every step copies its input state from page-locked host memory and its
    # result back.  Headline: dglm_run_ensemble, which overlaps member i's
    # compute with member i+1's host->device and member i-1's device->host
    # copies.  Also reported: the same steps as separate dglm_set_state /
    # dglm_step / dglm_get_state calls, each waiting for the previous one.
    nv, n = p.nvar, p.K * p.Np
    u0h = torch.from_numpy(np.ascontiguousarray(p.u0).reshape(nv, n))
    host_in = [torch.empty((nv, n), dtype=torch.float64, pin_memory=True) for _ in range(2)]
    host_out = [torch.empty((nv, n), dtype=torch.float64, pin_memory=True) for _ in range(2)]
    for h_ in host_in:
        h_.copy_(u0h)
    pin_in = [[h_[v].data_ptr() for v in range(nv)] for h_ in host_in]
    pin_out = [[h_[v].data_ptr() for v in range(nv)] for h_ in host_out]
    e2e_steps = max(4, a.steps)
    ens_in = [pin_in[i % 2] for i in range(e2e_steps)]
    ens_out = [pin_out[i % 2] for i in range(e2e_steps)]
    for _ in range(2):
        s.run_ensemble_ptrs(ens_in[:3], ens_out[:3], 1)
    barrier()
    t0 = time.perf_counter()
    s.run_ensemble_ptrs(ens_in, ens_out, 1)
    el = max_over_ranks(time.perf_counter() - t0)
    ens_launches = s.kernel_launches()
    for _ in range(2):
        s.set_state_ptrs(pin_in[0], 0)
        s.step(1)
        s.get_state_ptrs(pin_out[0], 0)
    barrier()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        s.set_state_ptrs(pin_in[i % 2], 0)     # H2D of the step's input state
        s.step(1)
        s.get_state_ptrs(pin_out[i % 2], 0)    # D2H of the step's result (synchronises)
    el_serial = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": world * per_step * e2e_steps / el, "unit": UNIT,
           "h2d_bytes_per_step": nv * n * 8, "d2h_bytes_per_step": nv * n * 8,
           "steps": e2e_steps, "ms_per_step": 1e3 * el / e2e_steps, "kernel_launches": ens_launches,
           "what": "dglm_run_ensemble: per step one state copied from page-locked host "
                   "memory, one CFL step, the result copied back; the copies of "
                   "neighbouring steps overlap the compute",
           "serial": {"value": world * per_step * e2e_steps / el_serial,
                      "ms_per_step": 1e3 * el_serial / e2e_steps,
                      "what": "dglm_set_state, dglm_step(1), dglm_get_state per step"}}
    s.close()

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(a, p, world),
        "roofline": roof, "e2e": e2e, "clocks": clk, "gpu_launches": launches,
    }
    if a.only is None and a.precision == "fp64":
        line["mixed"] = mixed_section(a, p, stream, ms_max / a.steps)
        line["face_maps"] = face_maps_section(a, p, stream)
        line["adjoint"] = adjoint_section(a, stream)
        if rank == 0:
            gb = gpu_baseline_section(a, p, rank)
            if "value" in gb:
                gb["ours_over_reference_gpu"] = value / world / gb["value"]
            line["gpu_baseline"] = gb
        line["precision"] = precision_section(a, stream)
        line["batch"] = batch_section(a, stream)
    if rank == 0 and not a.no_cpu_baseline:
        sample_steps = 1
        rate, kind, cores, secs = cpu_reference_rate(p, sample_steps)
        import oracle
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                                "sample": f"{sample_steps} LSERK step of the K={p.K} mesh "
                                          f"({secs:.1f} s)",
                                "compile": "g++ -O3 -std=c++11 -fopenmp -march="
                                           + oracle.ref_march(p.physics, p.N)}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
