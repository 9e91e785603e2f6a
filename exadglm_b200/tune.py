"""Autotuner for the fused stage kernel.

Each (physics, N) is compiled with several tile shapes ("variants": SIMT
register tiles, FP64 tensor-core DMMA tiles and persistent TMA-fed DMMA
tiles, see dglm_stage_fp64.cu).  ``tune(problem)`` times every variant's
stage kernel on the problem with CUDA events and returns the fastest; the
results are cached per (physics, N, precision, device name) in a JSON file
(``tuned.json`` next to this module, or $DGLM_TUNE_CACHE), which the Solver
reads to pick its default variant.
"""
from __future__ import annotations

import json
import re
import os

from . import capi

CACHE = os.environ.get("DGLM_TUNE_CACHE",
                       os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned.json"))


def _key(physics, N, precision, device_name):
    return f"{device_name}|{physics}|N{N}|{precision}"


def _device_name(device=0):
    import torch
    return torch.cuda.get_device_name(device)


def load_cache():
    if os.path.exists(CACHE):
        try:
            with open(CACHE) as f:
                return json.load(f)
        except (OSError, ValueError):
            return {}
    return {}


def cached_variant(physics, N, precision="fp64", device=0):
    """The cached best variant index for this device, or None."""
    try:
        name = _device_name(device)
    except Exception:
        return None
    ent = load_cache().get(_key(physics, N, precision, name))
    if ent is None:
        return None
    # match by description: indices move when variants are added; the
    # shared-memory size is left out of the match, since layout changes move
    # it without changing the tile shape
    descs = [_shape(d) for d in capi.variants(physics, N)]
    want = _shape(ent["desc"])
    return descs.index(want) if want in descs else None


def _shape(desc):
    """A variant description without its smem=<bytes> field."""
    return re.sub(r" smem=\d+", "", desc)


def time_variants(solver, reps=25):
    """Stage-kernel time (ms) of every variant on the solver's problem."""
    import torch
    p = solver.p
    stream = torch.cuda.Stream()
    solver.set_stream(stream.cuda_stream)
    out = []
    for v, desc in capi.variants(p.physics, p.N, solver.precision):
        solver.set_variant(v)
        solver.set_state(p.u0)
        solver.step(1)
        _, dt, _ = solver.time()
        for i in range(5):
            solver.stage(i, dt)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream.synchronize()
        e0.record(stream)
        for i in range(reps):
            solver.stage(i % 5, dt)
        e1.record(stream)
        e1.synchronize()
        out.append((e0.elapsed_time(e1) / reps, v, desc))
    solver.set_state(p.u0)
    return out


def tune(problem, precision="fp64", device=0, write=True, reps=25):
    """Times all variants on `problem`; returns (best_variant, timings) and
    records the winner in the cache."""
    solver = capi.Solver(problem, precision=precision, device=device, variant=-1)
    timings = time_variants(solver, reps)
    solver.close()
    best = min(timings)
    if write:
        cache = load_cache()
        cache[_key(problem.physics, problem.N, precision, _device_name(device))] = {
            "variant": best[1], "desc": best[2], "stage_ms": round(best[0], 5),
            "K": problem.K,
            "all": [{"variant": v, "desc": d, "stage_ms": round(t, 5)} for t, v, d in timings]}
        with open(CACHE, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    return best[1], timings


def main(argv=None):
    import argparse
    from . import problem as P
    ap = argparse.ArgumentParser(description="tune the stage kernel variants")
    ap.add_argument("--physics", default="euler", choices=["euler", "advection"])
    ap.add_argument("--orders", default="1-8")
    ap.add_argument("--dofs", type=float, default=2e7, help="target DOF count of the test mesh")
    ap.add_argument("--precisions", default="fp64,tf32x3,bf16x3,bf16x6",
                    help="modes to tune (those without variants for an order are skipped)")
    a = ap.parse_args(argv)
    lo, _, hi = a.orders.partition("-")
    for N in range(int(lo), int(hi or lo) + 1):
        nv = 5 if a.physics == "euler" else 1
        Np = (N + 1) * (N + 2) * (N + 3) // 6
        n = max(3, int(round((a.dofs / (6 * Np * nv)) ** (1 / 3))))
        prob = (P.euler_sine(n=n, N=N) if a.physics == "euler"
                else P.advection_gaussian(n=n, N=N))
        for prec in a.precisions.split(","):
            if not capi.variants(a.physics, N, prec):
                continue
            best, timings = tune(prob, precision=prec)
            print(f"{a.physics} N={N} K={prob.K} {prec}: best variant {best}")
            for t, v, d in sorted(timings):
                print(f"   {t:8.4f} ms  v{v}  {d}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
