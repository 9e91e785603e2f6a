"""The benchmark's roofline arithmetic: algorithmic bytes and FLOPs per
element-stage for the three single-mesh workloads, and the shared config
object of both arms."""
import argparse
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.mark.parametrize("nvar,N,adv,bytes_e,flops_e", [
    (5, 4, False, 6072, 57750),      # Euler N=4, K=196,608 (the benchmark workload)
    (5, 6, False, 14120, 305760),    # Euler N=6, K=663,552
    (1, 3, True, 1512, 4000),        # advection N=3, K=3,072
])
def test_bytes_and_flops_per_element_stage(nvar, N, adv, bytes_e, flops_e):
    b = load_bench()
    Np, Nfp = (N + 1) * (N + 2) * (N + 3) // 6, (N + 1) * (N + 2) // 2
    assert b.bytes_per_element_stage(nvar, Np, Nfp, advection=adv) == bytes_e
    assert b.flops_per_element_stage(nvar, Np, Nfp) == flops_e


def test_both_arms_share_the_config():
    b = load_bench()

    class P:
        N, K, Np, nvar = 4, 196608, 35, 5

    a = argparse.Namespace(n=32, precision="fp64")
    c = b.workload_config(a, P, 1)
    assert c["K"] == 196608 and c["N"] == 4 and c["parallelism"] == "replicas1"
    assert "K=196608" in c["workload"] and "l2" in c
    assert b.workload_config(a, P, 8)["parallelism"] == "replicas8"
    # roughly 1.194 GB of algorithmic traffic per stage of the benchmark workload
    assert b.bytes_per_element_stage(5, 35, 15) * 196608 == 1193803776
