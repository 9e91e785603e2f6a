"""Full-state snapshots and restart: a run interrupted at step S and continued
from its saved state (every field, t and the step counter) matches the
uninterrupted run bit for bit.  The reference has no restart (it writes only
u1 / u); the driver's ``--full-state`` keeps its file names and adds the other
fields and ``t_NNNNNNN.bin``."""
import os
import subprocess
from glob import glob

import numpy as np
import pytest

from exadglm_b200 import build as _build
from exadglm_b200 import problem as P
from test_launcher import notebook_launcher


def test_driver_rejects_restart_dir_without_step(tmp_path):
    if not os.path.exists(_build.MAIN):
        pytest.skip("dglm_main not built")
    r = subprocess.run([_build.MAIN, "--datain", str(tmp_path), "--dataout", str(tmp_path),
                        "--tmax", "1", "--restart-dir", str(tmp_path)],
                       stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    assert r.returncode == 2 and "--restart-step" in r.stderr


@pytest.mark.parametrize("flag,value,msg", [("--precision", "fp16", "unknown precision fp16"),
                                            ("--physics", "maxwell", "unknown physics maxwell"),
                                            ("--matrix-order", "x", "unknown matrix order x")])
def test_driver_rejects_unknown_values(tmp_path, flag, value, msg):
    """Flags with a fixed set of values fail instead of falling back."""
    if not os.path.exists(_build.MAIN):
        pytest.skip("dglm_main not built")
    r = subprocess.run([_build.MAIN, "--datain", str(tmp_path), "--dataout", str(tmp_path),
                        "--tmax", "1", flag, value],
                       stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    assert r.returncode == 2 and msg in r.stderr, r.stderr


def test_driver_rejects_mismatched_snapshots(tmp_path):
    """A field file of the wrong size or a time file of another step stops
    dglm_main before it touches the GPU."""
    if not os.path.exists(_build.MAIN):
        pytest.skip("dglm_main not built")
    from exadglm_b200.datain import field_name, time_name, write_full_state
    dg, _ = notebook_launcher(tmp_path, 5, nx=4, N=3, tmax=0.5)
    n = dg.Nelem * dg.Np
    snap = str(tmp_path / "snap")
    write_full_state(snap, 5, "euler", np.ones((5, n)), 0.1, 2)
    base = [_build.MAIN, "--datain", dg.datain_dir, "--dataout", str(tmp_path), "--physics",
            "euler", "--tmax", "1", "--matrix-order", "f", "--restart-dir", snap,
            "--restart-step", "5"]

    def run():
        return subprocess.run(base, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)

    np.ones(n + 1).tofile(os.path.join(snap, field_name(2, 5, "euler")))
    r = run()
    assert r.returncode != 0 and "expected" in r.stderr and field_name(2, 5, "euler") in r.stderr
    np.ones(n).tofile(os.path.join(snap, field_name(2, 5, "euler")))
    np.array([0.1, 6.0, 2.0]).tofile(os.path.join(snap, time_name(5)))
    r = run()
    assert r.returncode != 0 and "holds step 6" in r.stderr, r.stderr
    for bad in (-3.0, 2.5, np.nan):     # print interval: negative, fractional, NaN
        np.array([0.1, 5.0, bad]).tofile(os.path.join(snap, time_name(5)))
        r = run()
        assert r.returncode != 0 and "print interval" in r.stderr, (bad, r.stderr)


@pytest.mark.gpu
@pytest.mark.parametrize("phys", ["euler", "advection"])
def test_solver_restart_is_bitwise(phys):
    from exadglm_b200.capi import DglmError, Solver
    prob = (P.euler_sine(n=3, N=4, noise=1e-3, seed=1) if phys == "euler"
            else P.advection_gaussian(n=3, N=4, width2=0.05))
    a = Solver(prob)
    a.step(30)
    a.sync()
    ua, ta = a.get_state(), a.time()
    dta = a.dt_history(0, 30)

    b = Solver(prob)
    b.step(12)
    b.sync()
    u12, (t12, _, s12) = b.get_state(), b.time()
    b.close()
    c = Solver(prob)
    with pytest.raises(DglmError):
        c.set_time(-1.0, 0)
    c.set_state(u12)
    c.set_time(t12, s12)
    assert c.time()[0] == t12 and c.time()[2] == 12
    c.step(18)
    c.sync()
    uc, tc = c.get_state(), c.time()
    np.testing.assert_array_equal(uc, ua)
    assert tc[0] == ta[0] and tc[2] == ta[2] == 30
    np.testing.assert_array_equal(c.dt_history(12, 18), dta[12:])
    a.close()
    c.close()


@pytest.mark.gpu
def test_solver_full_state_files_restart_bitwise(tmp_path):
    """Solver.save_full_state at step 12, Solver.restart in a fresh handle,
    18 more steps: the state of the straight 30-step run, bit for bit."""
    from exadglm_b200.capi import Solver
    prob = P.euler_sine(n=3, N=4, noise=1e-3, seed=1)
    a = Solver(prob)
    a.step(30)
    ua, ta = a.get_state(), a.time()
    a.close()
    b = Solver(prob)
    b.step(12)
    assert b.save_full_state(str(tmp_path), print_interval=6) == 12
    b.close()
    c = Solver(prob)
    assert c.restart(str(tmp_path), 12)[1] == 12
    c.step(18)
    np.testing.assert_array_equal(c.get_state(), ua)
    assert c.time()[0] == ta[0] and c.time()[2] == 30
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("Nvar", [5, 1])
def test_driver_restart_is_bitwise(tmp_path, Nvar):
    """dglm_main --full-state, then --restart-dir/--restart-step from an
    intermediate snapshot: the same later snapshots, byte for byte, and the
    same printed steps."""
    dg, main = notebook_launcher(tmp_path, Nvar, nx=4, N=3, tmax=0.5)
    dg.build(verbose=0)
    physics = "euler" if Nvar == 5 else "advection"
    base = [_build.MAIN, "--datain", dg.datain_dir, "--physics", physics,
            "--tmax", "0.5", "--matrix-order", "f"]
    full = str(tmp_path / "full")
    rest = str(tmp_path / "rest")
    os.makedirs(full)
    os.makedirs(rest)
    r1 = subprocess.run(base + ["--dataout", full, "--full-state"],
                        stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    assert r1.returncode == 0, r1.stderr
    first = "u1_" if Nvar == 5 else "u_"
    steps = sorted(int(os.path.basename(f)[len(first):-4]) for f in glob(full + f"/{first}*.bin"))
    assert len(steps) >= 3 and steps[0] == 0
    fields = ["u%d_" % (v + 1) for v in range(5)] if Nvar == 5 else ["u_"]
    for s in steps:
        for f in fields + ["t_"]:
            assert os.path.exists(os.path.join(full, f"{f}{s:07d}.bin")), (f, s)
    S = steps[len(steps) // 2]
    r2 = subprocess.run(base + ["--dataout", rest, "--full-state", "--restart-dir", full,
                                "--restart-step", str(S)],
                        stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    assert r2.returncode == 0, r2.stderr
    later = [ln for ln in r1.stdout.splitlines() if int(ln.split(",")[0][6:]) > S]
    assert r2.stdout.splitlines() == later
    for s in steps:
        for f in fields + ["t_"]:
            name = f"{f}{s:07d}.bin"
            if s <= S:
                assert not os.path.exists(os.path.join(rest, name))
                continue
            with open(os.path.join(full, name), "rb") as x, open(os.path.join(rest, name), "rb") as y:
                assert x.read() == y.read(), name
