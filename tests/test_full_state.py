"""Full-state snapshot files (every variable plus t_NNNNNNN.bin) and the
host-side restart logic, on the CPU.  The GPU side of restart (dglm_set_time,
dglm_main --restart-dir) is covered by tests/test_restart.py."""
import os

import numpy as np
import pytest

from exadglm_b200 import datain as D
from exadglm_b200.capi import Solver


def test_names_keep_the_reference_snapshot_names():
    assert D.field_name(0, 30, "euler") == D.snapshot_name(30, "euler") == "u1_0000030.bin"
    assert D.field_name(4, 30, "euler") == "u5_0000030.bin"
    assert D.field_name(0, 809, "advection") == D.snapshot_name(809, "advection")
    assert D.time_name(1098) == "t_0001098.bin"
    for bad in ((5, 1, "euler"), (1, 1, "advection"), (0, -1, "euler"), (0, 10 ** 7, "euler")):
        with pytest.raises(ValueError):
            D.field_name(*bad)


@pytest.mark.parametrize("physics,nvar", [("euler", 5), ("advection", 1)])
def test_full_state_round_trip(tmp_path, physics, nvar):
    rng = np.random.default_rng(0)
    u = rng.standard_normal((nvar, 7 * 20))
    D.write_full_state(str(tmp_path), 120, physics, u, 0.3125, print_interval=40)
    D.write_full_state(str(tmp_path), 160, physics, 2 * u, 0.5, print_interval=40)
    got, t, step, pi = D.read_full_state(str(tmp_path), 120, physics, n=140)
    np.testing.assert_array_equal(got, u)
    assert (t, step, pi) == (0.3125, 120, 40)
    # the time file is three little-endian float64 values
    raw = np.fromfile(os.path.join(tmp_path, "t_0000120.bin"), dtype="<f8")
    np.testing.assert_array_equal(raw, [0.3125, 120.0, 40.0])
    assert D.full_state_steps(str(tmp_path), physics) == [120, 160]
    os.remove(os.path.join(tmp_path, D.field_name(nvar - 1, 160, physics)))
    assert D.full_state_steps(str(tmp_path), physics) == [120]


def test_full_state_rejects_wrong_sizes_and_steps(tmp_path):
    u = np.ones((5, 10))
    D.write_full_state(str(tmp_path), 3, "euler", u, 1.0)
    with pytest.raises(ValueError):
        D.read_full_state(str(tmp_path), 3, "euler", n=11)
    np.ones(4).tofile(os.path.join(tmp_path, "u3_0000003.bin"))
    with pytest.raises(ValueError):
        D.read_full_state(str(tmp_path), 3, "euler")
    D.write_full_state(str(tmp_path), 4, "euler", u, 1.0)
    os.replace(os.path.join(tmp_path, "t_0000004.bin"), os.path.join(tmp_path, "t_0000003.bin"))
    with pytest.raises(ValueError):
        D.read_full_state(str(tmp_path), 3, "euler")


class _FakeSolver:
    """The attributes Solver.save_full_state / restart use, without a GPU."""

    class p:
        physics, nvar, K, Np = "euler", 5, 4, 10

    def __init__(self):
        self.u = np.arange(200.0).reshape(5, 40)
        self.t, self.tstep = 0.75, 60

    def time(self):
        return self.t, 0.01, self.tstep

    def get_state(self):
        return self.u.copy()

    def set_state(self, u):
        self.u = np.array(u)

    def set_time(self, t, tstep):
        self.t, self.tstep = t, tstep


def test_solver_save_and_restart_logic(tmp_path):
    a = _FakeSolver()
    assert Solver.save_full_state(a, str(tmp_path), print_interval=20) == 60
    b = _FakeSolver()
    b.u[:] = 0
    b.t, b.tstep = 0.0, 0
    assert Solver.restart(b, str(tmp_path), 60) == (0.75, 60)
    np.testing.assert_array_equal(b.u, a.u)
    assert (b.t, b.tstep) == (0.75, 60)
    assert D.read_full_state(str(tmp_path), 60, "euler")[3] == 20


def test_launcher_command_carries_the_restart_flags(tmp_path):
    from exadglm_b200.launcher import DGLM3DSingleGPU
    param = {"CFL": 0.8, "gamma": 1.4, "tau_scale": 1.2, "interpN": 2, "dtype": "f8"}
    dg = DGLM3DSingleGPU(None, str(tmp_path / "work"), 3, 5, 1.0, param, 0)
    dg.make_work_dir()
    base = dg.command("euler_nopad_main")
    assert "--full-state" not in base and "--restart-dir" not in base
    cmd = dg.command("euler_nopad_main", full_state=True, restart_dir="/x/out", restart_step=300)
    assert cmd[:len(base)] == base
    assert cmd[len(base):] == ["--full-state", "--restart-dir", "/x/out", "--restart-step", "300"]
    with pytest.raises(ValueError):
        dg.command("euler_nopad_main", restart_dir="/x/out")
    with pytest.raises(ValueError):
        dg.command("advec_nopad_main")
