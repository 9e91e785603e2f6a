"""Problem set-ups: mesh + parameters + initial state.

The reference hard-codes its initial states in per-physics ``init.cpp``
files (euler_init.cpp:5-35, advec_init.cpp:5-25) that the launcher links in;
a different ``init`` unit is its mechanism for another case.  Here each case
is a function that returns a :class:`Problem`; the workloads used for
measurement are seeded synthetic states on periodic unit cubes:

* ``advection_gaussian`` -- N=3 on 8^3 x 6 tets, u0 = exp(-|x-c|^2/0.01),
  v = (1, 0.5, 0.25), CFL 0.5;
* ``euler_sine`` -- rho = 1 + 0.2 sin(2 pi (x+y+z)), v = (1, 0.5, 0.25),
  p = 1, gamma 1.4, CFL 0.4; N=4 on 32^3 x 6 tets is the headline workload;
* ``advection_notebook`` / ``euler_notebook`` -- the reference's own
  initial states and parameters (N=5, 6^3 hexes, CFL 0.8, T=2), used to pin
  against its published L2 errors.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .mesh import Mesh3D, UniformBox

PHYSICS = ("advection", "euler")


@dataclass
class Problem:
    physics: str
    N: int
    mesh: Mesh3D
    u0: np.ndarray                     # (nvar, K*Np)
    vel: np.ndarray | None = None      # (3, K*Np) advection velocity per node
    cfl: float = 0.8
    gamma: float = 1.4
    tau_scale: float = 1.2
    tmax: float = 1000.0
    name: str = ""
    extra: dict = field(default_factory=dict)

    @property
    def nvar(self):
        return 5 if self.physics == "euler" else 1

    @property
    def K(self):
        return self.mesh.Nelem

    @property
    def Np(self):
        return self.mesh.Np

    @property
    def Nfp(self):
        return self.mesh.Nfp

    def dof(self):
        return self.nvar * self.K * self.Np

    def datain_arrays(self):
        return self.mesh.datain_arrays()


def _nodes(mesh):
    return mesh.PX.ravel(), mesh.PY.ravel(), mesh.PZ.ravel()


def euler_state(rho, vx, vy, vz, p, gamma):
    """Conserved variables (rho, rho v, p/(gamma-1) + rho |v|^2 / 2)."""
    return np.stack([rho, rho * vx, rho * vy, rho * vz,
                     p / (gamma - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)])


def advection_gaussian(n=8, N=3, v=(1.0, 0.5, 0.25), center=(0.5, 0.5, 0.5), width2=0.01,
                       cfl=0.5, tau_scale=1.2, tmax=1000.0, mesh=None):
    mesh = mesh or Mesh3D(N, UniformBox(n + 1, n + 1, n + 1), high_order=False)
    x, y, z = _nodes(mesh)
    r2 = (x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2
    u0 = np.exp(-r2 / width2)[None, :]
    vel = np.stack([np.full_like(x, v[0]), np.full_like(x, v[1]), np.full_like(x, v[2])])
    return Problem("advection", N, mesh, u0, vel, cfl=cfl, tau_scale=tau_scale, tmax=tmax,
                   name=f"advection_gaussian_N{N}_n{n}")


def batch_instances(count=256, seed=0, n_range=(4, 24), orders=(2, 6), cfl=0.5,
                    tau_scale=1.2, tmax=1000.0):
    """Independent advection problems for batching, drawn from
    numpy.random.default_rng(seed): per instance n ~ U{n_range}, N ~ U{orders},
    v ~ U[-1, 1]^3, Gaussian centre ~ U[0, 1]^3, width w ~ U[0.05, 0.2],
    u0 = exp(-|x - c|^2 / w^2) on the periodic unit cube of n^3 x 6 tets.
    Meshes are shared between instances of the same (n, N); the velocity is
    a broadcast view (constant per instance)."""
    rng = np.random.default_rng(seed)
    meshes = {}
    out = []
    for i in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        N = int(rng.integers(orders[0], orders[1] + 1))
        v = rng.uniform(-1.0, 1.0, 3)
        c = rng.uniform(0.0, 1.0, 3)
        w = float(rng.uniform(0.05, 0.2))
        if (n, N) not in meshes:
            meshes[(n, N)] = Mesh3D(N, UniformBox(n + 1, n + 1, n + 1), high_order=False)
        mesh = meshes[(n, N)]
        x, y, z = _nodes(mesh)
        r2 = (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2
        u0 = np.exp(-r2 / (w * w))[None, :]
        vel = np.broadcast_to(v[:, None], (3, x.size))
        out.append(Problem("advection", N, mesh, u0, vel, cfl=cfl, tau_scale=tau_scale,
                           tmax=tmax, name=f"batch{i}_N{N}_n{n}"))
    return out


def euler_sine(n=32, N=4, v=(1.0, 0.5, 0.25), p=1.0, gamma=1.4, cfl=0.4, tau_scale=1.2,
               tmax=1000.0, noise=0.0, seed=0, mesh=None):
    mesh = mesh or Mesh3D(N, UniformBox(n + 1, n + 1, n + 1), high_order=False)
    x, y, z = _nodes(mesh)
    rho = 1 + 0.2 * np.sin(2 * np.pi * (x + y + z))
    one = np.ones_like(x)
    u0 = euler_state(rho, v[0] * one, v[1] * one, v[2] * one, p * one, gamma)
    if noise:
        u0 = u0 + noise * np.random.default_rng(seed).standard_normal(u0.shape)
    return Problem("euler", N, mesh, u0, None, cfl=cfl, gamma=gamma, tau_scale=tau_scale,
                   tmax=tmax, name=f"euler_sine_N{N}_n{n}")


def advection_notebook(nx=7, N=5, cfl=0.8, tmax=2.0):
    """The reference notebook case: u0 = sin(2 pi x) sin(2 pi y) sin(2 pi z),
    v = (1, 1, 1) (advec_init.cpp:5-25)."""
    mesh = Mesh3D(N, UniformBox(nx, nx, nx), high_order=True)
    x, y, z = _nodes(mesh)
    u0 = (np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y) * np.sin(2 * np.pi * z))[None, :]
    vel = np.ones((3, x.size))
    return Problem("advection", N, mesh, u0, vel, cfl=cfl, tmax=tmax,
                   name=f"advection_notebook_N{N}_nx{nx}")


def euler_notebook(nx=7, N=5, cfl=0.8, tmax=2.0):
    """The reference notebook case: rho = 1 + 0.2 sin(2 pi (x+y+z)),
    v = (1, -0.5, 1), p = 1 (euler_init.cpp:5-35)."""
    mesh = Mesh3D(N, UniformBox(nx, nx, nx), high_order=True)
    x, y, z = _nodes(mesh)
    rho = 1 + 0.2 * np.sin(2 * np.pi * (x + y + z))
    one = np.ones_like(x)
    u0 = euler_state(rho, one, -0.5 * one, one, one, 1.4)
    return Problem("euler", N, mesh, u0, None, cfl=cfl, tmax=tmax,
                   name=f"euler_notebook_N{N}_nx{nx}")


def exact_notebook(problem: Problem, t: float):
    """Exact solution of the notebook cases at time t on the order-(N+2)
    nodes (the notebooks' ref_solution cells)."""
    m = problem.mesh
    x, y, z = m.high_PX.ravel(), m.high_PY.ravel(), m.high_PZ.ravel()
    if problem.physics == "advection":
        v = (1.0, 1.0, 1.0)
    else:
        v = (1.0, -0.5, 1.0)
    xs = ((x - v[0] * t) + 1) % 1 - 1
    ys = ((y - v[1] * t) + 1) % 1 - 1
    zs = ((z - v[2] * t) + 1) % 1 - 1
    if problem.physics == "advection":
        return np.sin(2 * np.pi * xs) * np.sin(2 * np.pi * ys) * np.sin(2 * np.pi * zs)
    return 1 + 0.2 * np.sin(2 * np.pi * (xs + ys + zs))


def l2_error(problem: Problem, ref_high, u_first_var, apply_sqrt=True):
    """Mass-weighted L2 error against a solution given on the order-(N+2)
    nodes, vectorised form of dglm_3d_launcher.py:328-355."""
    m, ref = problem.mesh, problem.mesh.ref
    K, Np, hNp = problem.K, ref.Np, ref.high_Np
    un = np.asarray(u_first_var).reshape(K, Np) @ ref.interpM.T          # (K, hNp)
    E = np.asarray(ref_high).reshape(K, hNp) - un
    Eint = m.J * np.einsum("ki,ij,kj->k", E, ref.high_M, E)
    s = np.sum(Eint)
    return np.sqrt(s) if apply_sqrt else s
