"""B200-native explicit DGLM solver: the right-hand side and 5-stage
low-storage Runge-Kutta step of ExaDGLM (linear advection and compressible
Euler on tetrahedral meshes) as hand-written sm_100a CUDA behind the C ABI in
include/dglm.h.

Modules:
  refelem   reference-tetrahedron nodes and operators (WDr/WDs/WDt, LIFT, Fmask)
  mesh      uniform box meshes and their DG geometry (vmapP, metrics, normals)
  problem   problem set-ups (initial states, parameters) and the L2 error
  datain    the reference's datain/dataout binary formats, plus full-state
            snapshots (every variable and t) for restart
  capi      ctypes binding of libdglm.so (Solver and BatchSolver handles,
            ensembles with overlapped host copies, per-kernel entry points)
  adjoint   discrete adjoint behind torch.autograd (DGLMStep, evolve)
  tune      timing of the compiled tile shapes, tuned.json lookup
  launcher  drop-in for the reference's DGLM3DSingleGPU launcher class
  build     nvcc build of libdglm.so and the dglm_main driver
"""
__version__ = "0.1.0"
