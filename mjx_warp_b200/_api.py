"""The reference's stage functions (mujoco_warp/__init__.py:18-58) over the CUDA kernels.

Each function takes (Model, Data) like its reference counterpart, launches the corresponding
libmjb200.so entry point on the current torch CUDA stream and returns without synchronising, so
sequences of calls can be captured in a CUDA graph.  There is no CPU path: calling these on a
Data whose tensors live on the CPU, or without the built library, raises.
"""

from __future__ import annotations

import ctypes
import time as _time
from typing import Callable, Optional, Tuple

import numpy as np
import torch

from . import _abi
from .types import Data, Model

# launch forms (include/mjb200.h MJB_FORM_*): True / 1 the chosen form, False / 0 the plain
# one-kernel-per-stage form, 2 the single-kernel form
_FORMS = {0: _abi.MjbRunCfg(0, 0), 1: _abi.MjbRunCfg(1, 0), 2: _abi.MjbRunCfg(2, 0),
          3: _abi.MjbRunCfg(3, 0)}


def _form(fused) -> "_abi.MjbRunCfg":
  try:
    return _FORMS[int(fused)]
  except (KeyError, TypeError, ValueError):
    raise ValueError(f"unknown launch form {fused!r} (True/1 chosen, False/0 plain, 2 single, "
                     "3 precision)") from None


def _call(name: str, m: Model, d: Data, *extra) -> None:
  L = _abi.lib()
  mv = _abi.model_view(m)
  dv = _abi.data_view(d)
  rc = getattr(L, "mjb_" + name)(ctypes.byref(mv), ctypes.byref(dv), *extra, _abi.stream())
  _abi.check(rc, name)


def _integrator_check(m: Model) -> None:
  if m.opt.integrator == 1:
    raise NotImplementedError(f"integrator {m.opt.integrator} not implemented.")
  if m.opt.integrator not in (0, 3):
    raise NotImplementedError(f"integrator {m.opt.integrator} not implemented.")


def step(m: Model, d: Data, fused=True) -> None:
  """Advance simulation (forward.py:682-695).

  fused=True (or 1) runs the chosen form: the stage kernels of fwd_position .. fwd_acceleration
  forked over three streams, the persistent solver (keeping the Newton Hessian's factor while the
  active set is unchanged; one CTA per world for models with nv > 128) and one kernel for
  the integrator; fused=False (or 0) launches one kernel per reference stage and refactors
  the Hessian in every iteration, as the reference does; fused=2 runs the whole step of a world
  in one warp of a single kernel; fused=3 runs the chosen form with the Hessian and mass-matrix
  Cholesky factor-solves and the line-search coefficient sums in FP64 (the precision form; dense
  mass matrix with trees of up to 32 dofs, nv up to about 230).
  """
  _integrator_check(m)
  L = _abi.lib()
  rc = L.mjb_step(ctypes.byref(_abi.model_view(m)), ctypes.byref(_abi.data_view(d)),
                  ctypes.byref(_form(fused)), _abi.stream())
  _abi.check(rc, "step")
  d.time = d.time + m.opt.timestep


_STEP_IO_SHAPES = {"qpos": "nq", "qvel": "nv", "ctrl": "nu", "qacc_warmstart": "nv"}
_STEP_IO_OUT = {"qpos": (lambda m: (m.nq,)), "qvel": (lambda m: (m.nv,)),
                "qacc_warmstart": (lambda m: (m.nv,)), "xpos": (lambda m: (m.nbody, 3)),
                "xmat": (lambda m: (m.nbody, 3, 3)), "subtree_com": (lambda m: (m.nbody, 3)),
                "cvel": (lambda m: (m.nbody, 6)), "site_xpos": (lambda m: (m.nsite, 3))}


def step_io(m: Model, d: Data, nstep: int = 1, inputs: Optional[dict] = None,
            outputs=("qpos", "qvel"), out: Optional[dict] = None, fused=True) -> dict:
  """The step call of a host framework (an extension: the reference's callers write these copies
  around step themselves, e.g. contrib/jax_unroll.py:40-71 and the notebook's unrolled step):
  copies `inputs` (a dict over qpos, qvel, ctrl, qacc_warmstart of (nworld, n) CUDA tensors)
  into d, runs `nstep` steps, and copies the `outputs` fields (qpos, qvel, qacc_warmstart, xpos,
  xmat, subtree_com, cvel, site_xpos) out of d into `out`'s tensors (allocated when not given);
  returns the output dict.  One C call (mjb_step_io): no allocation besides `out`, no
  synchronisation, capturable in a CUDA graph.  d.time advances by nstep timesteps."""
  inputs = inputs or {}
  io = _abi.MjbStepIO()
  for k, t in inputs.items():
    if k not in _STEP_IO_SHAPES:
      raise ValueError(f"step_io: unknown input {k}")
    n = getattr(m, _STEP_IO_SHAPES[k])
    if tuple(t.shape) != (d.nworld, n) or t.dtype != torch.float32:
      raise ValueError(f"step_io: input {k} must be float32 of shape {(d.nworld, n)}")
    setattr(io, k, _abi._ptr(t.contiguous()))
  res = dict(out or {})
  for k in outputs:
    if k not in _STEP_IO_OUT:
      raise ValueError(f"step_io: unknown output {k}")
    shape = (d.nworld,) + _STEP_IO_OUT[k](m)
    t = res.get(k)
    if t is None:
      t = res[k] = torch.empty(shape, dtype=torch.float32, device=d.qpos.device)
    elif tuple(t.shape) != shape or t.dtype != torch.float32 or not t.is_contiguous():
      raise ValueError(f"step_io: output {k} must be a contiguous float32 tensor of shape {shape}")
    setattr(io, k + "_out", _abi._ptr(t))
  _integrator_check(m)
  rc = _abi.lib().mjb_step_io(ctypes.byref(_abi.model_view(m)), ctypes.byref(_abi.data_view(d)),
                              ctypes.byref(io), int(nstep), ctypes.byref(_form(fused)),
                              _abi.stream())
  _abi.check(rc, "step_io")
  d.time = d.time + nstep * m.opt.timestep
  return res


def step_phase(m: Model, d: Data, phase: int) -> None:
  """One phase of the chosen form's step (not in the reference): 0 = fwd_position ..
  fwd_acceleration, 1 = the constraint solver, 2 = integration.  Phases 0, 1, 2 in order equal
  step(m, d) except for d.time, which only step() advances."""
  L = _abi.lib()
  rc = L.mjb_step_phase(ctypes.byref(_abi.model_view(m)), ctypes.byref(_abi.data_view(d)),
                        int(phase), _abi.stream())
  _abi.check(rc, "step_phase")


def forward(m: Model, d: Data, fused=True) -> None:
  """Forward dynamics (forward.py:664-679); `fused` selects the launch form as in step()."""
  L = _abi.lib()
  rc = L.mjb_forward(ctypes.byref(_abi.model_view(m)), ctypes.byref(_abi.data_view(d)),
                     ctypes.byref(_form(fused)), _abi.stream())
  _abi.check(rc, "forward")


def fwd_position(m: Model, d: Data) -> None:
  """Position-dependent computations (forward.py:408-420)."""
  _call("fwd_position", m, d)


def fwd_velocity(m: Model, d: Data) -> None:
  """Velocity-dependent computations (forward.py:423-500)."""
  _call("fwd_velocity", m, d)


def fwd_actuation(m: Model, d: Data) -> None:
  """Actuation-dependent computations (forward.py:503-641)."""
  _call("fwd_actuation", m, d)


def fwd_acceleration(m: Model, d: Data) -> None:
  """Sum non-constraint forces and compute qacc_smooth (forward.py:644-661)."""
  _call("fwd_acceleration", m, d)


def euler(m: Model, d: Data) -> None:
  """Euler integrator, semi-implicit in velocity (forward.py:165-242)."""
  _call("euler", m, d)
  d.time = d.time + m.opt.timestep


def implicit(m: Model, d: Data) -> None:
  """Implicit-in-velocity integrator, implicitfast (forward.py:245-405)."""
  if m.opt.is_sparse:
    raise NotImplementedError("implicit integration needs the dense mass matrix")
  _call("implicit", m, d)
  d.time = d.time + m.opt.timestep


def kinematics(m: Model, d: Data) -> None:
  """Forward kinematics (smooth.py:32-145)."""
  _call("kinematics", m, d)


def com_pos(m: Model, d: Data) -> None:
  """Subtree CoM, cinert and cdof (smooth.py:148-245)."""
  _call("com_pos", m, d)


def crb(m: Model, d: Data) -> None:
  """Composite rigid body inertia and qM (smooth.py:248-314)."""
  _call("crb", m, d)


def factor_m(m: Model, d: Data) -> None:
  """Factorisation of qM into qLD (smooth.py:392-395)."""
  _call("factor_m", m, d)


def rne(m: Model, d: Data) -> None:
  """Bias forces by recursive Newton-Euler (smooth.py:398-466)."""
  _call("rne", m, d)


def transmission(m: Model, d: Data):
  """Actuator lengths and moments (smooth.py:469-536)."""
  if not m.nu:
    return d
  _call("transmission", m, d)


def com_vel(m: Model, d: Data) -> None:
  """cvel and cdof_dot (smooth.py:539-606)."""
  _call("com_vel", m, d)


def passive(m: Model, d: Data) -> None:
  """Joint springs and dampers (passive.py:27-108)."""
  _call("passive", m, d)


def solve_m(m: Model, d: Data, x: torch.Tensor, y: torch.Tensor) -> None:
  """x = inv(M) y with the factor in qLD (smooth.py:693-696)."""
  L = _abi.lib()
  rc = L.mjb_solve_m(ctypes.byref(_abi.model_view(m)), ctypes.byref(_abi.data_view(d)),
                     _abi._ptr(x), _abi._ptr(y), _abi.stream())
  _abi.check(rc, "solve_m")


def mul_m(m: Model, d: Data, res: torch.Tensor, vec: torch.Tensor, skip: Optional[torch.Tensor] = None) -> None:
  """res = M vec for worlds not skipped (support.py:35-137)."""
  L = _abi.lib()
  if skip is not None and skip.dtype == torch.bool:
    skip = skip.view(torch.uint8)
  rc = L.mjb_mul_m(ctypes.byref(_abi.model_view(m)), ctypes.byref(_abi.data_view(d)),
                   _abi._ptr(res), _abi._ptr(vec), _abi._ptr(skip), _abi.stream())
  _abi.check(rc, "mul_m")


def xfrc_accumulate(m: Model, d: Data, qfrc: torch.Tensor) -> None:
  """qfrc += Jacobian^T xfrc_applied (support.py:140-172)."""
  L = _abi.lib()
  rc = L.mjb_xfrc_accumulate(ctypes.byref(_abi.model_view(m)), ctypes.byref(_abi.data_view(d)),
                             _abi._ptr(qfrc), _abi.stream())
  _abi.check(rc, "xfrc_accumulate")


def collision(m: Model, d: Data) -> None:
  """Collision detection (collision_driver.py:525-547)."""
  _call("collision", m, d)


def nxn_broadphase(m: Model, d: Data) -> None:
  """All-pairs broadphase (collision_driver.py:458-512); appends to the collision_pair list."""
  _call("nxn_broadphase", m, d)


def sap_broadphase(m: Model, d: Data):
  """Sweep-and-prune broadphase (collision_driver.py:350-455)."""
  _call("sap_broadphase", m, d)
  return d


def primitive_narrowphase(m: Model, d: Data) -> None:
  """Primitive narrowphase over collision_pair (collision_primitive.py:271-274)."""
  _call("primitive_narrowphase", m, d)


def make_constraint(m: Model, d: Data) -> None:
  """Constraint rows for limits and pyramidal contacts (constraint.py:213-240)."""
  _call("make_constraint", m, d)


def solve(m: Model, d: Data) -> None:
  """Newton / CG constraint solve (solver.py:872-1000)."""
  _call("solve", m, d)


def world_status(d: Data) -> np.ndarray:
  """Per-world status bits (MJB_WS_* in include/mjb200.h); synchronises the stream."""
  out = np.zeros(d.nworld, dtype=np.uint32)
  rc = _abi.lib().mjb_world_status(ctypes.byref(_abi.data_view(d)), out.ctypes.data_as(ctypes.c_void_p),
                                   _abi.stream())
  _abi.check(rc, "world_status")
  return out


def benchmark(fn: Callable[[Model, Data], None], m: Model, d: Data, nstep: int = 1000,
              graph: bool = True) -> Tuple[float, float, int]:
  """Times nstep calls of fn(m, d) replayed from one captured CUDA graph (test_util.py:57-120).

  Returns (warmup seconds, run seconds, world-steps).
  """
  t0 = _time.perf_counter()
  fn(m, d)
  fn(m, d)
  torch.cuda.synchronize()
  t1 = _time.perf_counter()
  if graph:
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
      with torch.cuda.graph(g, stream=s):
        fn(m, d)
    torch.cuda.current_stream().wait_stream(s)
    run = g.replay
  else:
    run = lambda: fn(m, d)  # noqa: E731
  torch.cuda.synchronize()
  t2 = _time.perf_counter()
  for _ in range(nstep):
    run()
  torch.cuda.synchronize()
  t3 = _time.perf_counter()
  return t1 - t0, t3 - t2, d.nworld * nstep


def autotune(m: Model, d: Data) -> dict:
  """Picks the chosen form's launch parameters for this model and Data (an extension; the
  reference has no autotuner): times the chosen forward for every tree-stage lane count (8, 16,
  32 lanes per world) and solver CTA shape (for nv <= 32 the persistent one-warp-per-world
  solver's CTA width, 1, 2, 4 warps, with the Newton Hessian by FMAs or on the tensor pipe, then
  4 or 5 resident CTAs per SM for the best FMA setting; for
  nv > 32 the warps per world of the CTA solver, 2,
  4, 8, or one warp per world) on d's current worlds and keeps the fastest for later calls with
  the same nv and rows-per-world capacity on this device; reports the rows per world measured.
  d's qacc_warmstart is saved and restored around the trials; d is left as after one forward.
  Synchronises; call it before capturing a CUDA graph."""
  scratch = torch.empty_like(d.qacc_warmstart)
  out = _abi.MjbTune()
  rc = _abi.lib().mjb_autotune(ctypes.byref(_abi.model_view(m)), ctypes.byref(_abi.data_view(d)),
                               _abi._ptr(scratch), ctypes.byref(out), _abi.stream())
  _abi.check(rc, "autotune")
  return {"tree_lanes": out.tree_lanes, "solver_warps": out.solver_warps,
          "solver_cta_warps": out.solver_cta_warps, "hessian_tc": out.hessian_tc,
          "solver_ctas_per_sm": out.solver_ctas_per_sm, "ms_per_forward": out.ms_per_forward,
          "rows_per_world": out.rows_per_world}


def set_tune(m: Model, d: Data, tree_lanes: int = 16, solver_warps: int = 4,
             solver_cta_warps: int = 4, hessian_tc: bool = False,
             solver_ctas_per_sm: int = 0) -> None:
  """Pins the chosen form's launch parameters for this model and Data (an extension, as
  autotune): lanes per world of the tree-recursion stages (8, 16, 32), warps per CTA of the
  one-warp-per-world solver (1, 2, 4), its Newton Hessian on the tensor pipe in split TF32
  (hessian_tc, nv <= 32), its resident CTAs per SM with the FMA Hessian (solver_ctas_per_sm: 4
  or 5, 0 for the default 5) and warps per world of the CTA solver of models with nv > 32
  (2, 4, 8, 16, or 0 for one warp per world)."""
  t = _abi.MjbTune()
  t.tree_lanes, t.solver_warps, t.solver_cta_warps = tree_lanes, solver_warps, solver_cta_warps
  t.hessian_tc = int(bool(hessian_tc))
  t.solver_ctas_per_sm = solver_ctas_per_sm
  rc = _abi.lib().mjb_set_tune(ctypes.byref(_abi.model_view(m)), ctypes.byref(_abi.data_view(d)),
                               ctypes.byref(t))
  if rc == 1:
    raise ValueError(f"set_tune: unsupported setting {tree_lanes}, {solver_warps}, {solver_cta_warps}")
  _abi.check(rc, "set_tune")
