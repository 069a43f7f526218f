"""ORACLE — test infrastructure only (see oracle.cpp).

ctypes binding of the CPU restatement of the reference's batched step.  Imported by tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg; never by the product package.
The model description is derived here from the host model's raw arrays with this module's own
table builders (BFS levels, limited slide/hinge joints, tree blocks), independently of the
product's ``put_model``.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Dict, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")

STAGES = {
  "step": 0, "forward": 1, "fwd_position": 2, "fwd_velocity": 3, "fwd_actuation": 4,
  "fwd_acceleration": 5, "kinematics": 6, "com_pos": 7, "crb": 8, "factor_m": 9,
  "collision": 10, "nxn_broadphase": 11, "narrowphase": 12, "make_constraint": 13,
  "transmission": 14, "com_vel": 15, "passive": 16, "rne": 17, "solve": 18, "euler": 19,
  "implicit": 20, "forward_nosolve": 21, "sap_broadphase": 22,
}


def build(force: bool = False) -> str:
  """Compiles liboracle.so with g++ (OpenMP, no floating-point contraction)."""
  src = os.path.join(_HERE, "oracle.cpp")
  if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src):
    return LIB_PATH
  cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-shared", "-fPIC",
         "-o", LIB_PATH, src]
  subprocess.check_call(cmd)
  return LIB_PATH


_I = ctypes.POINTER(ctypes.c_int32)
_D = ctypes.POINTER(ctypes.c_double)


class OracleModelDesc(ctypes.Structure):
  _fields_ = (
    [(n, ctypes.c_int) for n in (
      "nq", "nv", "na", "nu", "nbody", "njnt", "ngeom", "nsite", "nmocap", "nlimit", "nlevel",
      "nblock", "integrator", "cone", "solver", "iterations", "ls_iterations", "disableflags",
      "ls_parallel", "nlsp", "actuator_affine_bias_gain")]
    + [(n, ctypes.c_double) for n in ("timestep", "impratio", "tolerance", "ls_tolerance",
                                      "meaninertia")]
    + [("gravity", ctypes.c_double * 3)]
    + [(n, _I) for n in ("body_tree", "body_treeadr", "body_parentid", "body_rootid",
                         "body_weldid", "body_jntnum", "body_jntadr", "body_dofnum",
                         "body_dofadr")]
    + [(n, _D) for n in ("body_pos", "body_quat", "body_ipos", "body_iquat", "body_mass",
                         "subtree_mass", "body_inertia", "body_invweight0")]
    + [(n, _I) for n in ("jnt_type", "jnt_qposadr", "jnt_dofadr", "jnt_bodyid", "jnt_limited",
                         "jnt_actfrclimited", "jnt_limited_slide_hinge_adr")]
    + [(n, _D) for n in ("jnt_solref", "jnt_solimp", "jnt_pos", "jnt_axis", "jnt_stiffness",
                         "jnt_range", "jnt_actfrcrange", "jnt_margin")]
    + [(n, _I) for n in ("dof_bodyid", "dof_jntid", "dof_parentid")]
    + [(n, _D) for n in ("dof_armature", "dof_damping", "dof_invweight0")]
    + [(n, _I) for n in ("block_adr", "block_size")]
    + [(n, _I) for n in ("geom_type", "geom_contype", "geom_conaffinity", "geom_condim",
                         "geom_bodyid", "geom_priority")]
    + [(n, _D) for n in ("geom_pos", "geom_quat", "geom_size", "geom_rbound", "geom_solmix",
                         "geom_solref", "geom_solimp", "geom_friction", "geom_margin",
                         "geom_gap")]
    + [("site_bodyid", _I)]
    + [(n, _D) for n in ("site_pos", "site_quat")]
    + [(n, _I) for n in ("actuator_trntype", "actuator_dyntype", "actuator_gaintype",
                         "actuator_biastype", "actuator_trnid", "actuator_actadr",
                         "actuator_ctrllimited", "actuator_forcelimited",
                         "actuator_actlimited")]
    + [(n, _D) for n in ("actuator_dynprm", "actuator_gainprm", "actuator_biasprm",
                         "actuator_ctrlrange", "actuator_forcerange", "actuator_actrange",
                         "actuator_gear")]
    + [(n, _D) for n in ("qpos0", "qpos_spring")]
  )


def _tables(mjm) -> Dict[str, np.ndarray]:
  """Derived tables, built from the raw model arrays (independently of put_model)."""
  nb = mjm.nbody
  depth = np.zeros(nb, dtype=int)
  for b in range(1, nb):
    depth[b] = depth[mjm.body_parentid[b]] + 1
  levels = [[b for b in range(nb) if depth[b] == d] for d in range(depth.max() + 1)]
  tree = np.array([b for lv in levels for b in lv], dtype=np.int32)
  treeadr = np.cumsum([0] + [len(lv) for lv in levels]).astype(np.int32)
  lim = np.nonzero(np.asarray(mjm.jnt_limited).astype(bool)
                   & ((np.asarray(mjm.jnt_type) == 2) | (np.asarray(mjm.jnt_type) == 3)))[0]
  corners = [i for i in range(mjm.nv) if mjm.dof_parentid[i] == -1]
  bsize = [(corners[i + 1] if i + 1 < len(corners) else mjm.nv) - corners[i]
           for i in range(len(corners))]
  smass = np.array(mjm.body_mass, dtype=float).copy()
  for i in range(nb - 1, -1, -1):  # includes the world adding into itself, as io.py:249-252
    smass[mjm.body_parentid[i]] += smass[i]
  return {"body_tree": tree, "body_treeadr": treeadr, "nlevel": len(levels),
          "jnt_limited_slide_hinge_adr": lim.astype(np.int32),
          "block_adr": np.array(corners, dtype=np.int32),
          "block_size": np.array(bsize, dtype=np.int32), "subtree_mass": smass}


class Oracle:
  """A batch of nworld worlds evaluated by the CPU restatement."""

  def __init__(self, mjm, nworld: int, precision: int = 64, ls_parallel: bool = False):
    build()
    self.lib = ctypes.CDLL(LIB_PATH)
    self.lib.oracle_create.restype = ctypes.c_void_p
    self.lib.oracle_create.argtypes = [ctypes.POINTER(OracleModelDesc), ctypes.c_int, ctypes.c_int]
    self.lib.oracle_destroy.argtypes = [ctypes.c_void_p]
    self.lib.oracle_run.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 4
    self.lib.oracle_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _D, _D, ctypes.c_int]
    self.lib.oracle_rows.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _I, _D, _D]
    self.lib.oracle_solver_scalar.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _D]
    self.mjm = mjm
    self.nworld = nworld
    self.precision = precision
    self._keep = []
    t = _tables(mjm)
    desc = OracleModelDesc()
    ints = dict(nq=mjm.nq, nv=mjm.nv, na=mjm.na, nu=mjm.nu, nbody=mjm.nbody, njnt=mjm.njnt,
                ngeom=mjm.ngeom, nsite=mjm.nsite, nmocap=mjm.nmocap,
                nlimit=len(t["jnt_limited_slide_hinge_adr"]), nlevel=t["nlevel"],
                nblock=len(t["block_adr"]), integrator=mjm.opt.integrator, cone=mjm.opt.cone,
                solver=mjm.opt.solver, iterations=mjm.opt.iterations,
                ls_iterations=mjm.opt.ls_iterations, disableflags=mjm.opt.disableflags,
                ls_parallel=int(ls_parallel), nlsp=mjm.opt.ls_iterations,
                actuator_affine_bias_gain=int(np.any(np.asarray(mjm.actuator_biastype) == 1)
                                              or np.any(np.asarray(mjm.actuator_gaintype) == 1)))
    for k, v in ints.items():
      setattr(desc, k, int(v))
    desc.timestep = mjm.opt.timestep
    desc.impratio = mjm.opt.impratio
    desc.tolerance = mjm.opt.tolerance
    desc.ls_tolerance = mjm.opt.ls_tolerance
    desc.meaninertia = mjm.stat.meaninertia
    for k in range(3):
      desc.gravity[k] = mjm.opt.gravity[k]
    for name, typ in OracleModelDesc._fields_:
      if typ not in (_I, _D):
        continue
      src = t[name] if name in t else getattr(mjm, name)
      if typ is _I:
        arr = np.ascontiguousarray(np.asarray(src, dtype=np.int32).reshape(-1))
        if arr.size == 0:
          arr = np.zeros(1, dtype=np.int32)
        setattr(desc, name, arr.ctypes.data_as(_I))
      else:
        arr = np.ascontiguousarray(np.asarray(src, dtype=np.float64).reshape(-1))
        if arr.size == 0:
          arr = np.zeros(1)
        setattr(desc, name, arr.ctypes.data_as(_D))
      self._keep.append(arr)
    self._desc = desc
    self.h = self.lib.oracle_create(ctypes.byref(desc), nworld, precision)

  def __del__(self):
    h = getattr(self, "h", None)
    if h:
      self.lib.oracle_destroy(h)
      self.h = None

  def run(self, stage: str = "step", nstep: int = 1, nthreads: int = 0, njmax_zero: bool = False):
    self.lib.oracle_run(self.h, STAGES[stage], nstep, nthreads, int(njmax_zero))

  def get(self, name: str, world: Optional[int] = None) -> np.ndarray:
    n = self.lib.oracle_field(self.h, name.encode(), None, None, -1 if world is None else world)
    if n < 0:
      raise KeyError(name)
    out = np.zeros(n)
    self.lib.oracle_field(self.h, name.encode(), out.ctypes.data_as(_D), None,
                          -1 if world is None else world)
    return out.reshape(1 if world is not None else self.nworld, -1)

  def set(self, name: str, value, world: Optional[int] = None) -> None:
    """Sets a per-world field: value is (nworld, n) or (n,) broadcast to every world."""
    value = np.asarray(value, dtype=np.float64)
    if world is None and (value.ndim < 2 or value.shape[0] != self.nworld):
      value = np.tile(value.reshape(1, -1), (self.nworld, 1))
    value = np.ascontiguousarray(value.reshape(-1))
    n = self.lib.oracle_field(self.h, name.encode(), None, value.ctypes.data_as(_D),
                              -1 if world is None else world)
    if n < 0:
      raise KeyError(name)

  def rows(self, name: str):
    """Returns (counts per world, concatenated rows as (total, width))."""
    counts = np.zeros(self.nworld, dtype=np.int32)
    n = self.lib.oracle_rows(self.h, name.encode(), counts.ctypes.data_as(_I), None, None)
    if n < 0:
      raise KeyError(name)
    out = np.zeros(n)
    self.lib.oracle_rows(self.h, name.encode(), counts.ctypes.data_as(_I), out.ctypes.data_as(_D),
                         None)
    total = int(counts.sum())
    return counts, out.reshape(total, -1) if total else out.reshape(0, max(1, n))

  def set_rows(self, name: str, counts, data) -> None:
    counts = np.ascontiguousarray(np.asarray(counts, dtype=np.int32))
    data = np.ascontiguousarray(np.asarray(data, dtype=np.float64).reshape(-1))
    if data.size == 0:
      data = np.zeros(1)
    n = self.lib.oracle_rows(self.h, name.encode(), counts.ctypes.data_as(_I), None,
                             data.ctypes.data_as(_D))
    if n < 0:
      raise KeyError(name)

  def scalar(self, name: str) -> np.ndarray:
    out = np.zeros(self.nworld)
    if self.lib.oracle_solver_scalar(self.h, name.encode(), out.ctypes.data_as(_D)) < 0:
      raise KeyError(name)
    return out


def closest_segments(a0, a1, b0, b1, precision: int = 64):
  """Closest points between segments a0-a1 and b0-b1 (math.py:209-242)."""
  build()
  lib = ctypes.CDLL(LIB_PATH)
  lib.oracle_closest_segments.argtypes = [_D] * 6 + [ctypes.c_int]
  arrs = [np.ascontiguousarray(np.asarray(x, dtype=np.float64)) for x in (a0, a1, b0, b1)]
  pa, pb = np.zeros(3), np.zeros(3)
  lib.oracle_closest_segments(*[a.ctypes.data_as(_D) for a in arrs], pa.ctypes.data_as(_D),
                              pb.ctypes.data_as(_D), precision)
  return pa, pb


def qacc_references(mjm, qpos, qvel, ctrl, warmstart, nthreads: int = 0, nperturb: int = 24,
                    seed: int = 0) -> dict:
  """qacc of one forward from the same per-world state by the restatement in FP64 and in FP32,
  plus how far the FP64 iterate is from convergence and how far rounding alone moves it.
  Returns a dict of per-world arrays: fp64, fp32 (qacc); fp64_unconverged = the FP64 iterate's
  distance from the converged FP64 solution (100 Newton / 50 line-search iterations); fp64_spread
  = the largest change of FP64 solves from inputs perturbed by up to one FP32 ulp (relative
  2^-23, 2 draws); fp32_worst = the largest error against FP64 of any FP32 realisation
  (unperturbed, or from such perturbed inputs, `nperturb` draws); all as
  ||x - y|| / max(||y||, 1)."""
  import copy

  def run(model, prec, inputs):
    o = Oracle(model, qpos.shape[0], prec)
    for k, v in inputs.items():
      o.set(k, v)
    o.run("forward", nthreads=nthreads)
    return o.get("qacc")

  base = {"qpos": qpos, "qvel": qvel, "qacc_warmstart": warmstart}
  if mjm.nu:
    base["ctrl"] = ctrl
  ref64 = run(mjm, 64, base)
  ref32 = run(mjm, 32, base)
  conv = copy.deepcopy(mjm)
  conv.opt.iterations, conv.opt.ls_iterations = 100, 50
  unconverged = rel_err(ref64, run(conv, 64, base))
  rng = np.random.default_rng(seed)
  spread = np.zeros(qpos.shape[0])
  worst32 = rel_err(ref32, ref64)
  for t in range(nperturb):
    pert = {k: v * (1.0 + rng.uniform(-1.0, 1.0, v.shape) * 2.0 ** -23) for k, v in base.items()}
    worst32 = np.maximum(worst32, rel_err(run(mjm, 32, pert), ref64))
    if t < 2:
      spread = np.maximum(spread, rel_err(run(mjm, 64, pert), ref64))
  return {"fp64": ref64, "fp32": ref32, "fp64_unconverged": unconverged, "fp64_spread": spread,
          "fp32_worst": worst32}


def rel_err(a, b) -> np.ndarray:
  """Per-world ||a - b|| / max(||b||, 1)."""
  a = np.asarray(a, dtype=np.float64).reshape(a.shape[0], -1)
  b = np.asarray(b, dtype=np.float64).reshape(b.shape[0], -1)
  e = np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1.0)
  return np.where(np.isfinite(e), e, np.inf)


def classify_qacc(q, refs: dict, tol: float = 1e-4) -> dict:
  """Splits the worlds where q (the device's qacc) misses FP64 by more than tol into: within tol of
  the FP32 restatement (the same miss as an FP32 implementation of the reference's algorithm
  makes); path-dependent (at these iteration counts the FP64 iterate is itself more than tol from
  the converged solution, so which line-search / active-set path the iterations take decides the
  result, or an FP32 realisation of the restatement from inputs within one ulp also misses, or
  FP64 moves by more than tol under such perturbations); and unexplained (none of these).
  refs: qacc_references' dict."""
  ref64, ref32 = refs["fp64"], refs["fp32"]
  e64 = rel_err(q, ref64)
  e32 = rel_err(q, ref32)
  o32 = rel_err(ref32, ref64)
  sensitive = ((refs["fp64_unconverged"] > tol) | (refs["fp32_worst"] > tol)
               | (refs["fp64_spread"] > tol))
  over = e64 > tol
  near32 = over & (e32 <= tol)
  sens = over & ~near32 & sensitive
  unexplained = over & ~near32 & ~sens
  return {"worlds": int(len(e64)), "frac_le_tol_vs_fp64": float(np.mean(~over)),
          "frac_le_tol_vs_fp32_restatement": float(np.mean(e32 <= tol)),
          "median_vs_fp64": float(np.median(e64)), "max_vs_fp64": float(e64.max()),
          "median_vs_fp32_restatement": float(np.median(e32)),
          "over_tol": int(over.sum()), "over_tol_within_tol_of_fp32_restatement": int(near32.sum()),
          "over_tol_path_dependent": int(sens.sum()), "over_tol_unexplained": int(unexplained.sum()),
          "fp32_restatement_frac_le_tol_vs_fp64": float(np.mean(o32 <= tol)),
          "unconverged_worlds": int(np.sum(refs["fp64_unconverged"] > tol)),
          "path_dependent_worlds": int(np.sum(sensitive)),
          "frac_le_tol_vs_fp64_in_converged_worlds":
              float(np.mean(~over[refs["fp64_unconverged"] <= tol]))
              if np.any(refs["fp64_unconverged"] <= tol) else None,
          "unexplained_worlds": {int(i): {"vs_fp64": float(e64[i]), "vs_fp32": float(e32[i]),
                                          "fp32_worst": float(refs["fp32_worst"][i]),
                                          "fp64_spread": float(refs["fp64_spread"][i]),
                                          "fp64_unconverged": float(refs["fp64_unconverged"][i])}
                                 for i in np.nonzero(unexplained)[0][:16]}}
