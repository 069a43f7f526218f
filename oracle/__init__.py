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
