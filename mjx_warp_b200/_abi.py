"""ctypes binding of libmjb200.so (include/mjb200.h).

The field lists below mirror struct MjbModel / MjbData in include/mjb200.h in declaration order
(tests/test_abi.py parses the header and checks them).  Views are filled from the torch tensors of
a Model / Data and cached until one of their fields is reassigned.
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
# MJX_WARP_B200_LIB selects another build of the library (e.g. one compiled with other options)
LIB_PATH = os.environ.get("MJX_WARP_B200_LIB") or os.path.join(_HERE, "libmjb200.so")

MODEL_INTS = ("nq", "nv", "na", "nu", "nbody", "njnt", "ngeom", "nsite", "nmocap", "nM", "nlimit",
              "nlevel", "nblock", "block_max", "npair_cand", "nlsp", "integrator", "cone", "solver",
              "iterations", "ls_iterations", "disableflags", "is_sparse", "ls_parallel",
              "actuator_affine_bias_gain", "precision")
MODEL_FLOATS = ("timestep", "impratio", "tolerance", "ls_tolerance", "meaninertia")
MODEL_PTRS = (
  "body_tree", "body_treeadr", "body_childadr", "body_childnum", "body_child", "body_subtreeend",
  "body_parentid", "body_rootid", "body_weldid", "body_jntnum", "body_jntadr", "body_dofnum",
  "body_dofadr",
  "body_pos", "body_quat", "body_ipos", "body_iquat", "body_mass", "subtree_mass", "body_inertia",
  "body_invweight0",
  "jnt_type", "jnt_qposadr", "jnt_dofadr", "jnt_bodyid", "jnt_limited", "jnt_actfrclimited",
  "jnt_limited_slide_hinge_adr",
  "jnt_solref", "jnt_solimp", "jnt_pos", "jnt_axis", "jnt_stiffness", "jnt_range",
  "jnt_actfrcrange", "jnt_margin",
  "dof_bodyid", "dof_jntid", "dof_parentid", "dof_Madr",
  "dof_armature", "dof_damping", "dof_invweight0",
  "block_adr", "block_size",
  "geom_type", "geom_contype", "geom_conaffinity", "geom_condim", "geom_bodyid", "geom_priority",
  "geom_pos", "geom_quat", "geom_size", "geom_rbound", "geom_solmix", "geom_solref", "geom_solimp",
  "geom_friction", "geom_margin", "geom_gap",
  "pair_cand",
  "site_bodyid",
  "site_pos", "site_quat",
  "actuator_trntype", "actuator_dyntype", "actuator_gaintype", "actuator_biastype",
  "actuator_trnid", "actuator_actadr", "actuator_ctrllimited", "actuator_forcelimited",
  "actuator_actlimited",
  "actuator_dynprm", "actuator_gainprm", "actuator_biasprm", "actuator_ctrlrange",
  "actuator_forcerange", "actuator_actrange", "actuator_gear",
  "qpos0", "qpos_spring",
  "alpha_candidate",
)

DATA_INTS = ("nworld", "nconmax", "njmax")
# (ABI field name, attribute path on the Python Data)
DATA_PTRS = (
  ("qpos", "qpos"), ("qvel", "qvel"), ("act", "act"), ("ctrl", "ctrl"), ("qacc", "qacc"),
  ("qacc_warmstart", "qacc_warmstart"), ("qfrc_applied", "qfrc_applied"),
  ("xfrc_applied", "xfrc_applied"),
  ("xpos", "xpos"), ("xquat", "xquat"), ("xmat", "xmat"), ("xipos", "xipos"), ("ximat", "ximat"),
  ("xanchor", "xanchor"), ("xaxis", "xaxis"), ("geom_xpos", "geom_xpos"),
  ("geom_xmat", "geom_xmat"), ("site_xpos", "site_xpos"), ("site_xmat", "site_xmat"),
  ("subtree_com", "subtree_com"), ("cinert", "cinert"), ("crb", "crb"), ("cdof", "cdof"),
  ("cvel", "cvel"), ("cdof_dot", "cdof_dot"), ("qM", "qM"), ("qLD", "qLD"),
  ("qLDiagInv", "qLDiagInv"),
  ("actuator_length", "actuator_length"), ("actuator_velocity", "actuator_velocity"),
  ("actuator_force", "actuator_force"), ("actuator_moment", "actuator_moment"),
  ("qfrc_bias", "qfrc_bias"), ("qfrc_spring", "qfrc_spring"), ("qfrc_damper", "qfrc_damper"),
  ("qfrc_passive", "qfrc_passive"), ("qfrc_actuator", "qfrc_actuator"),
  ("qfrc_smooth", "qfrc_smooth"), ("qfrc_constraint", "qfrc_constraint"),
  ("qacc_smooth", "qacc_smooth"), ("act_dot", "act_dot"), ("rne_cacc", "rne_cacc"),
  ("rne_cfrc", "rne_cfrc"),
  ("qfrc_integration", "qfrc_integration"), ("qacc_integration", "qacc_integration"),
  ("qM_integration", "qM_integration"), ("qLD_integration", "qLD_integration"),
  ("act_vel_integration", "act_vel_integration"),
  ("ncon", "ncon"), ("nefc", "nefc"), ("ncollision", "ncollision"),
  ("collision_pair", "collision_pair"), ("collision_worldid", "collision_worldid"),
  ("contact_dist", "contact.dist"), ("contact_pos", "contact.pos"),
  ("contact_frame", "contact.frame"), ("contact_includemargin", "contact.includemargin"),
  ("contact_friction", "contact.friction"), ("contact_solref", "contact.solref"),
  ("contact_solreffriction", "contact.solreffriction"), ("contact_solimp", "contact.solimp"),
  ("contact_dim", "contact.dim"), ("contact_geom", "contact.geom"),
  ("contact_efc_address", "contact.efc_address"), ("contact_worldid", "contact.worldid"),
  ("efc_worldid", "efc.worldid"),
  ("efc_J", "efc.J"), ("efc_pos", "efc.pos"), ("efc_margin", "efc.margin"), ("efc_D", "efc.D"),
  ("efc_aref", "efc.aref"), ("efc_force", "efc.force"), ("efc_Jaref", "efc.Jaref"),
  ("efc_jv", "efc.jv"), ("efc_quad", "efc.quad"),
  ("efc_active", "efc.active"),
  ("efc_Ma", "efc.Ma"), ("efc_grad", "efc.grad"), ("efc_grad_dot", "efc.grad_dot"),
  ("efc_Mgrad", "efc.Mgrad"), ("efc_search", "efc.search"), ("efc_search_dot", "efc.search_dot"),
  ("efc_gauss", "efc.gauss"), ("efc_cost", "efc.cost"), ("efc_prev_cost", "efc.prev_cost"),
  ("efc_gtol", "efc.gtol"), ("efc_mv", "efc.mv"), ("efc_quad_gauss", "efc.quad_gauss"),
  ("efc_h", "efc.h"), ("efc_alpha", "efc.alpha"), ("efc_prev_grad", "efc.prev_grad"),
  ("efc_prev_Mgrad", "efc.prev_Mgrad"), ("efc_beta", "efc.beta"),
  ("efc_solver_niter", "efc.solver_niter"),
  ("efc_done", "efc.done"),
  ("world_pairadr", "world_pairadr"), ("world_npair", "world_npair"),
  ("world_conadr", "world_conadr"), ("world_ncon", "world_ncon"),
  ("world_efcadr", "world_efcadr"), ("world_nefc", "world_nefc"),
  ("world_status", "world_status"),
  ("world_order", "world_order"), ("work_queue", "work_queue"),
)


class MjbModel(ctypes.Structure):
  _fields_ = ([(n, ctypes.c_int32) for n in MODEL_INTS]
              + [(n, ctypes.c_float) for n in MODEL_FLOATS]
              + [("gravity", ctypes.c_float * 3)]
              + [(n, ctypes.c_void_p) for n in MODEL_PTRS])


class MjbData(ctypes.Structure):
  _fields_ = ([(n, ctypes.c_int32) for n in DATA_INTS]
              + [(n, ctypes.c_void_p) for n, _ in DATA_PTRS])


class MjbTune(ctypes.Structure):
  _fields_ = [("tree_lanes", ctypes.c_int32), ("solver_warps", ctypes.c_int32),
              ("solver_cta_warps", ctypes.c_int32), ("hessian_tc", ctypes.c_int32),
              ("solver_ctas_per_sm", ctypes.c_int32), ("ms_per_forward", ctypes.c_float),
              ("rows_per_world", ctypes.c_float)]


class MjbRunCfg(ctypes.Structure):
  _fields_ = [("fused", ctypes.c_int32), ("worlds_per_block", ctypes.c_int32)]


STEP_IO_FIELDS = ("qpos", "qvel", "ctrl", "qacc_warmstart", "qpos_out", "qvel_out",
                  "qacc_warmstart_out", "xpos_out", "xmat_out", "subtree_com_out", "cvel_out",
                  "site_xpos_out")


class MjbStepIO(ctypes.Structure):
  _fields_ = [(n, ctypes.c_void_p) for n in STEP_IO_FIELDS]


_STAGES = ("kinematics", "com_pos", "crb", "factor_m", "rne", "transmission", "com_vel",
           "passive", "fwd_velocity", "fwd_actuation", "fwd_acceleration", "euler", "implicit",
           "nxn_broadphase", "fwd_position", "collision", "sap_broadphase",
           "primitive_narrowphase", "make_constraint", "solve")

_lib: Optional[ctypes.CDLL] = None


def lib() -> ctypes.CDLL:
  """Loads libmjb200.so; fails loudly when the CUDA library has not been built."""
  global _lib
  if _lib is not None:
    return _lib
  if not os.path.exists(LIB_PATH):
    raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m mjx_warp_b200.build`")
  L = ctypes.CDLL(LIB_PATH)
  pm, pd = ctypes.POINTER(MjbModel), ctypes.POINTER(MjbData)
  L.mjb_abi_version.restype = ctypes.c_int
  L.mjb_error_string.restype = ctypes.c_char_p
  L.mjb_error_string.argtypes = [ctypes.c_int]
  for n in ("mjb_step", "mjb_forward"):
    f = getattr(L, n)
    f.restype = ctypes.c_int
    f.argtypes = [pm, pd, ctypes.POINTER(MjbRunCfg), ctypes.c_void_p]
  for n in _STAGES:
    f = getattr(L, "mjb_" + n)
    f.restype = ctypes.c_int
    f.argtypes = [pm, pd, ctypes.c_void_p]
  L.mjb_solve_m.restype = ctypes.c_int
  L.mjb_solve_m.argtypes = [pm, pd, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
  L.mjb_mul_m.restype = ctypes.c_int
  L.mjb_mul_m.argtypes = [pm, pd, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
  L.mjb_xfrc_accumulate.restype = ctypes.c_int
  L.mjb_xfrc_accumulate.argtypes = [pm, pd, ctypes.c_void_p, ctypes.c_void_p]
  L.mjb_step_io.restype = ctypes.c_int
  L.mjb_step_io.argtypes = [pm, pd, ctypes.POINTER(MjbStepIO), ctypes.c_int,
                            ctypes.POINTER(MjbRunCfg), ctypes.c_void_p]
  L.mjb_step_phase.restype = ctypes.c_int
  L.mjb_step_phase.argtypes = [pm, pd, ctypes.c_int, ctypes.c_void_p]
  L.mjb_world_status.restype = ctypes.c_int
  L.mjb_world_status.argtypes = [pd, ctypes.c_void_p, ctypes.c_void_p]
  vp, ci, cf = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
  L.mjb_fd_perturb.restype = ctypes.c_int
  L.mjb_fd_perturb.argtypes = [pm, pd, pd, cf, ci, vp]
  L.mjb_fd_jacobian.restype = ctypes.c_int
  L.mjb_fd_jacobian.argtypes = [pm, pd, ci, cf, ci, vp, vp, vp]
  L.mjb_ctrl_vjp.restype = ctypes.c_int
  L.mjb_ctrl_vjp.argtypes = [pm, pd, vp, vp, vp]
  L.mjb_step_vjp.restype = ctypes.c_int
  L.mjb_step_vjp.argtypes = [pm, pd, vp, vp, vp, vp, vp, vp]
  L.mjb_autotune.restype = ctypes.c_int
  L.mjb_autotune.argtypes = [pm, pd, vp, ctypes.POINTER(MjbTune), vp]
  L.mjb_set_tune.restype = ctypes.c_int
  L.mjb_set_tune.argtypes = [pm, pd, ctypes.POINTER(MjbTune)]
  L.mjb_transition_vjp.restype = ctypes.c_int
  L.mjb_transition_vjp.argtypes = [pm, ci, vp, vp, vp, vp, vp, vp]
  if L.mjb_abi_version() != 7:
    raise RuntimeError("libmjb200.so ABI version mismatch")
  _lib = L
  return L


def check(rc: int, what: str) -> None:
  if rc != 0:
    msg = lib().mjb_error_string(rc).decode()
    if rc == 2:
      raise NotImplementedError(f"{what}: {msg}")
    raise RuntimeError(f"{what} failed ({rc}): {msg}")


def _ptr(t) -> int:
  if t is None:
    return 0
  if not isinstance(t, torch.Tensor):
    raise TypeError(f"expected a tensor, got {type(t)}")
  if t.numel() == 0:
    return 0
  if not t.is_cuda:
    raise RuntimeError("mjx_warp_b200 kernels need CUDA tensors; this Data/Model lives on the CPU")
  if not t.is_contiguous():
    raise ValueError("mjx_warp_b200 kernels need contiguous tensors")
  return t.data_ptr()


def model_view(m) -> MjbModel:
  """MjbModel for Model m, rebuilt when a field was reassigned; options refreshed every call."""
  v = m.__dict__.get("_view_cache")
  flags = int(m.opt.disableflags)
  if v is None or v._flags != flags:
    from .io import pair_candidates  # host-side table that depends on the current options
    pc = pair_candidates(m)
    object.__setattr__(m, "_pair_cand", pc)
    v = MjbModel()
    for n in MODEL_PTRS:
      if n == "pair_cand":
        setattr(v, n, _ptr(pc))
      else:
        setattr(v, n, _ptr(getattr(m, n)))
    v.npair_cand = pc.shape[0]
    v._flags = flags
    object.__setattr__(m, "_view_cache", v)
  for n in ("nq", "nv", "na", "nu", "nbody", "njnt", "ngeom", "nsite", "nmocap", "nM"):
    setattr(v, n, int(getattr(m, n)))
  v.nlimit = int(m.jnt_limited_slide_hinge_adr.shape[0])
  v.nlevel = int(m.body_treeadr.shape[0] - 1)
  v.nblock = int(m.block_adr.shape[0])
  v.block_max = int(m.__dict__.get("_block_max", -1))
  if v.block_max < 0:
    v.block_max = int(m.block_size.max().item()) if m.block_size.numel() else 0
    object.__setattr__(m, "_block_max", v.block_max)
  v.nlsp = int(m.nlsp)
  o = m.opt
  v.integrator, v.cone, v.solver = int(o.integrator), int(o.cone), int(o.solver)
  v.iterations, v.ls_iterations = int(o.iterations), int(o.ls_iterations)
  v.disableflags, v.is_sparse, v.ls_parallel = flags, int(bool(o.is_sparse)), int(bool(o.ls_parallel))
  v.actuator_affine_bias_gain = int(bool(m.actuator_affine_bias_gain))
  v.timestep, v.impratio = float(o.timestep), float(o.impratio)
  v.tolerance, v.ls_tolerance = float(o.tolerance), float(o.ls_tolerance)
  v.meaninertia = float(m.stat.meaninertia)
  g = o.gravity
  for k in range(3):
    v.gravity[k] = float(g[k])
  return v


def _get(d, path):
  obj = d
  for part in path.split("."):
    obj = getattr(obj, part, None)
    if obj is None:
      return None
  return obj


def data_view(d) -> MjbData:
  """MjbData for Data d, rebuilt when a field (or a contact / efc field) was reassigned."""
  v = d.__dict__.get("_view_cache")
  if v is None:
    v = MjbData()
    v.nworld, v.nconmax, v.njmax = int(d.nworld), int(d.nconmax), int(d.njmax)
    for abi, path in DATA_PTRS:
      setattr(v, abi, _ptr(_get(d, path)))
    object.__setattr__(d, "_view_cache", v)
  return v


def stream() -> int:
  return torch.cuda.current_stream().cuda_stream
