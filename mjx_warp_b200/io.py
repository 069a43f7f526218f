"""Host <-> device transfer: put_model, make_data, put_data, get_data_into.

Mirrors mujoco_warp/_src/io.py.  put_model validates the model like io.py:24-42, uploads every
array the kernels read as float32 / int32 torch tensors and derives the index tables the
reference builds (BFS body levels io.py:113-124, dense tree tiles :149-162, limited slide/hinge
joints :105-111, subtree mass :249-254, parallel line-search candidates :233) plus the B200
layout tables: children per body (bottom-up gathers instead of atomics), DFS subtree ranges
(ancestor tests in O(1)) and the statically filtered broadphase candidate pairs.
"""

from __future__ import annotations

import numpy as np
import torch

from . import types
from .types import Constraint, Contact, Data, Model

_SUPPORTED_INTEGRATORS = {0, 3}


def _device(device):
  if device is not None:
    return torch.device(device)
  return torch.device("cuda" if torch.cuda.is_available() else "cpu")


def is_sparse(mjm) -> bool:
  """support.py:29-32: AUTO picks the sparse path for nv >= 60."""
  if mjm.opt.jacobian == types.MJ_JAC_AUTO:
    return mjm.nv >= 60
  return mjm.opt.jacobian == types.MJ_JAC_SPARSE


def _f(x, dev):
  return torch.as_tensor(np.ascontiguousarray(np.asarray(x, dtype=np.float32)), device=dev)


def _i(x, dev):
  return torch.as_tensor(np.ascontiguousarray(np.asarray(x, dtype=np.int32)), device=dev)


def _bfs_levels(parentid):
  nb = len(parentid)
  depth = np.zeros(nb, dtype=int)
  bodies = {}
  for i in range(nb):
    depth[i] = depth[parentid[i]] + 1 if i > 0 else 0
    bodies.setdefault(depth[i], []).append(i)
  tree = np.concatenate([bodies[i] for i in range(len(bodies))])
  off = np.cumsum([0] + [len(bodies[i]) for i in range(len(bodies))])
  return tree.astype(np.int32), off.astype(np.int32)  # off has nlevel + 1 entries


def _static_pair_filter(mjm, filterparent, contype, conaffinity):
  """collision_driver.py:27-49 evaluated on the host for every geom pair, nxn order."""
  ng = mjm.ngeom
  bodyid = np.asarray(mjm.geom_bodyid)
  weld = np.asarray(mjm.body_weldid)
  parent = np.asarray(mjm.body_parentid)
  out = []
  for g1 in range(ng):
    for g2 in range(g1 + 1, ng):
      w1, w2 = weld[bodyid[g1]], weld[bodyid[g2]]
      wp1, wp2 = weld[parent[w1]], weld[parent[w2]]
      self_col = w1 == w2
      pc = filterparent and w1 != 0 and w2 != 0 and (w1 == wp2 or w2 == wp1)
      mask = (contype[g1] & conaffinity[g2]) or (contype[g2] & conaffinity[g1])
      if mask and not self_col and not pc:
        out.append((g1, g2))
  return np.array(out, dtype=np.int32).reshape(-1, 2)


def pair_candidates(m: Model) -> torch.Tensor:
  """Broadphase candidates for the model's current contype/conaffinity and FILTERPARENT flag."""
  filterparent = not (int(m.opt.disableflags) & types.DisableBit.FILTERPARENT)
  key = (filterparent, m.geom_contype.data_ptr(), m.geom_conaffinity.data_ptr())
  cache = m.__dict__.get("_pair_cache")
  if cache is not None and cache[0] == key:
    return cache[1]
  h = m._host
  pc = _static_pair_filter(h, filterparent, m.geom_contype.cpu().numpy(),
                           m.geom_conaffinity.cpu().numpy())
  t = _i(pc, m.geom_type.device)
  object.__setattr__(m, "_pair_cache", (key, t))
  return t


class _HostModel:
  """Host copies of the raw arrays the filter tables need."""

  def __init__(self, mjm):
    self.ngeom = mjm.ngeom
    self.geom_bodyid = np.asarray(mjm.geom_bodyid).copy()
    self.body_weldid = np.asarray(mjm.body_weldid).copy()
    self.body_parentid = np.asarray(mjm.body_parentid).copy()


def put_model(mjm, device=None) -> Model:
  """Uploads a compiled model (io.py:24-334)."""
  if mjm.neq > 0:
    raise NotImplementedError("Equality constraints are unsupported.")
  if mjm.nsensor > 0:
    raise NotImplementedError("Sensors are unsupported.")
  if mjm.ntendon > 0:
    raise NotImplementedError("Tendons are unsupported.")
  if mjm.opt.integrator not in _SUPPORTED_INTEGRATORS:
    raise NotImplementedError(f"Integrator: {mjm.opt.integrator} is unsupported.")
  if mjm.opt.cone != types.ConeType.PYRAMIDAL:
    raise NotImplementedError(f"Cone: {mjm.opt.cone} is unsupported.")
  if mjm.opt.solver not in (types.SolverType.CG, types.SolverType.NEWTON):
    raise NotImplementedError(f"Solver: {mjm.opt.solver} is unsupported.")

  dev = _device(device)
  m = Model()
  for n in ("nq", "nv", "na", "nu", "nbody", "njnt", "ngeom", "nsite", "nmocap", "nM", "nexclude"):
    object.__setattr__(m, n, int(getattr(mjm, n)))
  object.__setattr__(m, "nlsp", int(mjm.opt.ls_iterations))
  opt = types.Option(
    timestep=float(mjm.opt.timestep), impratio=float(mjm.opt.impratio),
    tolerance=float(mjm.opt.tolerance), ls_tolerance=float(mjm.opt.ls_tolerance),
    gravity=np.array(mjm.opt.gravity, dtype=np.float32), integrator=int(mjm.opt.integrator),
    cone=int(mjm.opt.cone), solver=int(mjm.opt.solver), iterations=int(mjm.opt.iterations),
    ls_iterations=int(mjm.opt.ls_iterations), disableflags=int(mjm.opt.disableflags),
    is_sparse=is_sparse(mjm), ls_parallel=False)
  object.__setattr__(m, "opt", opt)
  object.__setattr__(m, "stat", types.Statistic(meaninertia=float(mjm.stat.meaninertia)))
  object.__setattr__(m, "_host", _HostModel(mjm))

  nv, nb = mjm.nv, mjm.nbody
  parent = np.asarray(mjm.body_parentid)
  dof_parentid = np.asarray(mjm.dof_parentid)

  # BFS levels (io.py:113-124)
  body_tree, body_treeadr = _bfs_levels(parent)
  m.body_tree = _i(body_tree, dev)
  m.body_treeadr = _i(body_treeadr, dev)
  # children per body, DFS subtree ends
  children = [[] for _ in range(nb)]
  for b in range(1, nb):
    children[parent[b]].append(b)
  childadr = np.cumsum([0] + [len(c) for c in children])[:-1]
  m.body_childadr = _i(childadr, dev)
  m.body_childnum = _i([len(c) for c in children], dev)
  m.body_child = _i([b for c in children for b in c] or [0], dev)
  subtreeend = np.arange(nb) + 1
  for b in range(nb - 1, 0, -1):
    subtreeend[parent[b]] = max(subtreeend[parent[b]], subtreeend[b])
  m.body_subtreeend = _i(subtreeend, dev)

  # dof lower triangle / sparse index tables (io.py:76-103), kept for API parity
  tri_row, tri_col = np.tril_indices(nv)
  m.dof_tri_row = _i(tri_row, dev)
  m.dof_tri_col = _i(tri_col, dev)
  fi, fj = [], []
  for i in range(nv):
    j = i
    while j > -1:
      fi.append(i)
      fj.append(j)
      j = dof_parentid[j]
  m.qM_fullm_i = _i(fi, dev)
  m.qM_fullm_j = _i(fj, dev)
  mi, mj, madr = [], [], []
  for i in range(nv):
    a, j = int(mjm.dof_Madr[i]), i
    while True:
      a, j = a + 1, dof_parentid[j]
      if j == -1:
        break
      mi.append(i)
      mj.append(j)
      madr.append(a)
  m.qM_mulm_i = _i(mi, dev)
  m.qM_mulm_j = _i(mj, dev)
  m.qM_madr_ij = _i(madr, dev)

  # limited slide / hinge joints (io.py:105-111)
  jt = np.asarray(mjm.jnt_type)
  lim = np.nonzero(np.asarray(mjm.jnt_limited).astype(bool) & ((jt == 2) | (jt == 3)))[0]
  m.jnt_limited_slide_hinge_adr = _i(lim, dev)

  # dense tree tiles (io.py:149-162): one block per tree, in dof order
  corners = [i for i in range(nv) if dof_parentid[i] == -1]
  bsize = [(corners[k + 1] if k + 1 < len(corners) else nv) - corners[k] for k in range(len(corners))]
  m.block_adr = _i(corners, dev)
  m.block_size = _i(bsize, dev)
  tiles = {}
  for a, s in zip(corners, bsize):
    tiles.setdefault(s, []).append(a)
  keys = sorted(tiles)
  m.qLD_tile = _i([a for k in keys for a in tiles[k]], dev)
  m.qLD_tileadr = _i(np.cumsum([0] + [len(tiles[k]) for k in keys])[:-1], "cpu")
  m.qLD_tilesize = _i(keys, "cpu")

  m.alpha_candidate = _f(np.linspace(0.0, 1.0, max(int(mjm.opt.ls_iterations), 1)), dev)

  # subtree mass: the loop includes the world adding into itself (io.py:249-254)
  smass = np.array(mjm.body_mass, dtype=float)
  for i in range(nb - 1, -1, -1):
    smass[parent[i]] += smass[i]
  m.subtree_mass = _f(smass, dev)

  ints = ("body_parentid", "body_rootid", "body_weldid", "body_mocapid", "body_jntnum",
          "body_jntadr", "body_dofnum", "body_dofadr", "body_geomnum", "body_geomadr",
          "body_contype", "body_conaffinity", "jnt_type", "jnt_qposadr", "jnt_dofadr",
          "jnt_bodyid", "jnt_limited", "jnt_actfrclimited", "dof_bodyid", "dof_jntid",
          "dof_parentid", "dof_Madr", "geom_type", "geom_contype", "geom_conaffinity",
          "geom_condim", "geom_bodyid", "geom_priority", "geom_dataid", "site_bodyid",
          "actuator_trntype", "actuator_dyntype", "actuator_gaintype", "actuator_biastype",
          "actuator_trnid", "actuator_actadr", "actuator_ctrllimited", "actuator_forcelimited",
          "actuator_actlimited", "mesh_vertadr", "mesh_vertnum", "exclude_signature")
  floats = ("qpos0", "qpos_spring", "body_pos", "body_quat", "body_ipos", "body_iquat",
            "body_inertia", "body_mass", "body_invweight0", "jnt_solref", "jnt_solimp",
            "jnt_pos", "jnt_axis", "jnt_range", "jnt_margin", "jnt_stiffness",
            "jnt_actfrcrange", "dof_armature", "dof_damping", "dof_invweight0", "geom_pos",
            "geom_quat", "geom_size", "geom_priority_f", "geom_solmix", "geom_solref",
            "geom_solimp", "geom_friction", "geom_margin", "geom_gap", "geom_aabb",
            "geom_rbound", "mesh_vert", "site_pos", "site_quat", "actuator_ctrlrange",
            "actuator_forcerange", "actuator_gainprm", "actuator_biasprm", "actuator_gear",
            "actuator_actrange", "actuator_dynprm")
  for n in ints:
    setattr(m, n, _i(np.asarray(getattr(mjm, n)), dev))
  for n in floats:
    if n == "geom_priority_f":
      continue
    arr = np.asarray(getattr(mjm, n), dtype=np.float64)
    if n == "geom_aabb":
      arr = arr.reshape(mjm.ngeom, 2, 3)
    setattr(m, n, _f(arr, dev))

  # io.py:328-332
  object.__setattr__(m, "actuator_affine_bias_gain", bool(
    np.any(np.asarray(mjm.actuator_biastype) == types.BiasType.AFFINE)
    or np.any(np.asarray(mjm.actuator_gaintype) == types.GainType.AFFINE)))
  object.__setattr__(m, "_view_cache", None)
  return m


# ----------------------------------------------------------------------------------------------
# Data


def _data_arrays(mjm, nworld, nconmax, njmax, dev):
  """Field name -> zero tensor with the reference's logical shape (io.py:395-506)."""
  nq, nv, nu, na, nb, nj = mjm.nq, mjm.nv, mjm.nu, mjm.na, mjm.nbody, mjm.njnt
  ng, ns, nm = mjm.ngeom, mjm.nsite, mjm.nmocap
  f = lambda *s: torch.zeros(s, dtype=torch.float32, device=dev)  # noqa: E731
  i = lambda *s: torch.zeros(s, dtype=torch.int32, device=dev)  # noqa: E731
  W = nworld
  # the reference's layout: (nworld, 1, nM) for the sparse mass matrix, (nworld, nv, nv) dense
  mshape = (W, 1, int(mjm.nM)) if is_sparse(mjm) else (W, nv, nv)
  top = {
    "qpos": f(W, nq), "qvel": f(W, nv), "qacc_warmstart": f(W, nv), "qfrc_applied": f(W, nv),
    "mocap_pos": f(W, nm, 3), "mocap_quat": f(W, nm, 4), "qacc": f(W, nv),
    "xanchor": f(W, nj, 3), "xaxis": f(W, nj, 3), "xmat": f(W, nb, 3, 3), "xpos": f(W, nb, 3),
    "xquat": f(W, nb, 4), "xipos": f(W, nb, 3), "ximat": f(W, nb, 3, 3),
    "subtree_com": f(W, nb, 3), "geom_xpos": f(W, ng, 3), "geom_xmat": f(W, ng, 3, 3),
    "site_xpos": f(W, ns, 3), "site_xmat": f(W, ns, 3, 3), "cinert": f(W, nb, 10),
    "cdof": f(W, nv, 6), "ctrl": f(W, nu), "actuator_velocity": f(W, nu),
    "actuator_force": f(W, nu), "actuator_length": f(W, nu), "actuator_moment": f(W, nu, nv),
    "crb": f(W, nb, 10), "qM": f(*mshape), "qLD": f(*mshape), "act_dot": f(W, na),
    "act": f(W, na), "qLDiagInv": f(W, nv), "cvel": f(W, nb, 6), "cdof_dot": f(W, nv, 6),
    "qfrc_bias": f(W, nv), "qfrc_passive": f(W, nv), "qfrc_spring": f(W, nv),
    "qfrc_damper": f(W, nv), "qfrc_actuator": f(W, nv), "qfrc_smooth": f(W, nv),
    "qfrc_constraint": f(W, nv), "qacc_smooth": f(W, nv), "rne_cacc": f(W, nb, 6),
    "rne_cfrc": f(W, nb, 6), "xfrc_applied": f(W, nb, 6), "qfrc_integration": f(W, nv),
    "qacc_integration": f(W, nv), "qM_integration": f(*mshape), "qLD_integration": f(*mshape),
    "qLDiagInv_integration": f(W, nv), "act_vel_integration": f(W, nu),
    "sap_geom_sort": f(W, ng, 4), "sap_projection_lower": f(2 * W, ng),
    "sap_projection_upper": f(W, ng), "sap_sort_index": i(2 * W, ng), "sap_range": i(W, ng),
    "sap_cumulative_sum": i(W * ng),
    "sap_segment_index": torch.arange(0, (W + 1) * ng, max(ng, 1), dtype=torch.int64, device=dev)[: W + 1],
    "collision_pair": i(nconmax, 2), "collision_worldid": i(nconmax), "ncollision": i(1),
    "ncon": i(1), "nefc": i(1),
    "world_pairadr": i(W), "world_npair": i(W), "world_conadr": i(W), "world_ncon": i(W),
    "world_efcadr": i(W), "world_nefc": i(W), "world_status": torch.zeros(W, dtype=torch.int32, device=dev),
    "world_order": i(W), "work_queue": i(1),
  }
  contact = {
    "dist": f(nconmax), "pos": f(nconmax, 3), "frame": f(nconmax, 3, 3),
    "includemargin": f(nconmax), "friction": f(nconmax, 5), "solref": f(nconmax, 2),
    "solreffriction": f(nconmax, 2), "solimp": f(nconmax, 5), "dim": i(nconmax),
    "geom": i(nconmax, 2), "efc_address": i(nconmax), "worldid": i(nconmax),
  }
  nls = max(int(mjm.opt.ls_iterations), 1)
  efc = {
    "J": f(njmax, nv), "D": f(njmax), "pos": f(njmax), "aref": f(njmax), "force": f(njmax),
    "margin": f(njmax), "worldid": i(njmax), "Jaref": f(njmax), "Ma": f(W, nv), "grad": f(W, nv),
    "grad_dot": f(W), "Mgrad": f(W, nv), "search": f(W, nv), "search_dot": f(W), "gauss": f(W),
    "cost": f(W), "prev_cost": f(W), "solver_niter": i(W), "active": i(njmax), "gtol": f(W),
    "mv": f(W, nv), "jv": f(njmax), "quad": f(njmax, 3), "quad_gauss": f(W, 3),
    "h": f(W, nv, nv), "alpha": f(W), "prev_grad": f(W, nv), "prev_Mgrad": f(W, nv),
    "beta": f(W), "beta_num": f(W), "beta_den": f(W),
    "done": torch.zeros(W, dtype=torch.uint8, device=dev),
    "ls_done": torch.zeros(W, dtype=torch.uint8, device=dev), "p0": f(W, 3), "lo": f(W, 3),
    "lo_alpha": f(W), "hi": f(W, 3), "hi_alpha": f(W), "lo_next": f(W, 3), "lo_next_alpha": f(W),
    "hi_next": f(W, 3), "hi_next_alpha": f(W), "mid": f(W, 3), "mid_alpha": f(W),
    "cost_candidate": f(W, nls), "quad_total_candidate": f(W, nls, 3),
  }
  return top, contact, efc


def _assemble(mjm, nworld, nconmax, njmax, dev) -> Data:
  top, contact, efc = _data_arrays(mjm, nworld, nconmax, njmax, dev)
  d = Data()
  object.__setattr__(d, "nworld", int(nworld))
  object.__setattr__(d, "nconmax", int(nconmax))
  object.__setattr__(d, "njmax", int(njmax))
  object.__setattr__(d, "nl", 0)
  object.__setattr__(d, "time", 0.0)
  for k, v in top.items():
    setattr(d, k, v)
  c = Contact(d)
  for k, v in contact.items():
    object.__setattr__(c, k, types.as_device_array(v))
  e = Constraint(d)
  for k, v in efc.items():
    object.__setattr__(e, k, types.as_device_array(v))
  object.__setattr__(d, "contact", c)
  object.__setattr__(d, "efc", e)
  object.__setattr__(d, "_view_cache", None)
  return d


def make_data(mjm, nworld: int = 1, nconmax: int = -1, njmax: int = -1, device=None) -> Data:
  """Allocates a Data at qpos0 (io.py:395-506); nconmax / njmax default to 512 totals."""
  if nconmax == -1:
    nconmax = 512
  if njmax == -1:
    njmax = 512
  dev = _device(device)
  d = _assemble(mjm, nworld, nconmax, njmax, dev)
  d.qpos.copy_(torch.as_tensor(np.tile(np.asarray(mjm.qpos0, dtype=np.float32), (nworld, 1))))
  return d


def sparse_from_dense(mjm, M) -> np.ndarray:
  """The sparse layout (nM,) of a dense nv x nv mass matrix: row i's diagonal, then its entries
  against the dof's ancestors, at dof_Madr[i] (smooth.py:264-279)."""
  out = np.zeros(int(mjm.nM))
  parent = np.asarray(mjm.dof_parentid)
  for i in range(mjm.nv):
    a, j = int(mjm.dof_Madr[i]), i
    while j >= 0:
      out[a] = M[i, j]
      a, j = a + 1, parent[j]
  return out


def dense_from_sparse(mjm, Ms) -> np.ndarray:
  """The dense symmetric nv x nv matrix of a sparse-layout mass matrix (mj_fullM)."""
  M = np.zeros((mjm.nv, mjm.nv))
  parent = np.asarray(mjm.dof_parentid)
  for i in range(mjm.nv):
    a, j = int(mjm.dof_Madr[i]), i
    while j >= 0:
      M[i, j] = M[j, i] = Ms[a]
      a, j = a + 1, parent[j]
  return M


def factor_sparse_host(mjm, Ms) -> np.ndarray:
  """L'DL factor of a sparse-layout mass matrix in the same layout (mj_factorI), on the host."""
  L = np.array(Ms, dtype=float)
  parent = np.asarray(mjm.dof_parentid)
  madr = np.asarray(mjm.dof_Madr)
  rowlen = np.diff(np.append(madr, int(mjm.nM)))
  for k in range(mjm.nv - 1, -1, -1):
    mkk, mki, i = madr[k], madr[k] + 1, parent[k]
    while i >= 0:
      tmp = L[mki] / L[mkk] if L[mkk] != 0 else 0.0
      L[madr[i]:madr[i] + rowlen[i]] -= L[mki:mki + rowlen[i]] * tmp
      L[mki] = tmp
      i, mki = parent[i], mki + 1
  return L


def _dense_qM(mjm, mjd):
  qM = np.asarray(mjd.qM, dtype=float)
  if qM.ndim == 2:
    return qM
  import mujoco  # a real mujoco.MjData stores qM sparse

  full = np.zeros((mjm.nv, mjm.nv))
  mujoco.mj_fullM(mjm, full, mjd.qM)
  return full


def _dense_moment(mjm, mjd):
  am = np.asarray(mjd.actuator_moment, dtype=float)
  if am.ndim == 2 and am.shape == (mjm.nu, mjm.nv):
    return am
  import mujoco

  dense = np.zeros((mjm.nu, mjm.nv))
  mujoco.mju_sparse2dense(dense, mjd.actuator_moment, mjd.moment_rownnz, mjd.moment_rowadr,
                          mjd.moment_colind)
  return dense


def put_data(mjm, mjd, nworld: int = 1, nconmax: int = -1, njmax: int = -1, device=None) -> Data:
  """Replicates one host state to nworld worlds (io.py:509-725)."""
  ncon, nefc = int(mjd.ncon), int(mjd.nefc)
  if nconmax == -1:
    nconmax = max(512, ncon * nworld)
  if njmax == -1:
    njmax = max(512, nefc * nworld)
  if nworld * nefc > njmax:
    raise ValueError("nworld * nefc > njmax")
  if nworld * ncon > nconmax:
    raise ValueError("nworld * ncon > nconmax")
  dev = _device(device)
  d = _assemble(mjm, nworld, nconmax, njmax, dev)
  object.__setattr__(d, "nl", int(getattr(mjd, "nl", 0)))
  object.__setattr__(d, "time", float(mjd.time))

  def tile(name, value):
    t = getattr(d, name)
    v = torch.as_tensor(np.asarray(value, dtype=np.float32).reshape(t.shape[1:]))
    t.copy_(v.unsqueeze(0).expand_as(t))

  for n in ("qpos", "qvel", "qacc_warmstart", "qfrc_applied", "qacc", "act", "ctrl",
            "actuator_velocity", "actuator_force", "actuator_length", "qLDiagInv", "qfrc_bias",
            "qfrc_passive", "qfrc_spring", "qfrc_damper", "qfrc_actuator", "qfrc_smooth",
            "qfrc_constraint", "qacc_smooth", "act_dot"):
    tile(n, getattr(mjd, n))
  for n in ("mocap_pos", "mocap_quat", "xanchor", "xaxis", "xmat", "xpos", "xquat", "xipos",
            "ximat", "subtree_com", "geom_xpos", "geom_xmat", "site_xpos", "site_xmat", "cinert",
            "cdof", "crb", "cvel", "cdof_dot", "xfrc_applied"):
    tile(n, getattr(mjd, n))
  qM = _dense_qM(mjm, mjd)
  if is_sparse(mjm):
    Ms = sparse_from_dense(mjm, qM)
    tile("qM", Ms)
    tile("qLD", factor_sparse_host(mjm, Ms))
  else:
    tile("qM", qM)
    try:
      qLD = np.linalg.cholesky(qM) if np.any(qM) else np.zeros_like(qM)
    except np.linalg.LinAlgError:
      qLD = np.zeros_like(qM)
    tile("qLD", qLD)
  tile("actuator_moment", _dense_moment(mjm, mjd))

  # contacts and constraint rows: world i's block at [i * n, (i + 1) * n) (io.py:607-698)
  W = nworld
  if ncon:
    con = mjd.contact
    rep = lambda x, w: torch.as_tensor(np.repeat(np.asarray(x, dtype=np.float32).reshape(ncon, w), W, axis=0))  # noqa: E731
    n = W * ncon
    d.contact.dist[:n] = rep(con.dist, 1).reshape(-1)
    d.contact.pos[:n] = rep(con.pos, 3)
    d.contact.frame[:n] = rep(con.frame, 9).reshape(n, 3, 3)
    d.contact.includemargin[:n] = rep(con.includemargin, 1).reshape(-1)
    d.contact.friction[:n] = rep(con.friction, 5)
    d.contact.solref[:n] = rep(con.solref, 2)
    d.contact.solreffriction[:n] = rep(con.solreffriction, 2)
    d.contact.solimp[:n] = rep(con.solimp, 5)
    d.contact.dim[:n] = torch.as_tensor(np.repeat(np.asarray(con.dim, dtype=np.int32), W))
    d.contact.geom[:n] = torch.as_tensor(np.repeat(np.asarray(con.geom, dtype=np.int32).reshape(ncon, 2), W, axis=0))
    wid = np.repeat(np.arange(W, dtype=np.int32), ncon)
    d.contact.worldid[:n] = torch.as_tensor(wid)
    ea = np.concatenate([np.asarray(con.efc_address, dtype=np.int32) + k * ncon for k in range(W)])
    d.contact.efc_address[:n] = torch.as_tensor(ea)
    d.ncon.fill_(n)
    d.world_conadr.copy_(torch.arange(W, dtype=torch.int32) * ncon)
    d.world_ncon.fill_(ncon)
  if nefc:
    n = W * nefc
    J = np.asarray(mjd.efc_J, dtype=np.float32).reshape(nefc, mjm.nv)
    d.efc.J[:n] = torch.as_tensor(np.repeat(J, W, axis=0))
    for k in ("D", "pos", "aref", "force", "margin"):
      getattr(d.efc, k)[:n] = torch.as_tensor(np.repeat(np.asarray(getattr(mjd, "efc_" + k), dtype=np.float32), W))
    d.efc.worldid[:n] = torch.as_tensor(np.repeat(np.arange(W, dtype=np.int32), nefc))
    d.nefc.fill_(n)
    d.world_efcadr.copy_(torch.arange(W, dtype=torch.int32) * nefc)
    d.world_nefc.fill_(nefc)
  object.__setattr__(d, "_view_cache", None)
  return d


def get_data_into(result, mjm, d: Data) -> None:
  """Copies a single-world Data back into a host MjData (io.py:728-831)."""
  if d.nworld > 1:
    raise NotImplementedError("only nworld == 1 supported for now")
  ncon = int(min(d.ncon.numpy()[0], d.nconmax))
  nefc = int(min(d.nefc.numpy()[0], d.njmax))
  result.time = d.time
  for n in ("qpos", "qvel", "qacc_warmstart", "qfrc_applied", "mocap_pos", "mocap_quat", "qacc",
            "xanchor", "xaxis", "xpos", "xquat", "xipos", "subtree_com", "geom_xpos",
            "site_xpos", "cinert", "cdof", "crb", "qLDiagInv", "ctrl", "actuator_velocity",
            "actuator_force", "actuator_length", "cvel", "cdof_dot", "qfrc_bias", "qfrc_passive",
            "qfrc_spring", "qfrc_damper", "qfrc_actuator", "qfrc_smooth", "qfrc_constraint",
            "qacc_smooth", "act", "act_dot", "xfrc_applied"):
    setattr(result, n, getattr(d, n).numpy()[0].astype(np.float64).copy())
  for n in ("xmat", "ximat", "geom_xmat", "site_xmat"):
    setattr(result, n, getattr(d, n).numpy()[0].reshape(-1, 9).astype(np.float64))
  if is_sparse(mjm):  # io.py:803-805
    result.qM = d.qM.numpy()[0, 0].astype(np.float64)
    result.qLD = d.qLD.numpy()[0, 0].astype(np.float64)
  else:
    result.qM = d.qM.numpy()[0].astype(np.float64)
    result.qLD = d.qLD.numpy()[0].astype(np.float64)
  result.actuator_moment = d.actuator_moment.numpy()[0].astype(np.float64)
  result.ncon = ncon
  result.nefc = nefc
  c = result.contact
  c.dist = d.contact.dist.numpy()[:ncon].astype(np.float64)
  c.pos = d.contact.pos.numpy()[:ncon].astype(np.float64)
  c.frame = d.contact.frame.numpy()[:ncon].reshape(-1, 9).astype(np.float64)
  c.includemargin = d.contact.includemargin.numpy()[:ncon].astype(np.float64)
  c.friction = d.contact.friction.numpy()[:ncon].astype(np.float64)
  c.solref = d.contact.solref.numpy()[:ncon].astype(np.float64)
  c.solreffriction = d.contact.solreffriction.numpy()[:ncon].astype(np.float64)
  c.solimp = d.contact.solimp.numpy()[:ncon].astype(np.float64)
  c.dim = d.contact.dim.numpy()[:ncon].copy()
  c.geom = d.contact.geom.numpy()[:ncon].copy()
  c.efc_address = d.contact.efc_address.numpy()[:ncon].copy()
  result.efc_J = d.efc.J.numpy()[:nefc].astype(np.float64)
  for k in ("D", "pos", "aref", "force", "margin"):
    setattr(result, "efc_" + k, getattr(d.efc, k).numpy()[:nefc].astype(np.float64))
