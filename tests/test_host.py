"""Host-side logic: put_model / make_data / put_data, candidate pairs, ABI mirror, no CPU path."""

import ctypes
import re

import numpy as np
import pytest
import torch

import mjx_warp_b200 as mjw
from helpers import load
from mjx_warp_b200 import _abi, io, mjcf


def _arrays(d):
  out = {k: v for k, v in d.__dict__.items() if isinstance(v, torch.Tensor)}
  out.update({"contact." + k: v for k, v in d.contact.__dict__.items() if isinstance(v, torch.Tensor)})
  out.update({"efc." + k: v for k, v in d.efc.__dict__.items() if isinstance(v, torch.Tensor)})
  return out


def test_make_and_put_data_agree():
  """support_test.py:75-86: make_data and put_data expose the same fields with the same shapes."""
  mjm = load("pendula.xml")
  mjd = mjcf.MjData(mjm)
  a = _arrays(mjw.make_data(mjm, device="cpu"))
  b = _arrays(mjw.put_data(mjm, mjd, device="cpu"))
  assert a.keys() == b.keys()
  for k in a:
    assert a[k].shape == b[k].shape, k


def test_put_data_replicates_state_and_rows():
  mjm = load("humanoid.xml")
  mjd = mjcf.MjData(mjm)
  mjcf.mj_resetDataKeyframe(mjm, mjd, 0)
  mjd.qvel[:] = np.linspace(-1, 1, mjm.nv)
  mjd.ncon, mjd.nefc = 2, 3
  mjd.contact.dist = np.array([-0.1, -0.2])
  for k, w in (("pos", 3), ("frame", 9), ("friction", 5), ("solref", 2), ("solreffriction", 2), ("solimp", 5)):
    setattr(mjd.contact, k, np.zeros((2, w)))
  mjd.contact.includemargin = np.zeros(2)
  mjd.contact.dim = np.array([3, 3])
  mjd.contact.geom = np.array([[0, 1], [0, 2]])
  mjd.contact.efc_address = np.array([0, 1])
  mjd.efc_J = np.ones((3, mjm.nv))
  for k in ("D", "pos", "aref", "force", "margin"):
    setattr(mjd, "efc_" + k, np.arange(3.0))
  d = mjw.put_data(mjm, mjd, nworld=4, device="cpu")
  assert d.nconmax == 512 and d.njmax == 512
  np.testing.assert_allclose(d.qvel.numpy(), np.tile(mjd.qvel, (4, 1)), rtol=1e-6)
  assert int(d.ncon.numpy()[0]) == 8 and int(d.nefc.numpy()[0]) == 12
  np.testing.assert_array_equal(d.efc.worldid.numpy()[:12], np.repeat(np.arange(4), 3))
  np.testing.assert_array_equal(d.world_efcadr.numpy(), [0, 3, 6, 9])
  np.testing.assert_array_equal(d.world_ncon.numpy(), [2, 2, 2, 2])
  with pytest.raises(ValueError):
    mjw.put_data(mjm, mjd, nworld=4, njmax=8, device="cpu")


def test_put_model_tables():
  mjm = load("humanoid.xml")
  m = mjw.put_model(mjm, device="cpu")
  # BFS levels: depth 0 world, 1 torso, ..., 6 feet (io.py:113-124)
  assert m.body_treeadr.numpy().tolist() == [0, 1, 2, 6, 9, 13, 15, 17]
  assert m.block_adr.numpy().tolist() == [0] and m.block_size.numpy().tolist() == [27]
  assert m.jnt_limited_slide_hinge_adr.shape[0] == 21
  # subtree mass keeps the reference's doubled world entry (io.py:249-254)
  np.testing.assert_allclose(m.subtree_mass.numpy()[0], 2 * mjm.body_mass.sum(), rtol=1e-6)
  # children and DFS subtree ranges describe the same tree as body_parentid
  parent = mjm.body_parentid
  end = m.body_subtreeend.numpy()
  for b in range(1, mjm.nbody):
    a = b
    while a > 0:
      assert a <= b < end[a]
      a = parent[a]
  assert m.actuator_affine_bias_gain is False


def test_pair_candidates_follow_filter_and_flags():
  mjm = load("humanoid.xml")
  m = mjw.put_model(mjm, device="cpu")
  pc = io.pair_candidates(m).numpy()
  assert pc.shape == (161, 2) and np.all(pc[:, 0] < pc[:, 1])
  # order is the nxn element order (lexicographic in (g1, g2))
  keys = pc[:, 0] * 100 + pc[:, 1]
  assert np.all(np.diff(keys) > 0)
  m.opt.disableflags |= int(mjw.DisableBit.FILTERPARENT)
  assert io.pair_candidates(m).shape[0] > 161
  m.opt.disableflags &= ~int(mjw.DisableBit.FILTERPARENT)
  m.geom_conaffinity = torch.zeros_like(m.geom_conaffinity)
  assert io.pair_candidates(m).shape[0] == 0


def _header_fields(struct):
  text = open(_abi.os.path.join(_abi._HERE, "..", "include", "mjb200.h")).read()
  body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (struct, struct), text, re.S).group(1)
  body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
  names = []
  for decl in body.split(";"):
    decl = decl.strip()
    if not decl:
      continue
    decl = re.sub(r"^(const\s+)?(int32_t|float|uint8_t|uint32_t)\s*", "", decl)
    for part in decl.split(","):
      part = part.strip().lstrip("*").strip()
      names.append(re.sub(r"\[.*\]", "", part))
  return names


def test_abi_mirror_matches_header():
  assert [f[0] for f in _abi.MjbModel._fields_] == _header_fields("MjbModel")
  assert [f[0] for f in _abi.MjbData._fields_] == _header_fields("MjbData")
  assert [f[0] for f in _abi.MjbRunCfg._fields_] == _header_fields("MjbRunCfg")
  assert [f[0] for f in _abi.MjbTune._fields_] == _header_fields("MjbTune")


def test_library_exports_every_declared_entry_point():
  """libmjb200.so loads without a GPU and exports each function include/mjb200.h declares."""
  text = open(_abi.os.path.join(_abi._HERE, "..", "include", "mjb200.h")).read()
  names = re.findall(r"^\w[\w\s\*]*?\b(mjb_\w+)\(", text, re.M)
  assert len(names) >= 25
  lib = _abi.lib()
  for n in names:
    assert hasattr(lib, n), n
  assert lib.mjb_abi_version() == 7
  assert lib.mjb_error_string(0) == b"ok"


def test_cpu_tensors_are_refused():
  """No CPU fallback: stage functions on CPU tensors raise instead of computing."""
  mjm = load("pendula.xml")
  m = mjw.put_model(mjm, device="cpu")
  d = mjw.make_data(mjm, device="cpu")
  for fn in (mjw.step, mjw.forward, mjw.kinematics, mjw.solve):
    with pytest.raises(RuntimeError):
      fn(m, d)


def test_null_arguments_rejected():
  lib = _abi.lib()
  assert lib.mjb_step(None, None, None, None) == 1
  v = _abi.MjbData()
  v.nworld = 0
  mv = _abi.MjbModel()
  assert lib.mjb_kinematics(ctypes.byref(mv), ctypes.byref(v), None) == 0


def _fake_views(mjm):
  """MjbModel / MjbData views with the model's sizes and every Data pointer set to a dummy
  non-null address (never dereferenced: the calls below return before any launch)."""
  mv = _abi.MjbModel()
  for n in ("nq", "nv", "na", "nu", "nbody", "njnt", "ngeom", "nsite"):
    setattr(mv, n, int(getattr(mjm, n)))
  mv.nblock, mv.block_max = 1, mjm.nv
  mv.integrator, mv.solver, mv.iterations, mv.ls_iterations = 3, 2, 3, 4
  mv.actuator_affine_bias_gain = 1
  dv = _abi.MjbData()
  dv.nworld, dv.nconmax, dv.njmax = 4, 64, 256
  for name, _ in _abi.DATA_PTRS:
    setattr(dv, name, 0x1000)
  return mv, dv


@pytest.mark.parametrize("entry, field", [
  ("mjb_kinematics", "xpos"), ("mjb_kinematics", "geom_xmat"), ("mjb_com_pos", "cinert"),
  ("mjb_crb", "qM"), ("mjb_factor_m", "qLD"), ("mjb_transmission", "actuator_moment"),
  ("mjb_fwd_velocity", "rne_cfrc"), ("mjb_fwd_actuation", "actuator_force"),
  ("mjb_fwd_acceleration", "qfrc_smooth"), ("mjb_nxn_broadphase", "collision_pair"),
  ("mjb_primitive_narrowphase", "contact_frame"), ("mjb_make_constraint", "efc_J"),
  ("mjb_solve", "efc_Jaref"), ("mjb_euler", "qLD_integration"),
  ("mjb_implicit", "qfrc_integration"), ("mjb_implicit", "act_vel_integration"),
  ("mjb_forward", "cdof"), ("mjb_forward", "efc_Ma"), ("mjb_step", "qacc_integration"),
  ("mjb_fwd_position", "subtree_com"), ("mjb_collision", "contact_dist")])
def test_null_data_field_rejected(entry, field):
  """An entry point given a null Data field that one of its stages touches returns MJB_ERR_ARG
  before launching anything, instead of faulting on the device."""
  mjm = load("humanoid.xml", integrator=3)
  mv, dv = _fake_views(mjm)
  if entry == "mjb_euler":
    mv.integrator = 0
  setattr(dv, field, None)
  lib = _abi.lib()
  fn = getattr(lib, entry)
  if entry in ("mjb_forward", "mjb_step"):
    rc = fn(ctypes.byref(mv), ctypes.byref(dv), None, None)
  else:
    rc = fn(ctypes.byref(mv), ctypes.byref(dv), None)
  assert rc == 1, (entry, field, rc)


def test_step_io_rejects_mismatched_buffers():
  """step_io checks its buffers' shapes and types on the host before any device call."""
  mjm = load("pendula.xml")
  m = mjw.put_model(mjm, device="cpu")
  d = mjw.make_data(mjm, nworld=2, device="cpu")
  with pytest.raises(ValueError):
    mjw.step_io(m, d, inputs={"qpos": torch.zeros((3, mjm.nq))})
  with pytest.raises(ValueError):
    mjw.step_io(m, d, inputs={"qvel": torch.zeros((2, mjm.nv), dtype=torch.float64)})
  with pytest.raises(ValueError):
    mjw.step_io(m, d, outputs=("qacc",))
  with pytest.raises(ValueError):
    mjw.step_io(m, d, outputs=("xpos",), out={"xpos": torch.zeros((2, 3))})


def test_step_io_c_abi_argument_checks():
  """mjb_step_io returns MJB_ERR_ARG for a null io, a negative step count, or a requested copy
  into or out of a Data field that is null, before any copy or launch."""
  mjm = load("humanoid.xml", integrator=3)
  mv, dv = _fake_views(mjm)
  lib = _abi.lib()
  io = _abi.MjbStepIO()
  assert lib.mjb_step_io(ctypes.byref(mv), ctypes.byref(dv), None, 1, None, None) == 1
  assert lib.mjb_step_io(ctypes.byref(mv), ctypes.byref(dv), ctypes.byref(io), -1, None, None) == 1
  dv.ctrl = None
  io.ctrl = 0x2000
  assert lib.mjb_step_io(ctypes.byref(mv), ctypes.byref(dv), ctypes.byref(io), 1, None, None) == 1
  io.ctrl = None
  dv.site_xpos = None
  io.site_xpos_out = 0x2000
  mv.nsite = 1
  assert lib.mjb_step_io(ctypes.byref(mv), ctypes.byref(dv), ctypes.byref(io), 1, None, None) == 1
