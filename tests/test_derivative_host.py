"""Host-side logic of the derivatives (no GPU): which models the analytic step adjoint covers, and
the C entry points' argument checks."""

import ctypes

import numpy as np
import pytest

import mjx_warp_b200 as mjw
from helpers import load
from mjx_warp_b200 import _abi


def _expected_qpos_support(mjm):
  """The adjoint's coverage restated from the model's arrays."""
  if mjm.na or mjm.opt.jacobian == 1:
    return False
  jt, jb = np.asarray(mjm.jnt_type), np.asarray(mjm.jnt_bodyid)
  nj = np.asarray(mjm.body_jntnum)
  if any(nj[jb[j]] != 1 for j in range(mjm.njnt) if jt[j] == 1):
    return False
  if any(mjm.jnt_stiffness[j] != 0 for j in range(mjm.njnt) if jt[j] in (0, 1)):
    return False
  tid = np.asarray(mjm.actuator_trnid).reshape(mjm.nu, -1)[:, 0] if mjm.nu else []
  if any(jt[t] not in (2, 3) for t in tid):
    return False
  gb, wb = np.asarray(mjm.geom_bodyid), np.asarray(mjm.body_weldid)
  return all(wb[gb[g]] == 0 for g in range(mjm.ngeom) if mjm.geom_type[g] == 0)


@pytest.mark.parametrize("name", ["humanoid.xml", "sphere_chain.xml", "pendula.xml", "collision.xml"])
def test_qpos_vjp_support_follows_model_features(name):
  mjm = load(name)
  m = mjw.put_model(mjm, device="cpu")
  assert mjw.derivative.ctrl_vjp_supported(m)
  assert mjw.derivative.qpos_vjp_supported(m) == _expected_qpos_support(mjm)


def test_adjoint_needs_the_dense_mass_matrix():
  mjm = load("humanoid.xml", jacobian=1)  # sparse
  m = mjw.put_model(mjm, device="cpu")
  assert not mjw.derivative.ctrl_vjp_supported(m)
  assert not mjw.derivative.qpos_vjp_supported(m)


def test_humanoid_is_covered():
  m = mjw.put_model(load("humanoid.xml"), device="cpu")
  assert mjw.derivative.qpos_vjp_supported(m)


def test_step_vjp_entry_rejects_bad_arguments():
  lib = _abi.lib()
  assert lib.mjb_step_vjp(None, None, None, None, None, None, None, None) == 1
  assert lib.mjb_ctrl_vjp(None, None, None, None, None) == 1
  mv, dv = _abi.MjbModel(), _abi.MjbData()
  dv.nworld = 0
  # an empty batch is a no-op whatever the outputs
  assert lib.mjb_step_vjp(ctypes.byref(mv), ctypes.byref(dv), None, None, None, None, None, None) == 0


def test_segment_ring_shares_only_scratch():
  """The analytic rollout's per-step Data share the fields a step writes before it reads them and
  the adjoint never reads; everything the adjoint reads stays per step."""
  from mjx_warp_b200 import derivative
  mjm = load("humanoid.xml")
  ring = derivative._segment_ring(mjm, 2, 2 * 48, 2 * 80, 3)
  a, b = ring[0], ring[2]
  for name in derivative._RING_SHARED:
    if getattr(a, name, None) is not None:
      assert getattr(a, name) is getattr(b, name), name
  for name in derivative._RING_SHARED_EFC:
    assert getattr(a.efc, name) is getattr(b.efc, name), name
  for name in ("qpos", "qvel", "qM", "qLD_integration", "qacc", "qacc_integration", "cdof",
               "cinert", "cvel", "xpos", "xmat", "geom_xpos", "subtree_com", "actuator_moment"):
    assert getattr(a, name).data_ptr() != getattr(b, name).data_ptr(), name
  for name in ("h", "J", "D", "Jaref", "active", "pos", "margin"):
    assert getattr(a.efc, name).data_ptr() != getattr(b.efc, name).data_ptr(), name
  for name in ("pos", "frame", "dist", "geom"):
    assert getattr(a.contact, name).data_ptr() != getattr(b.contact, name).data_ptr(), name
