"""Smooth dynamics on the GPU vs the FP64 oracle (smooth_test.py, forward_test.py, support_test.py,
passive_test.py).  Tolerance: the reference's own atol = rtol = 5e-4 (_TOLERANCE * 10)."""

import numpy as np
import pytest
import torch

import mjx_warp_b200 as mjw
from helpers import (assert_close, dev, device_data, generic_state, humanoid, humanoid_state, load,
                     oracle)

pytestmark = pytest.mark.gpu

KIN = ("xpos", "xquat", "xmat", "xipos", "ximat", "xanchor", "xaxis", "geom_xpos", "geom_xmat",
       "site_xpos", "site_xmat")
COM = ("subtree_com", "cinert", "cdof")
VEL = ("actuator_velocity", "cvel", "cdof_dot", "qfrc_spring", "qfrc_damper", "qfrc_passive",
       "qfrc_bias")


def _setup(name, nworld=8, seed=0):
  mjm = load(name)
  qpos, qvel, ctrl = generic_state(mjm, nworld, seed)
  m = mjw.put_model(mjm)
  d = device_data(mjm, qpos, qvel, ctrl)
  o = oracle(mjm, qpos, qvel, ctrl, 64)
  return mjm, m, d, o


def _cmp(o, d, names):
  torch.cuda.synchronize()
  for n in names:
    assert_close(dev(getattr(d, n)), o.get(n), n)


@pytest.mark.parametrize("name", ["pendula.xml", "humanoid.xml", "sphere_chain.xml"])
def test_stage_chain(name):
  """Each stage function, run in the reference's order, matches the oracle's stage outputs."""
  mjm, m, d, o = _setup(name)
  mjw.kinematics(m, d)
  o.run("kinematics")
  _cmp(o, d, KIN if mjm.nsite else KIN[:-2])
  mjw.com_pos(m, d)
  o.run("com_pos")
  _cmp(o, d, COM)
  mjw.crb(m, d)
  o.run("crb")
  _cmp(o, d, ("crb", "qM"))
  mjw.factor_m(m, d)
  o.run("factor_m")
  _cmp(o, d, ("qLD",))
  mjw.transmission(m, d)
  o.run("transmission")
  if mjm.nu:
    _cmp(o, d, ("actuator_length", "actuator_moment"))
  mjw.fwd_velocity(m, d)
  o.run("fwd_velocity")
  _cmp(o, d, VEL)
  mjw.fwd_actuation(m, d)
  o.run("fwd_actuation")
  _cmp(o, d, ("actuator_force", "qfrc_actuator"))
  mjw.fwd_acceleration(m, d)
  o.run("fwd_acceleration")
  _cmp(o, d, ("qfrc_smooth",))
  # qacc_smooth = M^-1 qfrc_smooth: cond(M) ~ 3.6e3 for the humanoid, so an FP32 solve is only
  # good to ~cond * eps32 ~ 1e-3 (the FP32 oracle itself reaches 4.9e-4)
  assert_close(dev(d.qacc_smooth), o.get("qacc_smooth"), "qacc_smooth", rtol=2e-3, atol=2e-3)


def test_individual_stages_match_from_oracle_inputs():
  """rne / com_vel / passive alone, each fed the oracle's own inputs."""
  mjm, m, d, o = _setup("pendula.xml", nworld=4, seed=1)
  o.run("forward_nosolve")
  for n in ("cdof", "cinert", "qM", "qLD", "subtree_com", "xipos", "actuator_moment"):
    getattr(d, n).copy_(torch.as_tensor(o.get(n).reshape(getattr(d, n).shape), dtype=torch.float32))
  mjw.com_vel(m, d)
  mjw.passive(m, d)
  mjw.rne(m, d)
  _cmp(o, d, ("cvel", "cdof_dot", "qfrc_passive", "qfrc_bias"))


def test_disabled_flags():
  """PASSIVE / ACTUATION / GRAVITY disable flags zero their contributions like the reference."""
  for flag, fields in ((mjw.DisableBit.PASSIVE, ("qfrc_passive",)),
                       (mjw.DisableBit.ACTUATION, ("qfrc_actuator",)),
                       (mjw.DisableBit.GRAVITY, ("qfrc_bias",))):
    mjm = load("pendula.xml")
    mjm.opt.disableflags |= int(flag)
    qpos, qvel, ctrl = generic_state(mjm, 4, 2)
    m = mjw.put_model(mjm)
    d = device_data(mjm, qpos, qvel, ctrl)
    mjw.forward(m, d)
    o = oracle(mjm, qpos, qvel, ctrl, 64)
    o.run("forward")
    _cmp(o, d, fields)
    assert_close(dev(d.qacc_smooth), o.get("qacc_smooth"), "qacc_smooth", rtol=2e-3, atol=2e-3)
    if flag != mjw.DisableBit.GRAVITY:
      assert float(getattr(d, fields[0]).abs().max()) == 0.0


def test_solve_m_mul_m_xfrc():
  """support_test.py:43-73 and smooth_test.py:109-127."""
  mjm, m, d, o = _setup("pendula.xml", nworld=4, seed=3)
  mjw.forward(m, d)
  o.run("forward_nosolve")
  torch.cuda.synchronize()
  rng = np.random.default_rng(0)
  vec = rng.uniform(-1, 1, (4, mjm.nv))
  res = torch.zeros((4, mjm.nv), device="cuda")
  vt = torch.as_tensor(vec, dtype=torch.float32, device="cuda")
  skip = torch.zeros(4, dtype=torch.bool, device="cuda")
  skip[2] = True
  mjw.mul_m(m, d, res, vt, skip)
  qM = o.get("qM").reshape(4, mjm.nv, mjm.nv)
  want = np.einsum("wij,wj->wi", qM, vec)
  want[2] = 0.0
  assert_close(res.cpu().numpy(), want, "mul_m")
  x = torch.zeros_like(res)
  mjw.solve_m(m, d, x, vt)
  assert_close(x.cpu().numpy(), np.linalg.solve(qM, vec[..., None])[..., 0], "solve_m")
  xfrc = rng.normal(size=(4, mjm.nbody, 6))
  d.xfrc_applied.copy_(torch.as_tensor(xfrc, dtype=torch.float32))
  q = torch.zeros((4, mjm.nv), device="cuda")
  mjw.xfrc_accumulate(m, d, q)
  o.set("xfrc_applied", xfrc.reshape(4, -1))
  o.set("qfrc_applied", np.zeros((4, mjm.nv)))
  o.run("fwd_acceleration")
  base = o.get("qfrc_passive") - o.get("qfrc_bias") + o.get("qfrc_actuator")
  assert_close(q.cpu().numpy(), o.get("qfrc_smooth") - base, "xfrc_accumulate", atol=2e-3)


def test_humanoid_forward_all_fields():
  """fwd_position .. fwd_acceleration on the benchmark humanoid at many perturbed states."""
  mjm = humanoid()
  qpos, qvel, ctrl = humanoid_state(mjm, 64, seed=5)
  m = mjw.put_model(mjm)
  for fused in (1, 0, 2):
    d = device_data(mjm, qpos, qvel, ctrl)
    mjw.forward(m, d, fused=fused)
    o = oracle(mjm, qpos, qvel, ctrl, 64)
    o.run("forward")
    _cmp(o, d, KIN[:-2] + COM + ("crb", "qM", "qLD", "actuator_length", "actuator_moment") + VEL +
         ("actuator_force", "qfrc_actuator", "qfrc_smooth"))
    assert_close(dev(d.qacc_smooth), o.get("qacc_smooth"), "qacc_smooth", rtol=2e-3, atol=2e-3)
