"""MJCF-subset compiler: structure of the fixture models and the reference's rejections."""

import math

import numpy as np
import pytest

import mjx_warp_b200 as mjw
from helpers import fixtures, load
from mjx_warp_b200 import mjcf


def test_humanoid_structure():
  m = load("humanoid.xml")
  assert (m.nq, m.nv, m.nu, m.nbody, m.njnt, m.ngeom, m.nkey) == (28, 27, 21, 17, 22, 20, 3)
  assert m.opt.timestep == 0.005 and m.opt.iterations == 10 and m.opt.ls_iterations == 20
  assert m.opt.disableflags & mjw.DisableBit.EULERDAMP
  assert m.jnt_type[0] == mjw.JointType.FREE and np.all(m.jnt_type[1:] == mjw.JointType.HINGE)
  assert m.jnt_limited.sum() == 21
  assert np.all(m.body_mass[1:] > 0) and np.all(m.body_inertia[1:] > 0)
  assert m.stat.meaninertia > 0
  assert np.all(m.dof_invweight0 > 0) and np.all(m.body_invweight0[1:] > 0)
  # joint classes: solimplimit "0 .99 .01" over the built-in (0.5, 2) tail; ranges in radians
  np.testing.assert_allclose(m.jnt_solimp[1], [0.0, 0.99, 0.01, 0.5, 2.0])
  np.testing.assert_allclose(m.jnt_range[1], np.radians([-45, 45]))
  np.testing.assert_allclose(m.geom_friction[1], [0.7, 0.005, 0.0001])
  np.testing.assert_allclose(m.actuator_gear[5, 0], 120.0)
  np.testing.assert_allclose(np.linalg.norm(m.qpos0[3:7]), 1.0)
  # sparse-M addressing is consistent with the dof tree
  depth = [0] * m.nv
  for i in range(m.nv):
    depth[i] = 0 if m.dof_parentid[i] < 0 else depth[m.dof_parentid[i]] + 1
  assert m.nM == sum(d + 1 for d in depth)


def test_pendula_joint_zoo():
  m = load("pendula.xml")
  assert set(np.unique(m.jnt_type)) == {0, 1, 2, 3}
  assert m.nmocap == 2 and m.nsite == 5 and m.opt.disableflags & mjw.DisableBit.CONTACT
  # autolimits: a joint is limited exactly when it has a range
  has_range = np.any(m.jnt_range != 0, axis=1)
  np.testing.assert_array_equal(m.jnt_limited.astype(bool), has_range)
  # ball joints start at the identity quaternion
  for j in np.nonzero(m.jnt_type == 1)[0]:
    a = m.jnt_qposadr[j]
    np.testing.assert_allclose(m.qpos0[a:a + 4], [1, 0, 0, 0])


def test_capsule_inertia_matches_monte_carlo():
  """Capsule mass / inertia from geometry agree with a sampled solid capsule."""
  r, h = 0.05, 0.2
  mjm = mjcf.from_xml_string(
    f'<mujoco><worldbody><body><freejoint/><geom type="capsule" size="{r} {h}"/></body></worldbody></mujoco>')
  rng = np.random.default_rng(0)
  box = np.array([r, r, h + r])
  p = rng.uniform(-box, box, (400000, 3))
  zc = np.clip(p[:, 2], -h, h)
  inside = (p[:, 0] ** 2 + p[:, 1] ** 2 + (p[:, 2] - zc) ** 2) <= r * r
  vol = inside.mean() * np.prod(2 * box)
  q = p[inside]
  ixx = np.mean(q[:, 1] ** 2 + q[:, 2] ** 2) * 1000 * vol
  izz = np.mean(q[:, 0] ** 2 + q[:, 1] ** 2) * 1000 * vol
  assert abs(mjm.body_mass[1] - 1000 * vol) / mjm.body_mass[1] < 0.01
  np.testing.assert_allclose(mjm.body_inertia[1], [ixx, ixx, izz], rtol=0.02)


def test_fromto_and_zaxis_orientation():
  m = load("humanoid.xml")
  g = m.geom_names.index("thigh_right")
  # fromto="0 0 0 0 .01 -.34": z axis of the geom along the segment, centred on its midpoint
  from mjx_warp_b200.mjcf import _quat_to_mat
  z = _quat_to_mat(m.geom_quat[g])[:, 2]
  d = np.array([0, 0.01, -0.34])
  np.testing.assert_allclose(z, d / np.linalg.norm(d), atol=1e-12)
  np.testing.assert_allclose(m.geom_pos[g], d / 2, atol=1e-12)
  np.testing.assert_allclose(m.geom_size[g][:2], [0.06, np.linalg.norm(d) / 2])


def test_reference_fixture_quirks_parse():
  """constraints.xml has an attribute without a separating space; SAP model uses <!- comments."""
  m = load("constraints.xml")
  assert m.opt.impratio == 1.5 and m.nu == 3
  s = load(fixtures()["sap_model"])
  np.testing.assert_allclose(s.geom_rbound[1:], math.sqrt(3) * 0.5)


_EQUALITY = """<mujoco><worldbody>
  <body name="b1"><geom type="sphere" size=".1"/><freejoint/></body>
  <body name="b2"><geom type="sphere" size=".1"/><freejoint/></body></worldbody>
  <equality><connect body1="b1" body2="b2" anchor="0 0 0"/></equality></mujoco>"""
_SENSOR = """<mujoco><worldbody><body><geom type="sphere" size=".1"/><joint name="slide" type="slide"/>
  </body></worldbody><sensor><jointpos joint="slide"/></sensor></mujoco>"""
_TENDON = """<mujoco><worldbody><body><geom type="sphere" size=".1"/><site name="s0"/>
  <joint type="slide"/><body pos="0 0 .1"><geom type="sphere" size=".1"/><site name="s1"/></body>
  </body></worldbody><tendon><spatial><site site="s0"/><site site="s1"/></spatial></tendon></mujoco>"""


@pytest.mark.parametrize("xml", [_EQUALITY, _SENSOR, _TENDON])
def test_put_model_rejects_unsupported(xml):
  """io_test.py:27-91: equality constraints, sensors and tendons raise NotImplementedError."""
  mjm = mjcf.from_xml_string(xml)
  with pytest.raises(NotImplementedError):
    mjw.put_model(mjm, device="cpu")


def test_put_model_rejects_options():
  mjm = load("pendula.xml")
  mjm.opt.integrator = 1  # RK4
  with pytest.raises(NotImplementedError):
    mjw.put_model(mjm, device="cpu")
  mjm = load("pendula.xml")
  mjm.opt.cone = 1  # elliptic
  with pytest.raises(NotImplementedError):
    mjw.put_model(mjm, device="cpu")


def test_keyframe_reset():
  m = load("humanoid.xml")
  d = mjcf.MjData(m)
  mjcf.mj_resetDataKeyframe(m, d, 1)
  np.testing.assert_allclose(d.qpos, m.key_qpos[1])
  with pytest.raises(ValueError):
    mjcf.mj_resetDataKeyframe(m, d, 5)
