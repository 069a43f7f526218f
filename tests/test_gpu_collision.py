"""Collision and constraint rows on the GPU vs the oracle (collision_driver_test.py,
broad_phase_test.py, constraint_test.py).  Pair sets and contact / row counts are compared
exactly; pair sets bit-exactly when the oracle is fed the device's own geom poses."""

import numpy as np
import pytest
import torch

import mjx_warp_b200 as mjw
from helpers import (assert_close, dev, device_data, fixtures, generic_state, humanoid,
                     humanoid_state, load, oracle, world_rows)

pytestmark = pytest.mark.gpu


def _device_rows(d, kind, field, width):
  n, idx = world_rows(d, kind)
  t = field.cpu().numpy()[idx].reshape(len(idx), width) if len(idx) else np.zeros((0, width))
  return n, t


@pytest.mark.parametrize("name", ["box_plane", "plane_sphere", "sphere_sphere", "capsule_capsule",
                                  "plane_capsule"])
def test_primitives(name):
  """collision_driver_test.py:104-128 on the reference's own inline models."""
  mjm = load(fixtures()["primitive_models"][name])
  m = mjw.put_model(mjm)
  d = mjw.make_data(mjm, nworld=1)
  mjw.kinematics(m, d)
  mjw.collision(m, d)
  o = oracle(mjm, mjm.qpos0[None], np.zeros((1, mjm.nv)), np.zeros((1, 0)), 64)
  o.run("kinematics")
  o.run("collision")
  n, dist = _device_rows(d, "contact", d.contact.dist, 1)
  cnt, odist = o.rows("contact_dist")
  assert int(d.ncon.cpu()[0]) == n[0] == cnt[0] and n[0] > 0
  assert_close(dist, odist, "dist")
  _, pos = _device_rows(d, "contact", d.contact.pos, 3)
  assert_close(pos, o.rows("contact_pos")[1], "pos")
  _, frame = _device_rows(d, "contact", d.contact.frame, 9)
  assert_close(frame, o.rows("contact_frame")[1], "frame")
  for f, w in (("includemargin", 1), ("friction", 5), ("solref", 2), ("solimp", 5)):
    _, v = _device_rows(d, "contact", getattr(d.contact, f), w)
    assert_close(v, o.rows("contact_" + f)[1], f)


def test_nxn_keyframes_known_answers():
  """broad_phase_test.py:186-242 on the device: counts, pairs and type ordering."""
  mjm = load(fixtures()["nxn_model"])
  m = mjw.put_model(mjm)
  expect = {0: [], 1: [(0, 1)], 2: [(0, 1), (0, 2), (1, 2)], 3: [(3, 2)]}
  for key, pairs in expect.items():
    d = mjw.make_data(mjm, nworld=1)
    d.qpos.copy_(torch.as_tensor(mjm.key_qpos[key][None], dtype=torch.float32))
    mjw.kinematics(m, d)
    mjw.nxn_broadphase(m, d)
    nc = int(d.ncollision.cpu()[0])
    assert nc == len(pairs), key
    assert [tuple(p) for p in d.collision_pair.cpu().numpy()[:nc]] == pairs
  d = mjw.make_data(mjm, nworld=2)
  d.qpos.copy_(torch.as_tensor(np.stack([mjm.key_qpos[1], mjm.key_qpos[2]]), dtype=torch.float32))
  mjw.kinematics(m, d)
  mjw.nxn_broadphase(m, d)
  n, pairs = _device_rows(d, "pair", d.collision_pair, 2)
  assert int(d.ncollision.cpu()[0]) == 4 and list(n) == [1, 3]
  assert [tuple(p) for p in pairs] == [(0, 1), (0, 1), (0, 2), (1, 2)]
  assert list(d.collision_worldid.cpu().numpy()[d.world_pairadr.cpu().numpy()[1]:][:3]) == [1, 1, 1]


def test_sap_model_expected_pairs():
  """broad_phase_test.py:42-118: sap_broadphase finds exactly the expected 19 pairs."""
  f = fixtures()
  mjm = load(f["sap_model"])
  m = mjw.put_model(mjm)
  d = mjw.make_data(mjm, nworld=1)
  mjw.kinematics(m, d)
  mjw.sap_broadphase(m, d)
  nc = int(d.ncollision.cpu()[0])
  got = {tuple(sorted(p)) for p in d.collision_pair.cpu().numpy()[:nc]}
  assert nc == len(f["sap_expected_pairs"])
  assert got == {tuple(p) for p in f["sap_expected_pairs"]}


def _spheres_xml(n):
  """Project-written: a floor, two wall planes off the origin (x = +-0.5) and n free spheres of
  radius 0.05, so ngeom = n + 3."""
  bodies = "".join(f'<body pos="0 0 {0.2 + 0.1 * i}"><freejoint/><geom type="sphere" size="0.05"/></body>'
                   for i in range(n))
  return ('<mujoco><worldbody><geom type="plane" size="0 0 0.05"/>'
          '<geom type="plane" pos="0.5 0 0" zaxis="-1 0 0" size="0 0 0.05"/>'
          '<geom type="plane" pos="-0.5 0 0" zaxis="1 0 0" size="0 0 0.05"/>'
          f'{bodies}</worldbody></mujoco>')


def _scatter(mjm, nworld, seed, half=0.45, zmax=0.4):
  """Free bodies at x, y ~ U(-half, half), z ~ U(0.02, zmax), random orientations."""
  rng = np.random.default_rng(seed)
  qpos = np.tile(mjm.qpos0, (nworld, 1))
  for b in range(mjm.nq // 7):
    a = 7 * b
    qpos[:, a:a + 2] = rng.uniform(-half, half, (nworld, 2))
    qpos[:, a + 2] = rng.uniform(0.02, zmax, nworld)
    q = rng.normal(size=(nworld, 4))
    qpos[:, a + 3:a + 7] = q / np.linalg.norm(q, axis=1, keepdims=True)
  return qpos, np.zeros((nworld, mjm.nv)), np.zeros((nworld, 0))


@pytest.mark.parametrize("name", ["bin.xml", "spheres120", "spheres240"])
def test_sap_pair_lists_bit_exact(name):
  """Sweep-and-prune (collision_driver.py:350-455) on the device vs the oracle's restatement given
  the device's geom poses: identical pair lists, in the same sweep order, in every world.
  bin.xml (69 geoms, walls off the origin) calls sap_broadphase directly; the 123-geom model goes
  through collision(), which selects sweep-and-prune for ngeom > 100 as the reference does, and
  its contacts are compared too; with 240 spheres every world has more candidate pairs than the
  narrowphase keeps contact counts for between its counting and write passes (672), so the pairs
  past them are counted twice.  (These models are large enough for the reference's automatic
  sparse mass matrix; jacobian = 0 selects the dense one the kernels implement.)"""
  nsphere = 240 if name == "spheres240" else 120
  mjm = load("bin.xml", jacobian=0) if name == "bin.xml" else load(_spheres_xml(nsphere), jacobian=0)
  nworld = 64
  if name == "spheres240":  # packed into a 0.6 x 0.6 x 0.3 box: 876-979 pairs per world
    qpos, qvel, ctrl = _scatter(mjm, nworld, seed=5, half=0.3, zmax=0.3)
  else:
    qpos, qvel, ctrl = _scatter(mjm, nworld, seed=5)
  m = mjw.put_model(mjm)
  nconmax = (1024 if name == "spheres240" else 512) * nworld
  d = device_data(mjm, qpos, qvel, ctrl, nconmax=nconmax, njmax=64 * nworld)
  mjw.kinematics(m, d)
  if name == "bin.xml":
    mjw.sap_broadphase(m, d)
  else:
    assert mjm.ngeom > 100
    mjw.collision(m, d)
  torch.cuda.synchronize()
  assert np.all(mjw.world_status(d) == 0)
  o = oracle(mjm, qpos, qvel, ctrl, 32)
  o.set("geom_xpos", dev(d.geom_xpos))
  o.set("geom_xmat", dev(d.geom_xmat))
  o.run("sap_broadphase")
  cnt, opairs = o.rows("pair")
  n, pairs = _device_rows(d, "pair", d.collision_pair, 2)
  assert cnt.sum() > nworld
  if name == "spheres240":
    assert cnt.min() > 672
  np.testing.assert_array_equal(n, cnt)
  np.testing.assert_array_equal(pairs, opairs.astype(np.int32))
  if name != "bin.xml":
    o.run("narrowphase")
    ccnt, _ = o.rows("contact_dist")
    nc, geoms = _device_rows(d, "contact", d.contact.geom, 2)
    np.testing.assert_array_equal(nc, ccnt)
    np.testing.assert_array_equal(geoms, o.rows("contact_geom")[1].astype(np.int32))


def test_nxn_many_candidates_bit_exact():
  """nxn_broadphase with more candidate pairs than the 32 chunks of 32 whose test results the
  kernel keeps for its write pass (63 geoms: 1950 candidates), the rest tested again: the same
  pair lists as the oracle, in the same order, in every world, and the same contacts."""
  mjm = load(_spheres_xml(60), jacobian=0)
  assert mjm.ngeom <= 100
  nworld = 32
  qpos, qvel, ctrl = _scatter(mjm, nworld, seed=9, half=0.25, zmax=0.3)
  m = mjw.put_model(mjm)
  from mjx_warp_b200.io import pair_candidates
  assert pair_candidates(m).shape[0] > 32 * 32
  d = device_data(mjm, qpos, qvel, ctrl, nconmax=1024 * nworld, njmax=64 * nworld)
  mjw.kinematics(m, d)
  mjw.collision(m, d)
  torch.cuda.synchronize()
  assert np.all(mjw.world_status(d) == 0)
  o = oracle(mjm, qpos, qvel, ctrl, 32)
  o.set("geom_xpos", dev(d.geom_xpos))
  o.set("geom_xmat", dev(d.geom_xmat))
  o.run("nxn_broadphase")
  cnt, opairs = o.rows("pair")
  n, pairs = _device_rows(d, "pair", d.collision_pair, 2)
  assert cnt.sum() > nworld
  np.testing.assert_array_equal(n, cnt)
  np.testing.assert_array_equal(pairs, opairs.astype(np.int32))
  o.run("narrowphase")
  ccnt, _ = o.rows("contact_dist")
  nc, geoms = _device_rows(d, "contact", d.contact.geom, 2)
  np.testing.assert_array_equal(nc, ccnt)
  np.testing.assert_array_equal(geoms, o.rows("contact_geom")[1].astype(np.int32))


@pytest.mark.parametrize("name", ["humanoid.xml", "collision.xml"])
def test_pair_sets_bit_exact(name):
  """Given the device's geom poses, the oracle's FP32 nxn test selects the identical pair list,
  in the same canonical order, in every world."""
  mjm = humanoid() if name == "humanoid.xml" else load(name)
  nworld = 256
  if name == "humanoid.xml":
    qpos, qvel, ctrl = humanoid_state(mjm, nworld, seed=11)
  else:
    qpos, qvel, ctrl = generic_state(mjm, nworld, seed=11, qscale=0.15)
  m = mjw.put_model(mjm)
  d = device_data(mjm, qpos, qvel, ctrl)
  mjw.kinematics(m, d)
  mjw.collision(m, d)
  o = oracle(mjm, qpos, qvel, ctrl, 32)
  o.set("geom_xpos", dev(d.geom_xpos))
  o.set("geom_xmat", dev(d.geom_xmat))
  o.run("nxn_broadphase")
  cnt, opairs = o.rows("pair")
  n, pairs = _device_rows(d, "pair", d.collision_pair, 2)
  np.testing.assert_array_equal(n, cnt)
  np.testing.assert_array_equal(pairs, opairs.astype(np.int32))
  o.run("narrowphase")
  ccnt, _ = o.rows("contact_dist")
  nc, geoms = _device_rows(d, "contact", d.contact.geom, 2)
  np.testing.assert_array_equal(nc, ccnt)
  np.testing.assert_array_equal(geoms, o.rows("contact_geom")[1].astype(np.int32))


def test_collision_model_contacts():
  """Spheres, capsules and boxes on slide joints (collision.xml) vs the oracle."""
  mjm = load("collision.xml")
  m = mjw.put_model(mjm)
  qpos = mjm.key_qpos[0][None]
  d = mjw.make_data(mjm, nworld=1)
  d.qpos.copy_(torch.as_tensor(qpos, dtype=torch.float32))
  mjw.forward(m, d)
  o = oracle(mjm, qpos, np.zeros((1, mjm.nv)), np.zeros((1, 0)), 64)
  o.run("forward")
  n, dist = _device_rows(d, "contact", d.contact.dist, 1)
  cnt, odist = o.rows("contact_dist")
  assert list(n) == list(cnt) and cnt[0] > 0
  assert_close(dist, odist, "dist")


@pytest.mark.parametrize("name", ["humanoid.xml", "sphere_chain.xml"])
def test_constraint_rows(name):
  """constraint_test.py:39-56: efc_J / D / aref / pos / margin per world in canonical order."""
  mjm = humanoid() if name == "humanoid.xml" else load(name)
  nworld = 32
  if name == "humanoid.xml":
    qpos, qvel, ctrl = humanoid_state(mjm, nworld, seed=7)
  else:
    qpos, qvel, ctrl = generic_state(mjm, nworld, seed=7, qscale=1.2)
    qpos[:, 2] = 0.09  # the ball rests in contact with the floor
  m = mjw.put_model(mjm)
  d = device_data(mjm, qpos, qvel, ctrl)
  mjw.forward(m, d)
  o = oracle(mjm, qpos, qvel, ctrl, 64)
  o.run("forward")
  cnt, _ = o.rows("efc_D")
  n, idx = world_rows(d, "efc")
  np.testing.assert_array_equal(n, cnt)
  assert cnt.sum() > 0
  assert int(d.nefc.cpu()[0]) == cnt.sum()
  np.testing.assert_array_equal(d.efc.worldid.cpu().numpy()[idx], np.repeat(np.arange(nworld), n))
  for f in ("J", "pos", "margin"):
    assert_close(getattr(d.efc, f).cpu().numpy()[idx].reshape(len(idx), -1), o.rows("efc_" + f)[1], f)
  for f in ("D", "aref"):
    assert_close(getattr(d.efc, f).cpu().numpy()[idx].reshape(len(idx), -1), o.rows("efc_" + f)[1], f,
                 rtol=2e-3, atol=2e-3)


def test_overflow_sets_status_bits():
  """Capacity overflow drops a world's rows and flags it instead of writing out of bounds."""
  mjm = humanoid()
  qpos, qvel, ctrl = humanoid_state(mjm, 16, seed=1)
  m = mjw.put_model(mjm)
  d = device_data(mjm, qpos, qvel, ctrl, nconmax=40, njmax=40)
  mjw.step(m, d)
  st = mjw.world_status(d)
  assert np.any(st & 0x4) or np.any(st & 0x1)  # pair or contact overflow
  pair_over = (st & 0x4) != 0
  assert np.all(d.world_npair.cpu().numpy()[pair_over] == 0)
  kept = ~pair_over
  assert int(d.world_npair.cpu().numpy()[kept].sum()) <= 40
  assert np.all(np.isfinite(d.qpos.cpu().numpy()))
