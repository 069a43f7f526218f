"""Pins the CPU oracle to the known-answer vectors of the reference's own tests.

The vectors are read from tests/golden/reference_fixtures.json, which tests/golden/make_golden.py
extracted from the reference's test files (math_test.py, broad_phase_test.py).
"""

import numpy as np
import pytest

from helpers import fixtures, load
from oracle import Oracle, closest_segments


@pytest.mark.parametrize("precision", [64, 32])
def test_closest_segment_points(precision):
  """math_test.py:22-88 — closest points between segments."""
  for case in fixtures()["math_closest_segments"]:
    v = case["inputs"]
    pa, pb = closest_segments(v["a0"], v["a1"], v["b0"], v["b1"], precision)
    got = {"best_a": pa, "best_b": pb}
    for e in case["expected"]:
      tol = 0.5 * 10.0 ** (-e["places"])
      np.testing.assert_array_less(np.abs(got[e["var"]] - np.array(e["value"])), tol + 1e-12,
                                   err_msg=f"{case['name']} {e['var']}")


def _pairs_at(mjm, qpos, nworld=1, stage="nxn_broadphase"):
  o = Oracle(mjm, nworld, 32)
  o.set("qpos", qpos)
  o.run("kinematics")
  o.run(stage)
  cnt, pairs = o.rows("pair")
  return cnt, pairs.astype(int)


@pytest.mark.parametrize("stage", ["nxn_broadphase", "sap_broadphase"])
def test_sap_model_pairs(stage):
  """broad_phase_test.py:42-118: the 19 overlapping box / plane pairs at qpos0 (the reference
  checks its sweep-and-prune result against this brute-force list)."""
  f = fixtures()
  mjm = load(f["sap_model"])
  cnt, pairs = _pairs_at(mjm, mjm.qpos0, stage=stage)
  expected = {tuple(p) for p in f["sap_expected_pairs"]}
  got = {tuple(sorted(p)) for p in pairs}
  assert cnt[0] == len(expected)
  assert got == expected


def test_sap_matches_nxn_without_margins_or_offset_planes():
  """With zero margins and no planes, the sweep-and-prune overlap test is the nxn bounding test:
  the same pair set in every keyframe world of the nxn model (broad_phase_test.py:124-185)."""
  mjm = load(fixtures()["nxn_model"])
  qpos = np.stack([mjm.key_qpos[k] for k in range(mjm.key_qpos.shape[0])])
  cn, pn = _pairs_at(mjm, qpos, nworld=qpos.shape[0])
  cs, ps = _pairs_at(mjm, qpos, nworld=qpos.shape[0], stage="sap_broadphase")
  np.testing.assert_array_equal(cn, cs)
  off = np.concatenate([[0], np.cumsum(cn)])
  for w in range(len(cn)):
    assert {tuple(p) for p in pn[off[w]:off[w + 1]]} == {tuple(p) for p in ps[off[w]:off[w + 1]]}


def test_nxn_keyframes():
  """broad_phase_test.py:124-242: counts and (type-ordered) pairs per keyframe."""
  mjm = load(fixtures()["nxn_model"])
  expect = {0: [], 1: [(0, 1)], 2: [(0, 1), (0, 2), (1, 2)], 3: [(3, 2)]}
  for key, pairs in expect.items():
    cnt, got = _pairs_at(mjm, mjm.key_qpos[key])
    assert cnt[0] == len(pairs), key
    assert [tuple(p) for p in got] == pairs, key
  # two worlds (keyframes 1 and 2): four collisions, world order
  cnt, got = _pairs_at(mjm, np.stack([mjm.key_qpos[1], mjm.key_qpos[2]]), nworld=2)
  assert list(cnt) == [1, 3]
  assert [tuple(p) for p in got] == [(0, 1), (0, 1), (0, 2), (1, 2)]
  # contype / conaffinity incompatibility removes every pair
  mjm.geom_contype[:] = 0
  mjm.geom_conaffinity[:] = 1
  cnt, _ = _pairs_at(mjm, mjm.key_qpos[1])
  assert cnt[0] == 0


def test_disable_eulerdamp_velocity():
  """forward_test.py:130-145: with eulerdamp disabled, qvel = 1 + dt after euler with qacc = 1."""
  mjm = load("pendula.xml")
  mjm.opt.disableflags |= 1 << 14
  o = Oracle(mjm, 1, 64)
  o.set("qvel", np.ones(mjm.nv))
  o.set("qacc", np.ones(mjm.nv))
  o.run("euler")
  np.testing.assert_allclose(o.get("qvel")[0], 1 + mjm.opt.timestep)


def test_oracle_precisions_agree_on_smooth_dynamics():
  """float and double restatements agree on the smooth quantities of a perturbed humanoid."""
  from helpers import humanoid, humanoid_state

  mjm = humanoid()
  qpos, qvel, ctrl = humanoid_state(mjm, 8)
  res = {}
  for p in (32, 64):
    o = Oracle(mjm, 8, p)
    o.set("qpos", qpos)
    o.set("qvel", qvel)
    o.set("ctrl", ctrl)
    o.run("forward_nosolve")
    res[p] = {k: o.get(k) for k in ("xpos", "cinert", "qM", "qfrc_bias", "qacc_smooth")}
  for k in res[64]:
    np.testing.assert_allclose(res[32][k], res[64][k], rtol=5e-4, atol=5e-4, err_msg=k)
