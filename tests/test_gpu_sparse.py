"""The sparse mass matrix (the reference's layout when opt.is_sparse: qM and qLD as
(nworld, 1, nM), smooth.py:264-351, 609-652, support.py:96-137) on the GPU vs the dense path and
the oracle.  Models: pendula.xml (free, ball, slide and hinge trees), the humanoid and the bin
(nv = 384, which the reference's automatic choice runs sparse)."""

import numpy as np
import pytest
import torch

import mjx_warp_b200 as mjw
from helpers import dev, device_data, generic_state, humanoid, load, oracle, rel_err, world_rows
from mjx_warp_b200 import io
from mjx_warp_b200.types import MJ_JAC_DENSE, MJ_JAC_SPARSE

pytestmark = pytest.mark.gpu


def _pair(name, **opt):
  if name == "humanoid":
    dense, sparse = humanoid(), humanoid()
  else:
    dense, sparse = load(name), load(name)
  for k, v in opt.items():
    setattr(dense.opt, k, v)
    setattr(sparse.opt, k, v)
  dense.opt.jacobian, sparse.opt.jacobian = MJ_JAC_DENSE, MJ_JAC_SPARSE
  return dense, sparse


@pytest.mark.parametrize("name", ["pendula.xml", "humanoid"])
def test_sparse_mass_matrix_factor_solve_mul(name):
  dense, sparse = _pair(name)
  nworld = 8
  qpos, qvel, ctrl = generic_state(dense, nworld, seed=3, qscale=0.1)
  out = {}
  for tag, mjm in (("dense", dense), ("sparse", sparse)):
    m = mjw.put_model(mjm)
    d = device_data(mjm, qpos, qvel, ctrl)
    assert tuple(d.qM.shape) == ((nworld, 1, mjm.nM) if tag == "sparse" else (nworld, mjm.nv, mjm.nv))
    mjw.kinematics(m, d)
    mjw.com_pos(m, d)
    mjw.crb(m, d)
    mjw.factor_m(m, d)
    y = torch.as_tensor(np.random.default_rng(1).normal(size=(nworld, mjm.nv)), dtype=torch.float32,
                        device="cuda")
    x = torch.zeros_like(y)
    mjw.solve_m(m, d, x, y)
    r = torch.zeros_like(y)
    mjw.mul_m(m, d, r, y)
    torch.cuda.synchronize()
    out[tag] = (d.qM.cpu().numpy(), x.cpu().numpy(), r.cpu().numpy(), d.qLDiagInv.cpu().numpy())
  qd, xd, rd, _ = out["dense"]
  qs, xs, rs, dinv = out["sparse"]
  for w in range(nworld):
    np.testing.assert_array_equal(io.dense_from_sparse(sparse, qs[w, 0]), qd[w])  # same crb arithmetic
    L = io.factor_sparse_host(sparse, qs[w, 0].astype(np.float64))
    np.testing.assert_allclose(dinv[w], 1.0 / L[sparse.dof_Madr], rtol=1e-4)
  np.testing.assert_allclose(xs, xd, rtol=1e-4, atol=1e-5 * np.abs(xd).max())
  np.testing.assert_allclose(rs, rd, rtol=1e-5, atol=1e-6 * np.abs(rd).max())


@pytest.mark.parametrize("form", [0, 1, 2])
def test_sparse_steps_match_dense(form):
  """sphere_chain.xml (free sphere on the floor + a hinge chain; Euler with eulerdamp, Newton):
  sparse and dense steps agree in every launch form."""
  dense, sparse = _pair("sphere_chain.xml")
  nworld = 16
  rng = np.random.default_rng(0)
  qpos = np.tile(dense.qpos0, (nworld, 1))
  qpos[:, 7:] = rng.uniform(-0.1, 0.1, (nworld, 5))
  qpos[:, 2] = 0.09  # the ball touches the floor
  qvel = rng.normal(0, 0.1, (nworld, dense.nv))
  ctrl = rng.uniform(-1, 1, (nworld, dense.nu))
  res = {}
  for tag, mjm in (("dense", dense), ("sparse", sparse)):
    m = mjw.put_model(mjm)
    d = device_data(mjm, qpos, qvel, ctrl)
    for _ in range(10):
      mjw.step(m, d, fused=form)
    torch.cuda.synchronize()
    assert np.all(mjw.world_status(d) == 0)
    res[tag] = (dev(d.qpos), dev(d.qvel), int(d.nefc.cpu()[0]))
  assert res["sparse"][2] == res["dense"][2] > 0
  assert rel_err(res["sparse"][0], res["dense"][0]).max() < 1e-5
  assert rel_err(res["sparse"][1], res["dense"][1]).max() < 1e-3


def test_bin_auto_sparse_vs_fp64():
  """bin.xml with the reference's automatic choice (nv = 384 -> sparse) vs the FP64 oracle."""
  mjm = load("bin.xml", iterations=20, ls_iterations=20)
  assert mjw.is_sparse(mjm)
  nworld = 8
  rng = np.random.default_rng(1)
  qpos = np.tile(mjm.qpos0, (nworld, 1))
  for b in range(mjm.nbody - 1):
    a = 7 * b
    qpos[:, a:a + 2] = rng.uniform(-0.4, 0.4, (nworld, 2))
    qpos[:, a + 2] = rng.uniform(0.03, 0.35, nworld)
    q = rng.normal(size=(nworld, 4))
    qpos[:, a + 3:a + 7] = q / np.linalg.norm(q, axis=1, keepdims=True)
  qvel = rng.normal(0.0, 0.1, (nworld, mjm.nv))
  ctrl = np.zeros((nworld, 0))
  m = mjw.put_model(mjm)
  d = device_data(mjm, qpos, qvel, ctrl, nconmax=600 * nworld, njmax=512 * nworld)
  mjw.forward(m, d)
  o = oracle(mjm, qpos, qvel, ctrl, 64)
  o.run("forward")
  torch.cuda.synchronize()
  assert np.all(mjw.world_status(d) == 0)
  qm = np.stack([io.dense_from_sparse(mjm, v) for v in d.qM.cpu().numpy()[:, 0]])
  np.testing.assert_allclose(qm.reshape(nworld, -1), o.get("qM"), rtol=5e-4, atol=5e-4)
  assert rel_err(dev(d.qacc_smooth), o.get("qacc_smooth")).max() < 2e-3
  n_efc, _ = world_rows(d, "efc")
  np.testing.assert_array_equal(n_efc, o.rows("efc_D")[0])
  cg, co = d.efc.cost.cpu().numpy(), o.scalar("cost")
  assert np.all(cg <= co + 0.025 * np.abs(co) + 1e-3), (cg, co)
  assert np.median(rel_err(dev(d.qacc), o.get("qacc"))) < 1e-2
  for _ in range(3):
    mjw.step(m, d)
  torch.cuda.synchronize()
  assert np.all(np.isfinite(d.qpos.cpu().numpy())) and np.all(mjw.world_status(d) == 0)


def test_implicit_with_sparse_is_rejected():
  """forward.py:268 asserts the dense mass matrix for implicitfast."""
  _, sparse = _pair("humanoid")
  m = mjw.put_model(sparse)
  d = mjw.make_data(sparse, nworld=2)
  with pytest.raises(NotImplementedError):
    mjw.step(m, d)
  with pytest.raises(NotImplementedError):
    mjw.implicit(m, d)
