"""The uneven-contact configurations on the GPU vs the oracle, at sizes the oracle finishes quickly.

- bin.xml (64 free bodies in a 5-plane bin, nv = 384): packed states with 28-60 contacts and
  112-240 constraint rows per world, so one batch mixes very different row counts; the solver
  rows far exceed the 32 staged in shared memory and nv > 32 takes the generic path.
- humanoid_spheres.xml (humanoid + 16 free spheres, nv = 123): each world drops k ~ U{0..16}
  spheres next to the humanoid; the others are parked far away and never touch anything.

Both models have nv >= 60, for which the reference's automatic choice is the sparse mass matrix;
these tests select the dense one (jacobian = dense), the layout the kernels implement.
"""

import numpy as np
import pytest
import torch

import mjx_warp_b200 as mjw
from mjx_warp_b200.types import MJ_JAC_DENSE
from helpers import assert_close, dev, device_data, load, oracle, rel_err, world_rows

pytestmark = pytest.mark.gpu


def bin_state(mjm, nworld, seed):
  """Bodies at x, y ~ U(-0.4, 0.4), z ~ U(0.03, 0.35) with random orientations: overlapping
  packings with many contacts."""
  rng = np.random.default_rng(seed)
  qpos = np.tile(mjm.qpos0, (nworld, 1))
  for b in range(mjm.nbody - 1):
    a = 7 * b
    qpos[:, a:a + 2] = rng.uniform(-0.4, 0.4, (nworld, 2))
    qpos[:, a + 2] = rng.uniform(0.03, 0.35, nworld)
    q = rng.normal(size=(nworld, 4))
    qpos[:, a + 3:a + 7] = q / np.linalg.norm(q, axis=1, keepdims=True)
  qvel = rng.normal(0.0, 0.1, (nworld, mjm.nv))
  return qpos, qvel, np.zeros((nworld, 0))


def test_bin_uneven_rows_forward():
  mjm = load("bin.xml", iterations=20, ls_iterations=20, jacobian=MJ_JAC_DENSE)
  nworld = 8
  qpos, qvel, ctrl = bin_state(mjm, nworld, seed=1)
  m = mjw.put_model(mjm)
  d = device_data(mjm, qpos, qvel, ctrl, nconmax=600 * nworld, njmax=512 * nworld)
  mjw.forward(m, d)
  o = oracle(mjm, qpos, qvel, ctrl, 64)
  o.run("forward")
  torch.cuda.synchronize()
  assert np.all(mjw.world_status(d) == 0)
  for f in ("xpos", "cinert", "cdof", "qfrc_bias"):
    assert_close(dev(getattr(d, f)), o.get(f), f)
  qm = dev(d.qM)
  assert_close(qm, o.get("qM"), "qM")
  e = rel_err(dev(d.qacc_smooth), o.get("qacc_smooth"))
  assert e.max() < 2e-3, e.max()
  n_con, _ = world_rows(d, "contact")
  cnt, _ = o.rows("contact_dist")
  assert np.array_equal(n_con, cnt), (n_con, cnt)
  n_efc, _ = world_rows(d, "efc")
  ecnt, _ = o.rows("efc_D")
  np.testing.assert_array_equal(n_efc, ecnt)
  assert n_efc.min() > 64 and n_efc.max() > n_efc.min()
  cg, co = d.efc.cost.cpu().numpy(), o.scalar("cost")
  assert np.all(cg <= co + 0.025 * np.abs(co) + 1e-3), (cg, co)
  e = rel_err(dev(d.qacc), o.get("qacc"))
  assert np.median(e) < 1e-2, e


def test_bin_steps_stay_finite_and_forms_agree():
  """A short drop from the packed state: every form keeps every world finite and flag-free, and
  the chosen and plain forms give the same smooth accelerations."""
  mjm = load("bin.xml", iterations=5, ls_iterations=10, jacobian=MJ_JAC_DENSE)
  nworld = 8
  qpos, qvel, ctrl = bin_state(mjm, nworld, seed=2)
  m = mjw.put_model(mjm)
  out = {}
  for form in (1, 0):
    d = device_data(mjm, qpos, qvel, ctrl, nconmax=600 * nworld, njmax=512 * nworld)
    for _ in range(5):
      mjw.step(m, d, fused=form)
    torch.cuda.synchronize()
    assert np.all(np.isfinite(d.qpos.cpu().numpy())), form
    assert np.all(mjw.world_status(d) == 0), form
    out[form] = dev(d.qacc_smooth)
  assert_close(out[0], out[1], "qacc_smooth chosen vs plain", rtol=1e-3, atol=1e-3)


def humanoid_spheres_state(mjm, hum, nworld, seed):
  """Humanoid keyframe 0 + U(-0.05, 0.05); k ~ U{0..16} spheres dropped near it from
  z ~ U(0.1, 0.6), the rest parked 100 m away at 10 m height."""
  rng = np.random.default_rng(seed)
  qpos = np.zeros((nworld, mjm.nq))
  qpos[:, :hum.nq] = hum.key_qpos[0] + rng.uniform(-0.05, 0.05, (nworld, hum.nq))
  qpos[:, 3:7] /= np.linalg.norm(qpos[:, 3:7], axis=1, keepdims=True)
  nsph = (mjm.nq - hum.nq) // 7
  k = rng.integers(0, nsph + 1, nworld)
  for i in range(nsph):
    a = hum.nq + 7 * i
    active = i < k
    qpos[:, a] = np.where(active, rng.uniform(-0.6, 0.6, nworld), 100.0 + 2.0 * i)
    qpos[:, a + 1] = np.where(active, rng.uniform(-0.6, 0.6, nworld), 100.0)
    qpos[:, a + 2] = np.where(active, rng.uniform(0.1, 0.6, nworld), 10.0)
    qpos[:, a + 3] = 1.0
  qvel = rng.normal(0.0, 0.01, (nworld, mjm.nv))
  ctrl = rng.uniform(-0.4, 0.4, (nworld, mjm.nu))
  return qpos, qvel, ctrl, k


def test_humanoid_spheres_steps_vs_fp64():
  hum = load("humanoid.xml")
  mjm = load("humanoid_spheres.xml", integrator=3, timestep=0.005, iterations=10, ls_iterations=20,
             jacobian=MJ_JAC_DENSE)
  nworld = 16
  qpos, qvel, ctrl, k = humanoid_spheres_state(mjm, hum, nworld, seed=4)
  assert k.min() < k.max()
  m = mjw.put_model(mjm)
  d = device_data(mjm, qpos, qvel, ctrl, nconmax=96 * nworld, njmax=384 * nworld)
  o = oracle(mjm, qpos, qvel, ctrl, 64)
  mjw.forward(m, d)
  o.run("forward")
  torch.cuda.synchronize()
  e = rel_err(dev(d.qacc), o.get("qacc"))
  assert e.max() < 1e-3, e
  n_efc, _ = world_rows(d, "efc")
  ecnt, _ = o.rows("efc_D")
  np.testing.assert_array_equal(n_efc, ecnt)
  for _ in range(5):
    mjw.step(m, d)
  o.run("step", nstep=5)
  torch.cuda.synchronize()
  assert np.all(mjw.world_status(d) == 0)
  assert np.quantile(rel_err(dev(d.qvel), o.get("qvel")), 0.9) < 1e-3
  assert np.quantile(rel_err(dev(d.qpos), o.get("qpos")), 0.9) < 1e-4


def _bin_forward(mjm, qpos, qvel, ctrl, form, cta_warps=8, tc=False):
  nworld = qpos.shape[0]
  m = mjw.put_model(mjm)
  d = device_data(mjm, qpos, qvel, ctrl, nconmax=600 * nworld, njmax=512 * nworld)
  try:
    if form == 1:
      mjw.set_tune(m, d, solver_cta_warps=cta_warps, hessian_tc=tc)
    mjw.forward(m, d, fused=form)
    torch.cuda.synchronize()
  finally:
    mjw.set_tune(m, d)
  return d


@pytest.mark.parametrize("cta_warps, tc", [(2, False), (4, False), (8, False), (16, False),
                                           (2, True), (4, True)])
def test_cta_solver_factor(cta_warps, tc):
  """The chosen form's Newton Hessian factor for dense nv > 32 (one CTA of 2 / 4 / 8 / 16 warps per
  world; panel updates on the tensor pipe in split TF32; tc: the Hessian itself assembled there
  too) on the bin (nv = 384): with no solver
  iterations both forms factor the Hessian of the same active set (the warmstart's), so the
  chosen form's L must reproduce H = tril(qM) + J_a' D_a J_a and agree with the plain form's
  FP32 factor, and the Newton directions must agree."""
  mjm = load("bin.xml", iterations=0, ls_iterations=10, jacobian=MJ_JAC_DENSE)
  nworld = 6
  qpos, qvel, ctrl = bin_state(mjm, nworld, seed=5)
  dc = _bin_forward(mjm, qpos, qvel, ctrl, 1, cta_warps, tc)
  dp = _bin_forward(mjm, qpos, qvel, ctrl, 0)
  nv = mjm.nv
  Lc = np.tril(dc.efc.h.cpu().numpy().astype(np.float64))
  Lp = np.tril(dp.efc.h.cpu().numpy().astype(np.float64))
  qM = dc.qM.cpu().numpy().astype(np.float64)
  n, idx = world_rows(dc, "efc")
  J = dc.efc.J.cpu().numpy().astype(np.float64)
  D = dc.efc.D.cpu().numpy().astype(np.float64)
  act = dc.efc.active.cpu().numpy().astype(bool)
  start = 0
  for w in range(nworld):
    rows = idx[start:start + n[w]]
    start += n[w]
    rows = rows[act[rows]]
    H = np.tril(qM[w]) + np.tril(qM[w], -1).T + J[rows].T @ (D[rows, None] * J[rows])
    r = np.linalg.norm(Lc[w] @ Lc[w].T - H) / np.linalg.norm(H)
    assert r < 1e-5, (w, r)
    assert np.linalg.norm(Lc[w] - Lp[w]) / np.linalg.norm(Lp[w]) < 1e-4, w
  e = rel_err(dev(dc.efc.Mgrad), dev(dp.efc.Mgrad))
  assert e.max() < 1e-3, e


@pytest.mark.parametrize("cta_warps, tc", [(2, False), (4, False), (8, False), (16, False),
                                           (4, True)])
def test_cta_solver_vs_warp_solver_and_fp64(cta_warps, tc):
  """The whole Newton solve on the bin with the CTA solver against the plain form's
  one-warp-per-world solver and the FP64 oracle: the reference's cost acceptance (2.5 %,
  solver_test.py:127) in every world and the same qacc as the warp solver."""
  mjm = load("bin.xml", iterations=20, ls_iterations=20, jacobian=MJ_JAC_DENSE)
  nworld = 8
  qpos, qvel, ctrl = bin_state(mjm, nworld, seed=1)
  dc = _bin_forward(mjm, qpos, qvel, ctrl, 1, cta_warps, tc)
  dp = _bin_forward(mjm, qpos, qvel, ctrl, 0)
  o = oracle(mjm, qpos, qvel, ctrl, 64)
  o.run("forward")
  assert np.all(mjw.world_status(dc) == 0)
  cg, co = dc.efc.cost.cpu().numpy(), o.scalar("cost")
  assert np.all(cg <= co + 0.025 * np.abs(co) + 1e-3), (cg, co)
  assert np.median(rel_err(dev(dc.qacc), o.get("qacc"))) < 1e-2
  assert np.median(rel_err(dev(dc.qacc), dev(dp.qacc))) < 1e-2


def test_precision_form_humanoid_spheres():
  """The precision form for nv > 32 (the humanoid with 0-16 extra spheres, nv = 123): the CTA
  solver factors and solves the Newton Hessian in FP64 in shared memory and sums the line-search
  coefficients in FP64, the mass-matrix factor-solves run in FP64 per tree block; converged qacc
  within 1e-3 of FP64 in every world and no worse than the FP32 chosen form, and a few steps stay
  finite and flag-free."""
  hum = load("humanoid.xml")
  mjm = load("humanoid_spheres.xml", integrator=3, timestep=0.005, iterations=10, ls_iterations=20,
             jacobian=MJ_JAC_DENSE)
  nworld = 16
  qpos, qvel, ctrl, _ = humanoid_spheres_state(mjm, hum, nworld, seed=7)
  m = mjw.put_model(mjm)
  o = oracle(mjm, qpos, qvel, ctrl, 64)
  o.run("forward")
  err = {}
  for form in (1, 3):
    d = device_data(mjm, qpos, qvel, ctrl, nconmax=96 * nworld, njmax=384 * nworld)
    mjw.forward(m, d, fused=form)
    torch.cuda.synchronize()
    err[form] = rel_err(dev(d.qacc), o.get("qacc"))
  assert err[3].max() < 1e-3, err[3]
  assert np.median(err[3]) <= 1.5 * np.median(err[1]) + 1e-7, (np.median(err[3]), np.median(err[1]))
  for _ in range(3):
    mjw.step(m, d, fused=3)
  torch.cuda.synchronize()
  assert np.all(np.isfinite(d.qpos.cpu().numpy()))
  assert np.all(mjw.world_status(d) == 0)


def test_cta_solver_sparse_mass_matrix():
  """The CTA solver with the sparse mass matrix (the reference's automatic choice for nv >= 60):
  the bin's Newton solve against the dense CTA solve and the FP64 oracle (the reference's cost
  acceptance, solver_test.py:127), with the FMA and the tensor-core Hessian assembly."""
  from mjx_warp_b200.types import MJ_JAC_SPARSE

  nworld = 8
  mjd = load("bin.xml", iterations=20, ls_iterations=20, jacobian=MJ_JAC_DENSE)
  mjs = load("bin.xml", iterations=20, ls_iterations=20, jacobian=MJ_JAC_SPARSE)
  qpos, qvel, ctrl = bin_state(mjd, nworld, seed=1)
  dd = _bin_forward(mjd, qpos, qvel, ctrl, 1, 2)
  o = oracle(mjd, qpos, qvel, ctrl, 64)
  o.run("forward")
  co = o.scalar("cost")
  for tc in (False, True):
    ds = _bin_forward(mjs, qpos, qvel, ctrl, 1, 2, tc)
    assert np.all(mjw.world_status(ds) == 0)
    cg = ds.efc.cost.cpu().numpy()
    assert np.all(cg <= co + 0.025 * np.abs(co) + 1e-3), (tc, cg, co)
    assert np.median(rel_err(dev(ds.qacc), dev(dd.qacc))) < 1e-2, tc
