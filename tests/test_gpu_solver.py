"""Constraint solver on the GPU vs the oracle (solver_test.py).

Parity is checked where the problem is well posed: with enough Newton iterations the solve
converges and qacc must agree with the FP64 oracle to 1e-3 relative in every world (the measured
maximum is ~7e-5).  At the benchmark's 3 iterations the iterate is not converged and depends
discontinuously on its inputs (FP32 vs FP64 inputs alone move it by up to ~1e-1 in a few worlds),
so there the check is statistical plus the reference's own acceptance rule: the solver cost must
not exceed the oracle's by more than 2.5 % (solver_test.py:127).
"""

import numpy as np
import pytest
import torch

import mjx_warp_b200 as mjw
from helpers import (assert_close, dev, device_data, generic_state, humanoid, humanoid_state, load,
                     oracle, rel_err, world_rows)

pytestmark = pytest.mark.gpu


def _run(mjm, nworld, seed, fused=True, key=0, ls_parallel=False):
  qpos, qvel, ctrl = humanoid_state(mjm, nworld, seed=seed, key=key)
  m = mjw.put_model(mjm)
  m.opt.ls_parallel = ls_parallel
  d = device_data(mjm, qpos, qvel, ctrl)
  mjw.forward(m, d, fused=fused)
  from oracle import Oracle

  o = Oracle(mjm, nworld, 64, ls_parallel=ls_parallel)
  o.set("qpos", qpos)
  o.set("qvel", qvel)
  o.set("ctrl", ctrl)
  o.run("forward")
  torch.cuda.synchronize()
  return m, d, o


@pytest.mark.parametrize("fused", [1, 0, 2])
def test_newton_converged(fused):
  mjm = humanoid(iterations=10, ls_iterations=20)
  _, d, o = _run(mjm, 128, seed=3, fused=fused)
  e = rel_err(dev(d.qacc), o.get("qacc"))
  assert e.max() < 1e-3 and np.median(e) < 1e-5, (e.max(), np.median(e))
  e = rel_err(dev(d.qfrc_constraint), o.get("qfrc_constraint"))
  assert np.median(e) < 1e-4
  n, idx = world_rows(d, "efc")
  cnt, f = o.rows("efc_force")
  np.testing.assert_array_equal(n, cnt)
  ef = d.efc.force.cpu().numpy()[idx]
  assert np.median(np.abs(ef - f.ravel()) / np.maximum(np.abs(f.ravel()), 1.0)) < 1e-4


def test_keyframes_uneven_rows():
  """test_solve_batch (solver_test.py:134-326): worlds with different row counts in one batch."""
  mjm = humanoid(iterations=10, ls_iterations=20)
  for key in range(3):
    _, d, o = _run(mjm, 24, seed=key, key=key)
    e = rel_err(dev(d.qacc), o.get("qacc"))
    assert e.max() < 1e-3, (key, e.max())
  n, _ = world_rows(d, "efc")
  assert n.max() > n.min() or key == 2


@pytest.mark.parametrize("solver, iterations, ls_iterations, ls_parallel",
                         [(1, 25, 5, False), (2, 2, 4, True)])
def test_cg_and_parallel_linesearch(solver, iterations, ls_iterations, ls_parallel):
  """solver_test.py:70-127: CG and the parallel line search reach the oracle's cost."""
  mjm = humanoid(iterations=iterations, ls_iterations=ls_iterations, solver=solver)
  _, d, o = _run(mjm, 64, seed=4, ls_parallel=ls_parallel)
  cg, co = d.efc.cost.cpu().numpy(), o.scalar("cost")
  assert np.all(cg <= co + 0.025 * np.abs(co) + 1e-3), np.max(cg - co)
  e = rel_err(dev(d.qacc), o.get("qacc"))
  assert np.median(e) < 5e-2


def test_benchmark_setting_statistics():
  """3 Newton iterations (the nworld=8192 benchmark) from the keyframe states with no warmstart:
  most worlds agree to 1e-4 (measured 71 %); the cost is within the reference's 2.5 % acceptance
  in >= 98 % of worlds."""
  mjm = humanoid(iterations=3, ls_iterations=4)
  _, d, o = _run(mjm, 256, seed=5)
  e = rel_err(dev(d.qacc), o.get("qacc"))
  assert np.median(e) < 1e-4
  assert np.mean(e < 1e-4) > 0.66, np.mean(e < 1e-4)
  cg, co = d.efc.cost.cpu().numpy(), o.scalar("cost")
  ok = cg <= co + 0.025 * np.abs(co) + 1e-3
  assert ok.mean() >= 0.98, ok.mean()


@pytest.mark.parametrize("fused", [1, 0])
def test_benchmark_setting_vs_fp32_restatement(fused):
  """The benchmark's 3 Newton / 4 line-search iterations from states in contact (after 10 steps):
  every world whose qacc misses the FP64 restatement by more than 1e-4 is either within 1e-4 of
  the FP32 restatement (the FP32 implementation of the reference's algorithm misses the same
  way) or path-dependent: after 3 iterations the FP64 iterate itself is more than 1e-4 from the
  converged solution there (~30 % of these worlds), so which line-search and active-set path the
  iterations take decides the result, and rounding picks the path (FP32 runs of the
  restatement from inputs one ulp apart each miss in ~11 % of worlds, not the same ones).  In
  the worlds where 3 iterations do converge, the device agrees with FP64 to 1e-4."""
  import oracle as orc

  mjm = humanoid(iterations=3, ls_iterations=4)
  qpos, qvel, ctrl = humanoid_state(mjm, 256, seed=12)
  m = mjw.put_model(mjm)
  d = device_data(mjm, qpos, qvel, ctrl)
  for _ in range(10):
    mjw.step(m, d, fused=fused)
  torch.cuda.synchronize()
  host = {k: getattr(d, k).double().cpu().numpy() for k in ("qpos", "qvel", "ctrl", "qacc_warmstart")}
  refs = orc.qacc_references(mjm, host["qpos"], host["qvel"], host["ctrl"], host["qacc_warmstart"])
  mjw.forward(m, d, fused=fused)
  torch.cuda.synchronize()
  c = orc.classify_qacc(dev(d.qacc), refs)
  assert c["over_tol_unexplained"] == 0, c
  assert c["frac_le_tol_vs_fp64"] >= 0.8, c
  assert c["frac_le_tol_vs_fp64_in_converged_worlds"] >= 0.98, c


def test_tensor_core_hessian():
  """The chosen form with the Newton Hessian assembled on the tensor pipe in split TF32
  (set_tune(hessian_tc=True)) gives the FMA assembly's converged qacc and FP64's."""
  mjm = humanoid(iterations=10, ls_iterations=20)
  qpos, qvel, ctrl = humanoid_state(mjm, 128, seed=3)
  m = mjw.put_model(mjm)
  out = []
  for tc in (False, True):
    d = device_data(mjm, qpos, qvel, ctrl)
    try:
      mjw.set_tune(m, d, hessian_tc=tc)
      mjw.forward(m, d)
      torch.cuda.synchronize()
    finally:
      mjw.set_tune(m, d)
    out.append(dev(d.qacc))
  o = oracle(mjm, qpos, qvel, ctrl, 64)
  o.run("forward")
  e = rel_err(out[1], o.get("qacc"))
  assert e.max() < 1e-3 and np.median(e) < 1e-5, (e.max(), np.median(e))
  assert np.median(rel_err(out[1], out[0])) < 1e-5


def test_solve_standalone_matches_forward():
  """mjw.solve on rows left by forward reproduces the fused solve (index rebuilt from worldid)."""
  mjm = humanoid(iterations=10, ls_iterations=20)
  m, d, _ = _run(mjm, 32, seed=6)
  qacc = d.qacc.clone()
  ws = d.qacc_warmstart.clone()
  d.qacc_warmstart.copy_(torch.as_tensor(np.zeros((32, mjm.nv)), dtype=torch.float32))
  mjw.forward(m, d)  # recompute with zero warmstart
  d.qacc_warmstart.zero_()
  d.qacc.zero_()
  mjw.solve(m, d)
  torch.cuda.synchronize()
  e = rel_err(dev(d.qacc), dev(qacc))
  assert e.max() < 1e-3
  del ws


_MANY_ROWS = """
<mujoco model="footprint">
  <option timestep="0.002" solver="Newton" iterations="30" ls_iterations="30" tolerance="1e-10"/>
  <worldbody>
    <geom type="plane" size="0 0 1"/>
    <body pos="0 0 0.045">
      <freejoint/>
      {spheres}
    </body>
  </worldbody>
</mujoco>
"""


def test_many_rows_past_the_staged_capacity():
  """One body resting on 12 spheres: 48 pyramid rows in one world, more than the solver stages in
  shared memory, so the rows are read from global memory; forces must still match the oracle."""
  spheres = "\n".join(f'<geom type="sphere" size="0.05" pos="{0.1 * np.cos(a):.4f} {0.1 * np.sin(a):.4f} 0"/>'
                      for a in np.linspace(0, 2 * np.pi, 12, endpoint=False))
  mjm = load(_MANY_ROWS.format(spheres=spheres))
  qpos, qvel, ctrl = generic_state(mjm, 16, seed=7, qscale=0.003, vscale=0.01)
  m = mjw.put_model(mjm)
  d = device_data(mjm, qpos, qvel, ctrl)
  mjw.forward(m, d)
  o = oracle(mjm, qpos, qvel, ctrl, 64)
  o.run("forward")
  torch.cuda.synchronize()
  n, idx = world_rows(d, "efc")
  cnt, f = o.rows("efc_force")
  np.testing.assert_array_equal(n, cnt)
  assert n.min() > 32, n
  e = rel_err(dev(d.qacc), o.get("qacc"))
  assert e.max() < 1e-3, e.max()
  ef = d.efc.force.cpu().numpy()[idx]
  np.testing.assert_allclose(ef, f.ravel(), rtol=1e-3, atol=1e-3 * np.abs(f).max())


def test_reused_factor_matches_refactoring():
  """The chosen form keeps the Newton factor across iterations while the active set is unchanged;
  with a converged solve it must agree with the plain form, which refactors H in every iteration
  as the reference does."""
  mjm = humanoid(iterations=15, ls_iterations=20)
  qpos, qvel, ctrl = humanoid_state(mjm, 256, seed=11)
  m = mjw.put_model(mjm)
  out = []
  for form in (0, 1):
    d = device_data(mjm, qpos, qvel, ctrl)
    for _ in range(5):  # into contact, so the active sets change between iterations
      mjw.step(m, d, fused=0)
    mjw.forward(m, d, fused=form)
    torch.cuda.synchronize()
    out.append((dev(d.qacc), d.efc.cost.cpu().numpy()))
  e = rel_err(out[1][0], out[0][0])
  assert np.median(e) < 1e-5 and e.max() < 1e-3, (np.median(e), e.max())
  np.testing.assert_allclose(out[1][1], out[0][1], rtol=1e-4, atol=1e-4)
