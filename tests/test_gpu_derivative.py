"""Finite-difference transition Jacobians and the rollout adjoint on the GPU vs FP64 finite
differences of the oracle (the reference has no derivative API; the scheme is MuJoCo's
mjd_transitionFD).  Models: pendula.xml (free, ball, slide and hinge joints, motors, no contacts)
and the humanoid lifted 1 m above the floor (no contacts within the tested steps)."""

import numpy as np
import pytest
import torch

import mjx_warp_b200 as mjw
from helpers import device_data, generic_state, humanoid, humanoid_state, load, oracle

pytestmark = pytest.mark.gpu


# quaternion helpers (math.py:118-152): rotation about a local axis and the rotation-vector
# difference, for the oracle-side perturbations
def _qmul(u, v):
  return np.array([u[0] * v[0] - u[1] * v[1] - u[2] * v[2] - u[3] * v[3],
                   u[0] * v[1] + u[1] * v[0] + u[2] * v[3] - u[3] * v[2],
                   u[0] * v[2] - u[1] * v[3] + u[2] * v[0] + u[3] * v[1],
                   u[0] * v[3] + u[1] * v[2] - u[2] * v[1] + u[3] * v[0]])


def _qrot(q, axis, ang):
  r = np.concatenate([[np.cos(0.5 * ang)], np.sin(0.5 * ang) * np.asarray(axis, float)])
  out = _qmul(q, r)
  return out / np.linalg.norm(out)


def _qsub(qa, qb):
  dq = _qmul(np.array([qb[0], -qb[1], -qb[2], -qb[3]]), qa)
  if dq[0] < 0:
    dq = -dq
  s = np.linalg.norm(dq[1:])
  ang = 2.0 * np.arctan2(s, dq[0])
  return dq[1:] * (ang / s) if s > 0 else np.zeros(3)


def _tangent_diff(mjm, qa, qb):
  out = np.zeros(mjm.nv)
  for j in range(mjm.njnt):
    t, a, v = mjm.jnt_type[j], mjm.jnt_qposadr[j], mjm.jnt_dofadr[j]
    if t == 0:
      out[v:v + 3] = qa[a:a + 3] - qb[a:a + 3]
      out[v + 3:v + 6] = _qsub(qa[a + 3:a + 7], qb[a + 3:a + 7])
    elif t == 1:
      out[v:v + 3] = _qsub(qa[a:a + 4], qb[a:a + 4])
    else:
      out[v] = qa[a] - qb[a]
  return out


def _perturb(mjm, qpos, qvel, ctrl, col, delta):
  qpos, qvel, ctrl = qpos.copy(), qvel.copy(), ctrl.copy()
  nv = mjm.nv
  if col < nv:
    j = mjm.dof_jntid[col]
    t, a, r = mjm.jnt_type[j], mjm.jnt_qposadr[j], col - mjm.jnt_dofadr[j]
    if t == 0 and r < 3:
      qpos[a + r] += delta
    elif t in (0, 1):
      qa = a + 3 if t == 0 else a
      k = r - 3 if t == 0 else r
      qpos[qa:qa + 4] = _qrot(qpos[qa:qa + 4], np.eye(3)[k], delta)
    else:
      qpos[a] += delta
  elif col < 2 * nv:
    qvel[col - nv] += delta
  else:
    ctrl[col - 2 * nv] += delta
  return qpos, qvel, ctrl


def _oracle_fd(mjm, qpos, qvel, ctrl, eps=1e-6):
  """Centered FP64 finite differences of one oracle step, per world (na = 0 here)."""
  nworld, nv, nu = qpos.shape[0], mjm.nv, mjm.nu
  nx, ncol = 2 * nv, 2 * nv + nu
  A = np.zeros((nworld, nx, nx))
  B = np.zeros((nworld, nx, nu))
  for c in range(ncol):
    nxt = []
    for sgn in (1.0, -1.0):
      st = [_perturb(mjm, qpos[w], qvel[w], ctrl[w], c, sgn * eps) for w in range(nworld)]
      o = oracle(mjm, np.stack([s[0] for s in st]), np.stack([s[1] for s in st]),
                 np.stack([s[2] for s in st]), 64)
      o.run("step")
      nxt.append((o.get("qpos"), o.get("qvel")))
    for w in range(nworld):
      col = np.concatenate([_tangent_diff(mjm, nxt[0][0][w], nxt[1][0][w]),
                            nxt[0][1][w] - nxt[1][1][w]]) / (2 * eps)
      if c < nx:
        A[w, :, c] = col
      else:
        B[w, :, c - nx] = col
  return A, B


def _mid_range(mjm, qpos):
  """Moves every limited slide / hinge joint to the middle of its range (+ the state's offset
  from qpos0), away from the limit switch that finite differences would straddle."""
  qpos = qpos.copy()
  for j in range(mjm.njnt):
    if mjm.jnt_type[j] in (2, 3) and mjm.jnt_limited[j]:
      a = mjm.jnt_qposadr[j]
      lo, hi = mjm.jnt_range[j]
      qpos[:, a] += 0.5 * (lo + hi) - mjm.qpos0[a]
  return qpos


def _lifted_humanoid(mjm, nworld, seed):
  qpos, qvel, ctrl = humanoid_state(mjm, nworld, seed=seed)
  qpos[:, 2] += 1.0
  return qpos, qvel, ctrl


@pytest.mark.parametrize("name", ["pendula.xml", "humanoid"])
def test_transition_jacobians_vs_fp64_fd(name):
  if name == "humanoid":
    mjm = humanoid()
    qpos, qvel, ctrl = _lifted_humanoid(mjm, 3, seed=2)
  else:
    mjm = load(name)
    qpos, qvel, ctrl = generic_state(mjm, 3, seed=2, qscale=0.05, vscale=0.05)
    qpos = _mid_range(mjm, qpos)
  m = mjw.put_model(mjm)
  d = device_data(mjm, qpos, qvel, ctrl)
  fd = mjw.derivative.TransitionFD(mjm, m, 3, eps=1e-3, centered=True)
  A, B = fd(d)
  torch.cuda.synchronize()
  assert np.allclose(d.qpos.cpu().numpy(), qpos.astype(np.float32))  # base Data untouched
  Ar, Br = _oracle_fd(mjm, qpos, qvel, ctrl)
  A, B = A.cpu().numpy().astype(float), B.cpu().numpy().astype(float)
  for w in range(3):
    ea = np.linalg.norm(A[w] - Ar[w]) / np.linalg.norm(Ar[w])
    eb = np.linalg.norm(B[w] - Br[w]) / max(np.linalg.norm(Br[w]), 1e-12)
    assert ea < 2e-3 and eb < 2e-3, (w, ea, eb)


def test_forward_and_centered_differences_agree():
  mjm = load("pendula.xml")
  qpos, qvel, ctrl = generic_state(mjm, 4, seed=3, qscale=0.05, vscale=0.05)
  qpos = _mid_range(mjm, qpos)
  m = mjw.put_model(mjm)
  d = device_data(mjm, qpos, qvel, ctrl)
  Ac, Bc = (t.clone() for t in mjw.derivative.TransitionFD(mjm, m, 4, eps=1e-3, centered=True)(d))
  Af, Bf = mjw.derivative.TransitionFD(mjm, m, 4, eps=1e-3, centered=False)(d)
  assert torch.linalg.norm(Af - Ac) / torch.linalg.norm(Ac) < 2e-2
  assert torch.linalg.norm(Bf - Bc) / torch.linalg.norm(Bc) < 2e-2


@pytest.mark.parametrize("analytic", ["full", "qvel_ctrl", "ctrl", "none"])
def test_rollout_gradient_vs_fp64_central_fd(analytic):
  """d/d(ctrl, qvel0, qpos0) of ||root_pos_T - target||^2 + 1e-3 ||ctrl||^2 over an 8-step
  rollout (checkpoints every 4 steps) vs central FP64 differences of the oracle's loss, with the
  step's adjoint fully analytic, only its velocity and control columns analytic, only the
  controls analytic, or all by differences."""
  mjm = humanoid()
  nworld, T = 2, 8
  qpos, qvel, _ = _lifted_humanoid(mjm, nworld, seed=4)
  rng = np.random.default_rng(5)
  ctrl = rng.uniform(-0.4, 0.4, (T, nworld, mjm.nu))
  target = np.array([0.1, -0.1, 2.0])
  m = mjw.put_model(mjm)
  roll = mjw.derivative.Rollout(mjm, m, nworld, checkpoint=4, analytic=analytic)
  q0 = torch.tensor(qpos, dtype=torch.float32, device="cuda", requires_grad=True)
  v0 = torch.tensor(qvel, dtype=torch.float32, device="cuda", requires_grad=True)
  u = torch.tensor(ctrl, dtype=torch.float32, device="cuda", requires_grad=True)
  qT, _ = roll(q0, v0, u)
  tgt = torch.tensor(target, dtype=torch.float32, device="cuda")
  loss = ((qT[:, :3] - tgt) ** 2).sum() + 1e-3 * (u ** 2).sum()
  loss.backward()

  def loss64(qp, qv, cu):
    o = oracle(mjm, qp, qv, cu[0], 64)
    for t in range(T):
      o.set("ctrl", cu[t])
      o.run("step")
    return float(((o.get("qpos")[:, :3] - target) ** 2).sum() + 1e-3 * (cu ** 2).sum())

  h = 1e-5
  checks = []
  for (t, w, a) in [(0, 0, 3), (3, 1, 10), (7, 0, 20), (5, 1, 0)]:
    cp, cm = ctrl.copy(), ctrl.copy()
    cp[t, w, a] += h
    cm[t, w, a] -= h
    checks.append((u.grad[t, w, a].item(), (loss64(qpos, qvel, cp) - loss64(qpos, qvel, cm)) / (2 * h)))
  for (w, i) in [(0, 2), (1, 8), (0, 20)]:
    vp, vm = qvel.copy(), qvel.copy()
    vp[w, i] += h
    vm[w, i] -= h
    checks.append((v0.grad[w, i].item(), (loss64(qpos, vp, ctrl) - loss64(qpos, vm, ctrl)) / (2 * h)))
  for (w, i) in [(1, 0), (0, 2), (1, 10)]:  # root x, root z, a hinge
    pp, pm = qpos.copy(), qpos.copy()
    pp[w, i] += h
    pm[w, i] -= h
    checks.append((q0.grad[w, i].item(), (loss64(pp, qvel, ctrl) - loss64(pm, qvel, ctrl)) / (2 * h)))
  scale = max(abs(c[1]) for c in checks)
  for g, f in checks:
    assert abs(g - f) <= 1e-2 * abs(f) + 2e-3 * scale, checks


@pytest.mark.parametrize("case", ["lifted", "standing"])
def test_ctrl_vjp_matches_differences(case):
  """ctrl_vjp after a step equals B^T lam from centered differences of the same step, in the air
  and standing on the floor (contacts, the solve run to convergence)."""
  mjm = humanoid(iterations=30, ls_iterations=30)
  mjm.opt.tolerance = 1e-10
  nworld = 16
  if case == "lifted":
    qpos, qvel, ctrl = _lifted_humanoid(mjm, nworld, seed=6)
  else:
    qpos, qvel, ctrl = humanoid_state(mjm, nworld, seed=6)
  m = mjw.put_model(mjm)
  d = device_data(mjm, qpos, qvel, ctrl)
  if case == "standing":  # settle into contact with a warmstart
    for _ in range(10):
      mjw.step(m, d)
  fd = mjw.derivative.TransitionFD(mjm, m, nworld, eps=1e-3, centered=True)
  _, B = fd(d)
  B = B.clone()
  lam = torch.as_tensor(np.random.default_rng(7).normal(size=(nworld, 2 * mjm.nv)),
                        dtype=torch.float32, device="cuda")
  ref = torch.einsum("wij,wi->wj", B, lam)
  mjw.step(m, d)
  if case == "standing":
    assert int(d.nefc.cpu()[0]) > 0
  got = mjw.derivative.ctrl_vjp(m, d, lam)
  torch.cuda.synchronize()
  err = torch.linalg.norm(got - ref, dim=1) / torch.linalg.norm(ref, dim=1)
  assert float(torch.median(err)) < 1e-3 and float(err.max()) < (5e-3 if case == "lifted" else 5e-2), err


# ball, slide and hinge joints in a chain, a free sphere, dampers and motors; no contacts within
# the tested steps (nv = 11)
_JOINTS_XML = """
<mujoco>
  <option timestep="0.004" iterations="30" ls_iterations="30"/>
  <worldbody>
    <geom type="plane" size="2 2 0.1"/>
    <body pos="0 0 1.2">
      <joint name="ball" type="ball" damping="0.1"/>
      <geom type="capsule" fromto="0 0 0 0.05 0 -0.3" size="0.03"/>
      <body pos="0.05 0 -0.3">
        <joint name="slide" type="slide" axis="0 0.3 1" damping="0.2"/>
        <geom type="sphere" size="0.05"/>
        <body pos="0 0 -0.1">
          <joint name="hinge" type="hinge" axis="0 1 0.2" damping="0.05"/>
          <geom type="capsule" fromto="0 0 0 0.2 0.02 0" size="0.02"/>
        </body>
      </body>
    </body>
    <body pos="1 0 0.8">
      <freejoint/>
      <geom type="sphere" size="0.1"/>
    </body>
  </worldbody>
  <actuator>
    <motor joint="slide" gear="2"/>
    <motor joint="hinge" gear="0.5"/>
  </actuator>
</mujoco>
"""


def _vjp_case(case, nworld):
  """(mjm, qpos, qvel, ctrl, settle steps) for the analytic VJP tests, the solve converged."""
  if case in ("lifted", "standing"):
    mjm = humanoid(iterations=30, ls_iterations=30)
    fn = _lifted_humanoid if case == "lifted" else humanoid_state
    qpos, qvel, ctrl = fn(mjm, nworld, seed=6)
    settle = 10 if case == "standing" else 0
  elif case == "humanoid_spheres":  # nv = 123: the Hessian outside the warp tile
    from test_gpu_configs import humanoid_spheres_state
    mjm = load("humanoid_spheres.xml", integrator=3, timestep=0.005, iterations=30,
               ls_iterations=30, jacobian=0)
    qpos, qvel, ctrl, _ = humanoid_spheres_state(mjm, load("humanoid.xml"), nworld, seed=6)
    settle = 10
  else:
    mjm = load(_JOINTS_XML if case == "joints" else case)
    mjm.opt.iterations, mjm.opt.ls_iterations = 30, 30
    qpos, qvel, ctrl = generic_state(mjm, nworld, seed=6, qscale=0.05, vscale=0.5)
    qpos = _mid_range(mjm, qpos)
    settle = 5
  mjm.opt.tolerance = 1e-10
  return mjm, qpos, qvel, ctrl, settle


@pytest.mark.parametrize("case", ["lifted", "standing", "sphere_chain.xml", "joints",
                                  "humanoid_spheres"])
def test_step_vjp_matches_differences(case):
  """step_vjp after a step equals (A_q^T lam, A_v^T lam, B^T lam) from central FP64 differences
  of the oracle's step at the same state (A_q, A_v the qpos-tangent and velocity columns of A):
  the humanoid in the air and standing on the floor (implicitfast, contacts and limits), the
  sphere + chain (Euler with eulerdamp, damping, a resting contact), a ball / slide / hinge chain
  with a free body.  qvel_ctrl_vjp and ctrl_vjp give the same velocity and control gradients."""
  nworld = 4 if case == "humanoid_spheres" else 8
  mjm, qpos, qvel, ctrl, settle = _vjp_case(case, nworld)
  m = mjw.put_model(mjm)
  assert mjw.derivative.qpos_vjp_supported(m)
  d = device_data(mjm, qpos, qvel, ctrl)
  for _ in range(settle):
    mjw.step(m, d)
  nv = mjm.nv
  q64, v64 = (t.cpu().numpy().astype(np.float64) for t in (d.qpos, d.qvel))
  A, B = _oracle_fd(mjm, q64, v64, ctrl.astype(np.float32).astype(np.float64))
  lam_np = np.random.default_rng(7).normal(size=(nworld, 2 * nv))
  ref_q = np.einsum("wij,wi->wj", A[:, :, :nv], lam_np)
  ref_v = np.einsum("wij,wi->wj", A[:, :, nv:], lam_np)
  ref_u = np.einsum("wij,wi->wj", B, lam_np)
  lam = torch.as_tensor(lam_np, dtype=torch.float32, device="cuda")
  # the same products from the GPU's own transition Jacobians (MuJoCo's mjd_transitionFD scheme,
  # FP32, centered, eps 1e-3) at the same state
  Af, Bf = mjw.derivative.TransitionFD(mjm, m, nworld, eps=1e-3, centered=True)(d)
  fd_x = torch.einsum("wij,wi->wj", Af, lam).cpu().numpy()
  fd_u = torch.einsum("wij,wi->wj", Bf, lam).cpu().numpy()
  qvel_prev = d.qvel.clone()
  mjw.step(m, d)
  gq, gv, gu = mjw.derivative.step_vjp(m, d, qvel_prev, lam)
  gv2, gu2 = mjw.derivative.qvel_ctrl_vjp(m, d, qvel_prev, lam)
  gu3 = mjw.derivative.ctrl_vjp(m, d, lam)
  torch.cuda.synchronize()
  if case in ("standing", "humanoid_spheres"):
    assert int(d.nefc.cpu()[0]) > 0
  assert torch.equal(gu, gu2) and torch.equal(gu, gu3) and torch.equal(gv, gv2)
  gq, gv, gu = gq.cpu().numpy(), gv.cpu().numpy(), gu.cpu().numpy()
  rel = lambda g, r: np.linalg.norm(g - r, axis=1) / np.linalg.norm(r, axis=1)
  eq, ev, eu = rel(gq, ref_q), rel(gv, ref_v), rel(gu, ref_u)
  print(case, "qpos", np.median(eq), eq.max(), "qvel", np.median(ev), ev.max(), "ctrl",
        np.median(eu), eu.max())
  # velocity / control measured on a B200: max 1.5e-6 (lifted), 3.5e-5 (standing), 2.5e-5
  # (sphere chain), 1.1e-6
  assert ev.max() < 5e-4 and eu.max() < 5e-4, (ev, eu)
  assert eq.max() < 1e-3, eq
  # against the FP32 finite differences: their own error (rounding at eps 1e-3, and a velocity
  # perturbation moving aref by b eps ~ 0.1 can flip a limit row) bounds the agreement.  With
  # contacts, a 1e-3 perturbation of qpos or qvel switches contacts and rows, and the state
  # columns at eps 1e-3 are secants across the switches (measured: the FP64 differences at eps 1e-3
  # differ from those at 1e-6 by 2-39x in 3 of 4 standing worlds, while the GPU's agree with the
  # FP64 ones at 1e-3 to 5e-3); there only the control columns are compared.
  fx = rel(np.concatenate([gq, gv], 1), fd_x)
  fu = rel(gu, fd_u)
  print(case, "vs transitionFD (FP32)", np.median(fx), fx.max(), np.median(fu), fu.max())
  assert np.median(fu) < 2e-3, fu
  if case not in ("standing", "humanoid_spheres"):
    assert np.median(fx) < 2e-3, fx


def test_rollout_gradient_standing_vs_fp64_central_fd():
  """The analytic rollout gradient with the humanoid standing on the floor (contacts and limits
  in every step, the solve converged) vs central FP64 differences of the oracle's loss."""
  mjm = humanoid(iterations=30, ls_iterations=30)
  mjm.opt.tolerance = 1e-10
  nworld, T = 2, 8
  qpos, qvel, _ = humanoid_state(mjm, nworld, seed=4)
  rng = np.random.default_rng(5)
  ctrl = rng.uniform(-0.4, 0.4, (T, nworld, mjm.nu))
  target = np.array([0.1, -0.1, 1.0])
  m = mjw.put_model(mjm)
  roll = mjw.derivative.Rollout(mjm, m, nworld, checkpoint=4, analytic="full")
  q0 = torch.tensor(qpos, dtype=torch.float32, device="cuda", requires_grad=True)
  v0 = torch.tensor(qvel, dtype=torch.float32, device="cuda", requires_grad=True)
  u = torch.tensor(ctrl, dtype=torch.float32, device="cuda", requires_grad=True)
  qT, _ = roll(q0, v0, u)
  tgt = torch.tensor(target, dtype=torch.float32, device="cuda")
  loss = ((qT[:, :3] - tgt) ** 2).sum() + 1e-3 * (u ** 2).sum()
  loss.backward()

  def loss64(qp, qv, cu):
    o = oracle(mjm, qp, qv, cu[0], 64)
    for t in range(T):
      o.set("ctrl", cu[t])
      o.run("step")
    return float(((o.get("qpos")[:, :3] - target) ** 2).sum() + 1e-3 * (cu ** 2).sum())

  h = 1e-6
  checks = []
  for (t, w, a) in [(0, 0, 3), (3, 1, 10), (7, 0, 20), (5, 1, 0), (1, 0, 15)]:
    cp, cm = ctrl.copy(), ctrl.copy()
    cp[t, w, a] += h
    cm[t, w, a] -= h
    checks.append((u.grad[t, w, a].item(), (loss64(qpos, qvel, cp) - loss64(qpos, qvel, cm)) / (2 * h)))
  for (w, i) in [(0, 2), (1, 8), (0, 20)]:
    vp, vm = qvel.copy(), qvel.copy()
    vp[w, i] += h
    vm[w, i] -= h
    checks.append((v0.grad[w, i].item(), (loss64(qpos, vp, ctrl) - loss64(qpos, vm, ctrl)) / (2 * h)))
  for (w, i) in [(1, 0), (0, 2), (1, 10), (0, 12)]:  # root x, root z, hinges
    pp, pm = qpos.copy(), qpos.copy()
    pp[w, i] += h
    pm[w, i] -= h
    checks.append((q0.grad[w, i].item(), (loss64(pp, qvel, ctrl) - loss64(pm, qvel, ctrl)) / (2 * h)))
  print("standing rollout", checks)
  scale = max(abs(c[1]) for c in checks)
  for g, f in checks:
    assert abs(g - f) <= 1e-2 * abs(f) + 2e-3 * scale, checks


def test_rollout_backward_after_another_forward():
  """The analytic rollout keeps its last segment's steps from the forward pass; a second forward
  pass through the same Rollout before the first one's backward must not leak into it: the
  gradients equal those of a lone forward + backward."""
  mjm = humanoid()
  nworld, T = 4, 6
  qpos, qvel, _ = humanoid_state(mjm, nworld, seed=12)
  rng = np.random.default_rng(13)
  c1 = rng.uniform(-0.4, 0.4, (T, nworld, mjm.nu))
  c2 = rng.uniform(-0.4, 0.4, (T, nworld, mjm.nu))
  m = mjw.put_model(mjm)
  roll = mjw.derivative.Rollout(mjm, m, nworld, checkpoint=4, analytic="full")
  q0 = torch.tensor(qpos, dtype=torch.float32, device="cuda")
  v0 = torch.tensor(qvel, dtype=torch.float32, device="cuda")

  def grads(interleave):
    u = torch.tensor(c1, dtype=torch.float32, device="cuda", requires_grad=True)
    q = q0.clone().requires_grad_(True)
    qT, vT = roll(q, v0, u)
    if interleave:  # another rollout through the same workspace before the backward
      roll(q0, v0, torch.tensor(c2, dtype=torch.float32, device="cuda"))
    ((qT[:, :3] ** 2).sum() + (vT ** 2).sum()).backward()
    return u.grad.clone(), q.grad.clone()

  ua, qa = grads(False)
  ub, qb = grads(True)
  assert torch.isfinite(ua).all() and ua.abs().max() > 0
  torch.testing.assert_close(ub, ua, rtol=1e-5, atol=1e-7)
  torch.testing.assert_close(qb, qa, rtol=1e-5, atol=1e-7)


def test_step_vjp_without_constraint_capacity():
  """nv = 123 (the Hessian outside the warp tile): a step without constraint capacity
  (njmax = 0, the solver does not run) and a step with constraints disabled (the solver runs on
  no rows) have the same dynamics, so the adjoint -- which reuses the solver's factor only when
  the solver ran -- must agree between them."""
  from test_gpu_configs import humanoid_spheres_state
  nworld = 8
  out = []
  for case in ("njmax0", "disabled"):
    mjm = load("humanoid_spheres.xml", integrator=3, timestep=0.005, iterations=10,
               ls_iterations=10, jacobian=0)
    if case == "disabled":
      mjm.opt.disableflags |= 1  # DSBL_CONSTRAINT
    qpos, qvel, ctrl, _ = humanoid_spheres_state(mjm, load("humanoid.xml"), nworld, seed=9)
    m = mjw.put_model(mjm)
    d = mjw.make_data(mjm, nworld, nconmax=96 * nworld,
                      njmax=0 if case == "njmax0" else 256 * nworld)
    d.qpos.copy_(torch.as_tensor(qpos, dtype=torch.float32))
    d.qvel.copy_(torch.as_tensor(qvel, dtype=torch.float32))
    d.ctrl.copy_(torch.as_tensor(ctrl, dtype=torch.float32))
    lam = torch.as_tensor(np.random.default_rng(10).normal(size=(nworld, 2 * mjm.nv)),
                          dtype=torch.float32, device="cuda")
    qvel_prev = d.qvel.clone()
    mjw.step(m, d)
    out.append([g.clone() for g in mjw.derivative.step_vjp(m, d, qvel_prev, lam)])
  torch.cuda.synchronize()
  for a, b in zip(*out):
    assert torch.isfinite(a).all()
    torch.testing.assert_close(a, b, rtol=1e-4, atol=1e-5)


def test_rollout_overlapped_backward_matches_serial():
  """The analytic backward recomputing the next segment on a side stream (two rings of Data)
  gives the same gradients as the serial one, over three segments."""
  mjm = humanoid()
  nworld, T = 4, 12
  qpos, qvel, _ = humanoid_state(mjm, nworld, seed=14)
  ctrl = np.random.default_rng(15).uniform(-0.4, 0.4, (T, nworld, mjm.nu))
  m = mjw.put_model(mjm)
  grads = []
  for overlap in (False, True):
    roll = mjw.derivative.Rollout(mjm, m, nworld, checkpoint=4, analytic="full", overlap=overlap)
    assert bool(roll.seg2) == overlap
    u = torch.tensor(ctrl, dtype=torch.float32, device="cuda", requires_grad=True)
    q = torch.tensor(qpos, dtype=torch.float32, device="cuda", requires_grad=True)
    v = torch.tensor(qvel, dtype=torch.float32, device="cuda", requires_grad=True)
    qT, vT = roll(q, v, u)
    ((qT[:, :3] ** 2).sum() + (vT ** 2).sum()).backward()
    grads.append((u.grad.clone(), q.grad.clone(), v.grad.clone()))
  for a, b in zip(*grads):
    assert torch.isfinite(a).all()
    torch.testing.assert_close(b, a, rtol=1e-5, atol=1e-7)
