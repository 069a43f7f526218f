"""Derivatives of the batched step: finite-difference transition Jacobians on the GPU and a
rollout adjoint behind torch.autograd.

The reference (mujoco_warp 3.2.7) has no derivative API.  ``TransitionFD`` follows MuJoCo's
mjd_transitionFD scheme for a whole batch at once: every world's state is copied into
1 + ncol (forward differences) or 1 + 2 ncol (centered) slots of a second Data, one column per
slot is perturbed (``mjb_fd_perturb``), the slots advance by one step in a single launch
sequence, and the differences of their next states give, per world,

  A = dx'/dx  (nx x nx),  B = dx'/du  (nx x nu),  x = (qpos tangent, qvel, act), u = ctrl,

with nx = 2 nv + na and positions in the tangent space (free and ball joints rotate about local
axes, as mj_integratePos / mj_differentiatePos do).  ``rollout`` runs T steps forward, keeping
checkpoints every ``checkpoint`` steps, and its backward pass recomputes each segment's states
from its checkpoint and applies lam <- A^T lam, dL/du_t = B^T lam (``mjb_transition_vjp``) from
the last step to the first.  qacc_warmstart is part of each step's saved state but is not
differentiated (it is held fixed in every perturbed slot, as mjd_transitionFD does).

The velocity and control parts can instead be taken analytically (``qvel_ctrl_vjp``,
``mjb_qvel_ctrl_vjp``; ``ctrl_vjp`` for the controls alone): at the Newton solution the step's
velocity responds to qfrc_smooth and to the constraint reference through Mt^-1 M H^-1 (Mt the
integrator's matrix, H the solver's Hessian at its final active set), so both products need one
assembly and factorisation of H, two solves, a product and a reverse sweep of the bias-force
recursion per world; ``Rollout`` does this by default where it applies and differences only the
nv qpos columns.

The qpos columns are finite-difference derivatives, not an analytic adjoint: their cost is ncol (or
2 ncol) extra world-steps per world-step, and across a contact or active-set switch they
describe the secant of the switch.  They need a step that is (piecewise) smooth in its inputs:
a Newton solve stopped after 1-3 iterations returns an iterate that jumps when the active set
seen by an early iteration changes, and differences across those jumps make products of
transition Jacobians explode; run the solver to convergence (e.g. 10 iterations) when
differentiating.
"""

from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np
import torch

from . import _abi
from ._api import step
from .io import make_data
from .types import Data, Model

JNT_FREE, JNT_BALL = 0, 1


def _sizes(m: Model) -> Tuple[int, int]:
  nx = 2 * m.nv + m.na
  return nx, nx + m.nu


class TransitionFD:
  """Workspace for the transition Jacobians of `nworld` worlds of model `mjm` / `m`.

  Allocates a Data of nworld * K worlds (K = 1 + ncol, or 1 + 2 ncol when centered) once, with
  per-world pair / contact / constraint capacities `nconmax` / `njmax` (defaults: 64 and 128
  per world), and the output tensors A (nworld, nx, nx) and B (nworld, nx, nu).  eps is the
  perturbation size; in FP32 a value near 1e-3 balances truncation against rounding.
  """

  def __init__(self, mjm, m: Model, nworld: int, eps: float = 1e-3, centered: bool = True,
               nconmax: int = 64, njmax: int = 128, fused=True, state_only: bool = False,
               qpos_only: bool = False):
    self.m, self.nworld, self.eps, self.centered, self.fused = m, nworld, float(eps), centered, fused
    self.state_only, self.qpos_only = state_only, qpos_only
    self.nx, self.ncol = _sizes(m)
    if qpos_only:  # velocity and control columns are left to qvel_ctrl_vjp (A's other columns stay 0)
      self.ncol = m.nv
    elif state_only:  # the control columns are left to ctrl_vjp
      self.ncol = self.nx
    self.flags = (1 if centered else 0) | (2 if state_only else 0) | (4 if qpos_only else 0)
    self.K = 1 + self.ncol * (2 if centered else 1)
    n = nworld * self.K
    self.pert = make_data(mjm, n, nconmax=nconmax * n, njmax=njmax * n)
    dev = self.pert.qpos.device
    self.A = torch.zeros((nworld, self.nx, self.nx), dtype=torch.float32, device=dev)
    self.B = torch.zeros((nworld, self.nx, m.nu), dtype=torch.float32, device=dev)

  def __call__(self, d: Data) -> Tuple[torch.Tensor, torch.Tensor]:
    """Jacobians at d's current state and controls (d itself is not modified)."""
    if d.nworld != self.nworld:
      raise ValueError(f"workspace is for {self.nworld} worlds, Data has {d.nworld}")
    L = _abi.lib()
    mv = _abi.model_view(self.m)
    rc = L.mjb_fd_perturb(ctypes.byref(mv), ctypes.byref(_abi.data_view(d)),
                          ctypes.byref(_abi.data_view(self.pert)), self.eps, self.flags,
                          _abi.stream())
    _abi.check(rc, "fd_perturb")
    step(self.m, self.pert, fused=self.fused)
    rc = L.mjb_fd_jacobian(ctypes.byref(mv), ctypes.byref(_abi.data_view(self.pert)), self.nworld,
                           self.eps, self.flags, _abi._ptr(self.A), _abi._ptr(self.B),
                           _abi.stream())
    _abi.check(rc, "fd_jacobian")
    return self.A, self.B


def transition_vjp(m: Model, A: torch.Tensor, B: Optional[torch.Tensor], lam: torch.Tensor
                   ) -> Tuple[torch.Tensor, Optional[torch.Tensor]]:
  """(A^T lam, B^T lam) per world, on the device."""
  nworld, nx = lam.shape
  out = torch.empty_like(lam)
  gu = torch.empty((nworld, m.nu), dtype=lam.dtype, device=lam.device) if B is not None else None
  rc = _abi.lib().mjb_transition_vjp(ctypes.byref(_abi.model_view(m)), nworld, _abi._ptr(A),
                                     _abi._ptr(B) if B is not None else None,
                                     _abi._ptr(lam.contiguous()), _abi._ptr(out),
                                     _abi._ptr(gu) if gu is not None else None, _abi.stream())
  _abi.check(rc, "transition_vjp")
  return out, gu


def ctrl_vjp_supported(m: Model) -> bool:
  """Whether ctrl_vjp applies to m: dense mass matrix, no activations, and for
  implicitfast no velocity-dependent actuator gains or biases."""
  act_on = not (int(m.opt.disableflags) & (1 << 10)) and bool(m.actuator_affine_bias_gain)
  return (not m.opt.is_sparse and m.na == 0
          and not (int(m.opt.integrator) != 0 and act_on))


def ctrl_vjp(m: Model, d: Data, lam: torch.Tensor) -> torch.Tensor:
  """(d x' / d ctrl)^T lam per world, by implicit differentiation at the solver's final active set
  (mjb_ctrl_vjp): d must hold the step's results (call right after step); lam is the adjoint of
  the next state, (nworld, 2 nv) in (qpos tangent, qvel) order."""
  gu = torch.empty((d.nworld, m.nu), dtype=torch.float32, device=lam.device)
  rc = _abi.lib().mjb_ctrl_vjp(ctypes.byref(_abi.model_view(m)), ctypes.byref(_abi.data_view(d)),
                               _abi._ptr(lam.contiguous()), _abi._ptr(gu), _abi.stream())
  _abi.check(rc, "ctrl_vjp")
  return gu


def qpos_vjp_supported(m: Model) -> bool:
  """Whether step_vjp can give the qpos gradient for m: ctrl_vjp_supported, ball joints alone on
  their body, no stiffness on free / ball joints, actuators on hinge / slide joints, planes on
  bodies welded to the world (xfrc_applied is taken to be zero)."""
  if not ctrl_vjp_supported(m):
    return False
  cache = m.__dict__.get("_qpos_vjp_ok")
  if cache is None:
    jt = m.jnt_type.cpu().numpy()
    jb = m.jnt_bodyid.cpu().numpy()
    nj = m.body_jntnum.cpu().numpy()
    k = m.jnt_stiffness.cpu().numpy()
    ok = all(nj[jb[j]] == 1 for j in range(len(jt)) if jt[j] == JNT_BALL)
    ok &= not any(k[j] != 0 for j in range(len(jt)) if jt[j] in (JNT_FREE, JNT_BALL))
    if m.nu:
      tt = m.actuator_trntype.cpu().numpy()
      tid = m.actuator_trnid.cpu().numpy().reshape(m.nu, -1)[:, 0]
      ok &= bool(np.all(tt <= 1)) and all(jt[tid[a]] in (2, 3) for a in range(m.nu))
    gt = m.geom_type.cpu().numpy()
    gb = m.geom_bodyid.cpu().numpy()
    wb = m.body_weldid.cpu().numpy()
    ok &= all(wb[gb[g]] == 0 for g in range(len(gt)) if gt[g] == 0)
    cache = bool(ok)
    object.__setattr__(m, "_qpos_vjp_ok", cache)
  return cache


def step_vjp(m: Model, d: Data, qvel_prev: torch.Tensor, lam: torch.Tensor, qpos: bool = True,
             qvel: bool = True, ctrl: bool = True):
  """Adjoint of one step at the solver's final active set (mjb_step_vjp): for lam (nworld, 2 nv),
  the adjoint of the next state in (qpos tangent, qvel) order, returns (grad_qpos, grad_qvel,
  grad_ctrl) per world, each None unless requested; grad_qpos is in the qpos tangent space.  d
  holds the step's results (call right after step), qvel_prev (nworld, nv) the velocities the
  step started from."""
  if qpos and not qpos_vjp_supported(m):
    raise NotImplementedError("step_vjp: the qpos adjoint does not cover this model")
  dev = lam.device
  gq = torch.empty((d.nworld, m.nv), dtype=torch.float32, device=dev) if qpos else None
  gv = torch.empty((d.nworld, m.nv), dtype=torch.float32, device=dev) if qvel else None
  gu = torch.empty((d.nworld, m.nu), dtype=torch.float32, device=dev) if ctrl and m.nu else None
  P = lambda t: _abi._ptr(t) if t is not None else None
  rc = _abi.lib().mjb_step_vjp(ctypes.byref(_abi.model_view(m)), ctypes.byref(_abi.data_view(d)),
                               _abi._ptr(qvel_prev.contiguous()), _abi._ptr(lam.contiguous()),
                               P(gq), P(gv), P(gu), _abi.stream())
  _abi.check(rc, "step_vjp")
  return gq, gv, gu


def qvel_ctrl_vjp(m: Model, d: Data, qvel_prev: torch.Tensor, lam: torch.Tensor
                  ) -> Tuple[torch.Tensor, torch.Tensor]:
  """((d x' / d qvel)^T lam, (d x' / d ctrl)^T lam) per world (step_vjp without the qpos part)."""
  _, gv, gu = step_vjp(m, d, qvel_prev, lam, qpos=False)
  return gv, gu


def _quat_joints(m: Model):
  """(qpos address of each free / ball joint's quaternion, its first rotational dof)."""
  cache = m.__dict__.get("_quat_joint_cache")
  if cache is None:
    t = m.jnt_type.cpu().numpy()
    qa = m.jnt_qposadr.cpu().numpy()
    da = m.jnt_dofadr.cpu().numpy()
    adr, dof = [], []
    for j in range(t.shape[0]):
      if t[j] == JNT_FREE:
        adr.append(qa[j] + 3)
        dof.append(da[j] + 3)
      elif t[j] == JNT_BALL:
        adr.append(qa[j])
        dof.append(da[j])
    dev = m.jnt_type.device
    cache = (torch.as_tensor(adr, dtype=torch.long, device=dev),
             torch.as_tensor(dof, dtype=torch.long, device=dev))
    object.__setattr__(m, "_quat_joint_cache", cache)
  return cache


def _qpos_dof_map(m: Model) -> torch.Tensor:
  """For every non-quaternion qpos coordinate its dof (qpos and dof coordinates coincide there);
  -1 for quaternion coordinates."""
  cache = m.__dict__.get("_qpos_dof_cache")
  if cache is None:
    t = m.jnt_type.cpu().numpy()
    qa = m.jnt_qposadr.cpu().numpy()
    da = m.jnt_dofadr.cpu().numpy()
    mp = -np.ones(m.nq, dtype=np.int64)
    for j in range(t.shape[0]):
      if t[j] == JNT_FREE:
        mp[qa[j]:qa[j] + 3] = np.arange(da[j], da[j] + 3)
      elif t[j] != JNT_BALL:
        mp[qa[j]] = da[j]
    cache = torch.as_tensor(mp, device=m.jnt_type.device)
    object.__setattr__(m, "_qpos_dof_cache", cache)
  return cache


def _quat_basis(q: torch.Tensor) -> torch.Tensor:
  """q (..., 4) -> (..., 3, 4): q (x) (0, e_k) for k = x, y, z, the tangent directions at q."""
  w, x, y, z = q.unbind(-1)
  return torch.stack([torch.stack([-x, w, z, -y], -1),
                      torch.stack([-y, -z, w, x], -1),
                      torch.stack([-z, y, -x, w], -1)], -2)


def qpos_grad_to_tangent(m: Model, qpos: torch.Tensor, g: torch.Tensor) -> torch.Tensor:
  """dL/d(qpos coordinates) (nworld, nq) -> dL/d(tangent) (nworld, nv) at qpos: a quaternion's
  rotation delta about local axis k moves it by 0.5 q (x) (0, e_k)."""
  out = torch.zeros((g.shape[0], m.nv), dtype=g.dtype, device=g.device)
  mp = _qpos_dof_map(m)
  lin = mp >= 0
  out[:, mp[lin]] = g[:, lin]
  adr, dof = _quat_joints(m)
  for a, k in zip(adr.tolist(), dof.tolist()):
    basis = _quat_basis(qpos[:, a:a + 4])  # (nworld, 3, 4)
    out[:, k:k + 3] = 0.5 * torch.einsum("wkc,wc->wk", basis, g[:, a:a + 4])
  return out


def tangent_grad_to_qpos(m: Model, qpos: torch.Tensor, lam: torch.Tensor) -> torch.Tensor:
  """dL/d(tangent) (nworld, nv) -> dL/d(qpos coordinates) (nworld, nq) at unit quaternions: the
  tangent delta of a coordinate change dq is 2 vec(q* (x) dq), whose rows are q (x) (0, e_k)."""
  out = torch.zeros((lam.shape[0], m.nq), dtype=lam.dtype, device=lam.device)
  mp = _qpos_dof_map(m)
  lin = mp >= 0
  out[:, lin] = lam[:, mp[lin]]
  adr, dof = _quat_joints(m)
  for a, k in zip(adr.tolist(), dof.tolist()):
    basis = _quat_basis(qpos[:, a:a + 4])
    out[:, a:a + 4] = 2.0 * torch.einsum("wkc,wk->wc", basis, lam[:, k:k + 3])
  return out


_STATE = ("qpos", "qvel", "act", "qacc_warmstart")
# Data fields that a step writes before it reads them and that step_vjp does not read: the
# Data objects of a segment share one copy of each
_RING_SHARED = ("qLD", "qLDiagInv", "qM_integration", "qfrc_integration", "collision_pair",
                "collision_worldid", "sap_geom_sort", "sap_projection_lower", "sap_projection_upper",
                "sap_sort_index", "sap_range", "sap_cumulative_sum")
_RING_SHARED_EFC = ("quad", "jv", "force", "Ma", "grad", "Mgrad", "search", "mv", "prev_grad",
                    "prev_Mgrad")


def _segment_ring(mjm, nworld: int, nconmax: int, njmax: int, count: int):
  """`count` Data objects for the steps of one segment, sharing their scratch fields."""
  ring = [make_data(mjm, nworld, nconmax=nconmax, njmax=njmax)]
  for _ in range(count - 1):
    dk = make_data(mjm, nworld, nconmax=nconmax, njmax=njmax)
    for name in _RING_SHARED:
      if getattr(ring[0], name, None) is not None:
        setattr(dk, name, getattr(ring[0], name))
    for name in _RING_SHARED_EFC:
      if getattr(ring[0].efc, name, None) is not None:
        setattr(dk.efc, name, getattr(ring[0].efc, name))
    ring.append(dk)
  return ring


def _snapshot(d: Data):
  return tuple(getattr(d, k).clone() for k in _STATE)


def _snapshot_view(d: Data):
  return tuple(getattr(d, k) for k in _STATE)


def _restore(d: Data, s) -> None:
  for k, v in zip(_STATE, s):
    getattr(d, k).copy_(v)


def _backward_analytic(ctx, r, m, ctrl, lam, grad_ctrl):
  """The analytic backward over a rollout's segments, last to first: each segment's steps are
  recomputed once from its checkpoint into a ring of Data (the last segment's are kept from the
  forward pass when nothing stepped the ring since) and step_vjp runs back through them.  With a
  second ring and a side stream, the next segment's recomputation runs while the current segment's
  adjoint steps do."""
  T = ctrl.shape[0]
  bounds = lambda sg: (sg * r.checkpoint, min(T, (sg + 1) * r.checkpoint))

  def recompute(sg, ring, qbuf):
    t0, t1 = bounds(sg)
    for k, t in enumerate(range(t0, t1)):
      dk = ring[k]
      _restore(dk, ctx.ckpts[sg] if k == 0 else _snapshot_view(ring[k - 1]))
      qbuf[k].copy_(dk.qvel)
      dk.ctrl.copy_(ctrl[t])
      step(m, dk, fused=r.fused)

  kept = bool(ctx.kept_qvel) and ctx.generation == r._generation
  r._generation += 1  # the rings stop holding any forward pass's steps
  segs = list(reversed(range(len(ctx.ckpts))))
  overlap = bool(r.seg2)
  rings = [r.seg, r.seg2] if overlap else [r.seg, r.seg]
  main = torch.cuda.current_stream()
  ready = None  # the side stream's recomputation of the segment about to be differentiated
  for i, sg in enumerate(segs):
    ring, qbuf = rings[i % 2], r.qbuf[i % 2]
    if i == 0 and kept:
      qv = ctx.kept_qvel
    elif i == 0 or not overlap:
      recompute(sg, ring, qbuf)
      qv = qbuf
    else:
      main.wait_event(ready)
      qv = qbuf
    if overlap and i + 1 < len(segs):  # after the previous segment's adjoint steps, not this one's
      r.side.wait_stream(main)
      with torch.cuda.stream(r.side):
        recompute(segs[i + 1], rings[(i + 1) % 2], r.qbuf[(i + 1) % 2])
        ready = torch.cuda.Event()
        ready.record(r.side)
    t0, t1 = bounds(sg)
    for k in reversed(range(t1 - t0)):
      gq, gv, grad_ctrl[t0 + k] = step_vjp(m, ring[k], qv[k], lam)
      lam = torch.cat([gq, gv], 1)
  return lam


class _Rollout(torch.autograd.Function):
  @staticmethod
  def forward(ctx, qpos0, qvel0, ctrl, r):
    d, m = r.d, r.m
    T = ctrl.shape[0]
    d.qpos.copy_(qpos0)
    d.qvel.copy_(qvel0)
    d.act.zero_()
    d.qacc_warmstart.zero_()
    ckpts = []
    # with the analytic adjoint the last segment runs through the segment's Data, which keep its
    # steps for the backward pass (it then skips that segment's recomputation)
    full = r.analytic == "full"
    last0 = ((T - 1) // r.checkpoint) * r.checkpoint
    kept_qvel, cur = [], d
    for t in range(T):
      if t % r.checkpoint == 0:
        ckpts.append(_snapshot(cur))
      if full and t >= last0:
        dk = r.seg[t - last0]
        if dk is not cur:
          _restore(dk, _snapshot_view(cur))
        cur = dk
        kept_qvel.append(cur.qvel.clone())
      cur.ctrl.copy_(ctrl[t])
      step(m, cur, fused=r.fused)
    r._generation += 1
    ctx.generation, ctx.kept_qvel = r._generation, kept_qvel
    ctx.r, ctx.ckpts, ctx.qpos0, ctx.qpos_T = r, ckpts, qpos0.detach(), cur.qpos.clone()
    ctx.save_for_backward(ctrl)
    return cur.qpos.clone(), cur.qvel.clone()

  @staticmethod
  def backward(ctx, gq, gv):
    (ctrl,) = ctx.saved_tensors
    r, m, d = ctx.r, ctx.r.m, ctx.r.d
    T, nworld = ctrl.shape[0], ctrl.shape[1]
    nv, na = m.nv, m.na
    lam = torch.zeros((nworld, 2 * nv + na), dtype=torch.float32, device=ctrl.device)
    if gq is not None:
      lam[:, :nv] = qpos_grad_to_tangent(m, ctx.qpos_T, gq.float())
    if gv is not None:
      lam[:, nv:2 * nv] = gv.float()
    grad_ctrl = torch.zeros_like(ctrl)
    if r.analytic == "full":
      lam = _backward_analytic(ctx, r, m, ctrl, lam, grad_ctrl)
    # the finite-difference paths, segment by segment
    for seg in ([] if r.analytic == "full" else reversed(range(len(ctx.ckpts)))):
      t0, t1 = seg * r.checkpoint, min(T, (seg + 1) * r.checkpoint)
      _restore(d, ctx.ckpts[seg])
      states = []
      for t in range(t0, t1):  # recompute the segment's states from its checkpoint
        states.append(_snapshot(d))
        d.ctrl.copy_(ctrl[t])
        step(m, d, fused=r.fused)
      for t in reversed(range(t0, t1)):
        _restore(d, states[t - t0])
        d.ctrl.copy_(ctrl[t])
        if r.analytic == "qvel_ctrl":  # qpos columns by differences, the rest analytic
          A, _ = r.fd(d)
          qvel_prev = d.qvel.clone()
          step(m, d, fused=r.fused)
          gv, grad_ctrl[t] = qvel_ctrl_vjp(m, d, qvel_prev, lam)
          lam_q, _ = transition_vjp(m, A, None, lam)
          lam = torch.cat([lam_q[:, :nv], gv], 1)
        elif r.analytic == "ctrl":  # state columns by differences, controls by ctrl_vjp
          A, _ = r.fd(d)
          step(m, d, fused=r.fused)
          grad_ctrl[t] = ctrl_vjp(m, d, lam)
          lam, _ = transition_vjp(m, A, None, lam)
        else:
          A, B = r.fd(d)
          lam, gu = transition_vjp(m, A, B, lam)
          grad_ctrl[t] = gu
    grad_qpos0 = tangent_grad_to_qpos(m, ctx.qpos0, lam[:, :nv])
    grad_qvel0 = lam[:, nv:2 * nv].clone()
    return grad_qpos0, grad_qvel0, grad_ctrl, None


class Rollout:
  """Differentiable T-step rollout of `nworld` worlds from (qpos0, qvel0) under ctrl (T, nworld, nu).

  Calling it returns (qpos_T, qvel_T); gradients flow to qpos0 (per qpos coordinate), qvel0 and
  ctrl through finite-difference transition Jacobians (TransitionFD), with the forward states
  checkpointed every `checkpoint` steps and recomputed segment by segment in the backward pass.
  Each rollout starts from zero act and qacc_warmstart.  With the analytic adjoint and `overlap`
  (default: nworld <= 4096) the backward recomputes the next segment on a side stream, into a
  second ring of Data, while it differentiates the current one.  `analytic` picks which columns of the
  transition Jacobian are not differenced: "full" (the default where qpos_vjp_supported) takes
  every column from step_vjp, "qvel_ctrl" (the default where only ctrl_vjp_supported) takes the
  velocity and control parts from step_vjp and differences the nv qpos columns,
  "ctrl" differences the 2 nv state columns and takes the controls from ctrl_vjp, "none"
  differences all 2 nv + na + nu columns.
  """

  def __init__(self, mjm, m: Model, nworld: int, checkpoint: int = 8, eps: float = 1e-3,
               centered: bool = True, nconmax: int = 64, njmax: int = 128, fused=True,
               analytic: Optional[str] = None, overlap: Optional[bool] = None):
    self.m, self.checkpoint, self.fused = m, int(checkpoint), fused
    if analytic is None:
      analytic = ("full" if qpos_vjp_supported(m) else
                  "qvel_ctrl" if ctrl_vjp_supported(m) else "none")
    if analytic not in ("full", "qvel_ctrl", "ctrl", "none"):
      raise ValueError(f"analytic must be 'full', 'qvel_ctrl', 'ctrl' or 'none', got {analytic!r}")
    if analytic != "none" and not ctrl_vjp_supported(m):
      raise NotImplementedError("analytic step VJP: needs a dense mass matrix, na == 0 "
                                "and, for implicitfast, no affine actuator gains or biases")
    if analytic == "full" and not qpos_vjp_supported(m):
      raise NotImplementedError("analytic qpos adjoint: the model has a feature it does not cover")
    self.analytic = analytic
    self._generation = 0  # bumped whenever the segment's Data are stepped
    # the backward of the analytic adjoint keeps every step of a segment in its own Data (the
    # forward pass runs in the first of them)
    self.seg = _segment_ring(mjm, nworld, nconmax * nworld, njmax * nworld,
                             self.checkpoint) if analytic == "full" else []
    self.d = self.seg[0] if self.seg else make_data(mjm, nworld, nconmax=nconmax * nworld,
                                                     njmax=njmax * nworld)
    # a second ring lets the backward recompute one segment while it differentiates another:
    # by default for batches small enough to leave the GPU idle (up to 4096 worlds)
    if overlap is None:
      overlap = nworld <= 4096
    self.seg2 = _segment_ring(mjm, nworld, nconmax * nworld, njmax * nworld,
                              self.checkpoint) if (analytic == "full" and overlap) else []
    self.side = torch.cuda.Stream(device=self.d.qpos.device) if self.seg2 else None
    self.qbuf = [[torch.empty((nworld, m.nv), dtype=torch.float32, device=self.d.qpos.device)
                  for _ in range(self.checkpoint)] for _ in range(2)] if self.seg else []
    self.fd = None if analytic == "full" else TransitionFD(
        mjm, m, nworld, eps=eps, centered=centered, nconmax=nconmax, njmax=njmax, fused=fused,
        state_only=analytic == "ctrl", qpos_only=analytic == "qvel_ctrl")

  def __call__(self, qpos0: torch.Tensor, qvel0: torch.Tensor, ctrl: torch.Tensor):
    return _Rollout.apply(qpos0, qvel0, ctrl, self)


def rollout(mjm, m: Model, qpos0, qvel0, ctrl, checkpoint: int = 8, eps: float = 1e-3,
            centered: bool = True):
  """One-shot form of Rollout (allocates its workspaces)."""
  return Rollout(mjm, m, qpos0.shape[0], checkpoint=checkpoint, eps=eps, centered=centered)(
      qpos0, qvel0, ctrl)
