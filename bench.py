"""Benchmark: humanoid batched step, nworld=8192 per GPU, steps/s (one JSON line on rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--form chosen|plain|single|precision]

Workload: the reference's humanoid (27 dof, 21 motors) with implicitfast integration, dt=0.005,
Newton with 3 iterations and 4 line-search iterations, pyramidal condim-3 contacts; seeded
synthetic initial states (keyframe "squat" + U(-0.05, 0.05), qvel ~ N(0, 0.01),
ctrl ~ U(-0.4, 0.4)).  A "step" is one mjw.step over all worlds.

value: world-steps/s with the state resident in HBM, one captured CUDA graph of the step replayed
K times, in the chosen launch form (the stage kernels to fwd_acceleration forked over three
streams, the solver's world ordering + persistent k_solve_queue, k_integrate); `forms` gives the
same number for the plain one-kernel-per-stage form, the single-kernel form and the precision
form, measured in the same run.  e2e: the metric through the public API's host-framework call
(mjw.step_io, captured once per buffer in a CUDA graph and replayed) with, every step, the control
copied in from pinned host memory and qpos / qvel copied back.  roofline: the dominant kernel (the solver) timed with CUDA events around its own
launch (mjw.step_phase) over K steps, against the FP32 FMA peak measured in the same run
(mjb_fma_probe) and the measured HBM bandwidth; the bound is whichever takes longer.
Multi-GPU: one process per GPU, each owning its own 8192 worlds (replicas, weak scaling, no
collective on the data path); time is the maximum over ranks of CUDA-event time between barriers.

qacc_err (rank 0): one forward from the bench state in every launch form, checked against the
CPU restatement (the oracle, used only as the checker) in FP64 and FP32 on the first 256 worlds,
each miss over 1e-4 classified (oracle.classify_qacc).

grad (rank 0): grad-steps/s of the differentiation workload -- the same humanoid with the Newton
solve run to convergence (10 iterations), nworld=1024, a 32-step rollout, loss =
||root_pos_T - target||^2 + 1e-3 sum ||ctrl||^2, gradients w.r.t. the control sequence (32 x 21),
qpos0 and qvel0, checkpoints every 8 steps, by the analytic adjoint (and, for comparison, with
finite-difference columns); one forward + backward timed with CUDA events after one warm-up.

combined (rank 0): the humanoid with 0-16 extra spheres (nv = 123), 32768 worlds, a 16-step
rollout forward + analytic adjoint, in the chosen FP32 form and in the precision form.

bin (rank 0): the uneven-contact bin (nv = 384), 4096 worlds, 500 graph-replayed chosen-form
steps after autotuning, against the plain form launched eagerly.

cpu_baseline / --impl reference: the reference algorithm's CPU implementation available here --
the CPU restatement under oracle/, FP32, all host threads -- on the same 8192 worlds and the same
post-warm-up steps, repeated 3 times.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NWORLD = 8192
MODEL = os.path.join(ROOT, "tests", "golden", "models", "humanoid.xml")
METRIC = "humanoid nworld=8192 steps/s"
WORKLOAD = "humanoid step, implicitfast dt=0.005, Newton 3 it / ls 4, pyramidal condim 3"


def _model():
  from mjx_warp_b200 import mjcf

  mjm = mjcf.from_xml_path(MODEL)
  mjm.opt.integrator, mjm.opt.timestep = 3, 0.005
  mjm.opt.solver, mjm.opt.iterations, mjm.opt.ls_iterations = 2, 3, 4
  return mjm


def _state(mjm, start, count, seed=0):
  """Seeded per-world initial states; world w gets the same state however worlds are sharded."""
  from mjx_warp_b200.replicas import world_seeds

  qpos = np.empty((count, mjm.nq))
  qvel = np.empty((count, mjm.nv))
  ctrl = np.empty((count, mjm.nu))
  for i, s in enumerate(world_seeds(seed, start, count)):
    rng = np.random.default_rng(int(s))
    q = mjm.key_qpos[0] + rng.uniform(-0.05, 0.05, mjm.nq)
    q[3:7] /= np.linalg.norm(q[3:7])
    qpos[i], qvel[i], ctrl[i] = q, rng.normal(0, 0.01, mjm.nv), rng.uniform(-0.4, 0.4, mjm.nu)
  return qpos, qvel, ctrl


class _Clocks:
  """Samples nvidia-smi clocks and throttle reasons during the timed region."""

  FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
            "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
            "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

  def __init__(self, index):
    self.index = index
    self.rows = []
    self.proc = None

  def __enter__(self):
    try:
      self.proc = subprocess.Popen(
        ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
         "--format=csv,noheader,nounits", "-lms", "200"],
        stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
      threading.Thread(target=self._read, daemon=True).start()
    except OSError:
      self.proc = None
    return self

  def _read(self):
    for line in self.proc.stdout:
      self.rows.append([x.strip() for x in line.split(",")])

  def __exit__(self, *a):
    if self.proc:
      time.sleep(0.25)
      self.proc.terminate()
      try:
        self.proc.wait(timeout=2)
      except subprocess.TimeoutExpired:
        self.proc.kill()

  def summary(self):
    if not self.rows:
      return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
    sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
    mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
    names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    reasons = sorted({n for r in self.rows for n, v in zip(names, r[4:8]) if v == "Active"})
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
            "reasons": reasons, "samples": len(self.rows)}


def _bytes_of(t):
  return t.numel() * t.element_size()


def _algorithmic_bytes(d, mjm, ncon, nefc):
  """HBM bytes one step must move in full-Data mode: read the state, write every Data field the
  step produces (smooth quantities, contacts, constraint rows, solver vectors)."""
  W = d.nworld
  f = 4
  nq, nv, nu, nb, nj, ng, ns = mjm.nq, mjm.nv, mjm.nu, mjm.nbody, mjm.njnt, mjm.ngeom, mjm.nsite
  read_state = (nq + 2 * nv + nu + nv + 6 * nb) * f  # qpos, qvel, qacc_warmstart, ctrl, qfrc_applied, xfrc
  per_world_out = (nb * (3 + 4 + 9 + 3 + 9 + 3 + 10 + 10 + 6 + 6 + 6) + nj * 6 + ng * 12 + ns * 12
                   + nv * 6 * 2 + nv * nv * 2 + nu * (3 + nv) + nv * 14 + nq + nv * nv) * f
  contact_bytes = ncon * (1 + 3 + 9 + 1 + 5 + 2 + 2 + 5 + 1 + 2 + 1) * f
  efc_bytes = nefc * (nv + 10) * f
  return W * (read_state + per_world_out) + contact_bytes + efc_bytes


FORMS = {"plain": 0, "chosen": 1, "single": 2, "precision": 3}
LAUNCHES = {"plain": 16, "chosen": 16, "single": 2, "precision": 16}  # kernels per step (mjb200.cu run_* paths)


def _solver_bytes(mjm, nworld, nefc):
  """HBM bytes the solver must move: read qM, qfrc_smooth, qacc_smooth, qacc_warmstart and each
  row's J, D, aref; write qacc, qacc_warmstart, qfrc_constraint and the solver vectors (Ma, grad,
  Mgrad, search, mv, prev_grad, prev_Mgrad), per-world scalars (16) and each row's force, Jaref,
  active, jv and quad (3)."""
  nv = mjm.nv
  per_world = (nv * nv + 3 * nv) + (10 * nv + 16)
  per_row = (nv + 2) + 7
  return 4 * (nworld * per_world + nefc * per_row)


def _solver_flops(nv, rows, iters, ls_iters):
  """Algorithmic flops of one world's Newton solve, counted from the reference algorithm
  (solver.py:176-312, 737-869): (1 + I) Hessian assemblies and Cholesky factor-solves and I line
  searches, with R constraint rows, I Newton and L line-search iterations:
  (1 + I)(F_H + F_chol) + I(2 F_Mv + 2 F_Jv + F_ls), F_H = R nv (nv + 1) (symmetric J'DJ),
  F_chol = nv^3 / 3 + 2 nv^2, F_Mv = 2 nv^2, F_Jv = 2 R nv, F_ls = 24 L R."""
  f_h = rows * nv * (nv + 1)
  f_chol = nv ** 3 / 3.0 + 2.0 * nv * nv
  return (1 + iters) * (f_h + f_chol) + iters * (4.0 * nv * nv + 4.0 * rows * nv + 24.0 * ls_iters * rows)


def _step_flops(mjm, rows, pairs, contacts):
  """Algorithmic flops of one world-step: smooth dynamics (~600 per body, 60 per geom), collision
  (20 per broadphase pair, 150 per contact), constraint assembly (R (6 nv + 40)), the mass-matrix
  and integrator factor-solves (2 (nv^3 / 3 + 2 nv^2)) and the solve."""
  nv = mjm.nv
  return (600.0 * (mjm.nbody - 1) + 60.0 * mjm.ngeom + 20.0 * pairs + 150.0 * contacts
          + rows * (6.0 * nv + 40.0) + 2.0 * (nv ** 3 / 3.0 + 2.0 * nv * nv)
          + _solver_flops(nv, rows, mjm.opt.iterations, mjm.opt.ls_iterations))


def _fma_peaks(torch):
  """FP32 and FP64 FMA throughput of this GPU (TFLOP/s), best of 3 launches of mjb_fma_probe
  (8 independent FMA chains per thread, 8 CTAs of 256 threads per SM), CUDA events."""
  import ctypes

  from mjx_warp_b200 import _abi

  lib = _abi.lib()
  lib.mjb_fma_probe.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                ctypes.c_void_p]
  sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
  blocks = 8 * sms
  out = {}
  for name, fp64, iters in (("fp32_tflops", 0, 20000), ("fp64_tflops", 1, 4000)):
    sink = torch.empty(blocks * 256 * 2, dtype=torch.float64, device="cuda")
    best = 0.0
    for _ in range(4):
      a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
      a.record()
      _abi.check(lib.mjb_fma_probe(fp64, blocks, iters, sink.data_ptr(), _abi.stream()), "fma_probe")
      b.record()
      torch.cuda.synchronize()
      best = max(best, 2.0 * 8 * iters * blocks * 256 / (a.elapsed_time(b) * 1e-3) / 1e12)
    out[name] = best
  return out


STATE = ("qpos", "qvel", "act", "ctrl", "qacc_warmstart")


def _qacc_error(mjm, m, d, mjw, torch, restore, forms, sample=256):
  """qacc of one forward from the bench state (after the warm-up steps), per launch form, against
  the CPU restatement with the same solver settings on the first `sample` worlds (the oracle, used
  only as the checker): per-world ||qacc - ref|| / max(||ref||, 1) against its FP64 run and its
  FP32 run (the stand-in for an FP32 implementation of the reference's algorithm), and each world
  that misses FP64 by more than 1e-4 classified as within 1e-4 of the FP32 restatement,
  path-dependent (the FP64 iterate at these iteration counts is itself more than 1e-4 from the
  converged solution, or an FP32 run of the restatement from inputs within one ulp misses too,
  or FP64 moves by more than 1e-4 under such input perturbations) or unexplained."""
  import oracle

  restore()
  torch.cuda.synchronize()
  s = min(sample, d.nworld)
  host = {k: getattr(d, k)[:s].double().cpu().numpy() for k in ("qpos", "qvel", "ctrl",
                                                                "qacc_warmstart")}
  refs = oracle.qacc_references(mjm, host["qpos"], host["qvel"], host["ctrl"],
                                host["qacc_warmstart"], nthreads=os.cpu_count() or 1)
  out = {"vs": f"CPU restatement (FP64 and FP32), same solver settings "
               f"({mjm.opt.iterations} Newton it / ls {mjm.opt.ls_iterations}), tol 1e-4",
         "worlds": s}
  for name, f in forms.items():
    restore()
    mjw.forward(m, d, fused=f)
    q = d.qacc[:s].double().cpu().numpy()
    out[name] = oracle.classify_qacc(q, refs)
  restore()
  return out


def _stability(mjm, mjw, torch, nworld=1024, nstep=200):
  """Worlds that go non-finite within nstep steps of the benchmark configuration from the seeded
  initial states: the device (chosen form) against the CPU restatement in FP32 and in FP64 on the
  same worlds.  The 3-iteration implicitfast humanoid loses a few worlds in every arithmetic."""
  import oracle

  qpos, qvel, ctrl = _state(mjm, 0, nworld)
  m = mjw.put_model(mjm)
  d = mjw.make_data(mjm, nworld=nworld, nconmax=48 * nworld, njmax=80 * nworld)
  d.qpos.copy_(torch.as_tensor(qpos, dtype=torch.float32))
  d.qvel.copy_(torch.as_tensor(qvel, dtype=torch.float32))
  d.ctrl.copy_(torch.as_tensor(ctrl, dtype=torch.float32))
  for _ in range(nstep):
    mjw.step(m, d)
  torch.cuda.synchronize()
  out = {"worlds": nworld, "steps": nstep,
         "device": int(np.count_nonzero(mjw.world_status(d) & 0x8))}
  for prec in (32, 64):
    o = oracle.Oracle(mjm, nworld, prec)
    o.set("qpos", qpos)
    o.set("qvel", qvel)
    o.set("ctrl", ctrl)
    o.run("step", nstep=nstep, nthreads=os.cpu_count() or 1)
    q, v = o.get("qpos"), o.get("qvel")
    out[f"fp{prec}_restatement"] = int((~(np.isfinite(q).all(1) & np.isfinite(v).all(1))).sum())
  return out


def _grad_rate(mjw, torch, nworld=1024, horizon=32, checkpoint=8, reps=2, centered=True,
               analytic=None):
  """grad-steps/s of a differentiated rollout (see the module docstring).  The Newton solve runs
  to convergence (10 iterations, 10 line-search iterations): the 3-iteration iterate of the
  steps/s workload is discontinuous in its inputs, and differences across those jumps make the
  products of 32 transition Jacobians explode (measured: median max |dL/du| ~1e16 at 3
  iterations, ~6e-3 at 10 or 30)."""
  mjm = _model()
  mjm.opt.iterations, mjm.opt.ls_iterations = 10, 10
  qpos, qvel, ctrl0 = _state(mjm, 0, nworld, seed=1)
  m = mjw.put_model(mjm)
  roll = mjw.derivative.Rollout(mjm, m, nworld, checkpoint=checkpoint, eps=1e-3,
                                centered=centered, nconmax=48, njmax=80,
                                analytic=analytic)
  rng = np.random.default_rng(2)
  ctrl = np.repeat(ctrl0[None], horizon, axis=0) + rng.normal(0.0, 0.05, (horizon, nworld, mjm.nu))
  q0 = torch.tensor(qpos, dtype=torch.float32, device="cuda")
  v0 = torch.tensor(qvel, dtype=torch.float32, device="cuda")
  u0 = torch.tensor(ctrl, dtype=torch.float32, device="cuda")
  target = q0[:, :3] + torch.tensor([0.05, 0.0, 0.0], device="cuda")

  def once():
    q, v, u = (t.clone().requires_grad_(True) for t in (q0, v0, u0))
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    qT, _ = roll(q, v, u)
    loss = ((qT[:, :3] - target) ** 2).sum() + 1e-3 * (u ** 2).sum()
    e1.record()
    loss.backward()
    e2.record()
    torch.cuda.synchronize()
    ok = torch.isfinite(u.grad).all(2).all(0) & torch.isfinite(q.grad).all(1) & torch.isfinite(v.grad).all(1)
    gmax = u.grad.abs().amax(dim=(0, 2))[ok]
    return e0.elapsed_time(e1) * 1e-3, e1.elapsed_time(e2) * 1e-3, ok, gmax

  once()
  fwd = bwd = 0.0
  for _ in range(reps):
    f, b, ok, gmax = once()
    fwd, bwd = fwd + f / reps, bwd + b / reps
  t = fwd + bwd
  flags = mjw.world_status(roll.fd.pert) if roll.fd is not None else np.zeros(1, np.uint32)
  q = np.quantile(gmax.cpu().numpy(), [0.5, 0.99]) if gmax.numel() else [None, None]
  return {"value": nworld * horizon / t, "unit": "grad-steps/s",
          "config": {"nworld": nworld, "horizon": horizon, "checkpoint": checkpoint,
                     "wrt": "ctrl (32x21), qpos0, qvel0",
                     "method": ("analytic adjoint of the step (implicit differentiation at the Newton "
                                "solution, mjb_step_vjp), no finite differences" if roll.fd is None else
                                f"GPU finite-difference transition Jacobians ({'centered' if centered else 'forward'}, eps 1e-3, "
                                f"{roll.fd.K} world-steps per world-step"
                                + {"qvel_ctrl": ", qpos columns only; velocity and control gradients by implicit "
                                                "differentiation at the Newton solution",
                                   "ctrl": ", state columns only; control gradient by implicit differentiation "
                                           "at the Newton solution",
                                   "none": ""}[roll.analytic]
                                + ") + reverse recursion")},
          "solver": "Newton 10 it / ls 10 (converged)",
          "forward_ms": fwd * 1e3, "backward_ms": bwd * 1e3,
          "rollout_steps_per_s": nworld * horizon / fwd, "cost_vs_forward": t / fwd,
          "worlds_with_finite_grads": int(ok.sum()), "perturbed_worlds_flagged": int((flags != 0).sum()),
          "max_abs_dL_du_per_world": {"median": float(q[0]) if q[0] is not None else None,
                                      "p99": float(q[1]) if q[1] is not None else None}}


SPHERES_MODEL = os.path.join(ROOT, "tests", "golden", "models", "humanoid_spheres.xml")


def _spheres_state(mjm, hum, nworld, seed):
  """The humanoid's keyframe 0 + U(-0.05, 0.05); k ~ U{0..16} spheres dropped near it from
  z ~ U(0.1, 0.6), the others parked 100 m away at 10 m height (uneven contact counts)."""
  rng = np.random.default_rng(seed)
  qpos = np.zeros((nworld, mjm.nq))
  qpos[:, :hum.nq] = hum.key_qpos[0] + rng.uniform(-0.05, 0.05, (nworld, hum.nq))
  qpos[:, 3:7] /= np.linalg.norm(qpos[:, 3:7], axis=1, keepdims=True)
  nsph = (mjm.nq - hum.nq) // 7
  k = rng.integers(0, nsph + 1, nworld)
  for i in range(nsph):
    a = hum.nq + 7 * i
    act = i < k
    qpos[:, a] = np.where(act, rng.uniform(-0.6, 0.6, nworld), 100.0 + 2.0 * i)
    qpos[:, a + 1] = np.where(act, rng.uniform(-0.6, 0.6, nworld), 100.0)
    qpos[:, a + 2] = np.where(act, rng.uniform(0.1, 0.6, nworld), 10.0)
    qpos[:, a + 3] = 1.0
  return qpos, rng.normal(0.0, 0.01, (nworld, mjm.nv)), rng.uniform(-0.4, 0.4, (nworld, mjm.nu))


def _combined(mjw, torch, nworld=32768, horizon=16, checkpoint=4, reps=2, fused=True,
              plain=True, sample=16):
  """The combined form of the uneven-contact humanoid: humanoids with 0-16 extra free spheres
  (nv = 123), a 16-step rollout forward plus the analytic adjoint (d/d ctrl, qpos0, qvel0 of
  ||root_pos_T - target||^2 + 1e-3 ||ctrl||^2), checkpoints every 4 steps, in launch form `fused`
  (True: the chosen FP32 form; 3: the precision form, FP64 Hessian factor-solves and line-search
  sums); forward and backward world-steps/s, peak GPU memory of the differentiated rollout, qacc
  of one forward against the FP64 restatement on `sample` worlds, and (plain=True) the plain
  form's forward."""
  from mjx_warp_b200 import mjcf
  import oracle

  hum = mjcf.from_xml_path(MODEL)
  mjm = mjcf.from_xml_path(SPHERES_MODEL)
  mjm.opt.integrator, mjm.opt.timestep, mjm.opt.jacobian = 3, 0.005, 0
  mjm.opt.solver, mjm.opt.iterations, mjm.opt.ls_iterations = 2, 10, 10
  qpos, qvel, ctrl0 = _spheres_state(mjm, hum, nworld, seed=5)
  m = mjw.put_model(mjm)
  torch.cuda.synchronize()
  base = torch.cuda.memory_allocated()
  torch.cuda.reset_peak_memory_stats()
  roll = mjw.derivative.Rollout(mjm, m, nworld, checkpoint=checkpoint, nconmax=96, njmax=256,
                                fused=fused)
  rng = np.random.default_rng(6)
  ctrl = np.repeat(ctrl0[None], horizon, axis=0) + rng.normal(0.0, 0.05, (horizon, nworld, mjm.nu))
  q0 = torch.tensor(qpos, dtype=torch.float32, device="cuda")
  v0 = torch.tensor(qvel, dtype=torch.float32, device="cuda")
  u0 = torch.tensor(ctrl, dtype=torch.float32, device="cuda")
  target = q0[:, :3] + torch.tensor([0.05, 0.0, 0.0], device="cuda")

  def once():
    q, v, u = (t.clone().requires_grad_(True) for t in (q0, v0, u0))
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    qT, _ = roll(q, v, u)
    loss = ((qT[:, :3] - target) ** 2).sum() + 1e-3 * (u ** 2).sum()
    e1.record()
    loss.backward()
    e2.record()
    torch.cuda.synchronize()
    ok = torch.isfinite(u.grad).all(2).all(0) & torch.isfinite(q.grad).all(1)
    return e0.elapsed_time(e1) * 1e-3, e1.elapsed_time(e2) * 1e-3, int(ok.sum())

  once()
  fwd = bwd = 0.0
  for _ in range(reps):
    f, b, nok = once()
    fwd, bwd = fwd + f / reps, bwd + b / reps
  peak = torch.cuda.max_memory_allocated() - base
  status = mjw.world_status(roll.d)
  d = roll.d
  # qacc of one forward from the initial state against FP64 on a sample
  d.qpos.copy_(q0)
  d.qvel.copy_(v0)
  d.ctrl.copy_(u0[0])
  d.qacc_warmstart.zero_()
  mjw.forward(m, d, fused=fused)
  s = min(sample, nworld)
  qd = d.qacc[:s].double().cpu().numpy()
  o = oracle.Oracle(mjm, s, 64)
  o.set("qpos", qpos[:s])
  o.set("qvel", qvel[:s])
  o.set("ctrl", ctrl[0, :s])
  o.run("forward", nthreads=os.cpu_count() or 1)
  e = oracle.rel_err(qd, o.get("qacc"))
  out = {"workload": "humanoid + 0-16 free spheres per world (nv 123), implicitfast dt=0.005, "
                     "Newton 10 it / ls 10, dense mass matrix; 16-step rollout + analytic adjoint",
         "form": {True: "chosen", 3: "precision"}.get(fused, str(fused)),
         "nworld": nworld, "horizon": horizon, "checkpoint": checkpoint,
         "forward_steps_per_s": nworld * horizon / fwd,
         "backward_steps_per_s": nworld * horizon / bwd,
         "grad_steps_per_s": nworld * horizon / (fwd + bwd), "cost_vs_forward": (fwd + bwd) / fwd,
         "forward_ms": fwd * 1e3, "backward_ms": bwd * 1e3,
         "peak_gpu_memory_gb": peak / 1e9, "worlds_with_finite_grads": nok,
         "worlds_flagged": int((status != 0).sum()),
         "qacc_err_vs_fp64": {"worlds": s, "median": float(np.median(e)), "max": float(e.max()),
                              "frac_le_1e-4": float(np.mean(e <= 1e-4))}}
  if plain:  # the plain form's forward rollout of the same worlds (no checkpoints, no graph)
    step = lambda: mjw.step(m, d, fused=False)
    d.qpos.copy_(q0)
    d.qvel.copy_(v0)
    d.qacc_warmstart.zero_()
    d.ctrl.copy_(u0[0])
    step()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    d.qpos.copy_(q0)
    d.qvel.copy_(v0)
    d.qacc_warmstart.zero_()
    t0.record()
    for t in range(horizon):
      d.ctrl.copy_(u0[t])
      step()
    t1.record()
    torch.cuda.synchronize()
    out["plain_forward_steps_per_s"] = nworld * horizon / (t0.elapsed_time(t1) * 1e-3)
  del roll, d
  torch.cuda.empty_cache()
  return out


BIN_MODEL = os.path.join(ROOT, "tests", "golden", "models", "bin.xml")


def _bin_state(mjm, nworld, seed):
  """Bin bodies at x, y ~ U(-0.4, 0.4), z ~ U(0.03, 0.35), random orientations: overlapping
  packings with many contacts (uneven rows per world)."""
  rng = np.random.default_rng(seed)
  qpos = np.tile(mjm.qpos0, (nworld, 1))
  for b in range(mjm.nbody - 1):
    a = 7 * b
    qpos[:, a:a + 2] = rng.uniform(-0.4, 0.4, (nworld, 2))
    qpos[:, a + 2] = rng.uniform(0.03, 0.35, nworld)
    q = rng.normal(size=(nworld, 4))
    qpos[:, a + 3:a + 7] = q / np.linalg.norm(q, axis=1, keepdims=True)
  return qpos, rng.normal(0.0, 0.1, (nworld, mjm.nv)), np.zeros((nworld, 0))


def _bin_config(mjw, torch, nworld=4096, steps=500, plain_steps=10, sample=16):
  """The uneven-contact bin (48 spheres + 16 capsules in a 5-plane bin, nv = 384, Euler
  dt = 0.002, Newton 10 iterations / 10 line-search iterations, dense mass matrix): nworld worlds
  from seeded overlapping packings, the chosen form autotuned (mjw.autotune) and captured as a
  CUDA graph, replayed for `steps` steps; the plain one-launch-per-stage form launched eagerly
  from the same state for `plain_steps` steps.  Non-finite / overflow counts after the run, qacc
  of one forward from the final state against the FP64 restatement on `sample` worlds, and the
  solver's flop-bound roofline at the measured rows."""
  from mjx_warp_b200 import mjcf
  import oracle

  mjm = mjcf.from_xml_path(BIN_MODEL)
  mjm.opt.iterations, mjm.opt.ls_iterations, mjm.opt.jacobian = 10, 10, 0
  q, v, _ = _bin_state(mjm, nworld, seed=3)
  m = mjw.put_model(mjm)
  d = mjw.make_data(mjm, nworld, nconmax=600 * nworld, njmax=512 * nworld)
  d.qpos.copy_(torch.as_tensor(q, dtype=torch.float32))
  d.qvel.copy_(torch.as_tensor(v, dtype=torch.float32))
  tune = mjw.autotune(m, d)
  snap = {k: getattr(d, k).clone() for k in ("qpos", "qvel", "qacc_warmstart")}

  def restore():
    for k, t in snap.items():
      getattr(d, k).copy_(t)

  restore()
  g = torch.cuda.CUDAGraph()
  st = torch.cuda.Stream()
  st.wait_stream(torch.cuda.current_stream())
  with torch.cuda.stream(st):
    with torch.cuda.graph(g, stream=st):
      mjw.step(m, d)
  torch.cuda.current_stream().wait_stream(st)
  restore()
  torch.cuda.synchronize()
  e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
  e0.record()
  for _ in range(steps):
    g.replay()
  e1.record()
  torch.cuda.synchronize()
  chosen_s = e0.elapsed_time(e1) * 1e-3
  del g
  status = mjw.world_status(d)
  nefc = int(d.world_nefc.sum())
  rows = d.world_nefc.cpu().numpy()
  # one phase-timed step from the final state: the solver's share and its roofline
  a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
  mjw.step_phase(m, d, 0)
  a.record()
  mjw.step_phase(m, d, 1)
  b.record()
  mjw.step_phase(m, d, 2)
  torch.cuda.synchronize()
  solve_s = a.elapsed_time(b) * 1e-3
  rows_solve = int(d.world_nefc.sum()) / nworld
  fma = _fma_peaks(torch)
  flops = _solver_flops(mjm.nv, rows_solve, mjm.opt.iterations, mjm.opt.ls_iterations) * nworld
  # qacc of one forward from the final state against FP64 on a sample
  s = min(sample, nworld)
  host = {k: getattr(d, k)[:s].double().cpu().numpy() for k in ("qpos", "qvel", "qacc_warmstart")}
  mjw.forward(m, d)
  qd = d.qacc[:s].double().cpu().numpy()
  o = oracle.Oracle(mjm, s, 64)
  for k, t in host.items():
    o.set(k, t)
  o.run("forward", nthreads=os.cpu_count() or 1)
  e = oracle.rel_err(qd, o.get("qacc"))
  cost_ok = d.efc.cost[:s].cpu().numpy() <= o.scalar("cost") * 1.025 + 1e-3
  # the plain form, eager, from the same starting state
  restore()
  mjw.step(m, d, fused=False)
  restore()
  torch.cuda.synchronize()
  e0.record()
  for _ in range(plain_steps):
    mjw.step(m, d, fused=False)
  e1.record()
  torch.cuda.synchronize()
  plain_s = e0.elapsed_time(e1) * 1e-3
  return {"workload": "bin: 48 spheres + 16 capsules, nv 384, Euler dt 0.002, Newton 10 it / ls 10, "
                      "dense mass matrix, seeded overlapping packings",
          "nworld": nworld, "steps": steps, "autotuned": tune,
          "chosen": {"steps_per_s": nworld * steps / chosen_s, "ms_per_step": chosen_s / steps * 1e3,
                     "launch": "one captured CUDA graph per step, replayed"},
          "plain": {"steps_per_s": nworld * plain_steps / plain_s,
                    "ms_per_step": plain_s / plain_steps * 1e3, "steps": plain_steps,
                    "launch": "eager, one launch per stage"},
          "chosen_vs_plain": plain_s / plain_steps / (chosen_s / steps),
          "status_after": {"nonfinite_worlds": int(np.count_nonzero(status & 0x8)),
                           "overflow_worlds": int(np.count_nonzero(status & 0x7))},
          "rows_per_world": {"mean": nefc / nworld, "min": int(rows.min()), "max": int(rows.max())},
          "qacc_err_vs_fp64": {"worlds": s, "median": float(np.median(e)), "max": float(e.max()),
                               "frac_le_1e-4": float(np.mean(e <= 1e-4)),
                               "cost_within_2.5pct": float(np.mean(cost_ok))},
          "roofline": {"kernel": "k_solve_cta", "kernel_ms": solve_s * 1e3,
                       "flops_per_launch": flops, "achieved_tflops": flops / solve_s / 1e12,
                       "peak_tflops": fma["fp32_tflops"],
                       "frac": flops / solve_s / 1e12 / fma["fp32_tflops"], "bound": "fp32",
                       "rows_per_world": rows_solve}}


def _profile_case_bin(mjw, torch, nworld=512, cta_warps=2):
  """A small case of the bin for a profiler capture of the CTA solver: nworld worlds of
  _bin_config's bin from the same seeded packings, the CTA width pinned, one step then one
  forward (the capture's launch)."""
  from mjx_warp_b200 import mjcf

  mjm = mjcf.from_xml_path(BIN_MODEL)
  mjm.opt.iterations, mjm.opt.ls_iterations, mjm.opt.jacobian = 10, 10, 0
  q, v, _ = _bin_state(mjm, nworld, seed=3)
  m = mjw.put_model(mjm)
  d = mjw.make_data(mjm, nworld, nconmax=600 * nworld, njmax=512 * nworld)
  d.qpos.copy_(torch.as_tensor(q, dtype=torch.float32))
  d.qvel.copy_(torch.as_tensor(v, dtype=torch.float32))
  mjw.set_tune(m, d, solver_cta_warps=cta_warps)
  mjw.step(m, d)
  mjw.forward(m, d)
  torch.cuda.synchronize()
  return {"profile_case": "bin", "nworld": nworld, "cta_warps": cta_warps,
          "rows_per_world": float(d.world_nefc.float().mean()),
          "device_gb": torch.cuda.max_memory_allocated() / 1e9}


def _larger_models(mjw, torch, reps=3):
  """ms per step (chosen, plain) of the uneven-contact configurations: the bin (nv = 384, 4096
  worlds, Newton or CG 10 iterations, dense or sparse mass matrix) and the humanoid with 0-16
  extra spheres (nv = 123, 32768 worlds, implicitfast, Newton 3 iterations)."""
  from mjx_warp_b200 import mjcf

  def ms(m, mjm, q, v, u, nconmax, njmax, form):
    W = q.shape[0]
    d = mjw.make_data(mjm, W, nconmax=nconmax * W, njmax=njmax * W)
    d.qpos.copy_(torch.as_tensor(q, dtype=torch.float32))
    d.qvel.copy_(torch.as_tensor(v, dtype=torch.float32))
    if mjm.nu:
      d.ctrl.copy_(torch.as_tensor(u, dtype=torch.float32))
    mjw.step(m, d, fused=form)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
      mjw.step(m, d, fused=form)
    e1.record()
    torch.cuda.synchronize()
    return round(e0.elapsed_time(e1) / reps, 2)

  out = {}
  for label, jac, solver in (("bin, Newton, dense", 0, 2), ("bin, CG, dense", 0, 1),
                             ("bin, Newton, sparse", 1, 2), ("bin, CG, sparse", 1, 1)):
    mjm = mjcf.from_xml_path(BIN_MODEL)
    mjm.opt.iterations, mjm.opt.ls_iterations, mjm.opt.jacobian, mjm.opt.solver = 10, 10, jac, solver
    q, v, u = _bin_state(mjm, 4096, seed=3)
    m = mjw.put_model(mjm)
    out[label] = {"nworld": 4096, "ms_per_step_chosen": ms(m, mjm, q, v, u, 600, 512, 1),
                  "ms_per_step_plain": ms(m, mjm, q, v, u, 600, 512, 0)}
  hum = mjcf.from_xml_path(MODEL)
  mjm = mjcf.from_xml_path(SPHERES_MODEL)
  mjm.opt.integrator, mjm.opt.timestep, mjm.opt.jacobian = 3, 0.005, 0
  mjm.opt.solver, mjm.opt.iterations, mjm.opt.ls_iterations = 2, 3, 4
  q, v, u = _spheres_state(mjm, hum, 32768, seed=4)
  m = mjw.put_model(mjm)
  out["humanoid + 0-16 spheres, Newton 3"] = {
      "nworld": 32768, "ms_per_step_chosen": ms(m, mjm, q, v, u, 96, 384, 1),
      "ms_per_step_plain": ms(m, mjm, q, v, u, 96, 384, 0)}
  return out


def _graph_steps_per_s(torch, step, nworld, steps, barrier, restore):
  g = torch.cuda.CUDAGraph()
  s = torch.cuda.Stream()
  s.wait_stream(torch.cuda.current_stream())
  with torch.cuda.stream(s):
    with torch.cuda.graph(g, stream=s):
      step()
  torch.cuda.current_stream().wait_stream(s)
  restore()
  barrier()
  t0 = torch.cuda.Event(enable_timing=True)
  t1 = torch.cuda.Event(enable_timing=True)
  t0.record()
  for _ in range(steps):
    g.replay()
  t1.record()
  barrier()
  el = t0.elapsed_time(t1) / 1000.0
  del g
  return el


def run_ours(args):
  import torch

  import mjx_warp_b200 as mjw
  from mjx_warp_b200 import replicas

  rank, world_size, local_rank = replicas.dist_env()
  if world_size > 1:
    import datetime

    torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
  torch.cuda.set_device(local_rank)
  mjm = _model()
  nworld = args.nworld
  qpos, qvel, ctrl = _state(mjm, rank * nworld, nworld)
  m = mjw.put_model(mjm)
  d = mjw.make_data(mjm, nworld=nworld, nconmax=48 * nworld, njmax=80 * nworld)
  d.qpos.copy_(torch.as_tensor(qpos, dtype=torch.float32))
  d.qvel.copy_(torch.as_tensor(qvel, dtype=torch.float32))
  d.ctrl.copy_(torch.as_tensor(ctrl, dtype=torch.float32))
  form = FORMS[args.form]
  step = lambda: mjw.step(m, d, fused=form)  # noqa: E731

  def barrier():
    if world_size > 1:
      torch.distributed.barrier()
    torch.cuda.synchronize()

  for _ in range(args.warmup):
    step()
  # every measurement below starts from the state after the warm-up steps, so each times the
  # same K steps of the same trajectories
  barrier()
  snap = {k: getattr(d, k).clone() for k in STATE}

  def restore():
    for k, v in snap.items():
      getattr(d, k).copy_(v)

  # device-resident: one captured graph of the step, replayed K times
  g = torch.cuda.CUDAGraph()
  s = torch.cuda.Stream()
  s.wait_stream(torch.cuda.current_stream())
  with torch.cuda.stream(s):
    with torch.cuda.graph(g, stream=s):
      step()
  torch.cuda.current_stream().wait_stream(s)
  g.replay()
  restore()
  barrier()
  with _Clocks(local_rank) as clocks:
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(args.steps):
      g.replay()
    t1.record()
    barrier()
  elapsed = replicas.max_over_ranks(t0.elapsed_time(t1) / 1000.0, device="cuda")
  status = mjw.world_status(d)
  nonfinite = int(replicas.sum_over_ranks(int(np.count_nonzero(status & 0x8)), device="cuda"))
  overflow = int(replicas.sum_over_ranks(int(np.count_nonzero(status & 0x7)), device="cuda"))
  ncon = int(d.world_ncon.sum())
  nefc = int(d.world_nefc.sum())
  npair = int(d.world_npair.sum())

  # end to end through the public API's host-framework call (mjw.step_io: the control copied in,
  # one step, qpos / qvel copied out), with the control coming from pinned host memory and the
  # state going back to it every step
  # Transfers are double-buffered on a copy stream: step t's control is uploaded while step t - 1
  # computes, and step t's state is downloaded while step t + 1 computes (events order each
  # buffer's reuse); every step's bytes still cross PCIe inside the timed region.
  ctrl_h = torch.as_tensor(ctrl, dtype=torch.float32).pin_memory()
  ctrl_d = [torch.empty_like(d.ctrl) for _ in range(2)]
  io_out = [{"qpos": torch.empty_like(d.qpos), "qvel": torch.empty_like(d.qvel)} for _ in range(2)]
  qpos_h = torch.empty(d.qpos.shape, dtype=torch.float32).pin_memory()
  qvel_h = torch.empty(d.qvel.shape, dtype=torch.float32).pin_memory()
  copy = torch.cuda.Stream()
  main = torch.cuda.current_stream()
  # one captured CUDA graph of the step_io call per buffer pair, as a framework that calls it every
  # step would use it (the call is graph-capturable; the transfers stay outside, on the copy stream)
  io_graphs = []
  for b in range(2):
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
      mjw.step_io(m, d, 1, inputs={"ctrl": ctrl_d[b]}, outputs=("qpos", "qvel"), out=io_out[b],
                  fused=form)
    io_graphs.append(g)
  torch.cuda.synchronize()
  up = [torch.cuda.Event() for _ in range(2)]      # control t uploaded
  done = [torch.cuda.Event() for _ in range(2)]    # step t's outputs written / its control read
  down = [torch.cuda.Event() for _ in range(2)]    # outputs t downloaded
  restore()
  barrier()
  e0 = torch.cuda.Event(enable_timing=True)
  e1 = torch.cuda.Event(enable_timing=True)
  e0.record()
  with torch.cuda.stream(copy):
    ctrl_d[0].copy_(ctrl_h, non_blocking=True)
    up[0].record(copy)
  for t in range(args.steps):
    b = t & 1
    if t + 1 < args.steps:  # upload the next control once its buffer's last step is done
      with torch.cuda.stream(copy):
        if t >= 1:
          copy.wait_event(done[1 - b])
        ctrl_d[1 - b].copy_(ctrl_h, non_blocking=True)
        up[1 - b].record(copy)
    main.wait_event(up[b])
    if t >= 2:
      main.wait_event(down[b])  # step t - 2's outputs left this buffer
    io_graphs[b].replay()
    done[b].record(main)
    with torch.cuda.stream(copy):
      copy.wait_event(done[b])
      qpos_h.copy_(io_out[b]["qpos"], non_blocking=True)
      qvel_h.copy_(io_out[b]["qvel"], non_blocking=True)
      down[b].record(copy)
  main.wait_stream(copy)
  e1.record()
  barrier()
  e2e_elapsed = replicas.max_over_ranks(e0.elapsed_time(e1) / 1000.0, device="cuda")
  del io_graphs

  # the dominant kernel (the solver) timed around its own launch, same stream, K steps
  solve_ms = []
  if args.form == "plain":
    pre = lambda: (mjw.fwd_position(m, d), mjw.fwd_velocity(m, d), mjw.fwd_actuation(m, d),  # noqa: E731
                   mjw.fwd_acceleration(m, d))
    solve = lambda: mjw.solve(m, d)  # noqa: E731
    post = lambda: mjw.implicit(m, d)  # noqa: E731
  else:
    pre = lambda: mjw.step_phase(m, d, 0)  # noqa: E731
    solve = lambda: mjw.step_phase(m, d, 1)  # noqa: E731
    post = lambda: mjw.step_phase(m, d, 2)  # noqa: E731
  restore()
  barrier()
  for _ in range(args.steps):
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pre()
    a.record()
    solve()
    b.record()
    post()
    solve_ms.append((a, b))
  barrier()
  solve_s = replicas.max_over_ranks(float(np.mean([a.elapsed_time(b) for a, b in solve_ms])) / 1000.0,
                                    device="cuda")
  nefc_solve = int(d.world_nefc.sum())

  # the other launch forms on the same worlds, for the chosen-vs-plain comparison
  forms = {}
  for name, f in FORMS.items():
    if name == args.form:
      continue
    el = _graph_steps_per_s(torch, lambda: mjw.step(m, d, fused=f), nworld, args.steps, barrier,
                            restore)
    el = replicas.max_over_ranks(el, device="cuda")
    forms[name] = {"value": nworld * world_size * args.steps / el, "ms_per_step": el / args.steps * 1e3}

  accuracy = None
  stability = None
  if rank == 0 and not args.no_accuracy:
    accuracy = _qacc_error(mjm, m, d, mjw, torch, restore, FORMS)
    stability = _stability(mjm, mjw, torch)
  grad = None
  if rank == 0 and not args.no_grad:
    grad = _grad_rate(mjw, torch)
    for mode, key in (("qvel_ctrl", "qpos_columns_by_differences"),
                      ("none", "all_columns_by_differences")):
      other = _grad_rate(mjw, torch, analytic=mode)
      grad[key] = {k: other[k] for k in ("value", "unit", "cost_vs_forward", "worlds_with_finite_grads")}
      grad[key]["method"] = other["config"]["method"]

  combined = None
  if rank == 0 and not args.no_combined:
    combined = _combined(mjw, torch)
    combined["precision_form"] = _combined(mjw, torch, fused=3, plain=False)
  bin_cfg = None
  if rank == 0 and not args.no_bin:
    bin_cfg = _bin_config(mjw, torch)

  launches_per_step = LAUNCHES[args.form]
  total_worlds = nworld * world_size
  value = total_worlds * args.steps / elapsed
  alg = _solver_bytes(mjm, nworld, nefc_solve)
  step_alg = _algorithmic_bytes(d, mjm, ncon, nefc)
  peaks = {}
  try:
    with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
      peaks = json.load(f)
  except OSError:
    pass
  hbm = float(peaks.get("hbm_gbs", 6650.0))
  achieved = alg / solve_s / 1e9
  fma = _fma_peaks(torch)
  rows = nefc_solve / nworld
  solver_flops = _solver_flops(mjm.nv, rows, mjm.opt.iterations, mjm.opt.ls_iterations) * nworld
  flop_rate = solver_flops / solve_s / 1e12
  t_flop, t_hbm = solver_flops / (fma["fp32_tflops"] * 1e12), alg / (hbm * 1e9)
  flop_bound = t_flop >= t_hbm
  step_flops = _step_flops(mjm, nefc / nworld, npair / nworld, ncon / nworld) * nworld
  footprint = sum(_bytes_of(t) for t in list(d.arrays().values()) + list(d.contact.arrays().values())
                  + list(d.efc.arrays().values()))
  traffic = None
  tpath = os.path.join(ROOT, "profiles", "traffic.json")
  if os.path.exists(tpath):
    with open(tpath) as f:
      traffic = json.load(f).get(args.form, {}).get("dram_bytes_per_launch")
  line = {
    "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world_size, "steps": args.steps,
    "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1000.0, "higher_is_better": True,
    "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded states)",
    "config": {"workload": WORKLOAD, "nworld_per_gpu": nworld, "nv": mjm.nv, "form": args.form,
               "solver_reuses_factor": args.form != "plain",
               "nconmax": d.nconmax, "njmax": d.njmax,
               "l2": f"working set {footprint / 2**20:.0f} MiB per GPU > 126 MB L2, no flush",
               "parallelism": f"replicas x{world_size}"},
    "e2e": {"value": total_worlds * args.steps / e2e_elapsed, "unit": "steps/s",
            "h2d_bytes_per_step": _bytes_of(ctrl_h),
            "d2h_bytes_per_step": _bytes_of(qpos_h) + _bytes_of(qvel_h),
            "call": "mjw.step_io (mjb_step_io: ctrl in, one step, qpos / qvel out), one captured "
                    "CUDA graph of the call per buffer, replayed every step; transfers "
                    "double-buffered on a copy stream, overlapping the neighbouring steps"},
    "gpu_launches": launches_per_step * args.steps,
    "roofline": {"bound": "fp32" if flop_bound else "hbm",
                 "achieved": flop_rate if flop_bound else achieved,
                 "peak": fma["fp32_tflops"] if flop_bound else hbm,
                 "unit": "TFLOP/s" if flop_bound else "GB/s",
                 "frac": flop_rate / fma["fp32_tflops"] if flop_bound else achieved / hbm,
                 "traffic": traffic,
                 "kernel": "k_stage<S_SOLVE> (plain)" if args.form == "plain"
                           else "k_solve_queue",
                 "kernel_ms": solve_s * 1e3, "kernel_share_of_step": solve_s / (elapsed / args.steps),
                 "flops_per_launch": solver_flops, "algorithmic_bytes_per_launch": alg,
                 "t_min_us": {"fp32": t_flop * 1e6, "hbm": t_hbm * 1e6},
                 "hbm": {"achieved_gbs": achieved, "peak_gbs": hbm, "frac": achieved / hbm,
                         "peak_source": "measured (MEASURED_PEAKS.json)" if peaks else "fallback"},
                 "fp32": {"achieved_tflops": flop_rate, "peak_tflops": fma["fp32_tflops"],
                          "frac": flop_rate / fma["fp32_tflops"],
                          "peak_source": "measured in this run (mjb_fma_probe, FFMA)"},
                 "fp64_peak_tflops": fma["fp64_tflops"],
                 "rows_per_world": rows,
                 "step_flops": step_flops,
                 "step_achieved_tflops": step_flops / (elapsed / args.steps) / 1e12,
                 "step_algorithmic_bytes": step_alg,
                 "step_achieved_gbs": step_alg / (elapsed / args.steps) / 1e9},
    "forms": forms,
    "clocks": clocks.summary(),
    "status": {"nonfinite_worlds": nonfinite, "overflow_worlds": overflow,
               "mean_contacts_per_world": ncon / nworld, "mean_efc_rows_per_world": nefc / nworld},
  }
  if accuracy is not None:
    line["qacc_err"] = accuracy
  if stability is not None:
    line["status"]["nonfinite_within_200_steps"] = stability
  if grad is not None:
    line["grad"] = grad
  if combined is not None:
    line["combined"] = combined
  if bin_cfg is not None:
    line["bin"] = bin_cfg
  if rank == 0 and not args.no_cpu_baseline:
    line["cpu_baseline"] = cpu_baseline(mjm, args.steps, args.warmup, budget_s=args.cpu_seconds,
                                        nworld=nworld)
  del g
  if world_size > 1:
    torch.distributed.barrier()
    torch.distributed.destroy_process_group()
  if rank == 0:
    print(json.dumps(line), flush=True)


def cpu_baseline(mjm, steps, warmup, budget_s=10.0, nworld=NWORLD, repeats=3):
  """The CPU restatement (FP32, OpenMP over worlds, all host threads) on the GPU arm's workload:
  the same nworld worlds from the same seeded states, `warmup` untimed steps, then up to `steps`
  timed steps (as many as fit in about budget_s / repeats seconds), repeated `repeats` times from
  the same post-warm-up state; value = the median world-steps/s, with the repeats' spread."""
  from oracle import Oracle

  qpos, qvel, ctrl = _state(mjm, 0, nworld)
  o = Oracle(mjm, nworld, 32)
  o.set("qpos", qpos)
  o.set("qvel", qvel)
  o.set("ctrl", ctrl)
  cores = os.cpu_count() or 1
  t0 = time.perf_counter()
  o.run("step", nstep=max(1, warmup), nthreads=cores)
  per_step = (time.perf_counter() - t0) / max(1, warmup)
  k = int(max(1, min(steps, budget_s / repeats / max(per_step, 1e-6))))
  snap = {f: o.get(f) for f in ("qpos", "qvel", "qacc_warmstart")}
  rates = []
  for _ in range(repeats):
    for f, v in snap.items():
      o.set(f, v)
    t0 = time.perf_counter()
    o.run("step", nstep=k, nthreads=cores)
    rates.append(nworld * k / (time.perf_counter() - t0))
  med = statistics.median(rates)
  return {"value": med, "unit": "steps/s", "cores": cores, "kind": "port",
          "repeats": rates, "spread": (max(rates) - min(rates)) / med,
          "sample": (f"{nworld} worlds x {k} steps after {max(1, warmup)} warm-up steps, "
                     f"{repeats} repeats from the same state (median), FP32 CPU restatement")}


def run_reference(args):
  """Reference arm: the reference algorithm's CPU implementation (oracle/, the CPU restatement;
  MJWarp itself needs warp-lang and MuJoCo, neither installable here), same workload."""
  from mjx_warp_b200 import replicas

  rank, world_size, _ = replicas.dist_env()
  if rank != 0:
    return
  mjm = _model()
  cpu = cpu_baseline(mjm, args.steps, args.warmup,
                     budget_s=min(30.0, max(3.0, 0.05 * (args.steps + args.warmup))),
                     nworld=args.nworld)
  line = {
    "impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": "steps/s",
    "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup,
    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
    "data": "synthetic (seeded states)",
    "config": {"workload": WORKLOAD, "nworld_per_gpu": args.nworld, "form": "cpu"},
    "cpu_baseline": cpu,
    "e2e": {"value": cpu["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
  }
  print(json.dumps(line), flush=True)


def main():
  p = argparse.ArgumentParser()
  p.add_argument("--gpus", type=int, default=1)
  p.add_argument("--steps", type=int, default=200)
  p.add_argument("--warmup", type=int, default=10)
  p.add_argument("--impl", default="ours", choices=["ours", "reference"])
  p.add_argument("--form", default="chosen", choices=list(FORMS))
  p.add_argument("--nworld", type=int, default=NWORLD)
  p.add_argument("--cpu-seconds", type=float, default=10.0)
  p.add_argument("--no-cpu-baseline", action="store_true")
  p.add_argument("--no-accuracy", action="store_true")
  p.add_argument("--no-grad", action="store_true")
  p.add_argument("--no-combined", action="store_true")
  p.add_argument("--no-bin", action="store_true")
  p.add_argument("--profile-case", choices=["bin"],
                 help="run one small case for a profiler capture (bin: 512 worlds, the CTA solver's "
                      "launch is the forward's) and print one JSON line instead of the bench")
  p.add_argument("--larger-models", action="store_true",
                 help="print one JSON line of the uneven-contact configurations' step times instead")
  args = p.parse_args()
  if args.warmup < 3:
    args.warmup = 3
  if args.profile_case:
    import torch
    import mjx_warp_b200 as mjw
    print(json.dumps(_profile_case_bin(mjw, torch, nworld=min(args.nworld, 512))))
    return
  if args.larger_models:
    import torch
    import mjx_warp_b200 as mjw
    print(json.dumps({"larger_models": _larger_models(mjw, torch)}))
    return
  if args.impl == "reference":
    run_reference(args)
  else:
    run_ours(args)


if __name__ == "__main__":
  main()
