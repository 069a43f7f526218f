"""Shared test helpers: model loading, seeded batched states, oracle <-> device comparisons."""

import json
import os

import numpy as np
import torch

import mjx_warp_b200 as mjw
from mjx_warp_b200 import mjcf

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MODELS = os.path.join(GOLDEN, "models")


def fixtures():
  with open(os.path.join(GOLDEN, "reference_fixtures.json")) as f:
    return json.load(f)


def load(name, **opt):
  """Compiles tests/golden/models/<name> (or an MJCF string) and applies option overrides."""
  if name.lstrip().startswith("<"):
    mjm = mjcf.from_xml_string(name)
  else:
    mjm = mjcf.from_xml_path(os.path.join(MODELS, name))
  for k, v in opt.items():
    setattr(mjm.opt, k, v)
  return mjm


def humanoid(iterations=3, ls_iterations=4, integrator=3, timestep=0.005, solver=2):
  """The humanoid of the nworld=8192 benchmark: implicitfast, dt 0.005, Newton."""
  return load("humanoid.xml", iterations=iterations, ls_iterations=ls_iterations,
              integrator=integrator, timestep=timestep, solver=solver)


def humanoid_state(mjm, nworld, seed=0, key=0):
  """Seeded initial states: qpos = keyframe + U(-0.05, 0.05) (free-joint quat renormalised),
  qvel ~ N(0, 0.01), ctrl ~ U(-0.4, 0.4)."""
  rng = np.random.default_rng(seed)
  qpos = np.tile(mjm.key_qpos[key], (nworld, 1))
  qpos += rng.uniform(-0.05, 0.05, qpos.shape)
  qpos[:, 3:7] /= np.linalg.norm(qpos[:, 3:7], axis=1, keepdims=True)
  qvel = rng.normal(0.0, 0.01, (nworld, mjm.nv))
  ctrl = rng.uniform(-0.4, 0.4, (nworld, mjm.nu))
  return qpos, qvel, ctrl


def generic_state(mjm, nworld, seed=0, qscale=0.1, vscale=0.1):
  rng = np.random.default_rng(seed)
  qpos = np.tile(mjm.qpos0, (nworld, 1)).astype(float)
  adr = 0
  for j in range(mjm.njnt):
    t = mjm.jnt_type[j]
    a = mjm.jnt_qposadr[j]
    if t == 0:
      qpos[:, a:a + 3] += rng.uniform(-qscale, qscale, (nworld, 3))
      q = qpos[:, a + 3:a + 7] + rng.uniform(-qscale, qscale, (nworld, 4))
      qpos[:, a + 3:a + 7] = q / np.linalg.norm(q, axis=1, keepdims=True)
    elif t == 1:
      q = qpos[:, a:a + 4] + rng.uniform(-qscale, qscale, (nworld, 4))
      qpos[:, a:a + 4] = q / np.linalg.norm(q, axis=1, keepdims=True)
    else:
      qpos[:, a] += rng.uniform(-qscale, qscale, nworld)
    adr += 1
  qvel = rng.normal(0.0, vscale, (nworld, mjm.nv))
  ctrl = rng.uniform(-1.0, 1.0, (nworld, mjm.nu))
  return qpos, qvel, ctrl


def device_data(mjm, qpos, qvel, ctrl, nconmax=None, njmax=None, warmstart=None):
  nworld = qpos.shape[0]
  d = mjw.make_data(mjm, nworld=nworld, nconmax=nconmax or 64 * nworld, njmax=njmax or 256 * nworld,
                    device="cuda")
  d.qpos.copy_(torch.as_tensor(qpos, dtype=torch.float32))
  d.qvel.copy_(torch.as_tensor(qvel, dtype=torch.float32))
  if mjm.nu:
    d.ctrl.copy_(torch.as_tensor(ctrl, dtype=torch.float32))
  if warmstart is not None:
    d.qacc_warmstart.copy_(torch.as_tensor(warmstart, dtype=torch.float32))
  return d


def oracle(mjm, qpos, qvel, ctrl, precision=64, warmstart=None):
  from oracle import Oracle

  o = Oracle(mjm, qpos.shape[0], precision)
  o.set("qpos", qpos)
  o.set("qvel", qvel)
  if mjm.nu:
    o.set("ctrl", ctrl)
  if warmstart is not None:
    o.set("qacc_warmstart", warmstart)
  return o


def dev(t):
  return t.detach().cpu().numpy().astype(np.float64).reshape(t.shape[0], -1)


def world_rows(d, kind):
  """Per-world row arrays of the device's flat pairs / contacts / efc rows in world order."""
  if kind == "pair":
    adr, n = d.world_pairadr.cpu().numpy(), d.world_npair.cpu().numpy()
  elif kind == "contact":
    adr, n = d.world_conadr.cpu().numpy(), d.world_ncon.cpu().numpy()
  else:
    adr, n = d.world_efcadr.cpu().numpy(), d.world_nefc.cpu().numpy()
  idx = np.concatenate([np.arange(a, a + k) for a, k in zip(adr, n)]) if n.sum() else np.zeros(0, int)
  return n, idx


def assert_close(a, b, name, rtol=5e-4, atol=5e-4):
  np.testing.assert_allclose(a, b, rtol=rtol, atol=atol, err_msg=f"mismatch: {name}")


def rel_err(a, b):
  """Per-world relative error ||a - b|| / max(||b||, 1)."""
  a = np.asarray(a, dtype=np.float64).reshape(a.shape[0], -1)
  b = np.asarray(b, dtype=np.float64).reshape(b.shape[0], -1)
  return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1.0)
