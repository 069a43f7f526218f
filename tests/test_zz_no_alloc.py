"""mjb_implicit_noalloc: the implicitfast integrator for callers that cannot allocate.

A plugin that only receives its operand buffers, or a control loop that may not call cudaMalloc
once it runs, cannot provide the integrator's four per-world work arrays.  This entry point keeps
them in a fixed array inside libmjb200.so instead; the tests drive it through the C ABI with
those four MjbData fields set to null and check that two calls in a row advance the state
exactly as mjb_implicit (with caller-provided work arrays) does: on the motor-driven humanoid
(damping only) and on the pendula with affine position / velocity actuators, which exercise the
actuator velocity coefficients as well.
"""

import ctypes

import numpy as np
import pytest
import torch

import mjx_warp_b200 as mjw
from helpers import device_data, generic_state, humanoid, humanoid_state, load
from mjx_warp_b200 import _abi

pytestmark = pytest.mark.gpu


def _lib():
  lib = _abi.lib()
  lib.mjb_implicit_noalloc.restype = ctypes.c_int
  lib.mjb_implicit_noalloc.argtypes = [ctypes.POINTER(_abi.MjbModel), ctypes.POINTER(_abi.MjbData),
                                       ctypes.c_void_p]
  lib.mjb_implicit_noalloc_max_bytes.restype = ctypes.c_size_t
  return lib


def _view_without_work_arrays(d):
  v = _abi.MjbData()
  ctypes.pointer(v)[0] = _abi.data_view(d)
  v.qM_integration = None
  v.qLD_integration = None
  v.qfrc_integration = None
  v.act_vel_integration = None
  return v


def _affine_pendula():
  """The pendula with affine gains / biases on the velocity (forward_test.py:148-196's setup)."""
  rng = np.random.default_rng(0)
  mjm = load("pendula.xml", integrator=3)
  mjm.actuator_gainprm[:, 2] = rng.normal(scale=10, size=mjm.nu)
  mjm.actuator_gaintype[3] = 1
  mjm.actuator_gaintype[6] = 1
  mjm.actuator_biastype[0:3] = 1
  mjm.actuator_biastype[4:6] = 1
  mjm.actuator_biasprm[0:3, 2] = -1
  mjm.actuator_biasprm[4:6, 2] = -1
  mjm.actuator_ctrlrange[3:7] = 10.0
  mjm.actuator_gear[:] = 1.0
  nworld = 16
  qpos, _, _ = generic_state(mjm, nworld, 2)
  qvel = rng.uniform(-0.01, 0.01, (nworld, mjm.nv))
  ctrl = rng.normal(scale=10, size=(nworld, mjm.nu))
  return mjm, qpos, qvel, ctrl


def _humanoid():
  mjm = humanoid()
  qpos, qvel, ctrl = humanoid_state(mjm, 64, seed=21)
  return mjm, qpos, qvel, ctrl


@pytest.mark.parametrize("case", ["humanoid", "affine_pendula"])
def test_noalloc_matches_implicit_two_calls(case):
  lib = _lib()
  mjm, qpos, qvel, ctrl = _humanoid() if case == "humanoid" else _affine_pendula()
  assert case == "humanoid" or mjw.put_model(mjm).actuator_affine_bias_gain
  m = mjw.put_model(mjm)
  ref = device_data(mjm, qpos, qvel, ctrl)
  na = device_data(mjm, qpos, qvel, ctrl)
  mjw.forward(m, ref)
  mjw.forward(m, na)
  mv = _abi.model_view(m)
  nav = _view_without_work_arrays(na)
  stream = _abi.stream()
  for call in range(2):
    _abi.check(lib.mjb_implicit(ctypes.byref(mv), ctypes.byref(_abi.data_view(ref)), stream), "implicit")
    _abi.check(lib.mjb_implicit_noalloc(ctypes.byref(mv), ctypes.byref(nav), stream), "implicit_noalloc")
    torch.cuda.synchronize()
    for f in ("qpos", "qvel", "qacc_integration"):
      np.testing.assert_allclose(getattr(na, f).cpu().numpy(), getattr(ref, f).cpu().numpy(),
                                 rtol=5e-4, atol=5e-4, err_msg=f"call {call}: {f}")
  assert np.all(np.isfinite(na.qpos.cpu().numpy()))


def test_noalloc_rejects_oversize_batch():
  lib = _lib()
  mjm = humanoid()
  m = mjw.put_model(mjm)
  d = mjw.make_data(mjm, nworld=1)
  v = _view_without_work_arrays(d)
  per_world = (2 * mjm.nv * mjm.nv + mjm.nv + mjm.nu) * 4
  v.nworld = lib.mjb_implicit_noalloc_max_bytes() // per_world + 1
  rc = lib.mjb_implicit_noalloc(ctypes.byref(_abi.model_view(m)), ctypes.byref(v), _abi.stream())
  assert rc == 4  # MJB_ERR_SCRATCH
  assert b"scratch" in lib.mjb_error_string(rc)
