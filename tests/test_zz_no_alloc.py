"""mjb_implicit_noalloc: the implicitfast integrator for callers that cannot allocate.

A plugin that only receives its operand buffers, or a control loop that may not call cudaMalloc
once it runs, cannot provide the integrator's three per-world work arrays.  This entry point keeps
them in a fixed array inside libmjb200.so instead; the test drives it through the C ABI with
those three MjbData fields set to null and checks that two calls in a row advance the state
exactly as mjb_implicit (with caller-provided work arrays) does.
"""

import ctypes

import numpy as np
import pytest
import torch

import mjx_warp_b200 as mjw
from helpers import device_data, humanoid, humanoid_state
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
  return v


def test_noalloc_matches_implicit_two_calls():
  lib = _lib()
  mjm = humanoid()
  nworld = 64
  qpos, qvel, ctrl = humanoid_state(mjm, nworld, seed=21)
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
  per_world = (2 * mjm.nv * mjm.nv + mjm.nv) * 4
  v.nworld = lib.mjb_implicit_noalloc_max_bytes() // per_world + 1
  rc = lib.mjb_implicit_noalloc(ctypes.byref(_abi.model_view(m)), ctypes.byref(v), _abi.stream())
  assert rc == 4  # MJB_ERR_SCRATCH
  assert b"scratch" in lib.mjb_error_string(rc)
