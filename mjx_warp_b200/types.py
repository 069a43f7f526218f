"""Enums, constants and the device-side Model / Data containers.

The enum values are MuJoCo's (mjtDisableBit, mjtTrn, mjtDyn, mjtGain, mjtBias, mjtJoint,
mjtCone, mjtIntegrator, mjtGeom, mjtSolver), the same values the reference re-exports in
mujoco_warp/_src/types.py:27-201.  Model and Data keep the reference's field names and logical
shapes (mujoco_warp/_src/types.py:366-800); every array is a torch tensor, structured element
types (vec3, quat, mat33, spatial_vector, vec5, vec10) become trailing dimensions.
"""

from __future__ import annotations

import dataclasses
import enum
from typing import Any, Dict

import numpy as np
import torch

# mujoco.mjMINVAL / mjMINIMP / mjMAXIMP / mjNREF / mjNIMP (types.py:20-24)
MJ_MINVAL = 1e-15
MJ_MINIMP = 0.0001
MJ_MAXIMP = 0.9999
MJ_NREF = 2
MJ_NIMP = 5


class DisableBit(enum.IntFlag):
  """Disable default feature bitflags (mjtDisableBit; types.py:27-53)."""

  CONSTRAINT = 1 << 0
  EQUALITY = 1 << 1
  FRICTIONLOSS = 1 << 2
  LIMIT = 1 << 3
  CONTACT = 1 << 4
  PASSIVE = 1 << 5
  GRAVITY = 1 << 6
  CLAMPCTRL = 1 << 7
  WARMSTART = 1 << 8
  FILTERPARENT = 1 << 9
  ACTUATION = 1 << 10
  REFSAFE = 1 << 11
  SENSOR = 1 << 12
  MIDPHASE = 1 << 13
  EULERDAMP = 1 << 14


class TrnType(enum.IntEnum):
  """Actuator transmission type (types.py:56-66)."""

  JOINT = 0
  JOINTINPARENT = 1


class DynType(enum.IntEnum):
  """Actuator dynamics type (types.py:69-79)."""

  NONE = 0
  FILTEREXACT = 3


class GainType(enum.IntEnum):
  """Actuator gain type (types.py:82-92)."""

  FIXED = 0
  AFFINE = 1


class BiasType(enum.IntEnum):
  """Actuator bias type (types.py:95-105)."""

  NONE = 0
  AFFINE = 1


class JointType(enum.IntEnum):
  """Type of degree of freedom (types.py:108-127)."""

  FREE = 0
  BALL = 1
  SLIDE = 2
  HINGE = 3

  def dof_width(self) -> int:
    return {0: 6, 1: 3, 2: 1, 3: 1}[self.value]

  def qpos_width(self) -> int:
    return {0: 7, 1: 4, 2: 1, 3: 1}[self.value]


class ConeType(enum.IntEnum):
  """Friction cone type (types.py:130-138)."""

  PYRAMIDAL = 0


class IntegratorType(enum.IntEnum):
  """Integrator (types.py:141-151)."""

  EULER = 0
  IMPLICITFAST = 3


class GeomType(enum.IntEnum):
  """Geometry type (types.py:154-169)."""

  PLANE = 0
  SPHERE = 2
  CAPSULE = 3
  BOX = 6


class SolverType(enum.IntEnum):
  """Constraint solver algorithm (types.py:172-182)."""

  CG = 1
  NEWTON = 2


# values of mujoco enums that the reference rejects or never names
MJ_INT_RK4 = 1
MJ_INT_IMPLICIT = 2
MJ_JAC_DENSE = 0
MJ_JAC_SPARSE = 1
MJ_JAC_AUTO = 2
MJ_CONE_ELLIPTIC = 1
MJ_SOL_PGS = 0


class DeviceArray(torch.Tensor):
  """torch.Tensor with a Warp-style ``numpy()`` (device -> host copy).

  Reference callers read results with ``d.qpos.numpy()`` (smooth_test.py:51-61); a plain torch
  CUDA tensor refuses ``numpy()``, so every Model/Data array is wrapped in this subclass.
  """

  def numpy(self, *args, **kwargs):  # noqa: D102
    return torch.Tensor.numpy(self.detach().cpu().as_subclass(torch.Tensor), *args, **kwargs)


def as_device_array(t: torch.Tensor) -> DeviceArray:
  return t.as_subclass(DeviceArray)


@dataclasses.dataclass
class Option:
  """Physics options (types.py:218-250)."""

  timestep: float = 0.002
  impratio: float = 1.0
  tolerance: float = 1e-8
  ls_tolerance: float = 0.01
  gravity: Any = None
  integrator: int = 0
  cone: int = 0
  solver: int = 2
  iterations: int = 100
  ls_iterations: int = 50
  disableflags: int = 0
  is_sparse: bool = False
  ls_parallel: bool = False


@dataclasses.dataclass
class Statistic:
  """Model statistics in qpos0 (types.py:253-261)."""

  meaninertia: float = 1.0


# Data scalars copied into the cached C-ABI view (every other non-tensor field is host-only)
_VIEW_SCALARS = frozenset(("nworld", "nconmax", "njmax"))


class _Struct:
  """Attribute bag whose array fields are torch tensors.

  Assigning an array field (or a capacity) drops the cached C-ABI view of the owning Model/Data
  so it is rebuilt before the next kernel launch (callers may swap arrays, as
  solver_test.py:251-258 does with the reference's Data); host scalars such as ``time`` do not.
  """

  def __init__(self, owner=None):
    object.__setattr__(self, "_owner", owner)

  def __setattr__(self, name, value):
    is_tensor = isinstance(value, torch.Tensor)
    if is_tensor and not isinstance(value, DeviceArray):
      value = as_device_array(value)
    object.__setattr__(self, name, value)
    if not is_tensor and name not in _VIEW_SCALARS:
      return  # host scalars such as time do not enter the C-ABI view
    owner = self.__dict__.get("_owner")
    if owner is not None:
      owner._invalidate()
    elif hasattr(self, "_invalidate"):
      self._invalidate()

  def _invalidate(self):
    object.__setattr__(self, "_view_cache", None)

  def arrays(self) -> Dict[str, torch.Tensor]:
    return {k: v for k, v in self.__dict__.items() if isinstance(v, torch.Tensor)}


class Constraint(_Struct):
  """Constraint (efc) data: flat arrays over njmax rows tagged with worldid (types.py:264-363)."""


class Contact(_Struct):
  """Contact data: flat arrays over nconmax contacts tagged with worldid (types.py:615-645)."""


class Model(_Struct):
  """Read-only model shared by all worlds (types.py:366-612)."""

  def __init__(self):
    super().__init__(None)
    object.__setattr__(self, "_view_cache", None)


class Data(_Struct):
  """Per-world state and intermediates (types.py:648-800)."""

  def __init__(self):
    super().__init__(None)
    object.__setattr__(self, "_view_cache", None)


def np32(x) -> np.ndarray:
  return np.ascontiguousarray(np.asarray(x, dtype=np.float32))


def npi32(x) -> np.ndarray:
  return np.ascontiguousarray(np.asarray(x, dtype=np.int32))
