"""MJCF-subset model compiler: the stand-in for ``mujoco.MjModel.from_xml_*``.

The reference's ``put_model(mjm)`` (mujoco_warp/_src/io.py:24-334) consumes a compiled
``mujoco.MjModel``; ``put_data(mjm, mjd)`` (io.py:509-725) a ``mujoco.MjData``.  MuJoCo is not a
dependency of this package, so this module compiles the MJCF features the reference supports
(plane / sphere / capsule / box geoms; free / ball / slide / hinge joints; motor, position and
velocity actuators with JOINT / JOINTINPARENT transmission; default classes and childclass;
keyframes) into ``MjModel`` / ``MjData`` objects that carry the attribute names ``put_model`` and
``put_data`` read.  ``put_model`` also accepts a real ``mujoco.MjModel`` when one is importable.

The compiler follows MuJoCo's documented modelling conventions (MJCF reference documentation):
- bodies, joints, geoms, sites are numbered in depth-first XML order;
- angles in degrees unless ``<compiler angle="radian">``; euler sequence ``xyz`` (intrinsic);
- ``autolimits`` (default true): a joint / actuator is limited when it has a range;
- body inertia inferred from geoms at density 1000 when no ``<inertial>`` is given;
- ``fromto`` capsules: midpoint position, z axis along the segment, half-length from its length;
- ``mj_setConst`` quantities at qpos0: ``stat.meaninertia`` = mean diagonal of M,
  ``body_invweight0`` = mean translational / rotational diagonal of J M^-1 J^T at the body CoM,
  ``dof_invweight0`` = diagonal of M^-1 (averaged over the translational and rotational parts of
  free joints and over ball joints).
"""

from __future__ import annotations

import copy
import math
import os
import re
import xml.etree.ElementTree as ET
from typing import Dict, List, Optional

import numpy as np

from .types import (GeomType, JointType, MJ_JAC_AUTO, MJ_MINVAL)

_INT_NAMES = {"euler": 0, "rk4": 1, "implicit": 2, "implicitfast": 3}
_CONE_NAMES = {"pyramidal": 0, "elliptic": 1}
_SOLVER_NAMES = {"pgs": 0, "cg": 1, "newton": 2}
_JAC_NAMES = {"dense": 0, "sparse": 1, "auto": 2}
_GEOM_NAMES = {"plane": 0, "hfield": 1, "sphere": 2, "capsule": 3, "ellipsoid": 4,
               "cylinder": 5, "box": 6, "mesh": 7}
_JOINT_NAMES = {"free": 0, "ball": 1, "slide": 2, "hinge": 3}
_DISABLE_FLAGS = {"constraint": 0, "equality": 1, "frictionloss": 2, "limit": 3, "contact": 4,
                  "passive": 5, "gravity": 6, "clampctrl": 7, "warmstart": 8,
                  "filterparent": 9, "actuation": 10, "refsafe": 11, "sensor": 12,
                  "midphase": 13, "eulerdamp": 14}

# built-in element defaults (MJCF reference documentation)
_BUILTIN = {
  "geom": {"type": "sphere", "size": [0.0, 0.0, 0.0], "contype": 1, "conaffinity": 1,
           "condim": 3, "priority": 0, "friction": [1.0, 0.005, 0.0001], "solmix": 1.0,
           "solref": [0.02, 1.0], "solimp": [0.9, 0.95, 0.001, 0.5, 2.0], "margin": 0.0,
           "gap": 0.0, "density": 1000.0, "pos": [0.0, 0.0, 0.0]},
  "joint": {"type": "hinge", "pos": [0.0, 0.0, 0.0], "axis": [0.0, 0.0, 1.0],
            "range": [0.0, 0.0], "limited": "auto", "stiffness": 0.0, "damping": 0.0,
            "armature": 0.0, "margin": 0.0, "ref": 0.0, "springref": 0.0,
            "solreflimit": [0.02, 1.0], "solimplimit": [0.9, 0.95, 0.001, 0.5, 2.0],
            "actuatorfrclimited": "auto", "actuatorfrcrange": [0.0, 0.0]},
  "site": {"pos": [0.0, 0.0, 0.0], "size": [0.005, 0.005, 0.005]},
  "actuator": {"ctrllimited": "auto", "forcelimited": "auto", "actlimited": "auto",
               "ctrlrange": [0.0, 0.0], "forcerange": [0.0, 0.0], "actrange": [0.0, 0.0],
               "gear": [1.0, 0.0, 0.0, 0.0, 0.0, 0.0], "kp": 1.0, "kv": 0.0,
               "gainprm": [1.0] + [0.0] * 9, "biasprm": [0.0] * 10,
               "dynprm": [1.0] + [0.0] * 9, "gaintype": "fixed", "biastype": "none",
               "dyntype": "none"},
}
_VECTOR_ATTRS = {"size", "friction", "solref", "solimp", "pos", "axis", "range", "solreflimit",
                 "solimplimit", "actuatorfrcrange", "ctrlrange", "forcerange", "actrange",
                 "gear", "gainprm", "biasprm", "dynprm", "quat", "euler", "axisangle",
                 "xyaxes", "zaxis", "fromto", "diaginertia", "fullinertia"}
_ORIENT_ATTRS = ("quat", "axisangle", "euler", "xyaxes", "zaxis")
_ACTUATOR_TAGS = ("general", "motor", "position", "velocity")


class MjOption:
  """Subset of mjOption read by put_model (io.py:58-71)."""

  def __init__(self):
    self.timestep = 0.002
    self.impratio = 1.0
    self.tolerance = 1e-8
    self.ls_tolerance = 0.01
    self.gravity = np.array([0.0, 0.0, -9.81])
    self.integrator = 0
    self.cone = 0
    self.solver = 2
    self.iterations = 100
    self.ls_iterations = 50
    self.disableflags = 0
    self.enableflags = 0
    self.jacobian = MJ_JAC_AUTO


class MjStatistic:
  def __init__(self):
    self.meaninertia = 1.0


class MjModel:
  """Compiled model carrying the mujoco.MjModel attribute names that put_model reads."""

  def __init__(self):
    self.opt = MjOption()
    self.stat = MjStatistic()

  def __repr__(self):
    return (f"MjModel(nq={self.nq}, nv={self.nv}, nu={self.nu}, nbody={self.nbody}, "
            f"njnt={self.njnt}, ngeom={self.ngeom})")


class _Contact:
  def __init__(self):
    self.dist = np.zeros(0)
    self.pos = np.zeros((0, 3))
    self.frame = np.zeros((0, 9))
    self.includemargin = np.zeros(0)
    self.friction = np.zeros((0, 5))
    self.solref = np.zeros((0, 2))
    self.solreffriction = np.zeros((0, 2))
    self.solimp = np.zeros((0, 5))
    self.dim = np.zeros(0, dtype=np.int32)
    self.geom = np.zeros((0, 2), dtype=np.int32)
    self.efc_address = np.zeros(0, dtype=np.int32)


class MjData:
  """Host state with the mujoco.MjData attribute names put_data reads (io.py:509-725).

  Derived quantities start at zero; they are filled by running ``forward`` on the device and
  reading back with ``get_data_into``.  ``qM`` and ``qLD`` are kept dense (nv x nv) here, which
  is what the reference's dense path derives from MuJoCo's sparse storage (io.py:549-551).
  """

  def __init__(self, m: MjModel):
    nq, nv, nu, na, nb, nj = m.nq, m.nv, m.nu, m.na, m.nbody, m.njnt
    self.time = 0.0
    self.qpos = m.qpos0.copy()
    self.qvel = np.zeros(nv)
    self.act = np.zeros(na)
    self.ctrl = np.zeros(nu)
    self.qacc = np.zeros(nv)
    self.qacc_warmstart = np.zeros(nv)
    self.qfrc_applied = np.zeros(nv)
    self.xfrc_applied = np.zeros((nb, 6))
    self.mocap_pos = m.body_pos[m.body_mocapid >= 0][np.argsort(m.body_mocapid[m.body_mocapid >= 0])].copy() if m.nmocap else np.zeros((0, 3))
    self.mocap_quat = m.body_quat[m.body_mocapid >= 0][np.argsort(m.body_mocapid[m.body_mocapid >= 0])].copy() if m.nmocap else np.zeros((0, 4))
    self.xpos = np.zeros((nb, 3))
    self.xquat = np.zeros((nb, 4))
    self.xmat = np.zeros((nb, 9))
    self.xipos = np.zeros((nb, 3))
    self.ximat = np.zeros((nb, 9))
    self.xanchor = np.zeros((nj, 3))
    self.xaxis = np.zeros((nj, 3))
    self.geom_xpos = np.zeros((m.ngeom, 3))
    self.geom_xmat = np.zeros((m.ngeom, 9))
    self.site_xpos = np.zeros((m.nsite, 3))
    self.site_xmat = np.zeros((m.nsite, 9))
    self.subtree_com = np.zeros((nb, 3))
    self.cinert = np.zeros((nb, 10))
    self.crb = np.zeros((nb, 10))
    self.cdof = np.zeros((nv, 6))
    self.cvel = np.zeros((nb, 6))
    self.cdof_dot = np.zeros((nv, 6))
    self.qM = np.zeros((nv, nv))
    self.qLD = np.zeros((nv, nv))
    self.qLDiagInv = np.zeros(nv)
    self.actuator_length = np.zeros(nu)
    self.actuator_velocity = np.zeros(nu)
    self.actuator_force = np.zeros(nu)
    self.actuator_moment = np.zeros((nu, nv))
    self.qfrc_bias = np.zeros(nv)
    self.qfrc_spring = np.zeros(nv)
    self.qfrc_damper = np.zeros(nv)
    self.qfrc_passive = np.zeros(nv)
    self.qfrc_actuator = np.zeros(nv)
    self.qfrc_smooth = np.zeros(nv)
    self.qfrc_constraint = np.zeros(nv)
    self.qacc_smooth = np.zeros(nv)
    self.act_dot = np.zeros(na)
    self.ncon = 0
    self.nefc = 0
    self.nl = 0
    self.contact = _Contact()
    self.efc_J = np.zeros((0, nv))
    self.efc_D = np.zeros(0)
    self.efc_pos = np.zeros(0)
    self.efc_aref = np.zeros(0)
    self.efc_force = np.zeros(0)
    self.efc_margin = np.zeros(0)


def mj_resetData(m: MjModel, d: MjData) -> None:
  """Resets the state to qpos0 and zero velocities / controls (mj_resetData)."""
  fresh = MjData(m)
  d.__dict__.update(fresh.__dict__)


def mj_resetDataKeyframe(m: MjModel, d: MjData, key: int) -> None:
  """Resets the state to keyframe ``key`` (mj_resetDataKeyframe)."""
  if key < 0 or key >= m.nkey:
    raise ValueError(f"keyframe {key} out of range (nkey={m.nkey})")
  mj_resetData(m, d)
  d.time = float(m.key_time[key])
  d.qpos[:] = m.key_qpos[key]
  d.qvel[:] = m.key_qvel[key]
  d.act[:] = m.key_act[key]
  d.ctrl[:] = m.key_ctrl[key]


# ----------------------------------------------------------------------------------------------
# rotation helpers (float64)


def _quat_mul(a, b):
  return np.array([
    a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3],
    a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2],
    a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1],
    a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0],
  ])


def _quat_to_mat(q):
  w, x, y, z = q
  return np.array([
    [w * w + x * x - y * y - z * z, 2 * (x * y - w * z), 2 * (x * z + w * y)],
    [2 * (x * y + w * z), w * w - x * x + y * y - z * z, 2 * (y * z - w * x)],
    [2 * (x * z - w * y), 2 * (y * z + w * x), w * w - x * x - y * y + z * z],
  ])


def _mat_to_quat(r):
  # Shepperd's method
  tr = r[0, 0] + r[1, 1] + r[2, 2]
  if tr > 0:
    s = math.sqrt(tr + 1.0) * 2
    q = [0.25 * s, (r[2, 1] - r[1, 2]) / s, (r[0, 2] - r[2, 0]) / s, (r[1, 0] - r[0, 1]) / s]
  elif r[0, 0] > r[1, 1] and r[0, 0] > r[2, 2]:
    s = math.sqrt(1.0 + r[0, 0] - r[1, 1] - r[2, 2]) * 2
    q = [(r[2, 1] - r[1, 2]) / s, 0.25 * s, (r[0, 1] + r[1, 0]) / s, (r[0, 2] + r[2, 0]) / s]
  elif r[1, 1] > r[2, 2]:
    s = math.sqrt(1.0 + r[1, 1] - r[0, 0] - r[2, 2]) * 2
    q = [(r[0, 2] - r[2, 0]) / s, (r[0, 1] + r[1, 0]) / s, 0.25 * s, (r[1, 2] + r[2, 1]) / s]
  else:
    s = math.sqrt(1.0 + r[2, 2] - r[0, 0] - r[1, 1]) * 2
    q = [(r[1, 0] - r[0, 1]) / s, (r[0, 2] + r[2, 0]) / s, (r[1, 2] + r[2, 1]) / s, 0.25 * s]
  q = np.array(q)
  if q[0] < 0:
    q = -q
  return q / np.linalg.norm(q)


def _axis_angle_quat(axis, angle):
  axis = np.asarray(axis, dtype=float)
  n = np.linalg.norm(axis)
  if n < 1e-14:
    return np.array([1.0, 0.0, 0.0, 0.0])
  axis = axis / n
  return np.concatenate([[math.cos(angle / 2)], axis * math.sin(angle / 2)])


def _z_to_quat(vec):
  """Minimal rotation taking the z axis onto ``vec``."""
  vec = np.asarray(vec, dtype=float)
  vec = vec / np.linalg.norm(vec)
  axis = np.cross([0.0, 0.0, 1.0], vec)
  s = np.linalg.norm(axis)
  if s < 1e-10:
    axis = np.array([1.0, 0.0, 0.0])
  else:
    axis = axis / s
  ang = math.atan2(s, vec[2])
  return np.concatenate([[math.cos(ang / 2)], axis * math.sin(ang / 2)])


def _rot_vec(q, v):
  return _quat_to_mat(q) @ v


# ----------------------------------------------------------------------------------------------
# parsing


class _Compiler:

  def __init__(self, root: ET.Element, basedir: Optional[str]):
    self.root = root
    self.basedir = basedir
    comp = root.find("compiler")
    self.degree = True
    self.autolimits = True
    self.eulerseq = "xyz"
    if comp is not None:
      self.degree = comp.get("angle", "degree") == "degree"
      self.autolimits = comp.get("autolimits", "true") == "true"
      self.eulerseq = comp.get("eulerseq", "xyz")
    # default classes: name -> (parent name, {tag: attrs})
    self.classes: Dict[str, tuple] = {"main": (None, {})}
    for node in root.findall("default"):
      self._parse_default(node, None)

  # defaults ---------------------------------------------------------------------------------

  def _parse_default(self, node, parent):
    name = node.get("class", "main")
    attrs = {}
    for child in node:
      if child.tag == "default":
        continue
      tag = "actuator" if child.tag in _ACTUATOR_TAGS else child.tag
      attrs.setdefault(tag, {}).update(child.attrib)
      if child.tag in _ACTUATOR_TAGS:
        attrs[tag]["_shortcut"] = child.tag
    if name == "main" and parent is None:
      self.classes["main"] = (None, attrs)
    else:
      self.classes[name] = (parent if parent is not None else "main", attrs)
    for child in node:
      if child.tag == "default":
        self._parse_default(child, name)

  def _chain(self, cls):
    chain = []
    while cls is not None:
      if cls not in self.classes:
        raise ValueError(f"unknown default class '{cls}'")
      parent, attrs = self.classes[cls]
      chain.append(attrs)
      cls = parent
    return list(reversed(chain))

  def resolve(self, tag: str, elem: ET.Element, childclass: Optional[str]) -> dict:
    """Resolved attributes: built-in <- class chain <- element (vectors overlay partially)."""
    cls = elem.get("class", childclass or "main")
    out = copy.deepcopy(_BUILTIN.get(tag, {}))
    layers = [layer.get(tag, {}) for layer in self._chain(cls)] + [dict(elem.attrib)]
    orient_src = None
    for li, layer in enumerate(layers):
      if any(k in layer for k in _ORIENT_ATTRS):
        orient_src = li
      for k, v in layer.items():
        if k in ("class", "name", "childclass"):
          continue
        if k in _VECTOR_ATTRS:
          vals = [float(x) for x in v.split()]
          base = out.get(k)
          if isinstance(base, list) and k not in _ORIENT_ATTRS and k != "fromto":
            base = list(base)
            base[: len(vals)] = vals
            out[k] = base
          else:
            out[k] = vals
        else:
          out[k] = v
    # only the orientation given by the most specific layer counts
    if orient_src is not None:
      keep = [k for k in _ORIENT_ATTRS if k in layers[orient_src]]
      for k in _ORIENT_ATTRS:
        if k in out and k not in keep:
          del out[k]
    out["_name"] = elem.get("name")
    return out

  # orientation --------------------------------------------------------------------------------

  def _angle(self, a):
    return math.radians(a) if self.degree else a

  def orientation(self, attrs) -> np.ndarray:
    if "quat" in attrs:
      q = np.array(attrs["quat"], dtype=float)
      return q / np.linalg.norm(q)
    if "axisangle" in attrs:
      v = attrs["axisangle"]
      return _axis_angle_quat(v[:3], self._angle(v[3]))
    if "euler" in attrs:
      q = np.array([1.0, 0.0, 0.0, 0.0])
      for ax, ang in zip(self.eulerseq, attrs["euler"]):
        axis = {"x": [1, 0, 0], "y": [0, 1, 0], "z": [0, 0, 1]}[ax.lower()]
        r = _axis_angle_quat(axis, self._angle(ang))
        q = _quat_mul(q, r) if ax.islower() else _quat_mul(r, q)
      return q / np.linalg.norm(q)
    if "xyaxes" in attrs:
      v = attrs["xyaxes"]
      x = np.array(v[:3]) / np.linalg.norm(v[:3])
      y = np.array(v[3:6]) - x * np.dot(x, v[3:6])
      y = y / np.linalg.norm(y)
      z = np.cross(x, y)
      return _mat_to_quat(np.stack([x, y, z], axis=1))
    if "zaxis" in attrs:
      return _z_to_quat(attrs["zaxis"])
    return np.array([1.0, 0.0, 0.0, 0.0])


def _geom_inertia(gtype, size, density, mass_attr):
  """Mass and principal inertia (geom frame) of a solid geom."""
  if gtype == GeomType.SPHERE:
    r = size[0]
    vol = 4.0 / 3.0 * math.pi * r ** 3
    mass = density * vol if mass_attr is None else mass_attr
    i = 0.4 * mass * r * r
    return mass, np.array([i, i, i])
  if gtype == GeomType.CAPSULE:
    r, h = size[0], size[1]
    height = 2.0 * h
    vs = 4.0 / 3.0 * math.pi * r ** 3
    vc = math.pi * r * r * height
    if mass_attr is not None:
      dens = mass_attr / (vs + vc)
    else:
      dens = density
    ms, mc = dens * vs, dens * vc
    mass = ms + mc
    # cylinder about its centre + two hemispheres displaced to the cylinder ends
    ixy = mc * (3 * r * r + height * height) / 12.0 + ms * (0.4 * r * r + 0.25 * height * height + 0.375 * height * r)
    iz = mc * r * r / 2.0 + ms * 0.4 * r * r
    return mass, np.array([ixy, ixy, iz])
  if gtype == GeomType.BOX:
    a, b, c = size
    vol = 8.0 * a * b * c
    mass = density * vol if mass_attr is None else mass_attr
    return mass, mass / 3.0 * np.array([b * b + c * c, a * a + c * c, a * a + b * b])
  return 0.0, np.zeros(3)


def _rbound(gtype, size):
  if gtype == GeomType.SPHERE:
    return size[0]
  if gtype == GeomType.CAPSULE:
    return size[0] + size[1]
  if gtype == GeomType.BOX:
    return float(np.linalg.norm(size))
  return 0.0


def _aabb(gtype, size):
  if gtype == GeomType.SPHERE:
    return [0, 0, 0, size[0], size[0], size[0]]
  if gtype == GeomType.CAPSULE:
    return [0, 0, 0, size[0], size[0], size[0] + size[1]]
  if gtype == GeomType.BOX:
    return [0, 0, 0, size[0], size[1], size[2]]
  return [0, 0, 0, 0, 0, 0]


def _sanitize(xml: str) -> str:
  # tolerate two slips that MuJoCo's XML reader accepts: the single-dash comment ``<!- ... -->``
  # and a missing space between attributes (``type="ball"solreflimit=...``)
  xml = re.sub(r"<!-(?!-)[\s\S]*?-->", "", xml)
  return re.sub(r'(?<![=\s])"(?=[A-Za-z_])', '" ', xml)


def from_xml_string(xml: str, basedir: Optional[str] = None) -> MjModel:
  """Compiles an MJCF string into an MjModel."""
  root = ET.fromstring(_sanitize(xml))
  if root.tag != "mujoco":
    raise ValueError("root element must be <mujoco>")
  return _compile(root, basedir)


def from_xml_path(path: str) -> MjModel:
  """Compiles an MJCF file into an MjModel."""
  with open(path) as f:
    return from_xml_string(f.read(), os.path.dirname(os.path.abspath(path)))


def _compile(root: ET.Element, basedir) -> MjModel:
  c = _Compiler(root, basedir)
  m = MjModel()
  m.model_name = root.get("model", "")

  # options ------------------------------------------------------------------------------------
  opt = root.find("option")
  if opt is not None:
    f = lambda k, d: float(opt.get(k)) if opt.get(k) is not None else d  # noqa: E731
    m.opt.timestep = f("timestep", m.opt.timestep)
    m.opt.impratio = f("impratio", m.opt.impratio)
    m.opt.tolerance = f("tolerance", m.opt.tolerance)
    m.opt.ls_tolerance = f("ls_tolerance", m.opt.ls_tolerance)
    if opt.get("gravity") is not None:
      m.opt.gravity = np.array([float(x) for x in opt.get("gravity").split()])
    if opt.get("integrator") is not None:
      m.opt.integrator = _INT_NAMES[opt.get("integrator").lower()]
    if opt.get("cone") is not None:
      m.opt.cone = _CONE_NAMES[opt.get("cone").lower()]
    if opt.get("solver") is not None:
      m.opt.solver = _SOLVER_NAMES[opt.get("solver").lower()]
    if opt.get("jacobian") is not None:
      m.opt.jacobian = _JAC_NAMES[opt.get("jacobian").lower()]
    m.opt.iterations = int(f("iterations", m.opt.iterations))
    m.opt.ls_iterations = int(f("ls_iterations", m.opt.ls_iterations))
    flag = opt.find("flag")
    if flag is not None:
      for k, v in flag.attrib.items():
        if k in _DISABLE_FLAGS and v == "disable":
          m.opt.disableflags |= 1 << _DISABLE_FLAGS[k]

  # kinematic tree -----------------------------------------------------------------------------
  bodies: List[dict] = []
  joints: List[dict] = []
  geoms: List[dict] = []
  sites: List[dict] = []
  name2body: Dict[str, int] = {}
  name2jnt: Dict[str, int] = {}

  def add_body(elem, parent, childclass, is_world=False):
    bid = len(bodies)
    b = {"id": bid, "parent": parent, "name": elem.get("name", "world" if is_world else None),
         "pos": np.zeros(3), "quat": np.array([1.0, 0, 0, 0]), "mocap": False,
         "joints": [], "geoms": [], "sites": [], "inertial": None}
    if not is_world:
      attrs = {k: [float(x) for x in v.split()] if k in _VECTOR_ATTRS else v
               for k, v in elem.attrib.items()}
      b["pos"] = np.array(attrs.get("pos", [0.0, 0.0, 0.0]), dtype=float)
      b["quat"] = c.orientation(attrs)
      b["mocap"] = elem.get("mocap", "false") == "true"
      childclass = elem.get("childclass", childclass)
    bodies.append(b)
    if b["name"]:
      name2body[b["name"]] = bid
    for ch in elem:
      if ch.tag in ("joint", "freejoint"):
        if is_world:
          raise ValueError("joints cannot be attached to the world body")
        if ch.tag == "freejoint":
          a = {"type": "free", "pos": [0.0, 0.0, 0.0], "axis": [0.0, 0.0, 1.0],
               "range": [0.0, 0.0], "limited": "false", "stiffness": 0.0, "damping": 0.0,
               "armature": 0.0, "margin": 0.0, "ref": 0.0, "springref": 0.0,
               "solreflimit": [0.02, 1.0], "solimplimit": [0.9, 0.95, 0.001, 0.5, 2.0],
               "actuatorfrclimited": "false", "actuatorfrcrange": [0.0, 0.0],
               "_name": ch.get("name")}
        else:
          a = c.resolve("joint", ch, childclass)
        a["body"] = bid
        b["joints"].append(len(joints))
        if a["_name"]:
          name2jnt[a["_name"]] = len(joints)
        joints.append(a)
      elif ch.tag == "geom":
        a = c.resolve("geom", ch, childclass)
        a["body"] = bid
        b["geoms"].append(len(geoms))
        geoms.append(a)
      elif ch.tag == "site":
        a = c.resolve("site", ch, childclass)
        a["body"] = bid
        b["sites"].append(len(sites))
        sites.append(a)
      elif ch.tag == "inertial":
        b["inertial"] = {k: [float(x) for x in v.split()] if k in _VECTOR_ATTRS else v
                         for k, v in ch.attrib.items()}
    for ch in elem:
      if ch.tag == "body":
        add_body(ch, bid, childclass)

  wb = root.find("worldbody")
  if wb is None:
    wb = ET.Element("worldbody")
  add_body(wb, -1, None, is_world=True)
  # bodies must be ordered depth first: add_body recursed after listing its own elements, which
  # numbers children after the parent's geoms; re-derive geoms / joints / sites in body order.
  order_j = [j for b in bodies for j in b["joints"]]
  order_g = [g for b in bodies for g in b["geoms"]]
  order_s = [s for b in bodies for s in b["sites"]]
  joints = [joints[i] for i in order_j]
  geoms = [geoms[i] for i in order_g]
  sites = [sites[i] for i in order_s]
  name2jnt = {a["_name"]: i for i, a in enumerate(joints) if a["_name"]}

  nbody = len(bodies)
  njnt = len(joints)
  ngeom = len(geoms)
  nsite = len(sites)

  m.nbody, m.njnt, m.ngeom, m.nsite = nbody, njnt, ngeom, nsite
  m.body_names = [b["name"] for b in bodies]
  m.jnt_names = [j["_name"] for j in joints]
  m.geom_names = [g["_name"] for g in geoms]
  m.site_names = [s["_name"] for s in sites]

  # bodies
  m.body_parentid = np.array([max(b["parent"], 0) for b in bodies], dtype=np.int32)
  m.body_pos = np.array([b["pos"] for b in bodies])
  m.body_quat = np.array([b["quat"] for b in bodies])
  mocap = [b["id"] for b in bodies if b["mocap"]]
  m.nmocap = len(mocap)
  m.body_mocapid = np.full(nbody, -1, dtype=np.int32)
  for i, bid in enumerate(mocap):
    m.body_mocapid[bid] = i

  # joints, dofs, qpos
  jnt_type = np.array([_JOINT_NAMES[j["type"]] for j in joints], dtype=np.int32)
  m.jnt_type = jnt_type
  m.jnt_bodyid = np.array([j["body"] for j in joints], dtype=np.int32)
  qposadr, dofadr, nq, nv = [], [], 0, 0
  for t in jnt_type:
    qposadr.append(nq)
    dofadr.append(nv)
    nq += JointType(int(t)).qpos_width()
    nv += JointType(int(t)).dof_width()
  m.nq, m.nv = nq, nv
  m.jnt_qposadr = np.array(qposadr, dtype=np.int32)
  m.jnt_dofadr = np.array(dofadr, dtype=np.int32)
  m.jnt_pos = np.array([j["pos"] for j in joints]).reshape(njnt, 3)
  axes = []
  for j in joints:
    a = np.array(j["axis"], dtype=float)
    axes.append(a / np.linalg.norm(a))
  m.jnt_axis = np.array(axes).reshape(njnt, 3)
  m.jnt_stiffness = np.array([float(j["stiffness"]) for j in joints])
  m.jnt_margin = np.array([float(j["margin"]) for j in joints])
  m.jnt_solref = np.array([j["solreflimit"] for j in joints]).reshape(njnt, 2)
  m.jnt_solimp = np.array([j["solimplimit"] for j in joints]).reshape(njnt, 5)
  rng, lim = [], []
  for j, t in zip(joints, jnt_type):
    r = np.array(j["range"], dtype=float)
    if t in (JointType.HINGE, JointType.BALL):
      r = np.array([c._angle(x) for x in r])
    rng.append(r)
    limited = j["limited"]
    if limited == "auto":
      limited = c.autolimits and (r[0] != 0 or r[1] != 0)
    else:
      limited = limited == "true"
    lim.append(int(bool(limited)))
  m.jnt_range = np.array(rng).reshape(njnt, 2)
  m.jnt_limited = np.array(lim, dtype=np.int32)
  afl, afr = [], []
  for j in joints:
    r = np.array(j["actuatorfrcrange"], dtype=float)
    limited = j["actuatorfrclimited"]
    if limited == "auto":
      limited = c.autolimits and (r[0] != 0 or r[1] != 0)
    else:
      limited = limited == "true"
    afl.append(int(bool(limited)))
    afr.append(r)
  m.jnt_actfrclimited = np.array(afl, dtype=np.int32)
  m.jnt_actfrcrange = np.array(afr).reshape(njnt, 2)

  # bodies: joint / dof address tables
  m.body_jntnum = np.array([len(b["joints"]) for b in bodies], dtype=np.int32)
  m.body_jntadr = np.full(nbody, -1, dtype=np.int32)
  m.body_dofnum = np.zeros(nbody, dtype=np.int32)
  m.body_dofadr = np.full(nbody, -1, dtype=np.int32)
  jcount = 0
  for b in bodies:
    if b["joints"]:
      m.body_jntadr[b["id"]] = jcount
      m.body_dofadr[b["id"]] = dofadr[jcount]
      m.body_dofnum[b["id"]] = sum(JointType(int(jnt_type[jcount + k])).dof_width()
                                   for k in range(len(b["joints"])))
      jcount += len(b["joints"])

  dof_bodyid, dof_jntid = [], []
  for ji, t in enumerate(jnt_type):
    for _ in range(JointType(int(t)).dof_width()):
      dof_bodyid.append(m.jnt_bodyid[ji])
      dof_jntid.append(ji)
  m.dof_bodyid = np.array(dof_bodyid, dtype=np.int32)
  m.dof_jntid = np.array(dof_jntid, dtype=np.int32)
  # dof_parentid: previous dof of the same body, else last dof of the nearest ancestor with dofs
  dof_parentid = np.full(nv, -1, dtype=np.int32)
  for b in range(1, nbody):
    if m.body_dofnum[b] == 0:
      continue
    adr = m.body_dofadr[b]
    p = m.body_parentid[b]
    while p > 0 and m.body_dofnum[p] == 0:
      p = m.body_parentid[p]
    dof_parentid[adr] = m.body_dofadr[p] + m.body_dofnum[p] - 1 if p > 0 else -1
    for k in range(1, m.body_dofnum[b]):
      dof_parentid[adr + k] = adr + k - 1
  m.dof_parentid = dof_parentid
  madr, adr = [], 0
  for i in range(nv):
    madr.append(adr)
    depth, j = 0, dof_parentid[i]
    while j >= 0:
      depth += 1
      j = dof_parentid[j]
    adr += depth + 1
  m.dof_Madr = np.array(madr, dtype=np.int32)
  m.nM = adr
  dof_arm, dof_damp = [], []
  for j, t in zip(joints, jnt_type):
    for _ in range(JointType(int(t)).dof_width()):
      dof_arm.append(float(j["armature"]))
      dof_damp.append(float(j["damping"]))
  m.dof_armature = np.array(dof_arm)
  m.dof_damping = np.array(dof_damp)
  m.dof_frictionloss = np.zeros(nv)

  # root / weld / tree ids
  m.body_rootid = np.zeros(nbody, dtype=np.int32)
  m.body_weldid = np.zeros(nbody, dtype=np.int32)
  for b in range(1, nbody):
    p = m.body_parentid[b]
    m.body_rootid[b] = b if p == 0 else m.body_rootid[p]
    m.body_weldid[b] = b if m.body_jntnum[b] > 0 else m.body_weldid[p]
  m.body_treeid = np.full(nbody, -1, dtype=np.int32)
  ntree = 0
  roots_with_dofs = {}
  for b in range(1, nbody):
    r = m.body_rootid[b]
    # a tree is a child-of-world subtree that has dofs
    has = False
    bb = b
    while bb > 0:
      if m.body_dofnum[bb] > 0:
        has = True
        break
      bb = m.body_parentid[bb]
    if not has:
      # static body unless a descendant-independent chain has dofs (MuJoCo: -1 for static)
      continue
    if r not in roots_with_dofs:
      roots_with_dofs[r] = ntree
      ntree += 1
    m.body_treeid[b] = roots_with_dofs[r]
  m.ntree = ntree
  m.dof_treeid = np.array([m.body_treeid[b] for b in m.dof_bodyid], dtype=np.int32)

  # qpos0 / qpos_spring
  qpos0 = np.zeros(nq)
  qpos_spring = np.zeros(nq)
  for ji, (j, t) in enumerate(zip(joints, jnt_type)):
    a = qposadr[ji]
    if t == JointType.FREE:
      b = bodies[j["body"]]
      qpos0[a:a + 3] = b["pos"]
      qpos0[a + 3:a + 7] = b["quat"]
      qpos_spring[a:a + 7] = qpos0[a:a + 7]
    elif t == JointType.BALL:
      qpos0[a:a + 4] = [1, 0, 0, 0]
      qpos_spring[a:a + 4] = [1, 0, 0, 0]
    else:
      ref = float(j["ref"])
      if t == JointType.HINGE:
        ref = c._angle(ref)
      qpos0[a] = ref
      sref = float(j["springref"])
      qpos_spring[a] = c._angle(sref) if t == JointType.HINGE else sref
  m.qpos0 = qpos0
  m.qpos_spring = qpos_spring

  # geoms -------------------------------------------------------------------------------------
  g_type, g_size, g_pos, g_quat = [], [], [], []
  for g in geoms:
    t = _GEOM_NAMES[g["type"]]
    size = np.array(g["size"], dtype=float)
    if "fromto" in g and t in (GeomType.CAPSULE, GeomType.BOX, GeomType.CYLINDER if hasattr(GeomType, "CYLINDER") else -1):
      ft = np.array(g["fromto"], dtype=float)
      p0, p1 = ft[:3], ft[3:]
      pos = 0.5 * (p0 + p1)
      d = p1 - p0
      half = 0.5 * np.linalg.norm(d)
      quat = _z_to_quat(d)
      if t == GeomType.CAPSULE:
        size[1] = half
      else:
        if size[1] == 0:
          size[1] = size[0]
        size[2] = half
    else:
      pos = np.array(g["pos"], dtype=float)
      quat = c.orientation(g)
    if t == GeomType.BOX and size[1] == 0 and size[2] == 0:
      size[1] = size[2] = size[0]
    g_type.append(t)
    g_size.append(size)
    g_pos.append(pos)
    g_quat.append(quat)
  m.geom_type = np.array(g_type, dtype=np.int32)
  m.geom_size = np.array(g_size).reshape(ngeom, 3)
  m.geom_pos = np.array(g_pos).reshape(ngeom, 3)
  m.geom_quat = np.array(g_quat).reshape(ngeom, 4)
  m.geom_bodyid = np.array([g["body"] for g in geoms], dtype=np.int32)
  m.geom_contype = np.array([int(g["contype"]) for g in geoms], dtype=np.int32)
  m.geom_conaffinity = np.array([int(g["conaffinity"]) for g in geoms], dtype=np.int32)
  m.geom_condim = np.array([int(g["condim"]) for g in geoms], dtype=np.int32)
  m.geom_priority = np.array([int(g["priority"]) for g in geoms], dtype=np.int32)
  m.geom_solmix = np.array([float(g["solmix"]) for g in geoms])
  m.geom_solref = np.array([g["solref"] for g in geoms]).reshape(ngeom, 2)
  m.geom_solimp = np.array([g["solimp"] for g in geoms]).reshape(ngeom, 5)
  m.geom_friction = np.array([g["friction"] for g in geoms]).reshape(ngeom, 3)
  m.geom_margin = np.array([float(g["margin"]) for g in geoms])
  m.geom_gap = np.array([float(g["gap"]) for g in geoms])
  m.geom_rbound = np.array([_rbound(t, s) for t, s in zip(g_type, g_size)])
  m.geom_aabb = np.array([_aabb(t, s) for t, s in zip(g_type, g_size)], dtype=float).reshape(ngeom, 6)
  m.geom_dataid = np.full(ngeom, -1, dtype=np.int32)
  m.body_geomnum = np.array([len(b["geoms"]) for b in bodies], dtype=np.int32)
  m.body_geomadr = np.full(nbody, -1, dtype=np.int32)
  gcount = 0
  for b in bodies:
    if b["geoms"]:
      m.body_geomadr[b["id"]] = gcount
      gcount += len(b["geoms"])
  m.body_contype = np.zeros(nbody, dtype=np.int32)
  m.body_conaffinity = np.zeros(nbody, dtype=np.int32)
  for gi in range(ngeom):
    m.body_contype[m.geom_bodyid[gi]] |= m.geom_contype[gi]
    m.body_conaffinity[m.geom_bodyid[gi]] |= m.geom_conaffinity[gi]
  m.mesh_vertadr = np.zeros(0, dtype=np.int32)
  m.mesh_vertnum = np.zeros(0, dtype=np.int32)
  m.mesh_vert = np.zeros((0, 3))

  # sites
  m.site_bodyid = np.array([s["body"] for s in sites], dtype=np.int32)
  m.site_pos = np.array([s["pos"] for s in sites], dtype=float).reshape(nsite, 3)
  m.site_quat = np.array([c.orientation(s) for s in sites]).reshape(nsite, 4)

  # body inertia --------------------------------------------------------------------------------
  m.body_mass = np.zeros(nbody)
  m.body_inertia = np.zeros((nbody, 3))
  m.body_ipos = np.zeros((nbody, 3))
  m.body_iquat = np.tile([1.0, 0, 0, 0], (nbody, 1))
  for b in bodies[1:]:
    bid = b["id"]
    if b["inertial"] is not None:
      it = b["inertial"]
      m.body_mass[bid] = float(it["mass"])
      m.body_ipos[bid] = np.array(it.get("pos", [0, 0, 0]), dtype=float)
      if "fullinertia" in it:
        fi = it["fullinertia"]
        full = np.array([[fi[0], fi[3], fi[4]], [fi[3], fi[1], fi[5]], [fi[4], fi[5], fi[2]]])
        w, v = np.linalg.eigh(full)
        if np.linalg.det(v) < 0:
          v[:, 2] = -v[:, 2]
        m.body_inertia[bid] = w
        m.body_iquat[bid] = _mat_to_quat(v)
      else:
        m.body_inertia[bid] = np.array(it.get("diaginertia", [0, 0, 0]), dtype=float)
        m.body_iquat[bid] = c.orientation(it)
      continue
    items = []
    for gi in b["geoms"]:
      g = geoms[gi]
      t = m.geom_type[gi]
      if t == GeomType.PLANE:
        continue
      mass_attr = float(g["mass"]) if "mass" in g else None
      gm, gi_diag = _geom_inertia(t, m.geom_size[gi], float(g["density"]), mass_attr)
      items.append((gm, gi_diag, m.geom_pos[gi], m.geom_quat[gi]))
    if not items:
      continue
    if len(items) == 1:
      gm, gi_diag, gp, gq = items[0]
      m.body_mass[bid] = gm
      m.body_inertia[bid] = gi_diag
      m.body_ipos[bid] = gp
      m.body_iquat[bid] = gq
      continue
    mass = sum(it[0] for it in items)
    com = sum(it[0] * it[2] for it in items) / mass
    inert = np.zeros((3, 3))
    for gm, gi_diag, gp, gq in items:
      r = _quat_to_mat(gq)
      d = gp - com
      inert += r @ np.diag(gi_diag) @ r.T + gm * (np.dot(d, d) * np.eye(3) - np.outer(d, d))
    w, v = np.linalg.eigh(inert)
    if np.linalg.det(v) < 0:
      v[:, 2] = -v[:, 2]
    m.body_mass[bid] = mass
    m.body_inertia[bid] = w
    m.body_ipos[bid] = com
    m.body_iquat[bid] = _mat_to_quat(v)
  m.body_subtreemass = m.body_mass.copy()
  for b in range(nbody - 1, 0, -1):
    m.body_subtreemass[m.body_parentid[b]] += m.body_subtreemass[b]

  # actuators -----------------------------------------------------------------------------------
  acts = []
  act_elem = root.find("actuator")
  if act_elem is not None:
    for ae in act_elem:
      if ae.tag not in _ACTUATOR_TAGS:
        raise NotImplementedError(f"actuator <{ae.tag}> is unsupported")
      a = c.resolve("actuator", ae, None)
      a["_tag"] = ae.tag
      acts.append(a)
  nu = len(acts)
  m.nu = nu
  m.na = 0
  trntype, trnid, gear = [], [], []
  gaintype, biastype, dyntype, gainprm, biasprm, dynprm = [], [], [], [], [], []
  ctrllim, ctrlrange, forcelim, forcerange, actlim, actrange = [], [], [], [], [], []
  for a in acts:
    if "joint" in a:
      trntype.append(0)
      trnid.append([name2jnt[a["joint"]], -1])
    elif "jointinparent" in a:
      trntype.append(1)
      trnid.append([name2jnt[a["jointinparent"]], -1])
    else:
      raise NotImplementedError("only joint / jointinparent transmissions are supported")
    gear.append(np.array(a["gear"], dtype=float))
    gp = list(a["gainprm"])
    bp = list(a["biasprm"])
    tag = a["_tag"]
    if tag == "motor":
      gt, bt, gp, bp = 0, 0, [1.0] + [0.0] * 9, [0.0] * 10
    elif tag == "position":
      kp, kv = float(a["kp"]), float(a["kv"])
      gt, bt, gp, bp = 0, 1, [kp] + [0.0] * 9, [0.0, -kp, -kv] + [0.0] * 7
    elif tag == "velocity":
      kv = float(a["kv"]) if "kv" in a else 1.0
      gt, bt, gp, bp = 0, 1, [kv] + [0.0] * 9, [0.0, 0.0, -kv] + [0.0] * 7
    else:
      gt = {"fixed": 0, "affine": 1}[a["gaintype"]]
      bt = {"none": 0, "affine": 1}[a["biastype"]]
    if a.get("dyntype", "none") not in ("none",) and tag == "general":
      raise NotImplementedError("actuator dynamics other than none are unsupported")
    gaintype.append(gt)
    biastype.append(bt)
    dyntype.append(0)
    gainprm.append(gp)
    biasprm.append(bp)
    dynprm.append(list(a["dynprm"]))
    for lim_name, rng_name, lims, rngs in (("ctrllimited", "ctrlrange", ctrllim, ctrlrange),
                                           ("forcelimited", "forcerange", forcelim, forcerange),
                                           ("actlimited", "actrange", actlim, actrange)):
      r = np.array(a[rng_name], dtype=float)
      lv = a[lim_name]
      if lv == "auto":
        lv = c.autolimits and (r[0] != 0 or r[1] != 0)
      else:
        lv = lv == "true"
      lims.append(int(bool(lv)))
      rngs.append(r)
  m.actuator_trntype = np.array(trntype, dtype=np.int32)
  m.actuator_trnid = np.array(trnid, dtype=np.int32).reshape(nu, 2)
  m.actuator_gear = np.array(gear, dtype=float).reshape(nu, 6)
  m.actuator_gaintype = np.array(gaintype, dtype=np.int32)
  m.actuator_biastype = np.array(biastype, dtype=np.int32)
  m.actuator_dyntype = np.array(dyntype, dtype=np.int32)
  m.actuator_gainprm = np.array(gainprm, dtype=float).reshape(nu, 10)
  m.actuator_biasprm = np.array(biasprm, dtype=float).reshape(nu, 10)
  m.actuator_dynprm = np.array(dynprm, dtype=float).reshape(nu, 10)
  m.actuator_ctrllimited = np.array(ctrllim, dtype=np.int32)
  m.actuator_ctrlrange = np.array(ctrlrange, dtype=float).reshape(nu, 2)
  m.actuator_forcelimited = np.array(forcelim, dtype=np.int32)
  m.actuator_forcerange = np.array(forcerange, dtype=float).reshape(nu, 2)
  m.actuator_actlimited = np.array(actlim, dtype=np.int32)
  m.actuator_actrange = np.array(actrange, dtype=float).reshape(nu, 2)
  m.actuator_actadr = np.full(nu, -1, dtype=np.int32)
  m.actuator_actnum = np.zeros(nu, dtype=np.int32)
  m.actuator_names = [a["_name"] for a in acts]

  # features the reference rejects: counted so put_model can raise like io.py:25-32 ------------
  eq = root.find("equality")
  m.neq = len(list(eq)) if eq is not None else 0
  sens = root.find("sensor")
  m.nsensor = len(list(sens)) if sens is not None else 0
  ten = root.find("tendon")
  m.ntendon = len(list(ten)) if ten is not None else 0
  con = root.find("contact")
  excl = [e for e in con if e.tag == "exclude"] if con is not None else []
  m.nexclude = len(excl)
  sig = []
  for e in excl:
    b1, b2 = name2body[e.get("body1")], name2body[e.get("body2")]
    sig.append((min(b1, b2) << 16) + max(b1, b2))
  m.exclude_signature = np.array(sig, dtype=np.int32)

  # keyframes
  keys = root.find("keyframe")
  kl = [k for k in keys if k.tag == "key"] if keys is not None else []
  m.nkey = len(kl)
  m.key_names = [k.get("name") for k in kl]
  m.key_time = np.array([float(k.get("time", 0.0)) for k in kl])

  def kv(k, attr, n, default):
    v = k.get(attr)
    if v is None:
      return np.array(default, dtype=float)
    arr = np.array([float(x) for x in v.split()])
    if arr.size != n:
      raise ValueError(f"keyframe {attr} has {arr.size} values, expected {n}")
    return arr

  m.key_qpos = np.array([kv(k, "qpos", nq, qpos0) for k in kl]).reshape(len(kl), nq)
  m.key_qvel = np.array([kv(k, "qvel", nv, np.zeros(nv)) for k in kl]).reshape(len(kl), nv)
  m.key_act = np.zeros((len(kl), 0))
  m.key_ctrl = np.array([kv(k, "ctrl", nu, np.zeros(nu)) for k in kl]).reshape(len(kl), nu)

  _set_const(m)
  return m


# ----------------------------------------------------------------------------------------------
# mj_setConst at qpos0 (float64)


def _smooth_qpos0(m: MjModel):
  """Kinematics, subtree CoM, cdof and the dense mass matrix at qpos0 (float64, one world)."""
  nb, nv = m.nbody, m.nv
  xpos = np.zeros((nb, 3))
  xquat = np.tile([1.0, 0, 0, 0], (nb, 1))
  xipos = np.zeros((nb, 3))
  ximat = np.tile(np.eye(3), (nb, 1, 1))
  xanchor = np.zeros((m.njnt, 3))
  xaxis = np.zeros((m.njnt, 3))
  q = m.qpos0
  for b in range(1, nb):
    p = m.body_parentid[b]
    pos = _quat_to_mat(xquat[p]) @ m.body_pos[b] + xpos[p]
    quat = _quat_mul(xquat[p], m.body_quat[b])
    for j in range(m.body_jntadr[b], m.body_jntadr[b] + m.body_jntnum[b]):
      a = m.jnt_qposadr[j]
      t = m.jnt_type[j]
      if t == JointType.FREE:
        pos = q[a:a + 3].copy()
        quat = q[a + 3:a + 7].copy()
        xanchor[j] = pos
        xaxis[j] = m.jnt_axis[j]
        continue
      anchor = _rot_vec(quat, m.jnt_pos[j]) + pos
      axis = _rot_vec(quat, m.jnt_axis[j])
      if t == JointType.BALL:
        quat = _quat_mul(quat, q[a:a + 4])
        pos = anchor - _rot_vec(quat, m.jnt_pos[j])
      elif t == JointType.SLIDE:
        pos = pos + axis * (q[a] - m.qpos0[a])
      else:
        quat = _quat_mul(quat, _axis_angle_quat(m.jnt_axis[j], q[a] - m.qpos0[a]))
        pos = anchor - _rot_vec(quat, m.jnt_pos[j])
      xanchor[j] = anchor
      xaxis[j] = axis
    quat = quat / np.linalg.norm(quat)
    xpos[b] = pos
    xquat[b] = quat
    xipos[b] = pos + _rot_vec(quat, m.body_ipos[b])
    ximat[b] = _quat_to_mat(_quat_mul(quat, m.body_iquat[b]))
  # subtree com
  sc = xipos * m.body_mass[:, None]
  smass = m.body_mass.copy()
  for b in range(nb - 1, 0, -1):
    sc[m.body_parentid[b]] += sc[b]
    smass[m.body_parentid[b]] += smass[b]
  subtree_com = np.where(smass[:, None] > MJ_MINVAL, sc / np.maximum(smass[:, None], MJ_MINVAL), 0)
  # cdof
  cdof = np.zeros((nv, 6))
  for j in range(m.njnt):
    b = m.jnt_bodyid[j]
    d = m.jnt_dofadr[j]
    off = subtree_com[m.body_rootid[b]] - xanchor[j]
    xmat = _quat_to_mat(xquat[b])
    t = m.jnt_type[j]
    if t == JointType.FREE:
      for k in range(3):
        cdof[d + k, 3 + k] = 1.0
      for k in range(3):
        ax = xmat[:, k]
        cdof[d + 3 + k] = np.concatenate([ax, np.cross(ax, off)])
    elif t == JointType.BALL:
      for k in range(3):
        ax = xmat[:, k]
        cdof[d + k] = np.concatenate([ax, np.cross(ax, off)])
    elif t == JointType.SLIDE:
      cdof[d] = np.concatenate([np.zeros(3), xaxis[j]])
    else:
      cdof[d] = np.concatenate([xaxis[j], np.cross(xaxis[j], off)])
  # composite inertia in com frame, as 6x6 spatial matrices
  crb = np.zeros((nb, 6, 6))
  for b in range(1, nb):
    dif = xipos[b] - subtree_com[m.body_rootid[b]]
    rot = ximat[b] @ np.diag(m.body_inertia[b]) @ ximat[b].T
    mass = m.body_mass[b]
    cx = np.array([[0, -dif[2], dif[1]], [dif[2], 0, -dif[0]], [-dif[1], dif[0], 0]])
    crb[b, :3, :3] = rot - mass * cx @ cx
    crb[b, :3, 3:] = mass * cx
    crb[b, 3:, :3] = -mass * cx
    crb[b, 3:, 3:] = mass * np.eye(3)
  for b in range(nb - 1, 1, -1):
    p = m.body_parentid[b]
    if p > 0:
      crb[p] += crb[b]
  M = np.zeros((nv, nv))
  for i in range(nv):
    buf = crb[m.dof_bodyid[i]] @ cdof[i]
    M[i, i] = m.dof_armature[i] + cdof[i] @ buf
    j = m.dof_parentid[i]
    while j >= 0:
      M[i, j] = M[j, i] = cdof[j] @ buf
      j = m.dof_parentid[j]
  return xipos, subtree_com, cdof, M


def _set_const(m: MjModel) -> None:
  nv, nb = m.nv, m.nbody
  m.body_invweight0 = np.zeros((nb, 2))
  m.dof_invweight0 = np.zeros(nv)
  if nv == 0:
    m.stat.meaninertia = 1.0
    return
  xipos, subtree_com, cdof, M = _smooth_qpos0(m)
  m.stat.meaninertia = float(np.trace(M) / nv)
  Minv = np.linalg.inv(M)
  # ancestor dof sets per body
  for b in range(1, nb):
    cols = []
    bb = b
    while bb > 0:
      for k in range(m.body_dofnum[bb]):
        cols.append(m.body_dofadr[bb] + k)
      bb = m.body_parentid[bb]
    if not cols:
      continue
    J = np.zeros((6, nv))
    off = xipos[b] - subtree_com[m.body_rootid[b]]
    for dcol in cols:
      J[:3, dcol] = cdof[dcol, 3:] + np.cross(cdof[dcol, :3], off)
      J[3:, dcol] = cdof[dcol, :3]
    A = J @ Minv @ J.T
    m.body_invweight0[b, 0] = np.trace(A[:3, :3]) / 3.0
    m.body_invweight0[b, 1] = np.trace(A[3:, 3:]) / 3.0
  diag = np.diag(Minv)
  for j in range(m.njnt):
    d = m.jnt_dofadr[j]
    t = m.jnt_type[j]
    if t == JointType.FREE:
      m.dof_invweight0[d:d + 3] = diag[d:d + 3].mean()
      m.dof_invweight0[d + 3:d + 6] = diag[d + 3:d + 6].mean()
    elif t == JointType.BALL:
      m.dof_invweight0[d:d + 3] = diag[d:d + 3].mean()
    else:
      m.dof_invweight0[d] = diag[d]
