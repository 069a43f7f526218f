"""B200-native batched physics step with the MJWarp API (mujoco_warp/__init__.py:18-58).

Usage mirrors the reference:

    import mjx_warp_b200 as mjw
    mjm = mjw.mjcf.from_xml_path("humanoid.xml")   # or a mujoco.MjModel
    m = mjw.put_model(mjm)
    d = mjw.make_data(mjm, nworld=8192, nconmax=..., njmax=...)
    mjw.step(m, d)

Model and Data hold torch CUDA tensors with the reference's field names and logical shapes; the
stage functions launch the hand-written sm_100a kernels of libmjb200.so through its C ABI
(include/mjb200.h).
"""

from . import derivative as derivative
from . import mjcf as mjcf
from ._api import autotune as autotune
from ._api import set_tune as set_tune
from ._api import step_io as step_io
from ._api import benchmark as benchmark
from ._api import collision as collision
from ._api import com_pos as com_pos
from ._api import com_vel as com_vel
from ._api import crb as crb
from ._api import euler as euler
from ._api import factor_m as factor_m
from ._api import forward as forward
from ._api import fwd_acceleration as fwd_acceleration
from ._api import fwd_actuation as fwd_actuation
from ._api import fwd_position as fwd_position
from ._api import fwd_velocity as fwd_velocity
from ._api import implicit as implicit
from ._api import kinematics as kinematics
from ._api import make_constraint as make_constraint
from ._api import mul_m as mul_m
from ._api import nxn_broadphase as nxn_broadphase
from ._api import passive as passive
from ._api import primitive_narrowphase as primitive_narrowphase
from ._api import rne as rne
from ._api import sap_broadphase as sap_broadphase
from ._api import solve as solve
from ._api import solve_m as solve_m
from ._api import step as step
from ._api import step_phase as step_phase
from ._api import transmission as transmission
from ._api import world_status as world_status
from ._api import xfrc_accumulate as xfrc_accumulate
from .io import get_data_into as get_data_into
from .io import is_sparse as is_sparse
from .io import make_data as make_data
from .io import put_data as put_data
from .io import put_model as put_model
from .types import ConeType as ConeType
from .types import Contact as Contact
from .types import Data as Data
from .types import DisableBit as DisableBit
from .types import DynType as DynType
from .types import JointType as JointType
from .types import Model as Model
from .types import Option as Option
from .types import Statistic as Statistic
from .types import TrnType as TrnType
