"""B200-native (sm_100a) RK4 step of the AdS4 holographic superfluid.

The compute path is ``libhqt.so`` (CUDA kernels behind the C ABI of
``include/hqt.h``); this package adds the host-side seeding (Newton
stationary profiles, initial fields), the Python mirror of the step API and
MAT-v5 checkpoint I/O.  The directory name is not a Python identifier, so
import it with ``importlib.import_module("ads4-holographic-quantum-turbulence_b200")``.
"""
from . import seed
from ._lib import HQTError, NonfiniteEvolution
from .api import Ensemble, Simulation, StepInfo, assign_runs, from_device, to_device
from .checkpoint import load_checkpoint, save_checkpoint

__all__ = ["Simulation", "Ensemble", "assign_runs", "StepInfo", "HQTError", "NonfiniteEvolution", "seed",
           "to_device", "from_device", "save_checkpoint", "load_checkpoint"]
