"""B200-native region simulation loop of The Virtual Brain.

Host-side mirror of the reference's simulator interface over the sm_100a
kernels of libtvbk.so (include/tvbk.h):

    from tvb_b200 import models, coupling, integrators, monitors, noise
    from tvb_b200.connectivity import Connectivity
    from tvb_b200.simulator import Simulator
    from tvb_b200.sweep import ParameterSweep
"""
from . import _lib  # noqa: F401  (fails loudly when libtvbk.so is missing)
from . import coupling, equations, integrators, models, monitors, noise, patterns  # noqa: F401
from .connectivity import Connectivity  # noqa: F401

__version__ = '0.1.0'
