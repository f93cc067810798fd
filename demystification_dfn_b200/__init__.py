"""B200-native hot path of the DemystiFicatioN earthquake-cycle simulator.

The package keeps the reference's problem object model (``DemystiFicatioN``,
``Fault``, ``Hyperparameter``, ``Material_Loading``) and runs the per-stage
right-hand side (K.V stress transfer, rate-and-state friction, pore-pressure
diffusion) and the Cash-Karp RK45 driver in ``libdfn_b200.so`` on the GPU.
"""
from .problem import DemystiFicatioN, Fault, Hyperparameter, Material_Loading
from .layout import ProblemArrays, build_arrays

__all__ = ["DemystiFicatioN", "Fault", "Hyperparameter", "Material_Loading", "ProblemArrays", "build_arrays",
           "Simulation", "load_library"]


def load_library():
    from . import _lib

    return _lib.load()


def __getattr__(name):
    if name == "Simulation":
        from .simulation import Simulation

        return Simulation
    raise AttributeError(name)
