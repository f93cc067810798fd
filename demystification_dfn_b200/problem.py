"""Problem description with the reference's user-facing object model.

Mirrors the classes of ``wrapper_python/DemystiFicatioN.py`` (``Fault`` :10-240,
``Hyperparameter`` :245-268, ``Material_Loading`` :274-298, ``DemystiFicatioN``
:302-325) so that a script written for the reference builds the same problem
here: same attribute names, same defaults, same units (``Q`` in m/s, ``sigmaN``
negative in compression, ``theta`` holds psi = ln(theta*V0/Dc), ``index_injection``
1-based). Setting ``nb_element`` reallocates the per-element arrays and setting
``nb_source`` reallocates the source arrays, as in the reference.

``DemystiFicatioN.write(path)`` produces the reference's HDF5 ``config`` file
(layout of ``wrapper_python/DemystiFicatioN.py:330-422``) through the package's
own HDF5 writer.
"""
from __future__ import annotations

import numpy as np


class Fault:
    """One fault: geometry, friction, initial state, permeability, sources."""

    def __init__(self):
        self._nb_element = 1
        self._nb_source = 0
        self._alloc(1)
        self.Q = np.zeros(0)
        self.t_injection_beg = np.zeros(0)
        self.t_injection_end = np.zeros(0)
        self.index_injection = np.zeros(0, dtype=np.int64)

    def _alloc(self, n):
        # defaults of wrapper_python/DemystiFicatioN.py:55-82
        self.a = np.zeros(n)
        self.b = np.zeros(n)
        self.Dc = np.zeros(n)
        self.f0 = np.zeros(n)
        self.V0 = np.zeros(n)
        self.node = np.zeros((2, n + 1))
        self.sigmaN = np.zeros(n)
        self.V = np.zeros(n)
        self.theta = np.zeros(n)
        self.P = np.zeros(n)
        self.normal_loading_dot = np.zeros(n)
        self.shear_loading_dot = np.zeros(n)
        self.permeability = np.ones(n)
        self.Lk = np.zeros(n)
        self.Tk = np.zeros(n)
        self.kmin = np.zeros(n)
        self.kmax = np.zeros(n)
        self.Snk = np.zeros(n)

    @property
    def nb_element(self):
        return self._nb_element

    @nb_element.setter
    def nb_element(self, value):
        if not isinstance(value, (int, np.integer)):
            raise ValueError("The given value must be an integer")
        value = int(value)
        if value < 1:
            raise ValueError("The number of elements must be greater than 0")
        if value != self._nb_element:
            self._nb_element = value
            self._alloc(value)

    @property
    def nb_node(self):
        return self._nb_element + 1

    @nb_node.setter
    def nb_node(self, value):
        self.nb_element = value - 1

    @property
    def nb_source(self):
        return self._nb_source

    @nb_source.setter
    def nb_source(self, value):
        if not isinstance(value, (int, np.integer)):
            raise ValueError("The given value must be an integer")
        value = int(value)
        if value >= 1:
            self._nb_source = value
            self.Q = np.zeros(value)
            self.t_injection_beg = np.zeros(value)
            self.t_injection_end = np.zeros(value)
            self.index_injection = np.zeros(value, dtype=np.int64)
        elif value == 0:
            # the reference ignores 0 but keeps nb_source at its old value only
            # when it was never set; a fault without sources is written with 0
            self._nb_source = 0


class Hyperparameter:
    """Run options, defaults of wrapper_python/DemystiFicatioN.py:247-264."""

    def __init__(self):
        self.simulation_name = "test"
        self.fracture_mode = "modeII"
        self.static_kernel = "direct"
        self.friction_law = "RateStateAging"
        self.tol_solver = 1e-4
        self.freq_writing_file = 10
        self.max_it = 10
        self.stride_time = 1
        self.permeability_coupling = 0
        self.iprec = 4
        self.nb_fault = 1


class Material_Loading:
    """Material, remote loading and fluid constants (:276-298)."""

    def __init__(self):
        self.mu = 30e9
        self.cp = 5000.0
        self.cs = 3000.0
        self.Sigma31_dot = 0.0
        self.Sigma32_dot = 0.0
        self.Sigma11_dot = 0.0
        self.Sigma12_dot = 0.0
        self.Sigma22_dot = 0.0
        self.normal_loading_dot = 0.0
        self.shear_loading_dot = 0.001
        self.rock_comp = 1e-9
        self.fluid_comp = 1e-8
        self.fluid_density = 1000.0
        self.porosity = 0.1
        self.dyn_viscosity = 1e-3


class DemystiFicatioN:
    """A fault-network problem: ``hyperparameter``, ``material_loading``, ``faults``."""

    def __init__(self, nb_flt=1):
        self.hyperparameter = Hyperparameter()
        self.hyperparameter.nb_fault = nb_flt
        self.faults = [Fault() for _ in range(nb_flt)]
        self.material_loading = Material_Loading()

    @property
    def nb_fault(self):
        return self.hyperparameter.nb_fault

    @nb_fault.setter
    def nb_fault(self, value):
        self.hyperparameter.nb_fault = int(value)
        self.faults = [Fault() for _ in range(int(value))]

    def write(self, path_problem):
        """Write ``path_problem + 'config'`` in the reference's HDF5 layout."""
        from .hdf5 import write_config

        return write_config(self, path_problem)

    @classmethod
    def read(cls, config_path):
        """Build a problem from a reference HDF5 ``config`` file."""
        from .hdf5 import read_config

        return read_config(config_path)
