"""libaccint-b200: B200-native Rys-quadrature two-electron J/K engine.

Import with ``importlib.import_module("libaccint-public_b200")`` (the package
directory name is not a Python identifier).
"""
from ._lib import LibAccIntError, lib  # noqa: F401
from .basis import Atom, BasisSet, Shell, basis_data, cart_to_sph_matrix, point_charges  # noqa: F401
from .engine import (BatchedEngine, Engine, FockBuilder, GpuFockBuilder, Operator, ScreeningOptions, jk,  # noqa: F401
                     probe_fp64_peak)
from . import autograd, df, molecules, scf, workloads  # noqa: F401
