"""babelsim_b200: the BabelSim finite-volume SIMPLE hot path, native to NVIDIA B200.

The compute path is libbabelsim_b200.so (hand-written sm_100a CUDA kernels and
a C++17 host runtime behind the C ABI in include/babelsim_b200.h).  This
package loads it and offers the same vocabulary from Python.
"""
from ._lib import BsgError, lib  # noqa: F401
from .api import (Context, Equation, Field, LinearSystem, Mesh, Piso, Simple, div_flux, flux, grad,  # noqa: F401
                  interpolate, normal_gradient, options, solve_ldu, solver_config, write_results)
