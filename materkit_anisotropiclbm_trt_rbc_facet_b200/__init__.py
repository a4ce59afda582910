"""B200-native MaterKit coupled lattice-Boltzmann / phase-field step.

The compute path is ``libmkb200.so`` (hand-written sm_100a kernels behind the
C ABI of ``include/mkb200.h``); this package is its Python host side.
"""
from ._abi import MkError, MkParams, MkOptions, MkDiag, load as load_library  # noqa: F401
from .solver import (Solver, Ensemble, ensemble_params, case_params, initial_field, readParameters,  # noqa: F401
                     mkSpace, mkFluidsMRT, mkFluidsMultiphase)

__all__ = ["Solver", "Ensemble", "ensemble_params", "case_params", "initial_field", "readParameters", "mkSpace", "mkFluidsMRT",
           "mkFluidsMultiphase", "MkError", "MkParams", "MkOptions", "MkDiag", "load_library"]
