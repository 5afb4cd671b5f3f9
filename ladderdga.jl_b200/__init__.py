"""ladderdga_b200: the lDGA ladder hot path of LadderDGA.jl on NVIDIA B200 (sm_100a).

The package directory is named after the Julia project (``ladderdga.jl_b200``); import it as
``ladderdga_b200`` through the loader module at the repository root.
"""
from . import _lib, inputs, jld2, synthetic
from ._lib import (CH_D, CH_M, PREC_FP64, PREC_FP64_INV, PREC_MIXED, Context, LdgaError, LibraryMissing,
                   EXPORTS)
from .core import *  # noqa: F401,F403
from .core import __doc__ as _core_doc  # noqa: F401
from .inputs import (EnvironmentVars, ImpurityInput, calc_E_ED, load_impurity_input,  # noqa: F401
                     readConfig)
from .jld2 import jldopen  # noqa: F401

__version__ = "0.1.0"
