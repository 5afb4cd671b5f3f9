"""Import shim: loads the package directory ``ladderdga.jl_b200/`` (named after the Julia project,
which is not a valid Python identifier) as the module ``ladderdga_b200``."""
import importlib.util as _ilu
import os as _os
import sys as _sys

_pkg = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "ladderdga.jl_b200")
_spec = _ilu.spec_from_file_location("ladderdga_b200", _os.path.join(_pkg, "__init__.py"),
                                     submodule_search_locations=[_pkg])
_mod = _ilu.module_from_spec(_spec)
_sys.modules["ladderdga_b200"] = _mod
_spec.loader.exec_module(_mod)
