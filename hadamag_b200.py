"""Import shim: the package lives in the directory ``hadamag.jl_b200/`` (a name Python
cannot import directly); ``import hadamag_b200`` from the repository root loads it."""
import importlib.util
import os
import sys

_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hadamag.jl_b200")
_spec = importlib.util.spec_from_file_location("hadamag_b200", os.path.join(_DIR, "__init__.py"),
                                               submodule_search_locations=[_DIR])
_mod = importlib.util.module_from_spec(_spec)
sys.modules["hadamag_b200"] = _mod
_spec.loader.exec_module(_mod)
