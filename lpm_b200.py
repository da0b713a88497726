"""Import shim: exposes the package directory ``lpm-solver-trained-coarse-graining_b200/`` as ``lpm_b200``.

The directory name carries the upstream project name (hyphens are not valid in a Python module name), so this file
registers it under an importable name.  ``import lpm_b200`` then behaves like a regular package import, and submodules
resolve as ``lpm_b200.torch_lpm3d``, ``lpm_b200.lin3d`` and so on.
"""
import importlib.util
import os
import sys

_PKG_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lpm-solver-trained-coarse-graining_b200")
_spec = importlib.util.spec_from_file_location("lpm_b200", os.path.join(_PKG_DIR, "__init__.py"),
                                               submodule_search_locations=[_PKG_DIR])
_mod = importlib.util.module_from_spec(_spec)
sys.modules["lpm_b200"] = _mod
_spec.loader.exec_module(_mod)
