"""Import shim: exposes the package in ``taichi-spectral-render_b200/`` as ``spectral_b200``.

The package directory's name contains hyphens, which ``import`` cannot spell,
so this module loads it by path and registers it under the importable name.
"""
import importlib.util
import os
import sys

_PKG_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "taichi-spectral-render_b200")
_spec = importlib.util.spec_from_file_location("spectral_b200", os.path.join(_PKG_DIR, "__init__.py"),
                                               submodule_search_locations=[_PKG_DIR])
_mod = importlib.util.module_from_spec(_spec)
sys.modules["spectral_b200"] = _mod
_spec.loader.exec_module(_mod)
