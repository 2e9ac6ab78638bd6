"""Import name for the package directory ``sidon-autocorrelation-bound_b200/``.

The directory name is not a Python identifier, so ``import sidon_b200`` loads
it through this alias; submodules (``sidon_b200.kernels`` ...) resolve inside
that directory.
"""
import importlib.util as _ilu
import pathlib as _pl
import sys as _sys

_DIR = _pl.Path(__file__).resolve().parent / "sidon-autocorrelation-bound_b200"
_spec = _ilu.spec_from_file_location(__name__, _DIR / "__init__.py",
                                     submodule_search_locations=[str(_DIR)])
_mod = _ilu.module_from_spec(_spec)
_sys.modules[__name__] = _mod
_spec.loader.exec_module(_mod)
