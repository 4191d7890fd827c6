"""Import shim: loads the package directory ``bayesian-rans-uq_b200/`` (whose name is
not a Python identifier) as the module ``rans_uq_b200``."""
import importlib.util as _u
import pathlib as _p
import sys as _s

_pkg = _p.Path(__file__).resolve().with_name("bayesian-rans-uq_b200")
_spec = _u.spec_from_file_location("rans_uq_b200", _pkg / "__init__.py",
                                   submodule_search_locations=[str(_pkg)])
_mod = _u.module_from_spec(_spec)
_s.modules["rans_uq_b200"] = _mod
_spec.loader.exec_module(_mod)
