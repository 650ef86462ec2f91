"""Import shim: exposes the package directory ``3fold-field-engine_b200/`` as ``field_b200``.

The directory name is not a valid Python identifier, so ``import field_b200`` loads it through
this file and registers the package under that name; submodules then import normally
(``from field_b200.edt import PersistentPairEDT``).
"""
import importlib.util as _util
import sys as _sys
from pathlib import Path as _Path

_DIR = _Path(__file__).resolve().parent / "3fold-field-engine_b200"
_spec = _util.spec_from_file_location("field_b200", _DIR / "__init__.py", submodule_search_locations=[str(_DIR)])
_module = _util.module_from_spec(_spec)
_sys.modules["field_b200"] = _module
_spec.loader.exec_module(_module)
