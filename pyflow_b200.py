"""Import name of the package whose sources live in ``pyflow-public_b200/``.

``import pyflow_b200`` executes ``pyflow-public_b200/__init__.py`` as the
package ``pyflow_b200`` (the directory name itself is not a Python
identifier), so ``import pyflow_b200.solver`` and friends work as usual.
"""
import importlib.util
import os
import sys

_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                    "pyflow-public_b200")
_spec = importlib.util.spec_from_file_location(
    __name__, os.path.join(_DIR, "__init__.py"),
    submodule_search_locations=[_DIR])
_mod = importlib.util.module_from_spec(_spec)
sys.modules[__name__] = _mod
_spec.loader.exec_module(_mod)
