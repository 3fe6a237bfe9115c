"""Import name for the package directory i.sar.temporal_coherence_b200/.

The directory keeps the module's name, which is not a Python identifier;
``import tcoh_b200`` loads it as a package under this name.
"""
import importlib.util
import os
import sys

_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "i.sar.temporal_coherence_b200")
_spec = importlib.util.spec_from_file_location(
    "tcoh_b200", os.path.join(_DIR, "__init__.py"), submodule_search_locations=[_DIR]
)
_module = importlib.util.module_from_spec(_spec)
sys.modules["tcoh_b200"] = _module
_spec.loader.exec_module(_module)
