"""Import shim: the package lives in the directory ``weave-sim_b200/`` (a name Python cannot import directly); this
module loads it under the importable name ``weavesim_b200`` and replaces itself in ``sys.modules``."""
import importlib.util as _iu
import os as _os
import sys as _sys

_dir = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "weave-sim_b200")
_spec = _iu.spec_from_file_location(__name__, _os.path.join(_dir, "__init__.py"), submodule_search_locations=[_dir])
_mod = _iu.module_from_spec(_spec)
_sys.modules[__name__] = _mod
_spec.loader.exec_module(_mod)
