"""Load this package by path under the module name ``catabra_b200``.

The directory name (catabrafft.jl_b200) is not a Python identifier, so the
package cannot be imported with a plain ``import``.  ``load()`` imports it
from its own directory and registers it in ``sys.modules``; later calls
return the same module.  Callers outside the package reach this file by path:

    spec = importlib.util.spec_from_file_location("catabra_b200_load", path_to_this_file)
    mod = importlib.util.module_from_spec(spec); spec.loader.exec_module(mod)
    cb = mod.load()
"""
import importlib.util
import os
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
NAME = "catabra_b200"


def load():
    if NAME in sys.modules:
        return sys.modules[NAME]
    spec = importlib.util.spec_from_file_location(
        NAME, os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[NAME] = mod
    try:
        spec.loader.exec_module(mod)
    except BaseException:
        del sys.modules[NAME]
        raise
    return mod


def load_from(root):
    """Load the package that sits in ``root``/catabrafft.jl_b200."""
    path = os.path.join(root, "catabrafft.jl_b200", "_load.py")
    spec = importlib.util.spec_from_file_location("catabra_b200_load", path)
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.load()
