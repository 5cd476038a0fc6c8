"""Tests load the product through the package's own loader
(catabrafft.jl_b200/_load.py), under the module name ``catabra_b200``."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "catabrafft.jl_b200")


def load():
    spec = importlib.util.spec_from_file_location("catabra_b200_load", os.path.join(PKG_DIR, "_load.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.load()
