"""Imports this package from its folder (whose name is not an identifier).

    from loader import load_package   # with the package folder on sys.path
"""
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
NAME = "particle_mesh_b200"


def load_package():
    if NAME in sys.modules:
        return sys.modules[NAME]
    spec = importlib.util.spec_from_file_location(NAME, os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[NAME] = mod
    spec.loader.exec_module(mod)
    return mod
