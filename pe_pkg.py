"""Imports the ``photon-engine_b200`` package folder (its name is not a Python identifier) as
``photon_engine_b200``."""
import importlib.util
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parent
PKG_DIR = ROOT / "photon-engine_b200"


def load():
    if "photon_engine_b200" in sys.modules:
        return sys.modules["photon_engine_b200"]
    spec = importlib.util.spec_from_file_location("photon_engine_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["photon_engine_b200"] = mod
    spec.loader.exec_module(mod)
    return mod
