"""Import alias: ``import cls_b200`` loads the package directory
``complex-locomotion-skill-learning-via-differentiable-physics_b200/`` (whose
name is not a valid Python identifier) and registers it as ``cls_b200``."""
import importlib.util
import os
import sys

_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                    "complex-locomotion-skill-learning-via-differentiable-physics_b200")
_spec = importlib.util.spec_from_file_location(
    "cls_b200", os.path.join(_DIR, "__init__.py"), submodule_search_locations=[_DIR])
_module = importlib.util.module_from_spec(_spec)
sys.modules["cls_b200"] = _module
_spec.loader.exec_module(_module)
