"""samos_b200 -- B200-native (sm_100a) particle-dynamics hot path of SAMoS.

The compute path is libsamos_gpu.so (CUDA, C ABI in include/samos_gpu.h);
``engine`` binds it, ``plugins`` mirrors SAMoS's plugin factories and
conf-level commands on top of it.
"""
from . import engine, plugins  # noqa: F401
from .engine import Engine, EngineError  # noqa: F401
from .plugins import PluginError, Simulation  # noqa: F401

__all__ = ["Engine", "EngineError", "Simulation", "PluginError", "engine", "plugins"]
