"""Bempp boundary assembly on B200 GPUs (drop-in for the bempp-rs Python package).

Submodules load on first use (``bempp.function_space``, ``bempp.assembly``,
``bempp.sweep``, ``bempp.autograd``, ``bempp.shapes``), so that importing the pure-numpy
``bempp.shapes`` does not open the native library; any module that talks to the GPU
loads it (and fails loudly when it is missing).
"""

import importlib

_SUBMODULES = ("function_space", "assembly", "shapes", "sweep", "autograd")


def __getattr__(name):
    if name in _SUBMODULES:
        return importlib.import_module(f"bempp.{name}")
    raise AttributeError(f"module 'bempp' has no attribute {name!r}")
