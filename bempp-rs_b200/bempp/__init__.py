"""Bempp boundary assembly on B200 GPUs (drop-in for the bempp-rs Python package)."""

from bempp import function_space, assembly  # noqa: F401
