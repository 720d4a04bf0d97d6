"""fastcone_b200 -- B200-native (sm_100a) cone-beam CT projector / backprojector.

A drop-in for Fastcone's C ABI (libfastcone_b200.so exports the wrapper.c entry points) and
for its Python module (``fastcone_b200.fastcone``), plus torch-level device operators
(``fastcone_b200.ops``).
"""
from ._lib import FastconeError, lib  # noqa: F401
from .geometry import ConeGeometry  # noqa: F401

__all__ = ["ConeGeometry", "FastconeError", "lib"]
