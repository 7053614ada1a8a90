"""dopamine_b200 — sm_100a (B200) implementation of DOPAMINE's RK3W fractional-step hot path.

The product is the CUDA shared library built from dopamine_b200/csrc (C ABI in
include/dopamine_b200.h).  Python here is host plumbing: case set-up (cases.py), the ctypes
binding (solver.py) and the build recipe (build.py).
"""
from . import abi, cases  # noqa: F401

__all__ = ["abi", "cases"]
