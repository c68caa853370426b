"""B200-native (sm_100a) rebuild of the Eos ray-tracing render path.

Layout:
  csrc/       CUDA kernels (LBVH build, traversal, plain + wavefront renderers, adjoint)
              and the C ABI implementation, built into libeos_b200.so by build.py
  _lib.py     ctypes binding of include/eos_c.h
  api.py      Python view of the C ABI (contexts, resident scenes, render calls)
  scenes.py   seeded synthetic scenes and cameras of the benchmark workloads
  autotune.py per-scene-size tuning of block size / queue chunk / stack depth / leaf size

The C++ drop-in facade of the reference's Scene / Camera / DeviceRenderer API is the
header-only include/eos/eos.hpp over the same C ABI.
"""
from . import scenes  # noqa: F401

__all__ = ["scenes"]
