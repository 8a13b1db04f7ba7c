"""pantometry_b200 — B200-native stepping for pantometry's 3D explicit staggered grids.

The product is libpantometry_b200.so (sm_100a CUDA kernels and a C++ runtime behind the C ABI
in include/pantometry_gpu.h). This package is its Python face: `domains` mirrors the Rust
`Domain` implementations, `workloads` builds the seeded synthetic inputs. There is no CPU path:
if the library is missing, using any domain raises.
"""
from . import _native  # noqa: F401

__all__ = ["domains", "workloads", "build"]


def build(force=False, verbose=False):
    from .build import build as _build

    return _build(force=force, verbose=verbose)
