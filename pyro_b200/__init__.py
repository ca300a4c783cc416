"""pyro_b200 — B200-native (sm_100a) fire-simulation step of pyro.

The product is libpyro_b200.so (CUDA kernels + C ABI, include/pyro_sim.h);
this package holds its host-side mirror of the reference interface:

* scene  — TOML scenes, materials, the 576-byte parameter block, shapes
* sim    — `Sim` (new / step / read_stats / read_scalars) over the C ABI
* run    — the `--sim-only` frame loop: CFL substepping, statistics
           averaging, flame heights, `--slice` image
* poisson — the stand-alone pressure solver
"""
from . import _abi  # noqa: F401
from .scene import Scene, SceneError, MATERIALS, material  # noqa: F401

__all__ = ["Scene", "SceneError", "MATERIALS", "material", "build_library"]


def build_library(force: bool = False) -> str:
    from .build import build
    return build(force=force)
