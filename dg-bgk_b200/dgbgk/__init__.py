"""dgbgk: the DG-BGK transport-plus-collision sweep on B200 (sm_100a).

The compute path is lib/libdgbgk.so (hand-written CUDA, C ABI in
include/dgbgk.h); this package is its Python host side: case generators,
reference file formats and a thin Solver wrapper.
"""
from .cases import (CaseDef, RawMesh, cavity_case, cavity_mesh, channel_case, channel_mesh, config1, config2,
                    config3, config5, gll, node_scale, physical_params)
from .solver import Batch, Setup, Solver, setup_mesh, vspace

__all__ = ["Batch", "CaseDef", "RawMesh", "Setup", "Solver", "cavity_case", "cavity_mesh", "channel_case", "channel_mesh",
           "config1", "config2", "config3", "config5", "gll", "node_scale", "physical_params", "setup_mesh", "vspace"]
