"""B200 (sm_100a) implementation of the LBFS-IBM time step of LBFS-IBM-ADE-SP.

Host-side mirror of the reference's solver interface over the C ABI in
include/lbfs_b200.h; the compute runs only in the CUDA kernels of
liblbfs_b200.so (there is no CPU fallback).
"""
from . import _abi
from ._abi import LbfsError
from .mesh import PATCHES, UniformMesh, build_uniform_mesh, import_openfoam, uniform_counts, write_openfoam
from .rbc import Membrane, biconcave, build_springs, icosphere, red_cell, write_osay
from .solver import GpuSolver, StepParams

__all__ = ["_abi", "LbfsError", "PATCHES", "UniformMesh", "build_uniform_mesh", "uniform_counts", "write_openfoam", "import_openfoam", "Membrane",
           "biconcave", "build_springs", "icosphere", "red_cell", "write_osay", "GpuSolver", "StepParams"]
