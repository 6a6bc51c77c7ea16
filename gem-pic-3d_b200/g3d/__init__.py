"""Python mirror of the GEM-PIC-3D march API over libg3d (the sm_100a C-ABI of include/g3d.h)."""
from . import abi, configs
from .abi import PARTICLE_DTYPE, load_library
from .sim import G3DError, Simulation, sample_bunches

__all__ = ["abi", "configs", "PARTICLE_DTYPE", "load_library", "G3DError", "Simulation", "sample_bunches"]
