"""wavesim_b200: the modified Born series iteration loop of IvoVellekoop/wavesim
on NVIDIA B200 (sm_100a), behind the reference's own solver API.

``WaveSim`` / ``WaveSimVector`` / ``Source`` mirror the reference's MATLAB
classes; the loop runs in ``libwavesim_b200.so`` (C ABI:
include/wavesim_b200.h).  Importing the package loads the library and fails
if it has not been built.
"""
from ._lib import WaveSimError, lib  # noqa: F401  (fails loudly if the library is missing)
from .problem import Medium, PlaneWave, SimulationGrid, Source, efficient_size, symrange  # noqa: F401
from .simulation import WaveSim, WaveSimVector, nuttallwin, wiggle_perm  # noqa: F401
from .pstd import PSTD  # noqa: F401

__all__ = ["WaveSim", "WaveSimVector", "Source", "PlaneWave", "PSTD", "Medium", "SimulationGrid", "WaveSimError",
           "efficient_size", "symrange", "nuttallwin", "wiggle_perm"]
