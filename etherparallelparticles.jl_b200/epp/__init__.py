"""epp -- B200 (sm_100a) SPH time-step backend for EtherParallelParticles.jl.

Host-side mirror of the reference's Class / Algorithm interface for the SPH path; the device
work is done by libepp.so (C ABI in include/epp.h) through ctypes.
"""
from . import abi  # noqa: F401
from .classes import (ActivePair, Domain2D, Domain3D, NamedIndex, NeighbourSystem,  # noqa: F401
                      ParticleSystem, mapBasicIndex)
