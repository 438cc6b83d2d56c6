"""simtrack_b200: SimTrack's element-by-element 6D tracking path on NVIDIA B200.

The public surface mirrors SimTrack's construction API (simtrack.h): element
constructors, Line, Set_RefPartEnergy, Track.  Tracking runs in hand-written
sm_100a CUDA kernels behind the C ABI declared in include/simtrack_b200.h.
"""
from ._native import SimTrackError  # noqa: F401
from .api import *  # noqa: F401,F403

__version__ = "0.1.0"
