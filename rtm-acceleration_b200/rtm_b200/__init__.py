"""rtm_b200 -- Python host mirror of the B200 2D acoustic RTM engine.

The compute path is librtm_b200.so (hand-written sm_100a kernels behind a C
ABI, include/rtm_b200.h).  This package only marshals arguments, reads and
writes the reference's file formats and generates synthetic workloads.
"""
from .engine import (ENGINES, Engine, RTMError, RTMParams, ShotRecord, list_engines, make_engine,  # noqa: F401
                     max_stable_dt, mute_direct_wave, points_per_wavelength, ricker, stencil_coefficients)

__all__ = ["Engine", "RTMError", "RTMParams", "ShotRecord", "make_engine", "list_engines", "ENGINES",
           "stencil_coefficients", "max_stable_dt", "ricker", "points_per_wavelength", "mute_direct_wave"]
