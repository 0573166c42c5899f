"""ckmpm_b200: B200-native (sm_100a) CK-MPM substep engine.

The hot path (binning, block table, fused G2P/SVD/return-map/P2G, grid update)
runs in the CUDA library ckmpm_b200/_lib/libckmpm_b200.so through the C ABI of
include/ckmpm.h.  This package is the host-side mirror of the reference's
engine/material/model/config API; it has no CPU implementation of any kernel.
"""
from ._capi import CkmpmError, LIB_PATH
from .engine import (MPMConfig, MPMEngine, MPMMaterial, MPMModel, ParticleState, Scene, compute_lame_parameters,
                     evaluate_sound_speed, evaluate_timestep, load_scene_json)

__all__ = [
    "CkmpmError", "LIB_PATH", "MPMConfig", "MPMEngine", "MPMMaterial", "MPMModel", "ParticleState", "Scene",
    "compute_lame_parameters", "evaluate_sound_speed", "evaluate_timestep", "load_scene_json",
]
