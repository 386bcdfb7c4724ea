"""ffrb — host side of the B200 room solver (scene building, parameters,
C-ABI bindings, batched rooms and the serving loop).

The compute path lives in ``libffroom_cuda.so`` (sm_100a kernels behind the
C ABI declared in include/ffroom.h); ``_ffroom_core`` is the drop-in
pybind11 module with the reference's class surface.
"""
from .scene import (SceneConfig, RoomConfig, FanConfig, ObstacleConfig, OpeningConfig,
                    HeatPatchConfig, SolverConfig, RoomSpec, build_room, empty_room)
from .params import FluidParams, params_from_scene

__all__ = ["SceneConfig", "RoomConfig", "FanConfig", "ObstacleConfig", "OpeningConfig",
           "HeatPatchConfig", "SolverConfig", "RoomSpec", "build_room", "empty_room",
           "FluidParams", "params_from_scene"]
