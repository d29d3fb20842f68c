"""B200-native MPPI / PR-MPPI control step for the drone-race StratRace environment.

The compute lives in lib/libdrmppi.so (CUDA for sm_100a behind the C ABI of
include/drmppi.h); this package is the Python face of that ABI: ctypes types (abi),
track preprocessing (track), configuration presets (scenarios), the controller
classes mirroring the reference's include/controllers.h (controllers) and the
reference's wire protocol (protocol). The gradient path's torch op (grad) imports
torch and is loaded on demand: `import drone_race_b200.grad`.
"""
from . import abi, controllers, protocol, scenarios, track  # noqa: F401
