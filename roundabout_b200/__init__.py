"""roundabout_b200: B200-native vertical-physics hot path of Roundabout.

The compute lives in libvphys.so (hand-written CUDA for sm_100a behind the C
ABI of include/vphys.h); this package is the Python mirror of the
reference's python/rdb interface for that path: ctypes bindings (`_ffi`),
closure knobs (`config`), the `VerticalPhysics` driver (`column`) and the
seeded synthetic inputs (`synthetic`).
"""
from .config import default_config, hot_path_config  # noqa: F401

__all__ = ["default_config", "hot_path_config"]
