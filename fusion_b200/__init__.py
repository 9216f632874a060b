"""B200 (sm_100a) implementation of the per-frame dense RGB-D fusion path of
cnxyang/Fusion behind a C ABI (include/fusion_b200.h).

    from fusion_b200 import Session, config_c2
    s = Session(config_c2())
    r = s.grab(depth_u16, rgb_u8)      # one System::GrabImage
"""
from ._lib import FusionError, load  # noqa: F401
from .batch import Batch, mixed_config, mixed_population  # noqa: F401
from .system import (Session, System, config_c1, config_c2, config_dict, make_config,  # noqa: F401
                     reference_config)

__all__ = ["Session", "System", "Batch", "mixed_config", "mixed_population", "config_c1", "config_c2",
           "make_config", "reference_config", "config_dict", "FusionError", "load"]
