"""curig_b200 -- B200-native radio-interferometric gridder (ms2dirty / dirty2ms).

Drop-in for the Python surface of astronomical-data-processing/CuRIG
(python/curagridder/__init__.py:1-3): the reference-flavour vis2dirty /
dirty2vis and the Nifty-flavour ms2dirty / dirty2ms, all reaching the CUDA
library libcurafft.so through ctypes.  GridderPlan exposes the device-pointer
plan API.  Importing raises RuntimeError when the library is not built.
"""
from .curagridder import dirty2vis, vis2dirty  # noqa: F401
from .cursl import dirty2ms, ms2dirty  # noqa: F401
from .plan import DIRTY2MS, MS2DIRTY, GridderPlan  # noqa: F401


def release_memory() -> None:
    """Return the device memory the library keeps for its next calls (the
    current device's stream-ordered pool) to the driver.  Call it when no
    call or plan of the library is executing on the device."""
    from . import _lib
    _lib.check(_lib.lib.curig_release_memory(), "release_memory")
