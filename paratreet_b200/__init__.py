"""paratreet_b200 -- B200-native Barnes-Hut gravity path of ParaTreeT.

The compute lives in libpt_gravity.so (CUDA, sm_100a) behind the C ABI of
include/pt_gravity.h; this package holds the ctypes binding, a host-side
mirror of the reference's Gravity interface and seeded input generators.
"""
from . import ics  # noqa: F401

__all__ = ["ics", "gravity"]


def __getattr__(name):
    if name == "gravity":
        from . import gravity
        return gravity
    raise AttributeError(name)
