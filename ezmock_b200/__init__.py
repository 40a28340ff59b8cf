"""B200-native EZmock engine: the plain EZmock pipeline on the GPU behind the
reference's libEZmock C interface (include/EZmock.h) and a Python class with
the reference wrapper's methods (ezmock_b200.EZmock)."""
from .EZmock import EZmock

__all__ = ["EZmock"]
