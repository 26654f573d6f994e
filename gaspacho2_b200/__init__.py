"""B200-native GASPACHO2 sparse GP-LVM fit: CUDA kernels for sm_100a behind a C ABI
(include/gpl.h, libgpl_b200.so), with a host-side mirror of the reference driver."""
from ._lib import GplError, load  # noqa: F401
from .model import GPLVM  # noqa: F401

__all__ = ["GPLVM", "GplError", "load"]
