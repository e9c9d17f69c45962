"""terraneo_b200: B200 (sm_100a) matrix-free hot path of TerraNeo.

The CUDA library libterraneo_b200.so (built from terraneo_b200/csrc) is the
product; `terraneo_b200.shell` mirrors the reference's vector/operator
interface over its C ABI (include/terraneo_b200.h).
"""
from . import _capi  # noqa: F401

__all__ = ["_capi"]
