"""B200-native (sm_100a) nonhydrostatic hot path of ORCTM.

The product is the CUDA library liborctm_gpu.so behind the C ABI of
include/orctm_gpu.h; this package builds it (build.py), binds it (_lib.py),
mirrors the reference's routine interface (api.Instance) and generates the
seeded synthetic benchmark instances (configs.py).
"""
from .api import Instance  # noqa: F401
