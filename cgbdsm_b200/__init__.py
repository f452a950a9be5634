"""B200-native continuous subgraph matching (drop-in for the CGBDSM batched pipeline).

Native code lives in libcgbdsm.so (C ABI: include/cgbdsm.h); this package
holds the build script, a ctypes binding and the synthetic workloads.
"""
from .engine import CgbError, Engine, Gpma, MultiQuery, Producer, Server, load_library  # noqa: F401
