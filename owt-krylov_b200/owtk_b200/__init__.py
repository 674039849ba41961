"""Python access to the B200 OWT-Krylov solve path (ctypes over include/owtk.h).

`native` binds the C ABI of lib/libowtk_b200.so; `problems` generates the
seeded synthetic systems of the benchmark configurations.
"""
from . import native, problems  # noqa: F401
