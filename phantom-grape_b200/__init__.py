"""B200-native pairwise-force engine behind Phantom-GRAPE's GRAPE-5 / GRAPE-6 C APIs.

The product is the set of shared libraries built into ``lib/`` from ``csrc/`` (CUDA for
sm_100a + C++ host code, C ABI declared in the repository's ``include/``).  This Python
package only holds the ctypes mirror of those APIs (``ffi``) and the seeded synthetic
workloads (``workloads``) the tests and the benchmark use.

The directory name is not a valid Python identifier; import it as ``phantom_grape_b200``
through :func:`load` in ``__graft_entry__`` / ``tests/conftest.py``.
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")
LIBS = ("libpg5.so", "libpg5sym.so", "libpg5table.so", "libpg6.so", "libpgbtree.so", "libpgbpeak.so",
        "libpg5_newton.so", "libpg6_newton.so")

from . import ffi, shard, workloads  # noqa: E402,F401
