"""honee-4aiad_b200: B200-native matrix-free backend for HONEE's Newtonian ideal-gas operator.

The product is the shared library ``libceed_b200.so`` in this directory: a libCEED-compatible C API
(``include/ceed/ceed.h``) whose HONEE operators run as fused sm_100a kernels (``include/honee_b200.h``).
This Python package is a host-side mirror for tests, benchmarks and scripting:

* :mod:`.ceed`     -- ctypes binding of the libCEED API subset, used the way HONEE's C code uses it
* :mod:`.honee`    -- HONEE's operator set-up (SetupLibceed / QDataGet) expressed through that binding
* :mod:`.problem`  -- caller-side inputs: context structs with the reference defaults, box meshes, bases, states
* :mod:`.kernels`  -- direct binding of the kernel ABI on device pointers (torch tensors as device buffers)

The package is imported as ``importlib.import_module("honee-4aiad_b200")`` (its directory name has a dash).
Loading fails loudly when the compiled library is missing; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libceed_b200.so")

_lib = None


def build(force: bool = False) -> str:
    """Compile libceed_b200.so (nvcc for sm_100a + gcc) in place."""
    args = ["make", "-s", "-C", os.path.join(HERE, "csrc")]
    if force:
        subprocess.run(args + ["clean"], check=True)
    subprocess.run(args + ["-j8"], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    """The loaded backend library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {os.path.join(HERE, 'csrc')}` "
                               "(the backend has no CPU fallback)")
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def version() -> str:
    f = lib().hb_version
    f.restype = ctypes.c_char_p
    return f().decode()
