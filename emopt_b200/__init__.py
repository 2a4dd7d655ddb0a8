"""emopt_b200 -- B200-native (sm_100a) implementation of EMopt's 3D CW-FDTD hot path.

``emopt_b200.fdtd.FDTD`` is the drop-in for ``emopt.fdtd.FDTD`` and
``emopt_b200.fdtd_ctypes.libFDTD`` the drop-in for ``emopt.fdtd_ctypes.libFDTD``;
both sit on the CUDA library ``emopt_b200/FDTD.so`` (C ABI in
``include/emopt_fdtd.h``).  Importing the package does not load the library;
``emopt_b200.fdtd`` does, and fails loudly if it has not been built.
"""
__version__ = "0.1.0"


def __getattr__(name):
    if name == "FDTD":
        from .fdtd import FDTD
        return FDTD
    raise AttributeError(name)
