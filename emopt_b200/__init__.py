"""emopt_b200 -- B200-native (sm_100a) implementation of EMopt's 3D CW-FDTD hot path.

``emopt_b200.fdtd.FDTD`` is the drop-in for ``emopt.fdtd.FDTD`` and
``emopt_b200.fdtd_ctypes.libFDTD`` the drop-in for ``emopt.fdtd_ctypes.libFDTD``;
both sit on the CUDA library ``emopt_b200/FDTD.so`` (C ABI in
``include/emopt_fdtd.h``).  Around the solve, with the reference's names:
``emopt_b200.grid`` (layered materials), ``emopt_b200.misc``
(``DomainCoordinates``), ``emopt_b200.modes`` (``ModeFullVector`` on the GPU),
``emopt_b200.fomutils`` and ``emopt_b200.adjoint_method`` (adjoint sources
and drivers); ``emopt_b200.adjoint`` (autograd), ``emopt_b200.serving`` and
``emopt_b200.zslab`` are this package's own forms.  Importing the package
does not load the library; the modules that need it do, and fail loudly if
it has not been built.
"""
__version__ = "0.1.0"


def __getattr__(name):
    if name == "FDTD":
        from .fdtd import FDTD
        return FDTD
    raise AttributeError(name)
