"""ctypes binding of the B200 CW-FDTD library (``FDTD.so`` beside this module).

The first block declares exactly the argument and result types of the
reference binding (``emopt/fdtd_ctypes.py:14-149``): the library is loaded from
the same relative location and exports the same 32 symbols, so code written
against ``libFDTD`` works unchanged.  The second block declares the additions
of ``include/emopt_fdtd.h`` (destructor, error reporting, precision/kernel
switches and the device-resident ``FDTD_solve_cw``).
"""
from __future__ import annotations

import os
from ctypes import (POINTER, Structure, c_bool, c_char_p, c_double, c_int, c_longlong,
                    c_void_p, cdll, create_string_buffer)

import numpy as np
from numpy.ctypeslib import ndpointer

dir_path = os.path.dirname(os.path.realpath(__file__))
# EMOPT_B200_LIB selects another build of the library, e.g. FDTD_checked.so
# (index-checked stepping kernels, for debugging)
so_path = os.environ.get("EMOPT_B200_LIB") or os.path.join(dir_path, "FDTD.so")

if not os.path.exists(so_path):
    raise ImportError(
        f"{so_path} is missing: build the CUDA library first "
        "(python -m emopt_b200.build or __graft_entry__.build())")

libFDTD = cdll.LoadLibrary(so_path)

c_complex_p = ndpointer(np.complex128, ndim=1, flags="C")
c_double_p = ndpointer(np.double, ndim=1, flags="C")

# ---------------------------------------------------------- reference ABI
libFDTD.FDTD_new.argtypes = []
libFDTD.FDTD_new.restype = c_void_p
libFDTD.FDTD_set_wavelength.argtypes = [c_void_p, c_double]
libFDTD.FDTD_set_wavelength.restype = None
libFDTD.FDTD_set_physical_dims.argtypes = [c_void_p] + [c_double] * 6
libFDTD.FDTD_set_physical_dims.restype = None
libFDTD.FDTD_set_grid_dims.argtypes = [c_void_p, c_int, c_int, c_int]
libFDTD.FDTD_set_grid_dims.restype = None
libFDTD.FDTD_set_local_grid.argtypes = [c_void_p] + [c_int] * 6
libFDTD.FDTD_set_local_grid.restype = None
libFDTD.FDTD_set_dt.argtypes = [c_void_p, c_double]
libFDTD.FDTD_set_dt.restype = None
libFDTD.FDTD_set_complex_eps.argtypes = [c_void_p, c_bool]
libFDTD.FDTD_set_complex_eps.restype = None
libFDTD.FDTD_set_field_arrays.argtypes = [c_void_p] + [c_double_p] * 6
libFDTD.FDTD_set_field_arrays.restype = None
libFDTD.FDTD_set_mat_arrays.argtypes = [c_void_p] + [c_complex_p] * 6
libFDTD.FDTD_set_mat_arrays.restype = None
libFDTD.FDTD_update_H.argtypes = [c_void_p, c_int, c_double]
libFDTD.FDTD_update_H.restype = None
libFDTD.FDTD_update_E.argtypes = [c_void_p, c_int, c_double]
libFDTD.FDTD_update_E.restype = None
libFDTD.FDTD_set_pml_widths.argtypes = [c_void_p] + [c_int] * 6
libFDTD.FDTD_set_pml_widths.restype = None
libFDTD.FDTD_set_pml_properties.argtypes = [c_void_p] + [c_double] * 4
libFDTD.FDTD_set_pml_properties.restype = None
libFDTD.FDTD_build_pml.argtypes = [c_void_p]
libFDTD.FDTD_build_pml.restype = None
libFDTD.FDTD_reset_pml.argtypes = [c_void_p]
libFDTD.FDTD_reset_pml.restype = None
libFDTD.FDTD_set_t0_arrays.argtypes = [c_void_p] + [c_complex_p] * 6
libFDTD.FDTD_set_t0_arrays.restype = None
libFDTD.FDTD_set_t1_arrays.argtypes = [c_void_p] + [c_complex_p] * 6
libFDTD.FDTD_set_t1_arrays.restype = None
libFDTD.FDTD_calc_phase_2T.argtypes = [c_double] * 4
libFDTD.FDTD_calc_phase_2T.restype = c_double
libFDTD.FDTD_calc_phase_3T.argtypes = [c_double] * 6
libFDTD.FDTD_calc_phase_3T.restype = c_double
libFDTD.FDTD_calc_amplitude_2T.argtypes = [c_double] * 5
libFDTD.FDTD_calc_amplitude_2T.restype = c_double
libFDTD.FDTD_calc_amplitude_3T.argtypes = [c_double] * 7
libFDTD.FDTD_calc_amplitude_3T.restype = c_double
libFDTD.FDTD_capture_t0_fields.argtypes = [c_void_p]
libFDTD.FDTD_capture_t0_fields.restype = None
libFDTD.FDTD_capture_t1_fields.argtypes = [c_void_p]
libFDTD.FDTD_capture_t1_fields.restype = None
libFDTD.FDTD_calc_complex_fields_2T.argtypes = [c_void_p, c_double, c_double]
libFDTD.FDTD_calc_complex_fields_2T.restype = None
libFDTD.FDTD_calc_complex_fields_3T.argtypes = [c_void_p, c_double, c_double, c_double]
libFDTD.FDTD_calc_complex_fields_3T.restype = None
libFDTD.FDTD_add_source.argtypes = [c_void_p] + [c_complex_p] * 6 + [c_int] * 6 + [c_bool]
libFDTD.FDTD_add_source.restype = None
libFDTD.FDTD_clear_sources.argtypes = [c_void_p]
libFDTD.FDTD_clear_sources.restype = None
libFDTD.FDTD_set_source_properties.argtypes = [c_void_p, c_double, c_double]
libFDTD.FDTD_set_source_properties.restype = None
libFDTD.FDTD_src_func_t.argtypes = [c_void_p, c_int, c_double, c_double]
libFDTD.FDTD_src_func_t.restype = c_double
libFDTD.FDTD_set_bc.argtypes = [c_void_p, c_char_p]
libFDTD.FDTD_set_bc.restype = None
libFDTD.FDTD_copy_to_ghost_comm.argtypes = [c_double_p, c_complex_p, c_int, c_int, c_int]
libFDTD.FDTD_copy_to_ghost_comm.restype = None
libFDTD.FDTD_copy_from_ghost_comm.argtypes = [c_double_p, c_complex_p, c_int, c_int, c_int]
libFDTD.FDTD_copy_from_ghost_comm.restype = None

REFERENCE_SYMBOLS = (
    "FDTD_new", "FDTD_set_wavelength", "FDTD_set_physical_dims", "FDTD_set_grid_dims",
    "FDTD_set_local_grid", "FDTD_set_dt", "FDTD_set_complex_eps", "FDTD_set_field_arrays",
    "FDTD_set_mat_arrays", "FDTD_update_H", "FDTD_update_E", "FDTD_set_pml_widths",
    "FDTD_set_pml_properties", "FDTD_build_pml", "FDTD_reset_pml", "FDTD_set_t0_arrays",
    "FDTD_set_t1_arrays", "FDTD_calc_phase_2T", "FDTD_calc_amplitude_2T", "FDTD_calc_phase_3T",
    "FDTD_calc_amplitude_3T", "FDTD_capture_t0_fields", "FDTD_capture_t1_fields",
    "FDTD_calc_complex_fields_2T", "FDTD_calc_complex_fields_3T", "FDTD_add_source",
    "FDTD_clear_sources", "FDTD_set_source_properties", "FDTD_src_func_t", "FDTD_set_bc",
    "FDTD_copy_to_ghost_comm", "FDTD_copy_from_ghost_comm")


# --------------------------------------------------------------- additions
class SolveOptions(Structure):
    _fields_ = [("Tn", c_longlong), ("Nmax", c_double), ("rtol", c_double),
                ("conv_pts", POINTER(c_longlong)), ("nconv", c_int),
                ("fixed_steps", c_longlong), ("materials_unchanged", c_int),
                ("copy_t1", c_int), ("stop_nonfinite", c_int)]


class SolveResult(Structure):
    _fields_ = [("n_main", c_longlong), ("steps", c_longlong), ("A_change", c_double),
                ("phi_change", c_double), ("nprobes", c_longlong), ("device_ms", c_double),
                ("total_ms", c_double), ("launches", c_longlong), ("zchunk", c_int),
                ("status", c_int)]


FDTD_OK, FDTD_ERR_CUDA, FDTD_ERR_ARG, FDTD_ERR_NODEVICE, FDTD_NMAX, FDTD_NONFINITE = range(6)

libFDTD.FDTD_delete.argtypes = [c_void_p]
libFDTD.FDTD_delete.restype = None
libFDTD.FDTD_last_error.argtypes = [c_void_p, c_char_p, c_int]
libFDTD.FDTD_last_error.restype = c_int
libFDTD.FDTD_set_device.argtypes = [c_void_p, c_int]
libFDTD.FDTD_set_device.restype = c_int
libFDTD.FDTD_set_zchunk.argtypes = [c_void_p, c_int]
libFDTD.FDTD_set_zchunk.restype = c_int
libFDTD.FDTD_set_precision.argtypes = [c_void_p, c_int]
libFDTD.FDTD_set_precision.restype = c_int
libFDTD.FDTD_set_kernel.argtypes = [c_void_p, c_int]
libFDTD.FDTD_set_kernel.restype = c_int
libFDTD.FDTD_solve_cw.argtypes = [c_void_p, POINTER(SolveOptions), POINTER(SolveResult)]
libFDTD.FDTD_solve_cw.restype = c_int
libFDTD.FDTD_amp_phase_noalloc.argtypes = [c_int, c_void_p,
                                           ndpointer(np.complex128, flags="C_CONTIGUOUS"),
                                           c_longlong, c_char_p, c_int]
libFDTD.FDTD_amp_phase_noalloc.restype = c_int
NOALLOC_MAX_VALUES = 524288
libFDTD.FDTD_grad_eps.argtypes = [c_int, c_void_p, POINTER(c_void_p), POINTER(c_void_p), c_int,
                                  c_int, c_int, POINTER(c_int), c_int, c_void_p, c_char_p, c_int]
libFDTD.FDTD_grad_eps.restype = c_int
libFDTD.FDTD_serve_new.argtypes = [c_int, c_double, c_int, c_int]
libFDTD.FDTD_serve_new.restype = c_void_p
libFDTD.FDTD_serve_last_error.argtypes = [c_void_p, c_char_p, c_int]
libFDTD.FDTD_serve_last_error.restype = c_int
libFDTD.FDTD_serve_admit.argtypes = [c_void_p, c_void_p, POINTER(SolveOptions)]
libFDTD.FDTD_serve_admit.restype = c_int
libFDTD.FDTD_serve_advance.argtypes = [c_void_p]
libFDTD.FDTD_serve_advance.restype = c_int
libFDTD.FDTD_serve_finished.argtypes = [c_void_p, POINTER(c_void_p), c_int]
libFDTD.FDTD_serve_finished.restype = c_int
libFDTD.FDTD_serve_collect.argtypes = [c_void_p, POINTER(c_void_p), POINTER(SolveResult), c_int]
libFDTD.FDTD_serve_collect.restype = c_int
libFDTD.FDTD_serve_info.argtypes = [c_void_p, POINTER(c_double), POINTER(c_int)]
libFDTD.FDTD_serve_info.restype = c_int
libFDTD.FDTD_serve_delete.argtypes = [c_void_p]
libFDTD.FDTD_serve_delete.restype = None

# z slabs of a distributed solve (emopt_b200/zslab.py)
libFDTD.FDTD_set_stream.argtypes = [c_void_p, c_void_p]
libFDTD.FDTD_set_stream.restype = c_int
libFDTD.FDTD_slab_set.argtypes = [c_void_p, c_int, c_int, c_int, c_int]
libFDTD.FDTD_slab_set.restype = c_int
libFDTD.FDTD_slab_begin.argtypes = [c_void_p, POINTER(SolveOptions),
                                    ndpointer(np.int64, flags="C_CONTIGUOUS"), c_int]
libFDTD.FDTD_slab_begin.restype = c_int
libFDTD.FDTD_slab_step.argtypes = [c_void_p, c_longlong, c_int]
libFDTD.FDTD_slab_step.restype = c_int
libFDTD.FDTD_slab_step_part.argtypes = [c_void_p, c_longlong, c_int, c_int]
libFDTD.FDTD_slab_step_part.restype = c_int
libFDTD.FDTD_slab_halo.argtypes = [c_void_p, POINTER(c_void_p), POINTER(c_longlong)]
libFDTD.FDTD_slab_halo.restype = c_int
libFDTD.FDTD_slab_set_halo_source.argtypes = [c_void_p, POINTER(c_void_p)]
libFDTD.FDTD_slab_set_halo_source.restype = c_int
libFDTD.FDTD_slab_set_step.argtypes = [c_void_p, c_longlong]
libFDTD.FDTD_slab_set_step.restype = c_int
libFDTD.FDTD_slab_sample.argtypes = [c_void_p, POINTER(c_void_p)]
libFDTD.FDTD_slab_sample.restype = c_int
libFDTD.FDTD_slab_probe.argtypes = [c_void_p, c_longlong, POINTER(c_double), POINTER(c_double)]
libFDTD.FDTD_slab_probe.restype = c_int
libFDTD.FDTD_slab_capture.argtypes = [c_void_p, c_int]
libFDTD.FDTD_slab_capture.restype = c_int
libFDTD.FDTD_slab_finish.argtypes = [c_void_p, c_longlong, c_longlong]
libFDTD.FDTD_slab_finish.restype = c_int

libFDTD.FDTD_host_register.argtypes = [c_void_p, c_longlong]
libFDTD.FDTD_host_register.restype = c_int
libFDTD.FDTD_host_unregister.argtypes = [c_void_p]
libFDTD.FDTD_host_unregister.restype = c_int

# layered materials (emopt_b200/grid.py)
libFDTD.FDTD_structured_values.argtypes = [c_int, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                           c_void_p, c_void_p, c_int, c_void_p, c_int, c_void_p,
                                           c_int, c_double, c_double, c_double, c_int, c_int, c_int,
                                           c_int, c_int, c_int, c_double, c_double, c_double,
                                           c_void_p, c_char_p, c_int]
libFDTD.FDTD_structured_values.restype = c_int


class ModeLines(Structure):
    """FDTDModeLines: the plane's M x N points cut into lines (rows of
    constant y when sweep_y, else columns of constant x)."""
    _fields_ = [("M", c_int), ("N", c_int), ("sweep_y", c_int)]


libFDTD.FDTD_mode_last_error.argtypes = []
libFDTD.FDTD_mode_last_error.restype = c_char_p
libFDTD.FDTD_mode_assemble.argtypes = [c_void_p, c_int, c_void_p, c_double, c_double, c_double,
                                       c_double, c_double, c_void_p, c_char_p, c_void_p, c_void_p,
                                       c_void_p, c_void_p, c_void_p]
libFDTD.FDTD_mode_assemble.restype = c_int
libFDTD.FDTD_mode_bmul.argtypes = [c_void_p, c_int, c_void_p, c_double, c_void_p, c_void_p]
libFDTD.FDTD_mode_bmul.restype = c_int
libFDTD.FDTD_mode_lines_gemv.argtypes = [c_int, c_int, c_void_p, c_void_p, c_void_p, c_int, c_void_p,
                                         c_int, c_void_p, c_void_p, c_void_p]
libFDTD.FDTD_mode_lines_gemv.restype = c_int
libFDTD.FDTD_mode_couple.argtypes = [c_int, c_int, c_void_p, c_int, c_int, c_int, c_void_p, c_void_p,
                                     c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_double]
libFDTD.FDTD_mode_couple.restype = c_int
libFDTD.FDTD_mode_source.argtypes = [c_int, c_void_p, c_int, c_int, c_void_p, c_double, c_double,
                                     c_double, c_double, c_double, c_double, c_double, c_void_p,
                                     c_void_p, c_void_p, c_char_p, c_void_p]
libFDTD.FDTD_mode_source.restype = c_int

# The same library under a second handle whose array setters take raw
# pointers (device memory included); the reference-compatible bindings above
# accept numpy arrays only.
raw = cdll.LoadLibrary(so_path)
for _name in ("FDTD_set_mat_arrays", "FDTD_set_t0_arrays", "FDTD_set_t1_arrays"):
    getattr(raw, _name).argtypes = [c_void_p] + [c_void_p] * 6
    getattr(raw, _name).restype = None

# field access on the device (fieldops.py)
libFDTD.FDTD_interp_field.argtypes = [c_int, c_void_p, c_int, c_void_p, POINTER(c_int), c_void_p,
                                      c_char_p, c_int]
libFDTD.FDTD_interp_field.restype = c_int
libFDTD.FDTD_interp_field_T.argtypes = [c_int, c_void_p, c_int, c_void_p, POINTER(c_int), c_void_p,
                                        c_char_p, c_int]
libFDTD.FDTD_interp_field_T.restype = c_int
libFDTD.FDTD_dfdx_interp.argtypes = [c_int, c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_int,
                                     c_int, c_void_p, c_char_p, c_int]
libFDTD.FDTD_dfdx_interp.restype = c_int
libFDTD.FDTD_plane_flux.argtypes = [c_int, c_void_p, c_int, POINTER(c_void_p), POINTER(c_int),
                                    POINTER(c_int), c_void_p, c_char_p, c_int]
libFDTD.FDTD_plane_flux.restype = c_int

ADDED_SYMBOLS = ("FDTD_delete", "FDTD_last_error", "FDTD_set_device", "FDTD_set_zchunk",
                 "FDTD_set_precision", "FDTD_set_kernel", "FDTD_solve_cw",
                 "FDTD_amp_phase_noalloc", "FDTD_grad_eps", "FDTD_serve_new",
                 "FDTD_serve_last_error", "FDTD_serve_admit", "FDTD_serve_advance",
                 "FDTD_serve_finished", "FDTD_serve_collect", "FDTD_serve_info",
                 "FDTD_serve_delete", "FDTD_set_stream", "FDTD_slab_set", "FDTD_slab_begin",
                 "FDTD_slab_step", "FDTD_slab_step_part", "FDTD_slab_halo", "FDTD_slab_set_halo_source", "FDTD_slab_set_step", "FDTD_slab_sample", "FDTD_slab_probe",
                 "FDTD_slab_capture", "FDTD_slab_finish", "FDTD_structured_values",
                 "FDTD_host_register", "FDTD_host_unregister", "FDTD_mode_last_error",
                 "FDTD_mode_assemble", "FDTD_mode_bmul", "FDTD_mode_lines_gemv", "FDTD_mode_couple",
                 "FDTD_mode_source", "FDTD_interp_field", "FDTD_interp_field_T", "FDTD_dfdx_interp",
                 "FDTD_plane_flux")


class FDTDError(RuntimeError):
    """Raised when the library reports an error status."""


def last_error(handle) -> tuple[int, str]:
    buf = create_string_buffer(512)
    code = libFDTD.FDTD_last_error(handle, buf, 512)
    return code, buf.value.decode("utf-8", "replace")


def check(handle, what: str = "") -> None:
    """Raise FDTDError if the handle's last status is an error."""
    code, msg = last_error(handle)
    if code not in (FDTD_OK, FDTD_NMAX, FDTD_NONFINITE):
        raise FDTDError(f"{what}: {msg} (status {code})" if what else f"{msg} (status {code})")
