"""CPU tests of the C-ABI library: it loads without a GPU, exports every symbol
declared in include/emopt_fdtd.h, keeps the reference's ctypes signatures, and
its pure scalar entry points agree with the reference's known answers."""
import ctypes
import os
import re

import numpy as np
import pytest

from helpers import ROOT, golden


def header_symbols():
    text = open(os.path.join(ROOT, "include", "emopt_fdtd.h")).read()
    return sorted(set(re.findall(r"\b(FDTD_[A-Za-z0-9_]+)\s*\(", text)))


def test_library_exports_header_symbols():
    from emopt_b200 import fdtd_ctypes as ct
    lib = ctypes.CDLL(ct.so_path)
    syms = header_symbols()
    assert len(syms) == 74
    for s in syms:
        assert hasattr(lib, s), s
    assert set(ct.REFERENCE_SYMBOLS) | set(ct.ADDED_SYMBOLS) == set(syms)


def test_checked_library_exports_the_same_symbols():
    """FDTD_checked.so (index-checked stepping kernels) is a drop-in for FDTD.so."""
    from emopt_b200 import build
    lib = ctypes.CDLL(build.CHECKED)
    for s in header_symbols():
        assert hasattr(lib, s), s
    # EMOPT_B200_LIB selects it for the ctypes binding
    import subprocess
    import sys
    code = "import emopt_b200.fdtd_ctypes as ct, os; print(os.path.basename(ct.so_path))"
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         env=dict(os.environ, EMOPT_B200_LIB=build.CHECKED), timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "FDTD_checked.so"


def test_binding_declares_reference_symbols():
    """This package's binding declares the 32 reference symbols (the reference's
    own binding, unchanged, is driven in tests/test_reference_binding.py)."""
    from emopt_b200 import fdtd_ctypes as ct
    assert len(ct.REFERENCE_SYMBOLS) == 32
    for name in ct.REFERENCE_SYMBOLS:
        fn = getattr(ct.libFDTD, name)
        assert fn.argtypes is not None


def test_struct_layouts():
    from emopt_b200 import fdtd_ctypes as ct
    assert ctypes.sizeof(ct.SolveOptions) == 64
    assert ctypes.sizeof(ct.SolveResult) == 72


def test_scalar_entry_points_match_reference_kat():
    from emopt_b200 import fdtd_ctypes as ct
    lib = ct.libFDTD
    g = golden("kat_fit.npz")
    t, f = g["t"], g["f"]
    ph3 = np.array([lib.FDTD_calc_phase_3T(*t[q], *f[q]) for q in range(len(t))])
    am3 = np.array([lib.FDTD_calc_amplitude_3T(*t[q], *f[q], g["phase3"][q]) for q in range(len(t))])
    ph2 = np.array([lib.FDTD_calc_phase_2T(t[q, 0], t[q, 1], f[q, 0], f[q, 1]) for q in range(len(t))])
    am2 = np.array([lib.FDTD_calc_amplitude_2T(t[q, 0], t[q, 1], f[q, 0], f[q, 1], g["phase2"][q])
                    for q in range(len(t))])
    # same formulas, same libm on the host: identical
    np.testing.assert_array_equal(ph3, g["phase3"])
    np.testing.assert_array_equal(am3, g["amp3"])
    np.testing.assert_array_equal(ph2, g["phase2"])
    np.testing.assert_array_equal(am2, g["amp2"])
    h = lib.FDTD_new()
    lib.FDTD_set_source_properties(h, float(g["src_T"]), float(g["src_min"]))
    vals = [lib.FDTD_src_func_t(h, q, g["src_t"][q], g["src_phase"][q]) for q in range(len(g["src_t"]))]
    np.testing.assert_array_equal(vals, g["src_value"])
    lib.FDTD_delete(h)


def test_no_device_fails_loudly():
    """Without a GPU the handle reports FDTD_ERR_NODEVICE and the Python class raises."""
    from conftest import has_cuda
    if has_cuda():
        pytest.skip("a CUDA device is present")
    from emopt_b200 import fdtd_ctypes as ct
    from emopt_b200 import problems as P
    h = ct.libFDTD.FDTD_new()
    code, msg = ct.last_error(h)
    assert code == ct.FDTD_ERR_NODEVICE and "no CUDA device" in msg
    opt, res = ct.SolveOptions(), ct.SolveResult()
    opt.Tn = 10
    assert ct.libFDTD.FDTD_solve_cw(h, ctypes.byref(opt), ctypes.byref(res)) == ct.FDTD_ERR_NODEVICE
    ct.libFDTD.FDTD_delete(h)
    with pytest.raises(ct.FDTDError):
        P.make_solver(P.random_box(0))


def test_argument_errors_are_reported():
    from emopt_b200 import fdtd_ctypes as ct
    h = ct.libFDTD.FDTD_new()
    assert ct.libFDTD.FDTD_set_precision(h, 16) == ct.FDTD_ERR_ARG
    assert "precision" in ct.last_error(h)[1]
    assert ct.libFDTD.FDTD_set_kernel(h, 8) == ct.FDTD_ERR_ARG
    # the kernel ids the library keeps: auto, scalar, fused, vector, split
    for k in (0, 1, 3, 5, 6):
        assert ct.libFDTD.FDTD_set_kernel(h, k) == ct.FDTD_OK, k
    for k in (2, 4, 7, -1):
        assert ct.libFDTD.FDTD_set_kernel(h, k) == ct.FDTD_ERR_ARG, k
    assert "kernel must be" in ct.last_error(h)[1]
    ct.libFDTD.FDTD_delete(h)


def test_mode_entry_points_reject_bad_arguments():
    """The mode-solver entry points validate their arguments before any CUDA
    call and report FDTD_ERR_ARG with a message."""
    from emopt_b200 import fdtd_ctypes as ct
    lib = ct.libFDTD
    g = ct.ModeLines(0, 5, 1)
    assert lib.FDTD_mode_assemble(ctypes.byref(g), 0, None, 1.0, 1.0, 1.0, 3.0, 0.0, None, b"00",
                                  None, None, None, None, None) == ct.FDTD_ERR_ARG
    assert b"FDTD_mode_assemble" in lib.FDTD_mode_last_error()
    assert lib.FDTD_mode_bmul(None, 0, None, 1.0, None, None) == ct.FDTD_ERR_ARG
    dummy = ctypes.c_void_p(16)
    assert lib.FDTD_mode_lines_gemv(6, 0, None, dummy, dummy, 0, None, 6, dummy, None, dummy) == ct.FDTD_ERR_ARG
    assert lib.FDTD_mode_lines_gemv(6, 0, None, dummy, dummy, 1, None, 5, dummy, None, dummy) == ct.FDTD_ERR_ARG
    assert b"lines_gemv" in lib.FDTD_mode_last_error()
    assert lib.FDTD_mode_couple(6, 0, None, 1, 0, 2, dummy, dummy, dummy, dummy, dummy, dummy, dummy,
                                1.0) == ct.FDTD_ERR_ARG
    assert lib.FDTD_mode_source(0, None, 0, 3, dummy, 1.0, 0.0, 1.0, 0.0, 1.0, 1.0, 1.0, dummy, dummy,
                                dummy, b"00", dummy) == ct.FDTD_ERR_ARG


def test_header_struct_fields_match_binding(tmp_path):
    """Every field of the ctypes structures exists in the C structures of
    include/emopt_fdtd.h under the same name and at the same offset (a binding
    that drifted from the header would read or write the wrong bytes)."""
    import shutil
    import subprocess
    from emopt_b200 import fdtd_ctypes as ct
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    pairs = [("FDTDSolveOptions", ct.SolveOptions), ("FDTDSolveResult", ct.SolveResult),
             ("FDTDModeLines", ct.ModeLines)]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "emopt_fdtd.h"', 'int main(void) {']
    for cname, cls in pairs:
        for f in cls._fields_:
            lines.append('    printf("%%s %%s %%zu\\n", "%s", "%s", offsetof(%s, %s));' % (cname, f[0], cname, f[0]))
    lines += ['    return 0;', '}']
    src = tmp_path / "offsets.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "offsets"
    subprocess.run(["gcc", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {(a, b): int(c) for a, b, c in (ln.split() for ln in out if ln.strip())}
    for cname, cls in pairs:
        for f in cls._fields_:
            assert got[(cname, f[0])] == getattr(cls, f[0]).offset, (cname, f[0])


def test_header_compiles_and_struct_sizes_match_binding(tmp_path):
    """include/emopt_fdtd.h compiles as C and C++, and the structures the
    ctypes binding mirrors have the same sizes in C."""
    import shutil
    import subprocess
    from emopt_b200 import fdtd_ctypes as ct
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include "emopt_fdtd.h"\n'
                   'int main(void) { printf("%zu %zu %zu\\n", sizeof(FDTDSolveOptions), '
                   'sizeof(FDTDSolveResult), sizeof(FDTDModeLines)); return 0; }\n')
    exe = tmp_path / "sizes"
    inc = os.path.join(ROOT, "include")
    subprocess.run(["gcc", "-Wall", "-Werror", "-I", inc, str(src), "-o", str(exe)], check=True)
    subprocess.run(["g++", "-fsyntax-only", "-Wall", "-Werror", "-x", "c++", os.path.join(inc, "emopt_fdtd.h")],
                   check=True)
    sizes = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert sizes == [ctypes.sizeof(ct.SolveOptions), ctypes.sizeof(ct.SolveResult), ctypes.sizeof(ct.ModeLines)]
