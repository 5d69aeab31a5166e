"""A compiled C++ caller of include/axg.h (tests/cabi/axg_run_model.cpp).

The reference's time loop is C++, so the drop-in is bound from C++: the program includes only
the header and links libaxg.so. On the CPU the test compiles and links it (every symbol the
program uses resolves); on the GPU it runs the plain forward case (40 x 40 quads, nr = 5, the
axial moment source, 20 stations) through it and compares the displacement field and the
seismograms with the same run through the Python binding: bitwise equal (the same library
calls in the same order, with deterministic assembly so that the atomic sums cannot reorder).
"""
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cabi", "axg_run_model.cpp")


def _build(tmpdir):
    from axisem3d_b200.build import build
    lib = build()
    exe = os.path.join(str(tmpdir), "axg_run_model")
    libdir = os.path.dirname(lib)
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
                    "-L", libdir, "-laxg", "-Wl,-rpath," + libdir, "-o", exe], check=True)
    return exe


def _dump(m, path):
    """The model's arrays in the runner's dump format."""
    recs = [("dt", "d", [m.dt]), ("t0", "d", [m.t0]), ("sp_nr", "i", m.sp_nr), ("sp_mass", "d", m.sp_mass),
            ("sp_axial", "b", m.sp_axial), ("se_nr", "i", m.se_nr), ("se_pts", "i", m.se_pts),
            ("se_axial", "b", m.se_axial), ("se_geom", "d", m.se_geom), ("se_rheo", "i", m.se_rheo),
            ("se_mat_off", "l", m.se_mat_off), ("se_moduli", "d", m.se_moduli),
            ("ms_elem", "i", m.ms_elem), ("ms_nu", "i", m.ms_nu), ("ms_pat_off", "l", m.ms_pat_off),
            ("ms_pattern", "d", np.asarray(m.ms_pattern, np.complex128).view(np.float64)),
            ("ms_stf", "d", [[s.half_duration, s.decay_factor, s.time_shift, s.derivative_order] for s in m.ms_stf]),
            ("st_elem", "i", m.st_elem), ("st_w", "d", m.st_w), ("st_phi", "d", m.st_phi)]
    dt = {"d": np.float64, "i": np.int32, "l": np.int64, "b": np.uint8}
    with open(path, "wb") as f:
        for name, t, a in recs:
            a = np.ascontiguousarray(np.asarray(a, dt[t]).ravel())
            f.write(struct.pack("<I", len(name)) + name.encode() + t.encode() + struct.pack("<Q", a.size))
            f.write(a.tobytes())


def test_header_is_plain_c_and_links_from_c(built, tmp_path):
    """include/axg.h is an ISO C99 header (plain pointers, fixed-width integers, no C++): a C
    translation unit that takes the address of every declared entry point compiles with
    -std=c99 -pedantic -Werror and links against libaxg.so with the C driver, so C and Fortran
    (ISO_C_BINDING) callers can bind it as well as the reference's C++. Runs without a GPU (no
    entry point is called)."""
    import re
    from axisem3d_b200.build import build
    lib = build()
    hdr = open(os.path.join(ROOT, "include", "axg.h")).read()
    names = sorted(set(re.findall(r"\b(axg_[a-z0-9_]+)\s*\(", hdr)))
    src = os.path.join(str(tmp_path), "c_abi.c")
    with open(src, "w") as f:
        f.write('#include "axg.h"\n#include <stdio.h>\ntypedef void (*fn_t)(void);\nint main(void) {\n'
                "    fn_t fns[] = {\n")
        f.write("".join("        (fn_t)%s,\n" % n for n in names))
        f.write('    };\n    printf("%d\\n", (int)(sizeof fns / sizeof fns[0]));\n    return 0;\n}\n')
    exe = os.path.join(str(tmp_path), "c_abi")
    libdir = os.path.dirname(lib)
    subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    src, "-L", libdir, "-laxg", "-Wl,-rpath," + libdir, "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    assert int(out) == len(names) > 30


def test_cabi_program_compiles_and_links(built, tmp_path):
    exe = _build(tmp_path)
    assert os.access(exe, os.X_OK)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cabi_program_matches_python_binding(built, tmp_path, precision):
    from axisem3d_b200 import _lib as L
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    exe = _build(tmp_path)
    m = meshgen.cartesian_model()
    assert m.se_att is None and m.sp_mass_nr is None and m.cl_solid is None
    dump = os.path.join(str(tmp_path), "cfg0.bin")
    _dump(m, dump)
    nsteps = 300
    out = os.path.join(str(tmp_path), "run")
    r = subprocess.run([exe, dump, str(L.PRECISIONS[precision]), str(nsteps), out, "1"], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    u = np.fromfile(out + ".displ", np.float64).view(np.complex128)
    seis = np.fromfile(out + ".seis", np.float64).reshape(nsteps, len(m.st_elem), 3)
    with Solver(m, precision, deterministic=True) as s:
        s.run(nsteps)
        ref = s.get_field("displ")
        ref_seis = s.seismograms()
    assert np.abs(ref).max() > 0 and np.abs(ref_seis).max() > 0
    assert np.array_equal(u, ref)
    assert np.array_equal(seis, ref_seis)
