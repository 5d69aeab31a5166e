"""GPU test of axg_compute_stiffness_noalloc, the entry point for callers that cannot
allocate device memory (a process whose GPU memory another runtime already owns, such as
JAX/XLA with its up-front reservation, or code called back from such a runtime).

It must give what the existing axg_compute_stiffness gives on a handle at rest, on two
calls in a row: the fixed device array that holds the evaluation's SLS memory keeps the
previous call's contents, so each call has to clear it. Tolerances are those of the
stiffness parity tests (relative L2 over all point modes): FP64 1e-12, FP32 / mixed 1e-6.

The file sorts last so that a run stopping at its first failure has run everything else.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 1e-6, "mixed": 1e-6}


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _case(name):
    from axisem3d_b200 import meshgen
    return {
        # 3-D TI slices with 3 SLS (FULL): ~10.7 MB of SLS state in FP64
        "tiso_3d_full": lambda: meshgen.microbench_model(n_elem=150, nr_max=64, seed=21),
        # 1-D isotropic with FULL attenuation, on the axis
        "cart_iso_1d_full": lambda: meshgen.cartesian_model(
            nx=5, nz=4, nr=8, attenuation=dict(meshgen.default_sls(3), qkappa=57823.0, qmu=120.0)),
        # spherical shell: CG4 attenuation, RTZ frame, fluid layer (fluid pointers used)
        "sph_iso_3d_cg4_fluid": lambda: meshgen.spherical_model(n_theta=24, n_solid_layers=6,
                                                                n_fluid_layers=2, nr_max=40),
    }[name]()


def _call(s, xs, fs, xf=None, ff=None):
    """axg_compute_stiffness_noalloc through the C ABI; returns the status code."""
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
    return s.lib.axg_compute_stiffness_noalloc(s.h, ptr(xs), ptr(fs), ptr(xf), ptr(ff))


@pytest.mark.parametrize("precision", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("case", ["tiso_3d_full", "cart_iso_1d_full", "sph_iso_3d_cg4_fluid"])
def test_noalloc_stiffness_matches_compute_stiffness(built, case, precision):
    import torch
    from axisem3d_b200 import _lib as L, meshgen
    from axisem3d_b200.solver import Solver
    m = _case(case)
    fluid = len(m.fe_nr) > 0
    us = meshgen.random_displacement(m, seed=5)
    uf = meshgen.random_displacement(m, seed=6, solid=False) if fluid else None
    # the existing entry point on a freshly created handle
    with Solver(m, precision) as s:
        s.set_field(us, "displ")
        if fluid:
            s.set_field(uf, "displ", solid=False)
        s.compute_stiffness()
        ref_s = s.get_field("stiff")
        ref_f = s.get_field("stiff", solid=False) if fluid else None
    # the new entry point on caller-owned device buffers, twice in a row
    cdt = torch.complex128 if precision == "fp64" else torch.complex64
    dev = torch.device("cuda", 0)
    xs = torch.tensor(us, dtype=cdt, device=dev)
    fs = torch.zeros_like(xs)
    xf = torch.tensor(uf, dtype=cdt, device=dev) if fluid else None
    ff = torch.zeros_like(xf) if fluid else None
    with Solver(m, precision) as s:
        for call in range(2):
            fs.zero_()
            if fluid:
                ff.zero_()
            torch.cuda.synchronize()          # the engine's stream does not wait for torch's
            assert _call(s, xs, fs, xf, ff) == L.AXG_OK, s.lib.axg_last_error(s.h)
            s.synchronize()
            got = fs.cpu().numpy().astype(np.complex128)
            assert rel(got, ref_s) <= TOL[precision], (call, rel(got, ref_s))
            if fluid:
                gotf = ff.cpu().numpy().astype(np.complex128)
                assert rel(gotf, ref_f) <= TOL[precision], (call, rel(gotf, ref_f))
        # the handle's own stiffness field was not touched
        assert not np.any(s.get_field("stiff"))


def test_noalloc_rejects_state_beyond_the_fixed_array(built):
    """A model whose SLS state exceeds AXG_NOALLOC_SCRATCH_BYTES gets AXG_E_ARG with a
    message, before any work is queued."""
    import torch
    from axisem3d_b200 import _lib as L, meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.microbench_model(n_elem=2000, nr_max=64, seed=3)      # ~146 MB of FP64 state
    dev = torch.device("cuda", 0)
    with Solver(m, "mixed") as s:
        n = s.field_size()
        xs = torch.zeros(n, dtype=torch.complex64, device=dev)
        fs = torch.zeros_like(xs)
        torch.cuda.synchronize()
        assert _call(s, xs, fs) == L.AXG_E_ARG
        assert b"exceeds the fixed scratch" in s.lib.axg_last_error(s.h)
        s.synchronize()
        assert not torch.any(fs).item()
