"""Parity at the benchmark's full size: the stiffness microbenchmark of `bench.py` (200 000 TI
quads, nr log-uniform on [1, 64], 3-D slices, 3 SLS FULL, seed 1), through the C ABI, against
the FP64 oracle on the same model.

Two stiffness evaluations from one random displacement (the second starts from the SLS memory
the first left), as the reference's `SolidElement::computeStiff` would run them in two steps.
Bars: 1e-6 relative L2 over every point mode for the mixed and FP32 engines (the FP32 bar of
the stiffness forces), 1e-12 for the FP64 engine; the stiffness of every nr bucket is checked on its own as well, so an
error confined to the rare large-nr elements cannot hide in the norm of the whole field.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_ELEM = 200000
TOL = {"mixed": 1e-6, "fp32": 1e-6, "fp64": 1e-12}


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def fullsize(built):
    import oracle as O
    from axisem3d_b200 import meshgen
    m = meshgen.microbench_model(n_elem=N_ELEM, nr_max=64, seed=1)
    u = meshgen.random_displacement(m, seed=2)
    o = O.Oracle(m, "fp64", threads=os.cpu_count() or 1)
    o.set_field(u, "displ")
    o.compute_stiffness()
    first = o.get_field("stiff")
    o.set_field(np.zeros_like(u), "stiff")
    o.compute_stiffness()
    second = o.get_field("stiff")
    o.close()
    return m, u, first, second


def _point_slots(m, lo, hi):
    """Complex slots of the points whose largest nr lies in (lo, hi]."""
    nr = np.asarray(m.sp_nr, np.int64)
    nu = nr // 2 + 1
    first = np.concatenate([[0], np.cumsum(nu)[:-1]]) * 3
    sel = np.nonzero((nr > lo) & (nr <= hi))[0]
    cnt = nu[sel] * 3
    start = np.concatenate([[0], np.cumsum(cnt)[:-1]])
    return np.repeat(first[sel] - start, cnt) + np.arange(int(cnt.sum()))


@pytest.mark.parametrize("precision", ["mixed", "fp32", "fp64"])
def test_microbenchmark_full_size_matches_oracle(fullsize, precision):
    from axisem3d_b200.solver import Solver
    m, u, ref1, ref2 = fullsize
    assert m.n_solid_elements == N_ELEM
    with Solver(m, precision) as s:
        s.set_field(u, "displ")
        s.compute_stiffness()
        f1 = s.get_field("stiff")
        s.set_field(np.zeros_like(u), "stiff")
        s.compute_stiffness()
        f2 = s.get_field("stiff")
    assert np.abs(ref2).max() > 0
    tol = TOL[precision]
    assert rel(f1, ref1) <= tol, rel(f1, ref1)
    assert rel(f2, ref2) <= tol, rel(f2, ref2)
    for lo, hi in ((0, 3), (3, 9), (9, 25), (25, 64)):
        sl = _point_slots(m, lo, hi)
        if len(sl):
            assert rel(f2[sl], ref2[sl]) <= tol, (lo, hi, rel(f2[sl], ref2[sl]))
