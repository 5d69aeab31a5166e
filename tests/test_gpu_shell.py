"""GPU parity of the spherical-shell workload's generator at a reduced size.

The shell workload (half annulus r 3480-6371 km, a fluid layer 3480-3600 km under the
solid, a 2 % dlnVs random field of 200 km correlation sampled on every element's slices,
per-element nr from the field's azimuthal bandwidth in [3, 128], CG4 attenuation with
Q_mu = 300, a moment tensor with a 20 s Ricker wavelet) built with 48 x (2 fluid + 8 solid)
quads and run from rest through the engine's C ABI against the FP64 oracle: the
displacement of every solid and fluid point mode after the given steps.

Tolerances (relative L2): FP64 engine <= 1e-10; mixed (FP32 bulk, FP64 Newmark and SLS
state) <= 1e-4, the seismogram bar.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "mixed": 1e-4}


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def shell_case(built):
    import oracle as O
    from axisem3d_b200 import meshgen
    m = meshgen.spherical_model(n_theta=48, n_solid_layers=8, n_fluid_layers=2)
    nsteps = 120
    o = O.Oracle(m, "fp64", threads=16)
    o.run(nsteps)
    return m, nsteps, o.get_field("displ"), o.get_field("displ", solid=False), o.seismograms()


def test_reduced_shell_has_the_workload_features(shell_case):
    m = shell_case[0]
    assert len(m.fe_nr) > 0 and len(m.sf_solid) > 0          # fluid layer coupled to the solid
    assert m.se_nr.min() <= 9 and m.se_nr.max() >= 100       # nr spans the field's range
    assert np.all(m.se_is3d == 1) and np.all(m.se_att == 2)  # 3-D slices, CG4


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_reduced_shell_matches_oracle(shell_case, precision):
    from axisem3d_b200.solver import Solver
    m, nsteps, ref_s, ref_f, ref_seis = shell_case
    with Solver(m, precision) as s:
        s.run(nsteps)
        ds, df = s.get_field("displ"), s.get_field("displ", solid=False)
        seis = s.seismograms()
    assert np.abs(ref_s).max() > 0 and np.abs(ref_f).max() > 0
    assert rel(ds, ref_s) <= TOL[precision], rel(ds, ref_s)
    assert rel(df, ref_f) <= TOL[precision], rel(df, ref_f)
    assert seis.shape == ref_seis.shape
