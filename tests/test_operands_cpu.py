"""The engine's operand builder (libaxg.so, csrc/operands.cpp) against the oracle's own
restatement (oracle/axg_operands_oracle.cpp), on the workloads' meshes.

Both follow the reference's preloop: MappingLinear / MappingSpherical,
Quad::computeIntegralFactor (the axial GLJ branch with L'Hospital's rule on the axis),
Quad::createGradient, Quad::computeDt and AttBuilder. They are written separately, so a
wrong integral factor, Jacobian or 1/s in either one shows here even though the parity tests
feed both the engine and the oracle from one model. Tolerance: 1e-13 relative per operand
component (the two differ only in summation order).
"""
import numpy as np
import pytest

GEOM = ["dsdxii", "dsdeta", "dzdxii", "dzdeta", "inv_s", "ifact"]


def _pair(build):
    import oracle as O
    from axisem3d_b200 import meshgen
    with meshgen.operands(O.OracleOperands()):
        a = build(meshgen)
    b = build(meshgen)
    return a, b


def _check_geometry(ga, gb, tol=1e-13):
    ga, gb = np.asarray(ga), np.asarray(gb)
    assert ga.shape == gb.shape
    # the four inverse-Jacobian terms are measured against the element's largest one (on
    # rectangular quads two of them are zero up to cancellation noise); 1/s and the integral
    # factor entry by entry
    jscale = np.abs(gb[:, :4, :]).max(axis=(1, 2))[:, None]
    for c, name in enumerate(GEOM):
        x, y = ga[:, c, :], gb[:, c, :]
        scale = jscale if c < 4 else np.maximum(np.abs(y), np.abs(y).max(axis=1)[:, None] * 1e-3)
        err = float(np.max(np.abs(x - y) / scale))
        assert err <= tol, (name, err)


def test_spectral_tables_agree(built):
    import oracle as O
    from axisem3d_b200.solver import spectral_tables
    a, b = O.OracleOperands().tables(), spectral_tables()
    for k in ("pGLL", "pGLJ", "wGLL", "wGLJ", "gGLL", "gGLJ"):
        assert np.array_equal(np.asarray(a[k]).ravel(), np.asarray(b[k]).ravel()), k


@pytest.mark.parametrize("case", ["cartesian_axis", "microbench", "microbench_axial", "shell"])
def test_geometry_and_dt_agree(built, case):
    builders = {
        # plain forward case: the axis column uses the GLJ branch and L'Hospital's rule
        "cartesian_axis": lambda mg: mg.cartesian_model(nx=12, nz=10, nr=5),
        # the stiffness microbenchmark's perturbed quads (non-axial)
        "microbench": lambda mg: mg.microbench_model(n_elem=3000, nr_max=64, seed=7),
        "microbench_axial": lambda mg: mg.microbench_model(n_elem=400, nr_max=16, seed=8, axial_column=True),
        # spherical shell: MappingSpherical in all orientations, axis at both ends, fluid layer
        "shell": lambda mg: mg.spherical_model(n_theta=48, n_solid_layers=10, n_fluid_layers=2),
    }
    a, b = _pair(builders[case])
    _check_geometry(a.se_geom, b.se_geom)
    if len(getattr(b, "fe_geom", [])):
        _check_geometry(a.fe_geom, b.fe_geom)
    assert np.any(b.se_axial) == (case != "microbench")
    # masses are integral factor x density, summed over elements
    assert np.max(np.abs(a.sp_mass - b.sp_mass) / np.abs(b.sp_mass)) <= 1e-13
    # dt rounded to 4 significant figures comes out the same
    assert a.dt == b.dt


def test_attenuation_operands_agree(built):
    """AttBuilder: alpha, beta, gamma and the FULL unrelaxed moduli and defects."""
    import oracle as O
    from axisem3d_b200 import meshgen
    sls = meshgen.default_sls(5)
    e, o = meshgen.EngineOperands(), O.OracleOperands()
    for dt in (0.01, 0.37):
        for x, y in zip(e.att_alpha_beta_gamma(sls["w"], sls["y"], dt),
                        o.att_alpha_beta_gamma(sls["w"], sls["y"], dt)):
            assert np.max(np.abs(x - y) / np.abs(y)) <= 1e-14
    rng = np.random.Generator(np.random.PCG64(4))
    kp, mu = rng.uniform(1e10, 2e11, 500), rng.uniform(1e10, 8e10, 500)
    qk, qm = rng.uniform(200, 60000, 500), rng.uniform(50, 600, 500)
    for x, y in zip(e.att_moduli(sls["w"], sls["y"], sls["fmin"], sls["fmax"], sls["fref"], qk, qm, kp, mu),
                    o.att_moduli(sls["w"], sls["y"], sls["fmin"], sls["fmax"], sls["fref"], qk, qm, kp, mu)):
        assert np.max(np.abs(x - y) / np.abs(y)) <= 1e-13


def test_oracle_built_workload_needs_no_engine_library():
    """A workload built with the oracle's operands loads only the oracle's library: run in a
    fresh process, which then lists the shared objects it mapped."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys; sys.path[:0] = [%r, %r]\n"
            "import oracle as O\n"
            "from axisem3d_b200 import meshgen\n"
            "with meshgen.operands(O.OracleOperands()):\n"
            "    m = meshgen.microbench_model(n_elem=500, nr_max=32, seed=3)\n"
            "o = O.Oracle(m, 'fp32')\n"
            "o.compute_stiffness()\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('libaxg' in maps, 'liboracle' in maps)\n" % (root, os.path.join(root, "oracle")))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["False", "True"]
