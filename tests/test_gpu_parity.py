"""GPU parity: the CUDA engine, called through the C ABI, against the FP64 oracle.

Tolerances (relative L2 over all point modes, stated per test):
  per-step stiffness    FP64 engine <= 1e-12, FP32 / mixed engine <= 1e-6
  full steps            FP64 <= 1e-11; FP32 / mixed <= 1e-5 after 5 steps
  seismograms           every precision <= 1e-4 after the full plain-forward run
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_STIFF = {"fp64": 1e-12, "fp32": 1e-6, "mixed": 1e-6}


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _case(name):
    from axisem3d_b200 import meshgen
    mb = meshgen.microbench_model
    return {
        "cart_iso_1d_axial": lambda: meshgen.cartesian_model(nx=6, nz=6, nr=5),
        "cart_iso_1d_full": lambda: meshgen.cartesian_model(
            nx=5, nz=4, nr=8, attenuation=dict(meshgen.default_sls(3), qkappa=57823.0, qmu=120.0)),
        "tiso_3d_full": lambda: mb(n_elem=150, nr_max=64, seed=21),
        "tiso_3d_full_axial": lambda: mb(n_elem=60, nr_max=32, seed=22, axial_column=True),
        "tiso_1d_full": lambda: mb(n_elem=120, nr_max=64, seed=23, is3d=False),
        "iso_3d_elastic": lambda: mb(n_elem=100, nr_max=48, seed=24, rheology="iso", attenuation=None),
        "iso_1d_full_axial": lambda: mb(n_elem=60, nr_max=20, seed=25, rheology="iso", is3d=False,
                                        axial_column=True),
        "tiso_3d_cg4": lambda: mb(n_elem=60, nr_min=8, nr_max=8, seed=26, attenuation="cg4"),
        "tiso_1d_cg4": lambda: mb(n_elem=60, nr_min=6, nr_max=6, seed=27, attenuation="cg4", is3d=False),
        "aniso_3d": lambda: mb(n_elem=80, nr_max=40, seed=28, rheology="aniso", attenuation=None),
        "aniso_1d_axial": lambda: mb(n_elem=60, nr_max=16, seed=29, rheology="aniso", attenuation=None,
                                     is3d=False, axial_column=True),
        "nr1_only": lambda: mb(n_elem=40, nr_min=1, nr_max=1, seed=30),
    }[name]()


CASES = ["cart_iso_1d_axial", "cart_iso_1d_full", "tiso_3d_full", "tiso_3d_full_axial", "tiso_1d_full",
         "iso_3d_elastic", "iso_1d_full_axial", "tiso_3d_cg4", "tiso_1d_cg4", "aniso_3d",
         "aniso_1d_axial", "nr1_only"]


def _oracle_stiff(m, u, steps=1):
    import oracle as O
    o = O.Oracle(m, "fp64")
    o.set_field(u, "displ")
    for _ in range(steps):
        o.set_field(np.zeros_like(u), "stiff")
        o.compute_stiffness()
    return o.get_field("stiff")


@pytest.mark.parametrize("precision", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("case", CASES)
def test_stiffness_parity(built, case, precision):
    """Domain::computeStiffness through axg_compute_stiffness vs the FP64 oracle,
    two evaluations in a row (the second exercises the attenuation memory)."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = _case(case)
    u = meshgen.random_displacement(m, seed=5)
    ref1 = _oracle_stiff(m, u, 1)
    ref2 = _oracle_stiff(m, u, 2)
    with Solver(m, precision) as s:
        s.set_field(u, "displ")
        s.compute_stiffness()
        f1 = s.get_field("stiff")
        s.set_field(np.zeros_like(u), "stiff")
        s.compute_stiffness()
        f2 = s.get_field("stiff")
    assert rel(f1, ref1) <= TOL_STIFF[precision], rel(f1, ref1)
    assert rel(f2, ref2) <= TOL_STIFF[precision], rel(f2, ref2)


LARGE_NR = {
    # (nr_min, nr_max) per precision: FP64 up to 128 (the spherical-shell workload's range),
    # FP32 / mixed up to 256
    "fp64": (96, 128), "fp32": (200, 256), "mixed": (200, 256),
}


@pytest.mark.parametrize("precision", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("kind", ["tiso_3d_full", "tiso_1d_full", "aniso_3d_axial"])
def test_large_nr_mode_tiles(built, precision, kind):
    """Large nr: an element's modes no longer fit shared memory whole, so the gather /
    gradient and the quadrature run over tiles of modes and the slice phase over chunks of
    points. Two evaluations in a row against the FP64 oracle (the second exercises the SLS
    memory of every slice or mode)."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    lo, hi = LARGE_NR[precision]
    if kind == "tiso_3d_full":
        lo = hi          # every element at the largest nr: 128 in FP64, 256 in FP32 / mixed
    kw = {"tiso_3d_full": dict(),
          "tiso_1d_full": dict(is3d=False),
          "aniso_3d_axial": dict(rheology="aniso", attenuation=None, axial_column=True)}[kind]
    m = meshgen.microbench_model(n_elem=12, nr_min=lo, nr_max=hi, seed=31, **kw)
    assert m.se_nr.max() >= hi - 4
    u = meshgen.random_displacement(m, seed=6)
    ref1 = _oracle_stiff(m, u, 1)
    ref2 = _oracle_stiff(m, u, 2)
    with Solver(m, precision) as s:
        s.set_field(u, "displ")
        s.compute_stiffness()
        f1 = s.get_field("stiff")
        s.set_field(np.zeros_like(u), "stiff")
        s.compute_stiffness()
        f2 = s.get_field("stiff")
    assert rel(f1, ref1) <= TOL_STIFF[precision], rel(f1, ref1)
    assert rel(f2, ref2) <= TOL_STIFF[precision], rel(f2, ref2)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("fp32", 1e-5), ("mixed", 1e-5)])
def test_full_steps_parity(built, precision, tol):
    """Five full Newmark steps (sources, stiffness, BCs, mass, update) with
    attenuation, on the axis, vs the oracle's NewmarkTimeScheme loop."""
    import oracle as O
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.cartesian_model(nx=6, nz=6, nr=5,
                                attenuation=dict(meshgen.default_sls(3), qkappa=57823.0, qmu=100.0))
    u0 = meshgen.random_displacement(m, seed=8) * 1e-3
    o = O.Oracle(m, "fp64")
    o.set_field(u0, "displ")
    o.run(5)
    with Solver(m, precision) as s:
        s.set_field(u0, "displ")
        s.run(5, graph=True)
        for f in ("displ", "veloc", "accel"):
            assert rel(s.get_field(f), o.get_field(f)) <= tol, (f, rel(s.get_field(f), o.get_field(f)))
        assert s.step == 5


def test_graph_equals_eager_and_hooks(built):
    """One CUDA graph per step == eager launches == the individual Domain hooks (FP64)."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.cartesian_model(nx=5, nz=5, nr=5)
    u0 = meshgen.random_displacement(m, seed=9) * 1e-3
    out = []
    for mode in ("graph", "eager", "hooks"):
        with Solver(m, "fp64") as s:
            s.set_field(u0, "displ")
            if mode == "hooks":
                for t in range(4):
                    s.apply_sources(t)
                    s.compute_stiffness()
                    s.apply_bc_before_assembly()
                    s.record_stations(t)
                    s.apply_bc_after_assembly()
                    s.stiff_to_accel()
                    s.newmark_update()
            else:
                s.run(4, graph=(mode == "graph"))
            out.append((s.get_field("displ"), s.get_field("veloc")))
    for d, v in out[1:]:
        assert rel(d, out[0][0]) <= 1e-13 and rel(v, out[0][1]) <= 1e-13


@pytest.mark.parametrize("precision", ["fp64", "fp32", "mixed"])
def test_seismograms_plain_forward(built, precision):
    """Plain forward case (40 x 40 quads, nr = 5, axial moment tensor, 20 surface
    receivers, 2000 steps): seismogram rel-L2 vs the FP64 oracle <= 1e-4."""
    import oracle as O
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.cartesian_model()
    nsteps = 2000
    ref = _reference_seismograms(m, nsteps)
    with Solver(m, precision) as s:
        s.run(nsteps, graph=True)
        seis = s.seismograms()
    assert seis.shape == ref.shape
    err = rel(seis, ref)
    assert err <= 1e-4, err


_REF_CACHE = {}


def _reference_seismograms(m, nsteps):
    import oracle as O
    key = (m.meta["workload"], nsteps)
    if key not in _REF_CACHE:
        o = O.Oracle(m, "fp64", threads=8)
        o.run(nsteps)
        _REF_CACHE[key] = o.seismograms()
    return _REF_CACHE[key]


def test_error_paths(built):
    """Host-side validation: bad indices and out-of-order calls come back as
    AXG_E_* codes with the reference-style message; nothing faults."""
    import ctypes as C
    from axisem3d_b200 import _lib as L, meshgen
    from axisem3d_b200.solver import Solver, EngineError
    m = meshgen.cartesian_model(nx=3, nz=3, nr=5)
    bad = meshgen.cartesian_model(nx=3, nz=3, nr=5)
    bad.se_pts = bad.se_pts.copy()
    bad.se_pts[0, 0] = 10 ** 7
    with pytest.raises(EngineError) as ei:
        Solver(bad, "fp32")
    assert ei.value.code == L.AXG_E_ARG and "||" in str(ei.value)
    lib = L.lib()
    h = C.c_void_p()
    cfg = m.config("fp32")
    assert lib.axg_create(C.byref(cfg), C.byref(h)) == 0
    assert lib.axg_run(h, 1, 1) == L.AXG_E_STATE
    assert b"finalize" in lib.axg_last_error(h)
    lib.axg_destroy(h)
    dup = meshgen.cartesian_model(nx=3, nz=3, nr=5)
    dup.sponge_solid = (np.array([1, 1], np.int32), np.array([0.1, 0.2]))
    with pytest.raises(EngineError) as ei:
        Solver(dup, "fp32")
    assert ei.value.code == L.AXG_E_ARG and "twice" in str(ei.value)
    s = Solver(m, "fp32", stability_interval=1)
    u = np.zeros(s.field_size())
    u[0] = np.nan
    s.set_field(u.astype(complex), "displ")
    with pytest.raises(EngineError) as ei:
        s.run(2)
    assert ei.value.code == L.AXG_E_UNSTABLE
    s.close()


def test_launch_count_and_native_library(built):
    """The run launches the engine's own kernels, from the in-tree library."""
    from axisem3d_b200 import meshgen, _lib
    from axisem3d_b200.solver import Solver
    m = meshgen.cartesian_model(nx=4, nz=4, nr=5)
    with Solver(m, "fp32") as s:
        n0 = s.launch_count()
        s.run(3, graph=True)
        assert s.launch_count() - n0 >= 3 * 4
    import os
    maps = open("/proc/self/maps").read()
    assert os.path.realpath(_lib.LIB_PATH) in maps


SPH = {
    "sph_iso_3d_cg4_fluid": dict(n_theta=24, n_solid_layers=6, n_fluid_layers=2, nr_max=40),
    "sph_aniso_rtz_3d_fluid": dict(n_theta=16, n_solid_layers=4, n_fluid_layers=2, nr_max=24,
                                   rheology="aniso", attenuation=None),
    "sph_iso_1d_full_fluid": dict(n_theta=16, n_solid_layers=4, n_fluid_layers=2, nr_max=24,
                                  three_d=False, attenuation="full"),
}


@pytest.mark.parametrize("precision", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("case", sorted(SPH))
def test_spherical_shell_parity(built, case, precision):
    """Spherical mapping, both axes, fluid layer with solid-fluid coupling, RTZ
    rheology: solid and fluid stiffness of one evaluation, then five full steps."""
    import oracle as O
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.spherical_model(**SPH[case])
    us = meshgen.random_displacement(m, seed=3)
    uf = meshgen.random_displacement(m, seed=4, solid=False)
    o = O.Oracle(m, "fp64")
    o.set_field(us, "displ")
    o.set_field(uf, "displ", solid=False)
    o.compute_stiffness()
    ref_s, ref_f = o.get_field("stiff"), o.get_field("stiff", solid=False)
    tol = TOL_STIFF[precision]
    with Solver(m, precision) as s:
        s.set_field(us, "displ")
        s.set_field(uf, "displ", solid=False)
        s.compute_stiffness()
        assert rel(s.get_field("stiff"), ref_s) <= tol
        assert rel(s.get_field("stiff", solid=False), ref_f) <= tol
    o2 = O.Oracle(m, "fp64")
    o2.set_field(us * 1e-9, "displ")
    o2.set_field(uf * 1e-9, "displ", solid=False)
    o2.run(5)
    with Solver(m, precision) as s:
        s.set_field(us * 1e-9, "displ")
        s.set_field(uf * 1e-9, "displ", solid=False)
        s.run(5)
        tol5 = 1e-11 if precision == "fp64" else 1e-5
        assert rel(s.get_field("displ"), o2.get_field("displ")) <= tol5
        assert rel(s.get_field("displ", solid=False), o2.get_field("displ", solid=False)) <= tol5


def test_plain_and_autotuned_match(built):
    """The plain method (one bucket, eager launches) and the autotuned batched path
    compute the same steps."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.microbench_model(n_elem=300, nr_max=64, seed=41)
    u = meshgen.random_displacement(m, seed=2) * 1e-6
    out = []
    for kw in (dict(plain=True), dict(autotune=True), dict()):
        with Solver(m, "fp64", **kw) as s:
            s.set_field(u, "displ")
            s.run(3)
            out.append(s.get_field("displ"))
    assert rel(out[0], out[2]) <= 1e-13 and rel(out[1], out[2]) <= 1e-13


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_sources_equal_separate_runs(built, precision):
    """Several sources advanced as batched wavefields in the same launches give
    each source's own run (spherical shell with fluid, 21-Cij, RTZ)."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    base = meshgen.spherical_model(n_theta=16, n_solid_layers=4, n_fluid_layers=2, nr_max=24,
                                   rheology="aniso", attenuation=None)
    ens = meshgen.ensemble_model(base, nsrc=3, seed=5)
    with Solver(ens, precision) as s:
        s.run(40)
        d = s.get_field("displ").reshape(3, -1)
        seis = s.seismograms()
    tol = 1e-12 if precision == "fp64" else 1e-5
    for i in range(3):
        with Solver(meshgen.single_source(ens, i), precision) as s1:
            s1.run(40)
            assert rel(d[i], s1.get_field("displ")) <= tol
            assert rel(seis[:, i], s1.seismograms()) <= tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 1e-4), ("mixed", 1e-4)])
def test_absorbing_boundaries_parity(built, precision, tol):
    """Clayton conditions on the outer and bottom edges (a corner point carries one per
    boundary) and a Kosloff sponge: 800 steps of the plain forward, long enough for the
    waves to reach the boundaries, vs the oracle (displacement and seismograms)."""
    import oracle as O
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.cartesian_model(nx=8, nz=8, nr=5, nstations=6, absorbing=True,
                                attenuation=dict(meshgen.default_sls(3), qkappa=57823.0, qmu=200.0))
    assert len(np.unique(m.cl_solid["point"])) < len(m.cl_solid["point"])   # corner listed twice
    o = O.Oracle(m, "fp64", threads=4)
    o.run(800)
    with Solver(m, precision) as s:
        s.run(800)
        assert rel(s.get_field("displ"), o.get_field("displ")) <= 5 * tol
        assert rel(s.seismograms(), o.seismograms()) <= tol


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fluid_clayton_and_sponges_parity(built, precision):
    """ClaytonFluid1D on fluid points, sponges on both solid and fluid points of the
    spherical shell, five full steps vs the oracle."""
    import oracle as O
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.spherical_model(**SPH["sph_iso_1d_full_fluid"])
    rng = np.random.default_rng(7)
    nf = len(m.fp_nr)
    fpt = np.sort(rng.choice(nf, size=max(4, nf // 5), replace=False)).astype(np.int32)
    rvp = np.full(len(fpt), 1.0e7)
    m.cl_fluid = {"point": np.concatenate([fpt, fpt[:3]]),
                  "rho_vp": np.concatenate([rvp, rvp[:3]]),
                  "area": 0.05 * np.concatenate([m.fp_mass[fpt], m.fp_mass[fpt[:3]]]) * 1.0e7 / m.dt}
    spt = np.sort(rng.choice(len(m.sp_nr), size=len(m.sp_nr) // 4, replace=False)).astype(np.int32)
    m.sponge_solid = (spt, rng.uniform(0.0, 0.3 / m.dt, len(spt)))
    m.sponge_fluid = (fpt, rng.uniform(0.0, 0.3 / m.dt, len(fpt)))
    us = meshgen.random_displacement(m, seed=3) * 1e-9
    uf = meshgen.random_displacement(m, seed=4, solid=False) * 1e-9
    o = O.Oracle(m, "fp64")
    o.set_field(us, "displ")
    o.set_field(uf, "displ", solid=False)
    o.set_field(us, "veloc")
    o.set_field(uf, "veloc", solid=False)
    o.run(5)
    tol = 1e-11 if precision == "fp64" else 1e-5
    with Solver(m, precision) as s:
        s.set_field(us, "displ")
        s.set_field(uf, "displ", solid=False)
        s.set_field(us, "veloc")
        s.set_field(uf, "veloc", solid=False)
        s.run(5)
        for solid in (True, False):
            assert rel(s.get_field("displ", solid=solid), o.get_field("displ", solid=solid)) <= tol
            assert rel(s.get_field("veloc", solid=solid), o.get_field("veloc", solid=solid)) <= tol


def _mass3d_ocean_model():
    from axisem3d_b200 import meshgen
    m = meshgen.cartesian_model(nx=6, nz=6, nr=6,
                                attenuation=dict(meshgen.default_sls(3), qkappa=57823.0, qmu=100.0))
    meshgen.add_ocean_load(m, 6, 6, 100e3, tilt=0.3, seed=1)
    return meshgen.with_mass3d(m, amp=0.05, seed=2, exclude=m.ocean_load[0])


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("fp32", 1e-5), ("mixed", 1e-5)])
def test_mass3d_and_ocean_load_parity(built, precision, tol):
    """Mass3D points (per-slice masses: slices -> x 1/M_k -> Fourier, Mass3D.cpp:41-68) and
    MassOceanLoad1D surface points with tilted normals: five full steps vs the oracle."""
    import oracle as O
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = _mass3d_ocean_model()
    u0 = meshgen.random_displacement(m, seed=8) * 1e-3
    o = O.Oracle(m, "fp64")
    o.set_field(u0, "displ")
    o.run(5)
    with Solver(m, precision) as s:
        s.set_field(u0, "displ")
        s.run(5)
        for f in ("displ", "veloc", "accel"):
            assert rel(s.get_field(f), o.get_field(f)) <= tol, (f, rel(s.get_field(f), o.get_field(f)))


def test_mass3d_and_ocean_load_hooks_equal_graph(built):
    """The per-hook path (boundary conditions after assembly, then 1/M, as separate calls)
    gives the graph's steps on Mass3D and ocean-loaded points (FP64)."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = _mass3d_ocean_model()
    u0 = meshgen.random_displacement(m, seed=9) * 1e-3
    out = []
    for mode in ("graph", "hooks"):
        with Solver(m, "fp64") as s:
            s.set_field(u0, "displ")
            if mode == "hooks":
                for t in range(4):
                    s.apply_sources(t)
                    s.compute_stiffness()
                    s.apply_bc_before_assembly()
                    s.record_stations(t)
                    s.apply_bc_after_assembly()
                    s.stiff_to_accel()
                    s.newmark_update()
            else:
                s.run(4)
            out.append((s.get_field("displ"), s.get_field("veloc")))
    assert rel(out[1][0], out[0][0]) <= 1e-13 and rel(out[1][1], out[0][1]) <= 1e-13


def test_ocean_load_errors(built):
    """A 1-D ocean load on a Mass3D point, or twice on one point: host-side errors."""
    from axisem3d_b200 import _lib as L, meshgen
    from axisem3d_b200.solver import Solver, EngineError
    m = meshgen.cartesian_model(nx=3, nz=3, nr=4)
    meshgen.add_ocean_load(m, 3, 3, 100e3)
    bad3d = meshgen.with_mass3d(m, seed=1)          # ocean points get 3-D masses too
    with pytest.raises(EngineError) as ei:
        Solver(bad3d, "fp32")
    assert ei.value.code == L.AXG_E_ARG and "3-D ocean load" in str(ei.value)
    pt, mo, th = m.ocean_load
    m.ocean_load = (np.concatenate([pt, pt[:1]]), np.concatenate([mo, mo[:1]]), np.concatenate([th, th[:1]]))
    with pytest.raises(EngineError) as ei:
        Solver(m, "fp32")
    assert ei.value.code == L.AXG_E_ARG and "twice" in str(ei.value)


def _abc3d_model():
    from axisem3d_b200 import meshgen
    m = meshgen.spherical_model(n_theta=16, n_solid_layers=4, n_fluid_layers=2, nr_max=24, three_d=True)
    meshgen.add_absorbing3d(m, seed=3)
    # ClaytonFluid3D on a seeded subset of fluid points (synthetic values: parity only)
    rng = np.random.default_rng(11)
    fpt = np.sort(rng.choice(len(m.fp_nr), size=len(m.fp_nr) // 5, replace=False)).astype(np.int32)
    nr = np.asarray(m.fp_nr)[fpt]
    off = np.concatenate([[0], np.cumsum(nr)[:-1]]).astype(np.int64)
    tot = int(nr.sum())
    mass = np.asarray(m.fp_mass)[np.repeat(fpt, nr)]
    m.cl3_fluid = {"point": fpt, "offset": off, "rho_vp": np.full(tot, 1.0e7),
                   "area": 0.05 * mass * 1.0e7 / m.dt * rng.uniform(0.5, 1.5, tot)}
    return m


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("fp32", 1e-5), ("mixed", 1e-5)])
def test_absorbing3d_parity(built, precision, tol):
    """ClaytonSolid3D (per-slice impedances, tilted normals) on the outer surface of a 3-D
    shell, ClaytonFluid3D on fluid points and 3-D sponges (nr gammas per point): five full
    steps vs the oracle."""
    import oracle as O
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = _abc3d_model()
    us = meshgen.random_displacement(m, seed=3) * 1e-9
    uf = meshgen.random_displacement(m, seed=4, solid=False) * 1e-9
    o = O.Oracle(m, "fp64")
    for which in ("displ", "veloc"):
        o.set_field(us, which)
        o.set_field(uf, which, solid=False)
    o.run(5)
    with Solver(m, precision) as s:
        for which in ("displ", "veloc"):
            s.set_field(us, which)
            s.set_field(uf, which, solid=False)
        s.run(5)
        for solid in (True, False):
            for f in ("displ", "veloc"):
                got, ref = s.get_field(f, solid=solid), o.get_field(f, solid=solid)
                assert rel(got, ref) <= tol, (solid, f, rel(got, ref))


def test_absorbing3d_hooks_equal_graph_and_errors(built):
    """The per-hook path equals the graph with 3-D boundaries (FP64); a point with a 1-D and
    a 3-D sponge, and per-slice arrays too short for a point's nr, are host-side errors."""
    from axisem3d_b200 import _lib as L, meshgen
    from axisem3d_b200.solver import Solver, EngineError
    m = _abc3d_model()
    us = meshgen.random_displacement(m, seed=5) * 1e-9
    out = []
    for mode in ("graph", "hooks"):
        with Solver(m, "fp64") as s:
            s.set_field(us, "displ")
            s.set_field(us, "veloc")
            if mode == "hooks":
                for t in range(4):
                    s.apply_sources(t)
                    s.compute_stiffness()
                    s.apply_bc_before_assembly()
                    s.record_stations(t)
                    s.apply_bc_after_assembly()
                    s.stiff_to_accel()
                    s.newmark_update()
            else:
                s.run(4)
            out.append((s.get_field("displ"), s.get_field("veloc")))
    assert rel(out[1][0], out[0][0]) <= 1e-13 and rel(out[1][1], out[0][1]) <= 1e-13
    both = _abc3d_model()
    p0 = both.sponge3d_solid[0][:1]
    both.sponge_solid = (p0, np.array([0.01]))
    with pytest.raises(EngineError) as ei:
        Solver(both, "fp32")
    assert ei.value.code == L.AXG_E_ARG and "twice" in str(ei.value)
    short = _abc3d_model()
    c = dict(short.cl3_solid)
    c["offset"] = c["offset"] + 1
    short.cl3_solid = c
    with pytest.raises(EngineError) as ei:
        Solver(short, "fp32")
    assert ei.value.code == L.AXG_E_ARG and "Incompatible sizes" in str(ei.value)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_wavefield_scanning_matches_oracle(built, precision):
    """Wavefield scanning (Scanning1D peaks of the displacement's Fourier series, every 4 steps)
    on a shell excited by an off-axis source: the per-point nr it reports vs the oracle's.
    In FP64 the two agree at every point; in mixed precision a peak whose H2 or truncation
    test sits within rounding of a threshold may differ, so 99 % of the points must agree and
    none by more than one mode pair."""
    import oracle as O
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    base = meshgen.spherical_model(n_theta=24, n_solid_layers=6, n_fluid_layers=2, nr_max=40, three_d=False,
                                   attenuation=None)
    m = meshgen.single_source(meshgen.ensemble_model(base, nsrc=1, seed=3, periods=(20.0, 20.0)), 0)
    m.scanning = dict(tol_fourier_h1=1e-2, rel_tol_h1=0.1, abs_tol_h1=1e-12, max_num_peaks=10, interval=4)
    o = O.Oracle(m, "fp64", threads=4)
    o.run(400)
    ref_s, ref_f = o.scanning_nr()
    with Solver(m, precision) as s:
        s.run(400)
        got_s, got_f = s.scanning_nr()
    assert (ref_s > 1).sum() > len(ref_s) // 4          # the waves reached most points
    for got, ref in ((got_s, ref_s), (got_f, ref_f)):
        if precision == "fp64":
            assert np.array_equal(got, ref), np.nonzero(got != ref)
        else:
            assert np.mean(got == ref) >= 0.99 and np.max(np.abs(got - ref)) <= 2


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_wavefield_scanning_prescribed_history(built, precision):
    """The prescribed history of the oracle pin (modes 0..3 filled, amplitudes 1, 2, 3, 2, 1
    at five scans) through axg_set_field and axg_record_stations: nr = 9 at every point."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.cartesian_model(nx=3, nz=3, nr=16)
    m.ms_elem = np.zeros(0, np.int32)
    m.ms_nu = np.zeros(0, np.int32)
    m.ms_pat_off = np.zeros(0, np.int64)
    m.ms_pattern = np.zeros(0, np.complex128)
    m.ms_stf = []
    m.scanning = dict(tol_fourier_h1=1e-2, rel_tol_h1=0.1, abs_tol_h1=1e-12, max_num_peaks=10, interval=1)
    nu = 16 // 2 + 1
    pattern = np.zeros((len(m.sp_nr), nu, 3), np.complex128)
    pattern[:, :4, :] = 1.0 + 0.5j
    with Solver(m, precision) as s:
        for t, amp in enumerate((1.0, 2.0, 3.0, 2.0, 1.0)):
            s.set_field((amp * pattern).ravel(), "displ")
            s.record_stations(t)
        s_nr, _ = s.scanning_nr()
    assert np.all(s_nr == 9), np.unique(s_nr)


def _ocean3d_model():
    from axisem3d_b200 import meshgen
    m = meshgen.cartesian_model(nx=6, nz=6, nr=6,
                                attenuation=dict(meshgen.default_sls(3), qkappa=57823.0, qmu=100.0))
    meshgen.add_ocean_load3d(m, 6, 6, 100e3, seed=2)
    return meshgen.with_mass3d(m, amp=0.05, seed=2)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("fp32", 1e-5), ("mixed", 1e-5)])
def test_ocean_load3d_parity(built, precision, tol):
    """MassOceanLoad3D (per-slice ocean masses and tilted normals) on surface points whose own
    masses are 3-D: five full steps vs the oracle; the per-hook path equals the graph."""
    import oracle as O
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = _ocean3d_model()
    u0 = meshgen.random_displacement(m, seed=8) * 1e-3
    o = O.Oracle(m, "fp64")
    o.set_field(u0, "displ")
    o.run(5)
    with Solver(m, precision) as s:
        s.set_field(u0, "displ")
        s.run(5)
        for f in ("displ", "veloc", "accel"):
            assert rel(s.get_field(f), o.get_field(f)) <= tol, (f, rel(s.get_field(f), o.get_field(f)))
    if precision == "fp64":
        with Solver(m, "fp64") as s:
            s.set_field(u0, "displ")
            for t in range(5):
                s.apply_sources(t)
                s.compute_stiffness()
                s.apply_bc_before_assembly()
                s.record_stations(t)
                s.apply_bc_after_assembly()
                s.stiff_to_accel()
                s.newmark_update()
            assert rel(s.get_field("displ"), o.get_field("displ")) <= tol


PRT_GPU = {
    "cart_iso_1d_full": (lambda m: m.cartesian_model(nx=5, nz=4, nr=8, attenuation=dict(
        m.default_sls(3), qkappa=57823.0, qmu=120.0)), False),
    "tiso_3d_full_prt3d": (lambda m: m.microbench_model(n_elem=60, nr_max=32, seed=22, axial_column=True), True),
    "tiso_3d_full_prt1d": (lambda m: m.microbench_model(n_elem=60, nr_max=32, seed=23), False),
    "sph_aniso_rtz": (lambda m: m.spherical_model(n_theta=16, n_solid_layers=4, n_fluid_layers=2, nr_max=24,
                                                  rheology="aniso", attenuation=None), False),
    "sph_iso_rtz_cg4": (lambda m: m.spherical_model(n_theta=16, n_solid_layers=4, n_fluid_layers=2,
                                                    nr_max=24), False),
}


@pytest.mark.parametrize("precision", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("case", sorted(PRT_GPU))
def test_prt_stiffness_parity(built, case, precision):
    """Solid elements with particle relabelling (1-D and 3-D factors, on the axis, RTZ frame,
    FULL / CG4 attenuation): two stiffness evaluations vs the oracle, the tolerances of the
    other stiffness tests."""
    import oracle as O
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    build, three_d = PRT_GPU[case]
    m = build(meshgen)
    meshgen.add_prt(m, amp=0.05, three_d=three_d, seed=4)
    u = meshgen.random_displacement(m, seed=5)
    uf = meshgen.random_displacement(m, seed=6, solid=False) if len(m.fp_nr) else None
    ref = []
    o = O.Oracle(m, "fp64")
    o.set_field(u, "displ")
    if uf is not None:
        o.set_field(uf, "displ", solid=False)
    for _ in range(2):
        o.set_field(np.zeros_like(u), "stiff")
        o.compute_stiffness()
        ref.append(o.get_field("stiff"))
    with Solver(m, precision) as s:
        s.set_field(u, "displ")
        if uf is not None:
            s.set_field(uf, "displ", solid=False)
        for k in range(2):
            s.set_field(np.zeros_like(u), "stiff")
            s.compute_stiffness()
            got = s.get_field("stiff")
            assert rel(got, ref[k]) <= TOL_STIFF[precision], (k, rel(got, ref[k]))


def test_prt_full_steps_and_errors(built):
    """Five full steps of a PRT model (mixed precision) vs the oracle; a 3-D PRT on a 1-D
    element and a PRT on an element listed twice are host-side errors."""
    import oracle as O
    from axisem3d_b200 import _lib as L, meshgen
    from axisem3d_b200.solver import Solver, EngineError
    m = meshgen.cartesian_model(nx=6, nz=6, nr=5,
                                attenuation=dict(meshgen.default_sls(3), qkappa=57823.0, qmu=100.0))
    meshgen.add_prt(m, elements=np.arange(0, 36, 2), amp=0.05, seed=7)
    u0 = meshgen.random_displacement(m, seed=8) * 1e-3
    o = O.Oracle(m, "fp64")
    o.set_field(u0, "displ")
    o.run(5)
    with Solver(m, "mixed") as s:
        s.set_field(u0, "displ")
        s.run(5)
        assert rel(s.get_field("displ"), o.get_field("displ")) <= 1e-5
    bad = meshgen.cartesian_model(nx=3, nz=3, nr=5)
    meshgen.add_prt(bad, three_d=True)
    with pytest.raises(EngineError) as ei:
        Solver(bad, "fp32")
    assert ei.value.code == L.AXG_E_ARG and "3-D PRT on a 1-D element" in str(ei.value)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("three_d", [False, True])
def test_fluid_prt_parity(built, precision, three_d):
    """Fluid elements with PRT factors in the RTZ frame of a spherical shell (1-D elements
    with 1-D factors; 3-D elements with per-slice K and 3-D factors): fluid stiffness vs the
    oracle."""
    import copy
    import oracle as O
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.spherical_model(n_theta=16, n_solid_layers=4, n_fluid_layers=2, nr_max=24)
    if three_d:
        nr = np.asarray(m.fe_nr)
        K = np.asarray(m.fe_moduli).reshape(-1, 25)
        m = copy.copy(m)
        m.fe_is3d = np.ones(len(nr), np.uint8)
        m.fe_moduli = np.concatenate([
            (np.tile(K[e], (nr[e], 1)) * (1 + 0.02 * np.sin(np.arange(nr[e])))[:, None]).ravel()
            for e in range(len(nr))])
        m.fe_mat_off = np.concatenate([[0], np.cumsum(nr * 25)[:-1]]).astype(np.int64)
    meshgen.add_prt_fluid(m, amp=0.05, three_d=three_d, seed=2)
    uf = meshgen.random_displacement(m, seed=6, solid=False)
    o = O.Oracle(m, "fp64")
    o.set_field(uf, "displ", solid=False)
    o.compute_stiffness()
    ref = o.get_field("stiff", solid=False)
    with Solver(m, precision) as s:
        s.set_field(uf, "displ", solid=False)
        s.compute_stiffness()
        assert rel(s.get_field("stiff", solid=False), ref) <= TOL_STIFF[precision]


@pytest.mark.parametrize("mode", ["hooks", "chunks"])
def test_table_stf_without_padding_to_the_last_step(built, mode):
    """A StreamSTF table with padding NONE whose last sample is the time of the last step the
    run takes: the run needs no time beyond the table, so it completes, per hook or in chunks
    of 7 steps (StreamSTF::getValue throws only for a time the run asks for), and matches the
    oracle; one step more asks for a time past the table and raises."""
    import math
    import oracle as O
    from axisem3d_b200 import meshgen
    from axisem3d_b200.model import STF
    from axisem3d_b200.solver import EngineError, Solver
    m = meshgen.cartesian_model(nx=5, nz=5, nr=5)
    n = 40
    t = m.t0 + np.arange(n) * m.dt
    v = (1. - 2. * (math.pi * 2.0 * (t - t[n // 3])) ** 2) * np.exp(-(math.pi * 2.0 * (t - t[n // 3])) ** 2)
    m.ms_stf = [STF(table=(t, v), padding=0)]
    o = O.Oracle(m, "fp64")
    o.run(n)
    ref = o.get_field("displ")
    with Solver(m, "fp64") as s:
        if mode == "hooks":
            for k in range(n):
                s.apply_sources(k)
                s.compute_stiffness()
                s.apply_bc_before_assembly()
                s.record_stations(k)
                s.apply_bc_after_assembly()
                s.stiff_to_accel()
                s.newmark_update()
        else:
            for _ in range(n // 7):
                s.run(7)
            s.run(n % 7)
            assert s.step == n
        assert np.abs(ref).max() > 0 and rel(s.get_field("displ"), ref) <= 1e-11
        with pytest.raises(EngineError):
            if mode == "hooks":
                s.apply_sources(n)
            else:
                s.run(1)


# lucky numbers above the FFT threshold (nr > 64): every radix of the slice FFTs (4, 2, 3, 5,
# 7, 11, 13) and plans of two to four passes
FFT_NR = [66, 70, 75, 77, 78, 81, 88, 91, 98, 99, 104, 105, 110, 117, 120, 125, 126, 128]


@pytest.mark.parametrize("precision", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("kind", ["tiso_3d_full", "iso_3d_cg4", "aniso_3d_axial"])
def test_slice_fft_parity(built, precision, kind):
    """3-D elements of large nr take the slice FFTs (mixed-radix Stockham passes in shared
    memory, component pairs as complex signals) instead of the direct sums: two evaluations
    against the FP64 oracle's direct DFT."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    kw = {"tiso_3d_full": dict(nr_choices=FFT_NR),
          "iso_3d_cg4": dict(nr_choices=[117], rheology="iso", attenuation="cg4"),
          "aniso_3d_axial": dict(nr_choices=FFT_NR, rheology="aniso", attenuation=None, axial_column=True)}[kind]
    m = meshgen.microbench_model(n_elem=60, seed=32, **kw)
    assert m.se_nr.min() > 64
    u = meshgen.random_displacement(m, seed=7)
    ref1 = _oracle_stiff(m, u, 1)
    ref2 = _oracle_stiff(m, u, 2)
    with Solver(m, precision) as s:
        s.set_field(u, "displ")
        s.compute_stiffness()
        f1 = s.get_field("stiff")
        s.set_field(np.zeros_like(u), "stiff")
        s.compute_stiffness()
        f2 = s.get_field("stiff")
    assert rel(f1, ref1) <= TOL_STIFF[precision], rel(f1, ref1)
    assert rel(f2, ref2) <= TOL_STIFF[precision], rel(f2, ref2)


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_deterministic_assembly_is_bitwise_reproducible(built, precision):
    """axg_config.deterministic: coloured element launches make the assembled stiffness and
    the fields bitwise identical from run to run (the reference's serial scatter is
    deterministic, SolidPoint.hpp:101-109), and equal to the atomic path within the FP32
    tolerance. 3-D TI with FULL SLS, a fluid-free microbenchmark with many shared points, and
    the spherical shell with its fluid layer."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    for m, nsteps in ((meshgen.microbench_model(n_elem=800, nr_max=40, seed=44), 4),
                      (meshgen.spherical_model(n_theta=24, n_solid_layers=6, n_fluid_layers=2, nr_max=24), 20)):
        u = meshgen.random_displacement(m, seed=3) * 1e-6
        runs = []
        for det in (True, True, False):
            with Solver(m, precision, deterministic=det) as s:
                s.set_field(u, "displ")
                s.run(nsteps)
                runs.append((s.get_field("displ"), s.get_field("stiff")))
        (d1, k1), (d2, k2), (d3, k3) = runs
        assert np.array_equal(d1, d2) and np.array_equal(k1, k2)
        assert rel(d1, d3) <= 1e-5 and rel(k1, k3) <= 1e-5


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 1e-5), ("mixed", 1e-5)])
@pytest.mark.parametrize("mode", [0, 1])
def test_engine_patch_test(built, mode, precision, tol):
    """The patch test on the CUDA path itself, not only through the oracle: a Cartesian-linear
    (uniform-strain) field in a homogeneous medium leaves no force off the box's outer boundary,
    axis points included after their axial projection. Mode 0: u_s = a s, u_z = b z; mode 1:
    the shear u_x = a z, u_z = b x (coefficients a z / 2, i a z / 2, b s / 2)."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    from test_oracle_pins import _axial_projection
    m = meshgen.cartesian_model(nx=6, nz=5, nr=5)
    nu = np.asarray(m.sp_nr) // 2 + 1
    first = np.concatenate([[0], np.cumsum(nu)[:-1]])
    rows = first + mode
    s, z = m.sp_coords[:, 0], m.sp_coords[:, 1]
    u = np.zeros((int(nu.sum()), 3), complex)
    if mode == 0:
        u[rows, 0], u[rows, 2] = 1e-3 * s, -2e-3 * z
    else:
        u[rows, 0], u[rows, 1], u[rows, 2] = 0.5e-3 * z, 0.5e-3j * z, 0.7e-3 * s
    with Solver(m, precision) as h:
        h.set_field(u.ravel(), "displ")
        h.compute_stiffness()
        f = h.get_field("stiff").reshape(-1, 3)[rows]
    width, height = s.max(), -z.min()
    eps = 1e-9 * max(width, height)
    axis = s < eps
    boundary = (np.abs(s - width) < eps) | (np.abs(z) < eps) | (np.abs(z + height) < eps)
    f[axis] = _axial_projection(f[axis], mode)
    fb = np.linalg.norm(f[boundary])
    assert fb > 0 and np.any(~boundary & axis)
    assert np.linalg.norm(f[~boundary]) <= tol * fb, np.linalg.norm(f[~boundary]) / fb
