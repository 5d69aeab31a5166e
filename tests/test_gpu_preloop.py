"""GPU tests of the whole simulation path from the reference's input formats: Exodus mesh +
inparam files -> preloop -> engine time loop -> station files, against the oracle run on the
same preloop model.

Cases (meshes written at test time by tests/exodus_fixture.py):
  box    Cartesian 10 x 8 quads, axis, FULL attenuation, moment tensor on the axis, five
         surface receivers (DISTANCE_AZIMUTH, spz frame, ASCII_STATION)
  shell  spherical half annulus 24 x 7 quads with a fluid layer, solid-fluid coupling, both
         axis ends, CG4 attenuation, Clayton + sponge at the bottom, eight receivers given by
         latitude / longitude (RTZ frame, ASCII_CHANNEL)
Tolerance (relative L2 over each group's traces): FP64 1e-10, FP32 / mixed 1e-4.
"""
import math
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import exodus_fixture as fx  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-4, "mixed": 1e-4}


def _box(d):
    from axisem3d_b200 import meshgen
    sls = dict(meshgen.default_sls(3, fmin=0.1, fmax=2.0), qkappa=57823.0, qmu=120.0)
    desc = fx.cartesian_box(10, 8, 100e3, 80e3, 2700.0, 5800.0, 3460.0, attenuation=sls, minimum_period=1.0)
    st = [("S%d" % k, "XX", 100e3 * k / 5, 0.0, 0.0) for k in range(1, 6)]
    return fx.write_inputs(d, desc, nr=5, depth=10e3, mt=(1e18, -3e17, 2e17, 4e17, -1e17, 5e17), hdur=1.0,
                           decay=math.pi, order="RICKER", courant=0.6, record_length=8.0, stations=st,
                           attenuation="FULL", fmt="ASCII_STATION")


def _shell(d):
    from axisem3d_b200 import meshgen
    r_edges = [3480e3, 3540e3, 3600e3, 4200e3, 4800e3, 5400e3, 6000e3, 6371e3]
    layers = [dict(RHO=9900., VP=8000., VS=0., QMU=0., QKAPPA=57823.)] * 2 + \
        [dict(RHO=5500. - 300 * k, VP=13000. - 600 * k, VS=7000. - 300 * k, QMU=300., QKAPPA=57823.)
         for k in range(5)]
    sls = meshgen.default_sls(3, fmin=1 / 80., fmax=1 / 5.)
    desc = fx.spherical_shell(24, r_edges, 2, layers, attenuation=sls, minimum_period=20.0,
                              discontinuities=[3480e3, 3600e3, 6371e3])
    st = [("S%02d" % k, "XX", 90. - 170. * k / 9, 0.0, 0.0) for k in range(1, 9)]
    return fx.write_inputs(d, desc, nr=8, depth=100e3, mt=(1e20, -2e19, 3e19, 5e19, -4e19, 1e19), hdur=10.0,
                           decay=1.628, order="RICKER", courant=0.6, record_length=200., stations=st,
                           horizontal="LATITUDE_LONGITUDE", frame="RTZ", attenuation="CG4",
                           boundaries=["BOTTOM"], clayton=True, sponge=True, spans=[0.05], lucky=True,
                           bound_nr=True, fmt="ASCII_CHANNEL")


def _oracle_traces(sim):
    import oracle as O
    from axisem3d_b200 import output
    o = O.Oracle(sim.model, "fp64")
    o.run(sim.nsteps)
    seis = o.seismograms()
    o.close()
    out = {}
    for g in sim.groups:
        steps, rows = output.group_records(g, sim.nsteps, sim.t0, sim.dt, sim.model.st_interval)
        u = np.transpose(seis[rows][:, g.first:g.first + len(g.keys), :], (1, 0, 2))
        out[g.name] = (sim.t0 + steps * sim.dt,
                       output.group_channels(u, None, g.channels, g.frame, g.theta, g.baz, g.phi, sim.cartesian))
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("case", ["box", "shell"])
def test_simulation_matches_oracle(built, tmp_path, case, precision):
    from axisem3d_b200 import simulation
    d = (_box if case == "box" else _shell)(str(tmp_path / "input"))
    res = simulation.run(d, str(tmp_path / "output"), precision=precision)
    ref = _oracle_traces(res.sim)
    assert set(ref) == set(res.traces)
    for name, (t_ref, w_ref) in ref.items():
        t, w = res.traces[name]
        assert np.array_equal(t, t_ref)
        assert np.abs(w_ref).max() > 0
        err = float(np.linalg.norm(w - w_ref) / np.linalg.norm(w_ref))
        assert err <= TOL[precision], (name, err)
    # the files hold the returned traces
    g = res.sim.groups[0]
    gd = tmp_path / "output" / "stations" / g.name
    times, data = res.traces[g.name]
    assert np.allclose(np.loadtxt(gd / "data_time.ascii"), times)
    if g.fmt == "ASCII_STATION":
        got = np.loadtxt(gd / (g.keys[0] + ".ascii"))
        assert np.allclose(got.reshape(len(times), -1), data[0].T, rtol=1e-6, atol=1e-6 * np.abs(data).max())
    else:
        got = np.loadtxt(gd / "dir_rank0" / (g.channels[0] + ".ascii"))
        assert np.allclose(got, data[:, 0].T, rtol=1e-6, atol=1e-6 * np.abs(data).max())


def test_simulation_max_steps(built, tmp_path):
    from axisem3d_b200 import simulation
    d = _box(str(tmp_path / "input"))
    res = simulation.run(d, None, precision="fp32", max_steps=17)
    assert res.sim.nsteps == 17
    t, w = next(iter(res.traces.values()))
    assert len(t) == 17 and w.shape[-1] == 17


def _element_displ_grad(m, field, e):
    """The displacement U [order, 3, 5, 5] of solid element e (orders < nr/2 + 1 of the
    element, collectDisplFromPoints) and its computeGrad9 (GradientQuadrature.hpp:177-202,
    L'Hopital rows :421-459) g [order, 9, 5, 5], g[c * 3 + d] = d_d u_c, from the point field."""
    from axisem3d_b200.solver import spectral_tables
    t = spectral_tables()
    gll, glj = t["gGLL"].reshape(5, 5), t["gGLJ"].reshape(5, 5)      # [k, i] = l_k'(x_i)
    nu_p = np.asarray(m.sp_nr) // 2 + 1
    off = np.concatenate([[0], np.cumsum(nu_p)[:-1]])
    f = field.reshape(-1, 3)
    nu = int(m.se_nr[e]) // 2 + 1
    pts = m.se_pts[e]
    U = np.zeros((nu, 3, 5, 5), np.complex128)
    for q in range(25):
        p = pts[q]
        n = min(nu, nu_p[p])
        U[:n, :, q // 5, q % 5] = f[off[p]:off[p] + n]
    gx = glj if m.se_axial[e] else gll
    X = np.einsum("ki,ackj->acij", gx, U)
    Y = np.einsum("kj,acik->acij", gll, U)
    sx, se, zx, ze, inv_s = (m.se_geom[e, k].reshape(5, 5) for k in range(5))
    al = np.arange(nu)[:, None, None]
    A = np.stack([1j * al * U[:, 0] - U[:, 1], 1j * al * U[:, 1] + U[:, 0], 1j * al * U[:, 2]], axis=1)
    g = np.zeros((nu, 9, 5, 5), np.complex128)
    for c in range(3):
        g[:, c * 3 + 0] = X[:, c] * ze + Y[:, c] * zx
        g[:, c * 3 + 2] = X[:, c] * se + Y[:, c] * sx
        g[:, c * 3 + 1] = A[:, c] * inv_s
    if m.se_axial[e]:
        ax = np.einsum("k,ackj->acj", gx[:, 0], A)
        ay = np.einsum("kj,ack->acj", gll, A[:, :, 0, :])
        for c in range(3):
            g[:, c * 3 + 1, 0, :] += ax[:, c] * ze[0] + ay[:, c] * zx[0]
    return U, g


def _grad9_at_stations(m, field):
    """computeGrad9 of the field at the points of each station's element, interpolated like
    the displacement (Station::interpolate): [station, 9]. Also returns the interpolated
    displacement."""
    out_g, out_u = [], []
    for s, e in enumerate(m.st_elem):
        U, g = _element_displ_grad(m, field, e)
        nu = U.shape[0]
        w = m.st_w[s].reshape(5, 5)
        z = np.where(np.arange(nu) == 0, 1.0, 2.0) * np.exp(1j * np.arange(nu) * m.st_phi[s])
        out_g.append(np.real(np.einsum("a,akij,ij->k", z, g, w)))
        out_u.append(np.real(np.einsum("a,akij,ij->k", z, U, w)))
    return np.array(out_g), np.array(out_u)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_station_gradient_matches_numpy_restatement(built, tmp_path, precision):
    """Gradient records against computeGrad9 restated in numpy on the oracle's displacement,
    for stations on the surface, inside the box and on the axis (the L'Hopital row)."""
    import oracle as O
    from axisem3d_b200 import preloop
    from axisem3d_b200.solver import Solver
    d = _box(str(tmp_path / "input"))
    with open(os.path.join(d, "STATIONS.txt"), "a") as f:
        f.write("AX XX 0.0 0.0 0.0 30000.0\n")         # on the axis, 30 km deep
        f.write("IN XX 37000.0 0.0 0.0 41000.0\n")     # inside an element
    p = os.path.join(d, "inparam.output.yaml")
    with open(p) as f:
        txt = f.read()
    with open(p, "w") as f:
        f.write(txt.replace("channels: [U]", "channels: [U, G, E_I1, R]"))
    sim = preloop.build(d, max_steps=40)
    m = sim.model
    assert m.st_gradient
    with Solver(m, precision) as s:
        s.run(sim.nsteps)
        grad = s.station_gradients()
        seis = s.seismograms()
    o = O.Oracle(m, "fp64")
    ref_g, ref_u = [], []
    for k in range(sim.nsteps):
        g, u = _grad9_at_stations(m, o.get_field("displ"))
        ref_g.append(g)
        ref_u.append(u)
        o.run(1)
    o_seis = o.seismograms()
    o.close()
    ref_g, ref_u = np.array(ref_g), np.array(ref_u)
    # the restatement reproduces the oracle's own station displacement (timing and weights)
    assert np.abs(ref_u - o_seis).max() <= 1e-12 * np.abs(o_seis).max()
    assert np.abs(ref_g).max() > 0
    tol = 1e-10 if precision == "fp64" else 1e-4
    for k in range(len(m.st_elem)):
        err = np.linalg.norm(grad[:, k] - ref_g[:, k]) / np.linalg.norm(ref_g)
        assert err <= tol, (k, err)
    assert np.linalg.norm(seis - o_seis) / np.linalg.norm(o_seis) <= tol


def _with_3d(d, case):
    """Add a 3-D model to a box or shell input directory (grids written here)."""
    if case == "box":
        x, y, dep = np.linspace(-120., 120., 7), np.linspace(-120., 120., 5), np.linspace(0., 90., 4)
        X, Y, D = np.meshgrid(x, y, dep, indexing="ij")
        fx.write_grid_v3d(os.path.join(d, "m3d.nc"), {"x": x, "y": y, "depth": dep},
                          {"dvs": 0.01 + 2e-4 * X - 3e-4 * Y + 4e-4 * D, "drho": -0.02 + 1e-4 * X + 2e-4 * D},
                          ["depth", "x", "y"])
        fx.add_3d_models(d, [fx.model3d_yaml("blob", "m3d.nc", "XY_CARTESIAN", "DEPTH", ["x", "y", "depth"],
                                             [1, 2, 0], [("VS", "dvs", 1.0, "REF1D"),
                                                         ("RHO", "drho", 0.5, "REF1D")])])
    else:
        lat, lon, dep = np.linspace(-90., 90., 7), np.linspace(-180., 180., 9), np.linspace(0., 2000., 5)
        LA, LO, DE = np.meshgrid(lat, lon, dep, indexing="ij")
        fx.write_grid_v3d(os.path.join(d, "ll.nc"), {"lat": lat, "lon": lon, "dep": dep},
                          {"dv": 0.02 + 1e-4 * LA - 5e-5 * LO + 1e-5 * DE}, ["lat", "lon", "dep"])
        fx.add_3d_models(d, [fx.model3d_yaml("sh", "ll.nc", "LATITUDE_LONGITUDE", "DEPTH", ["lat", "lon", "dep"],
                                             [0, 1, 2], [("VSH", "dv", 1.0, "REF1D"),
                                                         ("RHO", "dv", -0.5, "REF1D")])])
    return d


@pytest.mark.parametrize("precision", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("case", ["box", "shell"])
def test_simulation_with_3d_models_matches_oracle(built, tmp_path, case, precision):
    """3-D elements (per-slice moduli and attenuation), transversely isotropic evolution and
    Mass3D points from StructuredGridV3D models, through the whole path."""
    from axisem3d_b200 import simulation
    d = _with_3d((_box if case == "box" else _shell)(str(tmp_path / "input")), case)
    res = simulation.run(d, None, precision=precision)
    m = res.sim.model
    assert m.se_is3d.any() and m.sp_mass_nr is not None and (m.sp_mass_nr > 1).any()
    ref = _oracle_traces(res.sim)
    for name, (t_ref, w_ref) in ref.items():
        t, w = res.traces[name]
        assert np.array_equal(t, t_ref) and np.abs(w_ref).max() > 0
        err = float(np.linalg.norm(w - w_ref) / np.linalg.norm(w_ref))
        assert err <= TOL[precision], (name, err)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_3d_model_at_absorbing_boundaries_matches_oracle(built, tmp_path, precision):
    """A 3-D model reaching the box's Clayton (right, bottom) and sponge layers: 3-D Clayton
    conditions and 3-D sponge gammas from the preloop, against the oracle."""
    from axisem3d_b200 import meshgen, simulation
    sls = dict(meshgen.default_sls(3, fmin=0.1, fmax=2.0), qkappa=57823.0, qmu=120.0)
    desc = fx.cartesian_box(10, 8, 100e3, 80e3, 2700.0, 5800.0, 3460.0, attenuation=sls, minimum_period=1.0)
    st = [("S%d" % k, "XX", 100e3 * k / 5, 0.0, 0.0) for k in range(1, 6)]
    d = fx.write_inputs(str(tmp_path / "input"), desc, nr=5, depth=10e3, mt=(1e18, -3e17, 2e17, 4e17, -1e17, 5e17),
                        hdur=1.0, decay=math.pi, order="RICKER", courant=0.6, record_length=8.0, stations=st,
                        attenuation="FULL", boundaries=["RIGHT", "BOTTOM"], clayton=True, sponge=True,
                        spans=[0.1, 0.1])
    d = _with_3d(d, "box")
    res = simulation.run(d, None, precision=precision)
    m = res.sim.model
    assert m.cl3_solid is not None and m.sponge3d_solid is not None
    ref = _oracle_traces(res.sim)
    for name, (t_ref, w_ref) in ref.items():
        t, w = res.traces[name]
        err = float(np.linalg.norm(w - w_ref) / np.linalg.norm(w_ref))
        assert err <= TOL[precision], (name, err)


SCAN_NR_YAML = """type_Nr: CONSTANT
bound_Nr_by_inplane: false
constant: 8
wavefield_scanning:
    enable_scanning: true
    output_file: scan_nr.nc
    threshold_Fourier_convergence: 1e-2
    relative_amplitude_skipped: 0.1
    advanced:
        absolute_amplitude_skipped: 1e-12
        max_num_peaks: 10
        vertex_only: true
        num_steps_per_mesh_period: 12
"""


def test_scanning_file_and_pointwise_nr_round_trip(built, tmp_path):
    """Wavefield scanning from inparam.nr.yaml writes the reference's scanning file
    (pointwise_sz, pointwise_Nr, starting_Nr_for_scanning) with the oracle's scanned Nr; a
    second preloop reads it as a POINTWISE Nr field and puts those values on the vertices."""
    import oracle as O
    from scipy.io import netcdf_file
    from axisem3d_b200 import preloop, simulation
    d = _box(str(tmp_path / "input"))
    with open(os.path.join(d, "inparam.nr.yaml"), "w") as f:
        f.write(SCAN_NR_YAML)
    out = str(tmp_path / "output")
    res = simulation.run(d, out, precision="fp64")
    m = res.sim.model
    assert m.scanning is not None
    nc = netcdf_file(os.path.join(out, "scan_nr.nc"), "r", mmap=False)
    sz = np.array(nc.variables["pointwise_sz"][:])
    nr_scan = np.array(nc.variables["pointwise_Nr"][:])
    nr0 = np.array(nc.variables["starting_Nr_for_scanning"][:])
    nc.close()
    o = O.Oracle(m, "fp64")
    o.run(res.sim.nsteps)
    ref_s, _ = o.scanning_nr()
    o.close()
    pts = m.scanning["solid_points"]
    assert len(nr_scan) == len(pts) and np.all(nr0 == 8)
    assert np.array_equal(nr_scan, ref_s[pts]) and nr_scan.max() > 1
    with open(os.path.join(d, "inparam.nr.yaml"), "w") as f:
        f.write("type_Nr: POINTWISE\nbound_Nr_by_inplane: false\npointwise:\n    nc_data_file: %s\n"
                "    multip_factor: 1.\n" % os.path.join(out, "scan_nr.nc"))
    m2 = preloop.build(d).model
    look = {(round(c[0], 3), round(c[1], 3)): k for k, c in enumerate(m2.sp_coords)}
    got = np.array([m2.sp_nr[look[(round(a, 3), round(b, 3))]] for a, b in sz])
    assert np.array_equal(got, nr_scan)


def _with_geometry(d, case):
    """Add geometric (undulation) and ocean-load 3-D models to a box or shell input directory:
    box: a Moho-like undulation 300 cos(phi) m between 10 and 70 km depth and an ocean whose
    sum(rho * depth) varies with phi; shell: a latitude / longitude undulation between 100
    and 800 km depth and an ocean on half of the globe; shell_ellipticity: WGS84 flattening
    with the Ellipticity model."""
    if case == "box":
        s = np.linspace(0, 200e3, 11)
        ph = np.linspace(0, 2 * np.pi, 9)
        fx.write_grid_v3d(os.path.join(d, "und.nc"), {"s": s, "phi": ph},
                          {"dz": 300.0 * np.cos(ph)[None, :] * np.ones((11, 1))}, ["s", "phi"])
        fx.write_grid_v3d(os.path.join(d, "sea.nc"), {"s": s, "phi": ph},
                          {"srd": 4e6 * (1 + 0.5 * np.sin(ph))[None, :] * np.ones((11, 1))}, ["s", "phi"])
        fx.add_3d_models(d, [fx.geometric_yaml("moho", "und.nc", "DISTANCE_AZIMUTH", "DEPTH", ["s", "phi"], [0, 1],
                                               "dz", 40e3, 10e3, 70e3),
                             fx.ocean_yaml("sea", "sea.nc", "DISTANCE_AZIMUTH", ["s", "phi"], [0, 1], "srd")])
    elif case == "shell":
        lat, lon = np.linspace(-90, 90, 19), np.linspace(-180, 180, 37)
        fx.write_grid_v3d(os.path.join(d, "moho.nc"), {"lat": lat, "lon": lon},
                          {"dz": 2000.0 * np.cos(np.radians(lat))[:, None] * np.sin(np.radians(lon))[None, :]},
                          ["lat", "lon"])
        fx.write_grid_v3d(os.path.join(d, "sea.nc"), {"lat": lat, "lon": lon},
                          {"srd": np.maximum(0, 4e6 * np.sin(np.radians(lon)))[None, :] * np.ones((19, 1))},
                          ["lat", "lon"])
        fx.add_3d_models(d, [fx.geometric_yaml("moho", "moho.nc", "LATITUDE_LONGITUDE", "DEPTH", ["lat", "lon"],
                                               [0, 1], "dz", 400e3, 100e3, 800e3, angle_unit="degree"),
                             fx.ocean_yaml("sea", "sea.nc", "LATITUDE_LONGITUDE", ["lat", "lon"], [0, 1], "srd",
                                           angle_unit="degree")])
    elif case == "shell_cmb":
        # undulation that varies with phi on the solid-fluid boundary (3600 km radius):
        # SolidFluidCoupling3D
        lat, lon = np.linspace(-90, 90, 19), np.linspace(-180, 180, 37)
        fx.write_grid_v3d(os.path.join(d, "cmb.nc"), {"lat": lat, "lon": lon},
                          {"dz": 1500.0 * np.cos(np.radians(lat))[:, None] * np.cos(np.radians(lon))[None, :]},
                          ["lat", "lon"])
        fx.add_3d_models(d, [fx.geometric_yaml("cmb", "cmb.nc", "LATITUDE_LONGITUDE", "RADIUS", ["lat", "lon"],
                                               [0, 1], "dz", 3600e3, 3500e3, 3800e3, angle_unit="degree")])
    else:
        fx.add_3d_models(d, [fx.ellipticity_yaml("ellipticity")])
        p = os.path.join(d, "inparam.model.yaml")
        with open(p) as f:
            txt = f.read()
        with open(p, "w") as f:
            f.write(txt.replace("flattening_on_surface: SPHERE", "flattening_on_surface: WGS84"))
    return d


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["box", "shell", "shell_ellipticity", "shell_cmb"])
def test_simulation_with_geometric_and_ocean_models_matches_oracle(built, tmp_path, case, precision):
    """Undulated geometry through the whole path: particle relabelling (1-D and 3-D, solid
    and fluid elements), the PRT Jacobian on the masses, 3-D ocean loads, slice-wise dt."""
    from axisem3d_b200 import simulation
    d = _with_geometry((_box if case == "box" else _shell)(str(tmp_path / "input")), case)
    res = simulation.run(d, None, precision=precision)
    m = res.sim.model
    assert m.prt is not None and len(m.prt["element"]) > 0
    if case in ("box", "shell"):
        assert m.prt["is3d_prt"].any() and m.ocean_load3d is not None
    if case == "shell_cmb":
        assert m.sf3 is not None and len(m.sf3["solid"]) > 0
    ref = _oracle_traces(res.sim)
    for name, (t_ref, w_ref) in ref.items():
        t, w = res.traces[name]
        assert np.array_equal(t, t_ref) and np.abs(w_ref).max() > 0
        err = float(np.linalg.norm(w - w_ref) / np.linalg.norm(w_ref))
        assert err <= TOL[precision], (name, err)


def _pressure_source(d, depth=2831e3):
    """Turn the input's moment tensor into a FLUID_PRESSURE source inside the fluid layer."""
    p = os.path.join(d, "inparam.source.yaml")
    with open(p) as f:
        txt = f.read()
    i = txt.index("depth:")
    j = txt.index("\n", i)
    txt = txt[:i] + "depth: %r" % depth + txt[j:]
    i = txt.index("type: MOMENT_TENSOR")
    j = txt.index("unit:", i)
    txt = txt[:i] + "type: FLUID_PRESSURE\n            data: [1e12]\n            " + txt[j:]
    with open(p, "w") as f:
        f.write(txt)
    return d


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fluid_pressure_source_matches_oracle(built, tmp_path, precision):
    """FLUID_PRESSURE (Mechanism::release's pressure pattern, FluidPressure::apply) in the
    shell's fluid layer: the pressure goes to the fluid acceleration after the mass term."""
    from axisem3d_b200 import simulation
    d = _pressure_source(_shell(str(tmp_path / "input")))
    res = simulation.run(d, None, precision=precision)
    m = res.sim.model
    assert len(m.ps_elem) == 1 and len(m.ms_elem) == 0
    ref = _oracle_traces(res.sim)
    for name, (t_ref, w_ref) in ref.items():
        t, w = res.traces[name]
        assert np.array_equal(t, t_ref) and np.abs(w_ref).max() > 0
        err = float(np.linalg.norm(w - w_ref) / np.linalg.norm(w_ref))
        assert err <= TOL[precision], (name, err)


def _table_stf(d, cls="StreamSTF", padding="FIRST_LAST"):
    """Replace the Gaussian STF of the input's source by a table: a Ricker-like wavelet
    sampled every 0.37 s (not a multiple of dt), as an ascii file or a NetCDF file."""
    t = np.arange(-3.0, 9.0, 0.37)
    v = (1. - 2. * (math.pi * 0.8 * (t - 1.)) ** 2) * np.exp(-(math.pi * 0.8 * (t - 1.)) ** 2)
    if cls == "StreamSTF":
        with open(os.path.join(d, "stf.txt"), "w") as f:
            f.write("# time value\n")
            for a, b in zip(t, v):
                f.write("%.17g %.17g\n" % (a, b))
        spec = "class_name: StreamSTF\n            ascii_data_file: stf.txt\n"
    else:
        fx.write_grid_v3d(os.path.join(d, "stf.nc"), {"time": t}, {"stf": v}, ["time"])
        spec = ("class_name: NetCDF_STF\n            nc_data_file: stf.nc\n            nc_var_times: time\n"
                "            nc_var_data: stf\n            chunk_size: NONE\n")
    p = os.path.join(d, "inparam.source.yaml")
    with open(p) as f:
        txt = f.read()
    i = txt.index("class_name: GaussianSTF")
    j = txt.index("use_derivative_integral:", i)
    j = txt.index("\n", j) + 1
    txt = txt[:i] + spec + "            padding: %s\n" % padding + txt[j:]
    with open(p, "w") as f:
        f.write(txt)
    return d, t, v


@pytest.mark.parametrize("cls", ["StreamSTF", "NetCDF_STF"])
def test_table_stf_matches_oracle(built, tmp_path, cls):
    """StreamSTF / NetCDF_STF: the table is interpolated at the accumulated step times (in
    the engine's STF table and in the oracle alike); the run starts at the first sample."""
    from axisem3d_b200 import simulation
    d, t, v = _table_stf(_box(str(tmp_path / "input")), cls)
    res = simulation.run(d, None, precision="fp64", max_steps=60)
    sim = res.sim
    st = sim.model.ms_stf[0]
    assert st.table is not None and st.padding == 1 and st.pad_first == int(cls == "NetCDF_STF")
    assert sim.t0 == math.floor(t[0] / sim.dt) * sim.dt
    ref = _oracle_traces(sim)
    for name, (t_ref, w_ref) in ref.items():
        tt, w = res.traces[name]
        assert np.array_equal(tt, t_ref) and np.abs(w_ref).max() > 0
        err = float(np.linalg.norm(w - w_ref) / np.linalg.norm(w_ref))
        assert err <= TOL["fp64"], (name, err)
