"""CPU tests of mesh and input ingestion (hdf5, exodus, inparam, preloop, output).

Pins, in order of strength:
  - a Cartesian Exodus fixture (the box of meshgen.cartesian_model, written as an Exodus file)
    gives the model meshgen builds directly: masses, operands, moduli, source pattern and
    station weights to round-off, and the oracle's seismograms of both models agree to 1e-10;
  - the reference's own example meshes (read when the reference tree is present): all open, and
    the PREM global mesh integrates to Earth's mass without the outer core;
  - a spherical shell fixture: closed-form solid volume, axis and interface counts;
  - geodesy identities, output file round trips and the error paths of unsupported inputs.
"""
import glob
import math
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import exodus_fixture as fx  # noqa: E402

# the reference checkout's examples directory, named by AXISEM3D_REFERENCE (the checkout root);
# the tests that read it are skipped where it is not set
REF = os.path.join(os.environ.get("AXISEM3D_REFERENCE", ""), "examples")
have_ref = pytest.mark.skipif(not os.environ.get("AXISEM3D_REFERENCE") or not os.path.isdir(REF),
                              reason="AXISEM3D_REFERENCE (reference checkout with examples) not set")

NX, NZ, W, H, R = 10, 8, 100e3, 80e3, 6371e3


def _box_dir(tmp, attenuation=None, storage="element_nodes"):
    from axisem3d_b200 import meshgen
    ref = meshgen.cartesian_model(nx=NX, nz=NZ, width=W, height=H, nr=5, nstations=5, source_depth=10e3,
                                  attenuation=attenuation)
    desc = fx.cartesian_box(NX, NZ, W, H, 2700.0, 5800.0, 3460.0, surface=R, storage=storage,
                            attenuation=attenuation, minimum_period=1.0)
    st = [("S%d" % k, "XX", W * k / 5, 0.0, 0.0) for k in range(1, 6)]
    d = fx.write_inputs(str(tmp), desc, nr=5, depth=10e3, mt=ref.meta["moment"], hdur=1.0, decay=math.pi,
                        order="RICKER", courant=0.6, record_length=1.0, stations=st,
                        attenuation="FULL" if attenuation else "NONE")
    return d, ref


def _point_perm(m, ref):
    rmap = {(round(c[0], 3), round(c[1] + R, 3)): i for i, c in enumerate(ref.sp_coords)}
    return np.array([rmap[(round(c[0], 3), round(c[1], 3))] for c in m.sp_coords])


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("storage", ["element_nodes", "elements"])
def test_box_exodus_gives_the_meshgen_model(tmp_path, storage):
    from axisem3d_b200 import preloop
    d, ref = _box_dir(tmp_path, storage=storage)
    m = preloop.build(d).model
    perm = _point_perm(m, ref)
    assert m.dt == ref.dt
    assert np.array_equal(perm[m.se_pts], ref.se_pts)
    assert np.array_equal(m.sp_axial, ref.sp_axial[perm]) and np.array_equal(m.sp_nr, ref.sp_nr[perm])
    assert _rel(m.sp_mass, ref.sp_mass[perm]) < 1e-12
    assert _rel(m.se_geom, ref.se_geom) < 1e-12
    assert _rel(m.se_moduli, ref.se_moduli) < 1e-14
    assert np.array_equal(m.ms_elem, ref.ms_elem) and _rel(m.ms_pattern, ref.ms_pattern) < 1e-14
    assert m.ms_stf == ref.ms_stf
    assert np.array_equal(m.st_elem, ref.st_elem) and _rel(m.st_w, ref.st_w) < 1e-14


def test_box_with_full_attenuation_gives_the_meshgen_model(tmp_path):
    from axisem3d_b200 import meshgen, preloop
    sls = dict(meshgen.default_sls(3, fmin=0.1, fmax=2.0), qkappa=57823.0, qmu=120.0)
    d, ref = _box_dir(tmp_path, attenuation=sls)
    m = preloop.build(d).model
    assert m.dt == ref.dt
    assert _rel(m.se_moduli, ref.se_moduli) < 1e-13
    assert _rel(m.se_att_moduli, ref.se_att_moduli) < 1e-13
    assert np.allclose(m.att_alpha, ref.att_alpha, rtol=0, atol=1e-15)
    assert np.allclose(m.att_beta, ref.att_beta, rtol=1e-13) and np.allclose(m.att_gamma, ref.att_gamma, rtol=1e-13)


def test_box_seismograms_of_both_models_agree_in_the_oracle(built, tmp_path):
    import oracle as O
    from axisem3d_b200 import preloop
    d, ref = _box_dir(tmp_path)
    m = preloop.build(d).model
    ref.t0 = m.t0            # the preloop starts at floor(t0 / dt) dt, as main.cpp does
    out = []
    for mod in (m, ref):
        o = O.Oracle(mod, "fp64")
        o.run(60)
        out.append(o.seismograms())
        o.close()
    assert np.abs(out[1]).max() > 0
    assert _rel(out[0], out[1]) < 1e-10


def _shell_dir(tmp, rho_solid=None, attenuation="CG4"):
    from axisem3d_b200 import meshgen
    r_edges = [3480e3, 3540e3, 3600e3, 4200e3, 4800e3, 5400e3, 6000e3, 6371e3]
    layers = [dict(RHO=9900., VP=8000., VS=0., QMU=0., QKAPPA=57823.)] * 2 + \
        [dict(RHO=rho_solid or 5500. - 300 * k, VP=13000. - 600 * k, VS=7000. - 300 * k, QMU=300.,
              QKAPPA=57823.) for k in range(5)]
    sls = meshgen.default_sls(3, fmin=1 / 80., fmax=1 / 5.)
    desc = fx.spherical_shell(24, r_edges, 2, layers, attenuation=sls, minimum_period=20.0,
                              discontinuities=[3480e3, 3600e3, 6371e3])
    st = [("S%02d" % k, "XX", 90. - 170. * k / 9, 0.0, 0.0) for k in range(1, 9)]
    return fx.write_inputs(str(tmp), desc, nr=8, depth=100e3, mt=(1e20, -2e19, 3e19, 5e19, -4e19, 1e19),
                           hdur=10.0, decay=1.628, order="RICKER", courant=0.6, record_length=200., stations=st,
                           horizontal="LATITUDE_LONGITUDE", frame="RTZ", attenuation=attenuation,
                           boundaries=["BOTTOM", "RIGHT"], clayton=True, sponge=True, spans=[0.05, 0.05],
                           lucky=True, bound_nr=True), r_edges


def test_shell_volume_axis_and_interface(tmp_path):
    from axisem3d_b200 import preloop
    d, r_edges = _shell_dir(tmp_path, rho_solid=4000.0)
    sim = preloop.build(d)
    m = sim.model
    # solid mass = rho * 4/3 pi (R^3 - r_sf^3); the points carry it divided by 2 pi
    vol = 4. / 3. * math.pi * (r_edges[-1] ** 3 - r_edges[2] ** 3)
    assert abs(m.sp_mass.sum() * 2 * math.pi / (4000.0 * vol) - 1.0) < 1e-6
    # both axis columns are axial (the south one after the side-3 rotation)
    assert int(m.se_axial.sum()) == 2 * 5 and int(m.fe_axial.sum()) == 2 * 2
    assert len(m.sf_solid) == 4 * 24 + 1
    # Clayton on the fluid bottom, sponge over the lowest 5 % of the radius span
    assert m.cl_fluid is not None and m.cl_solid is None
    assert m.sponge_fluid is not None and m.sponge_solid is not None
    assert sim.info["abc_keys"] == ["BOTTOM"] and sim.info["attenuation"] == "CG4"
    # station longitude 0 -> phi 0; theta = epicentral distance
    g = sim.groups[0]
    assert np.allclose(g.phi, 0.0) and np.allclose(g.theta, np.radians(170. * np.arange(1, 9) / 9), atol=1e-12)


@have_ref
def test_reference_meshes_open():
    from axisem3d_b200 import hdf5
    from axisem3d_b200.exodus import ExodusMesh
    files = sorted(set(glob.glob(REF + "/**/*.e", recursive=True)))
    assert len(files) >= 10
    for f in files:
        h = hdf5.File(f)
        for ds in h.datasets.values():
            ds.read()
        m = ExodusMesh(f)
        assert m.connectivity.min() == 0 and m.connectivity.max() == m.num_nodes - 1
        assert len(m.radial_coords) >= 2


@have_ref
def test_reference_prem_mesh_mass():
    """PREM: Earth 5.974e24 kg minus the outer core 1.841e24 kg in the solid elements."""
    from axisem3d_b200 import preloop
    sim = preloop.build(REF + "/01_S362ANI_EMC_global/input1D", skip_unsupported_channels=True)
    m = sim.model
    assert abs(m.sp_mass.sum() * 2 * math.pi / 4.133e24 - 1.0) < 3e-3
    assert sim.info["skipped_channels"] == [] and m.st_gradient     # E_I1 and R3 need gradients
    assert len(m.ms_elem) == 1 and m.ms_nu[0] == 3 and m.ms_stf[0].derivative_order == -1


def test_unsupported_inputs_raise(tmp_path):
    from axisem3d_b200 import preloop
    d, _ = _box_dir(tmp_path)
    p = os.path.join(d, "inparam.output.yaml")
    with open(p) as f:
        txt = f.read()
    with open(p, "w") as f:
        f.write(txt.replace("channels: [U]", "channels: [U, E_I1, S11]"))
    with pytest.raises(preloop.PreloopError, match="S11"):
        preloop.build(d)
    sim = preloop.build(d, skip_unsupported_channels=True)
    assert sim.info["skipped_channels"] == ["S11"] and sim.groups[0].channels == ["U1", "U2", "U3", "E_I1"]
    p = os.path.join(d, "inparam.model.yaml")
    with open(p) as f:
        txt = f.read()
    with open(p, "w") as f:
        f.write(txt.replace("list_of_3D_models: []", "list_of_3D_models:\n    - moho:\n        activated: true\n"
                                                      "        class_name: SphericalHarmonicsG3D\n"))
    with pytest.raises(preloop.PreloopError, match="SphericalHarmonicsG3D is not supported"):
        preloop.build(d)


def test_lucky_numbers():
    from axisem3d_b200.preloop import is_lucky, next_lucky
    assert [n for n in range(1, 30) if not is_lucky(n)] == [17, 19, 23, 29]
    assert not is_lucky(11 * 13) and is_lucky(11 * 8) and not is_lucky(11 * 11)
    assert next_lucky(17) == 18 and next_lucky(127) == 128


def test_geodesy_round_trip_and_back_azimuth(tmp_path):
    from axisem3d_b200.exodus import ExodusMesh
    from axisem3d_b200.inparam import Inparam
    from axisem3d_b200.preloop import Geodesy
    d, _ = _shell_dir(tmp_path)
    p = os.path.join(d, "inparam.source.yaml")
    with open(p) as f:
        txt = f.read()
    with open(p, "w") as f:
        f.write(txt.replace("latitude_longitude: [90., 0.]", "latitude_longitude: [37.91, -77.93]"))
    inp = Inparam(d)
    geo = Geodesy(ExodusMesh(os.path.join(d, "mesh.e")), inp)
    rng = np.random.default_rng(3)
    llr = np.stack([rng.uniform(-80, 80, 20), rng.uniform(-170, 170, 20), np.full(20, 6.0e6)], axis=1)
    spz = geo.llr2spz(llr, True)
    back = geo.spz2llr(spz, True, False)
    assert np.allclose(back[:, :2], llr[:, :2], atol=1e-9) and np.allclose(back[:, 2], 6.0e6)
    # back azimuth against the spherical-trigonometry formula (no flattening on a sphere)
    la1, lo1 = np.radians(37.91), np.radians(-77.93)
    la2, lo2 = np.radians(llr[:, 0]), np.radians(llr[:, 1])
    baz = np.arctan2(np.sin(lo1 - lo2) * np.cos(la1),
                     np.cos(la2) * np.sin(la1) - np.sin(la2) * np.cos(la1) * np.cos(lo1 - lo2))
    got = geo.back_azimuth(llr, True)
    assert np.allclose(np.angle(np.exp(1j * (got - baz))), 0.0, atol=1e-9)


def test_semi_spherical_quad_area():
    """sum of ifact / s over the points = the area of a quad with one curved edge."""
    from axisem3d_b200 import _lib as L, meshgen
    r0, r1, t0, t1 = 1000.0, 1500.0, 0.3, 0.5
    # straight inner edge, curved outer edge (nodes 2-3 on r1)
    n = np.array([r0 * math.sin(t0), r0 * math.cos(t0), r0 * math.sin(t1), r0 * math.cos(t1),
                  r1 * math.sin(t1), r1 * math.cos(t1), r1 * math.sin(t0), r1 * math.cos(t0)])
    g, sz = meshgen.geometry_batch(n[None, :], np.zeros(1, np.uint8), L.AXG_MAP_SEMI_SPHERICAL)
    area = float(np.sum(g[0, 5] / sz[0, 0]))
    exact = 0.5 * r1 * r1 * (t1 - t0) - 0.5 * r0 * r0 * math.sin(t1 - t0)
    assert abs(area / exact - 1.0) < 1e-9
    # corners map onto the nodes
    out = np.zeros(6)
    for k, (xi, eta) in enumerate([(-1, -1), (1, -1), (1, 1), (-1, 1)]):
        assert L.lib().axg_quad_map(L.AXG_MAP_SEMI_SPHERICAL, n.ctypes.data_as(L.P_f64), xi, eta,
                                    out.ctypes.data_as(L.P_f64)) == 0
        assert np.allclose(out[:2], n[2 * k:2 * k + 2], atol=1e-9)


def test_output_formats_round_trip(tmp_path):
    from scipy.io import netcdf_file
    from axisem3d_b200 import output
    from axisem3d_b200.preloop import StationGroup
    rng = np.random.default_rng(0)
    data = rng.normal(size=(3, 2, 37))
    times = np.arange(37) * 0.25 - 2.0
    for fmt in ("ASCII_STATION", "ASCII_CHANNEL", "NETCDF"):
        g = StationGroup(name="g_" + fmt, keys=["XX.A", "XX.B", "YY.C"], channels=["U1", "U3"], frame="RTZ",
                         interval=1, tmin=-9e9, tmax=9e9, fmt=fmt, buffer_size=10, first=0)
        output.write_group(str(tmp_path), g, times, data, 16)
        gd = tmp_path / "stations" / g.name
        if fmt == "NETCDF":
            nc = netcdf_file(str(gd / "axisem3d_synthetics.nc.rank0"), "r", mmap=False)
            assert np.allclose(nc.variables["data_wave"][:], data)
            assert np.allclose(nc.variables["data_time"][:], times)
            nc.close()
            continue
        assert np.allclose(np.loadtxt(gd / "data_time.ascii"), times)
        if fmt == "ASCII_STATION":
            for k, key in enumerate(g.keys):
                assert np.allclose(np.loadtxt(gd / (key + ".ascii")), data[k].T, rtol=1e-15)
        else:
            for c, ch in enumerate(g.channels):
                assert np.allclose(np.loadtxt(gd / "dir_rank0" / (ch + ".ascii")), data[:, c].T, rtol=1e-15)
            assert (gd / "dir_rank0" / "list_station.info").read_text().split() == g.keys


def test_tensor_rotation_identities():
    """Rotated gradients are R G R^T, and the strain of the rotated gradient is the rotated
    strain (the Voigt round trip of Station::rotate for 6-component fields)."""
    from axisem3d_b200 import output
    rng = np.random.default_rng(1)
    g = rng.normal(size=(2, 4, 9))
    u = rng.normal(size=(2, 4, 3))
    th, baz, phi = np.array([0.3, 1.2]), np.array([0.5, -0.7]), np.array([0.1, 0.2])
    for frame in ("RTZ", "ENZ", "xyz"):
        gr = output.rotate_field(g, frame, th, baz, phi, False)
        ur = output.rotate_field(u, frame, th, baz, phi, False)
        for k in range(2):
            R = output.rotate_field(np.eye(3)[None], frame, th[k:k + 1], baz[k:k + 1], phi[k:k + 1], False)[0].T
            assert np.allclose(ur[k], u[k] @ R.T)
            assert np.allclose(gr[k].reshape(4, 3, 3), R @ g[k].reshape(4, 3, 3) @ R.T)
        e = output.strain_from_gradient(g)
        e[..., 3:] *= .5
        er = output.rotate_field(e, frame, th, baz, phi, False)
        er[..., 3:] *= 2.
        assert np.allclose(er, output.strain_from_gradient(gr))


def test_rotation_frames():
    from axisem3d_b200.output import rotate_displacement
    # a purely radial (outward) displacement at colatitude theta: spz = (sin, 0, cos)
    th = np.array([0.3, 1.1])
    u = np.stack([np.sin(th), np.zeros(2), np.cos(th)], axis=1)[:, None, :]
    rtz = rotate_displacement(u, "RTZ", th, np.zeros(2), np.zeros(2), False)
    assert np.allclose(rtz[:, 0], [[0, 0, 1], [0, 0, 1]], atol=1e-15)
    # ENZ with back azimuth 0 (source due north): R points south, T east
    e = np.array([[[1.0, 0.0, 0.0]]])
    enz = rotate_displacement(e, "ENZ", np.array([0.0]), np.array([0.0]), np.array([0.0]), False)
    assert np.allclose(enz[0, 0], [0, -1, 0], atol=1e-15)


# ------------------------------------------------------------------ 3-D models ---
def _lin_box(x, y, d):
    return 0.01 + 2e-4 * x - 3e-4 * y + 4e-4 * d        # per km


def _lin_rho(x, y, d):
    return -0.02 + 1e-4 * x + 2e-4 * d


def _box3d_dir(tmp, props=None, fluid_vs=False):
    desc = fx.cartesian_box(NX, NZ, W, H, 2700.0, 5800.0, 3460.0, surface=R)
    st = [("S%d" % k, "XX", W * k / 5, 0.0, 0.0) for k in range(1, 6)]
    d = fx.write_inputs(str(tmp), desc, nr=5, depth=10e3, mt=(1e18, -3e17, 2e17, 4e17, -1e17, 5e17),
                        record_length=2.0, stations=st)
    x = np.linspace(-120., 120., 7)
    y = np.linspace(-120., 120., 5)
    dep = np.linspace(0., 90., 4)
    X, Y, D = np.meshgrid(x, y, dep, indexing="ij")
    fx.write_grid_v3d(os.path.join(d, "m3d.nc"), {"x": x, "y": y, "depth": dep},
                      {"dvs": _lin_box(X, Y, D), "drho": _lin_rho(X, Y, D)}, ["depth", "x", "y"])
    props = props or [("VS", "dvs", 1.0, "REF1D"), ("RHO", "drho", 0.5, "REF1D")]
    fx.add_3d_models(d, [fx.model3d_yaml("blob", "m3d.nc", "XY_CARTESIAN", "DEPTH", ["x", "y", "depth"],
                                         [1, 2, 0], props)])
    return d


def test_3d_model_moduli_and_masses_are_exact(tmp_path):
    """A grid linear in (x, y, depth) is interpolated exactly: every slice of every element
    carries rho (1 + 0.5 drho) and vs (1 + dvs) of the 1-D values, and the points carry the
    per-slice masses (Mass3D)."""
    from axisem3d_b200 import preloop
    d = _box3d_dir(tmp_path)
    m = preloop.build(d).model
    m1 = preloop.build(_box_dir(tmp_path / "plain")[0]).model
    assert m.se_is3d.all() and m.sp_mass_nr is not None
    for e in (0, 37, 79):
        nr = int(m.se_nr[e])
        off = m.se_mat_off[e]
        lam = m.se_moduli[off:off + nr * 25].reshape(nr, 25)
        mu = m.se_moduli[off + nr * 25:off + 2 * nr * 25].reshape(nr, 25)
        pts = m.se_pts[e]
        s_, z_ = m.sp_coords[pts, 0], m.sp_coords[pts, 1]
        phi = 2 * np.pi * np.arange(nr) / nr
        xx = s_[None] * np.cos(phi)[:, None] / 1e3
        yy = s_[None] * np.sin(phi)[:, None] / 1e3
        dd = (R - z_)[None] / 1e3
        rho = 2700.0 * (1 + 0.5 * _lin_rho(xx, yy, dd))
        mu_ref = rho * (3460.0 * (1 + _lin_box(xx, yy, dd))) ** 2
        assert np.allclose(mu, mu_ref, rtol=1e-13)
        assert np.allclose(lam, rho * 5800.0 ** 2 - 2 * mu_ref, rtol=1e-13)
    # Mass3D: the per-slice density times the summed integral factors (1-D mass / 2700)
    perm = {(round(c[0], 3), round(c[1], 3)): i for i, c in enumerate(m1.sp_coords)}
    for p in range(0, len(m.sp_nr), 97):
        nr = int(m.sp_mass_nr[p])
        vals = m.sp_mass[m.sp_mass_off[p]:m.sp_mass_off[p] + nr]
        s_, z_ = m.sp_coords[p]
        phi = 2 * np.pi * np.arange(nr) / nr
        rho = 2700.0 * (1 + 0.5 * _lin_rho(s_ * np.cos(phi) / 1e3, s_ * np.sin(phi) / 1e3, (R - z_) / 1e3))
        ref = rho * m1.sp_mass[perm[(round(s_, 3), round(z_, 3))]] / 2700.0
        assert np.allclose(vals, ref if nr > 1 else ref[:1], rtol=1e-12)


def test_3d_model_lat_lon_and_iso_to_tiso(tmp_path):
    """LATITUDE_LONGITUDE / DEPTH grid on the shell (mesh pole at the source at the north
    pole, so latitude = 90 - theta and longitude = phi): a VSH model on isotropic elements
    turns them transversely isotropic (VSV = VS, VSH = VS (1 + dv)); the fluid layer and the
    deepest mantle lie outside the grid and stay 1-D."""
    from axisem3d_b200 import _lib as L, preloop
    d, r_edges = _shell_dir(tmp_path / "in", attenuation="NONE")
    lat = np.linspace(-90., 90., 7)
    lon = np.linspace(-180., 180., 9)
    dep = np.linspace(0., 2000., 5)
    LA, LO, DE = np.meshgrid(lat, lon, dep, indexing="ij")
    dv = 0.02 + 1e-4 * LA - 5e-5 * LO + 1e-5 * DE
    fx.write_grid_v3d(os.path.join(d, "ll.nc"), {"lat": lat, "lon": lon, "dep": dep}, {"dv": dv},
                      ["lat", "lon", "dep"])
    fx.add_3d_models(d, [fx.model3d_yaml("sh", "ll.nc", "LATITUDE_LONGITUDE", "DEPTH", ["lat", "lon", "dep"],
                                         [0, 1, 2], [("VSH", "dv", 1.0, "REF1D")])])
    sim = preloop.build(d)
    m = sim.model
    ti = m.se_rheo == L.AXG_TISO
    assert ti.any() and m.se_is3d[ti].all() and not m.se_is3d[~ti].any()
    assert not m.fe_is3d.any()
    # N = rho VSH^2 on the slices of one TI element against the closed form
    e = int(np.nonzero(ti)[0][len(np.nonzero(ti)[0]) // 2])
    nr = int(m.se_nr[e])
    off = m.se_mat_off[e]
    pts = m.se_pts[e]
    s_, z_ = m.sp_coords[pts, 0], m.sp_coords[pts, 1]
    r_ = np.hypot(s_, z_)
    th = np.degrees(np.arccos(z_ / r_))
    phi = 2 * np.pi * np.arange(nr) / nr
    lo = np.degrees(np.where(phi > np.pi, phi - 2 * np.pi, phi))
    dvr = 0.02 + 1e-4 * (90. - th)[None] - 5e-5 * lo[:, None] + 1e-5 * ((6371e3 - r_) / 1e3)[None]
    Lm = m.se_moduli[off + 3 * nr * 25:off + 4 * nr * 25].reshape(nr, 25)
    N = m.se_moduli[off + 4 * nr * 25:off + 5 * nr * 25].reshape(nr, 25)
    inside = ((6371e3 - r_) / 1e3) <= 2000.0                 # points below the grid keep 1-D values
    ref = np.where(inside[None], (1 + dvr) ** 2, 1.0)
    assert inside.any() and (~inside).any()
    assert np.allclose(N / Lm, ref, rtol=1e-12)


def test_3d_model_errors(tmp_path):
    from axisem3d_b200 import preloop
    d = _box3d_dir(tmp_path / "c", props=[("C11", "dvs", 1.0, "ABS")])
    with pytest.raises(preloop.PreloopError, match="Cij"):
        preloop.build(d)
    # a VS model reaching into the fluid layer of the shell
    d2, _ = _shell_dir(tmp_path / "s")
    lat, lon, dep = np.linspace(-90., 90., 3), np.linspace(-180., 180., 3), np.linspace(0., 3000., 3)
    fx.write_grid_v3d(os.path.join(d2, "ll.nc"), {"lat": lat, "lon": lon, "dep": dep},
                      {"dv": np.full((3, 3, 3), 0.01)}, ["lat", "lon", "dep"])
    fx.add_3d_models(d2, [fx.model3d_yaml("deep", "ll.nc", "LATITUDE_LONGITUDE", "DEPTH", ["lat", "lon", "dep"],
                                          [0, 1, 2], [("VS", "dv", 1.0, "REF1D")])])
    with pytest.raises(preloop.PreloopError, match="Unacceptable property key: VS"):
        preloop.build(d2)


def test_ti_absorbing_boundaries_use_voigt_velocities(tmp_path):
    """Material::getPointwiseRhoVpVs: Clayton rho vp / rho vs of a transversely isotropic
    element are the Voigt averages of kappa and mu, not VPV / VSV (homogeneous TI layers, so
    the nodal interpolation is exact)."""
    from axisem3d_b200 import preloop
    r_edges = [5000e3, 5500e3, 6000e3, 6371e3]
    lay = dict(RHO=3300., VPV=8000., VPH=8400., VSV=4400., VSH=4700., ETA=0.9)
    desc = fx.spherical_shell(12, r_edges, 0, [lay] * 3, discontinuities=[5000e3, 6371e3])
    d = fx.write_inputs(str(tmp_path), desc, nr=4, depth=100e3, record_length=20., boundaries=["BOTTOM"],
                        clayton=True, sponge=False, spans=[0.05])
    m = preloop.build(d).model
    A, C, Lm, N = (lay["RHO"] * lay[k] ** 2 for k in ("VPH", "VPV", "VSV", "VSH"))
    F = lay["ETA"] * (A - 2 * Lm)
    kp = (4 * A + C + 4 * F - 4 * N) / 9.
    mu = (A + C - 2 * F + 6 * Lm + 5 * N) / 15.
    assert m.cl_solid is not None
    assert np.allclose(m.cl_solid["rho_vp"], np.sqrt((kp + 4. / 3. * mu) * lay["RHO"]), rtol=1e-12)
    assert np.allclose(m.cl_solid["rho_vs"], np.sqrt(mu * lay["RHO"]), rtol=1e-12)


# ------------------------------------------------------------------ Nr fields ---
def _set_nr(d, text):
    with open(os.path.join(d, "inparam.nr.yaml"), "w") as f:
        f.write(text)


def test_nr_fields(tmp_path):
    """ANALYTICAL (linear in depth between control depths), STRUCTURED (bilinear on an (s, z)
    grid, out-of-range value outside) and POINTWISE (inverse-distance average of the 4
    nearest control points, exact on a control point) at the mesh nodes."""
    from axisem3d_b200 import preloop
    from axisem3d_b200.exodus import ExodusMesh
    from axisem3d_b200.inparam import Inparam
    d, _ = _box_dir(tmp_path)
    mesh = ExodusMesh(os.path.join(d, "mesh.e"))
    depth = R - mesh.coords[:, 1]
    _set_nr(d, "type_Nr: ANALYTICAL\nbound_Nr_by_inplane: false\nanalytical:\n"
               "    code_ID: depth-dependent (AxiSEM3D default)\n    depth_dependent_AxiSEM3D_default:\n"
               "        control_depths: [0., 40e3, 80e3]\n        Nr_at_control_depths: [40, 20, 8]\n")
    geo = preloop.Geodesy(mesh, Inparam(d))
    nr = preloop._nr_field(mesh, Inparam(d), geo)
    ref = np.where(depth <= 40e3, 40 - 20 * depth / 40e3, 20 - 12 * (depth - 40e3) / 40e3)
    assert np.array_equal(nr, np.floor(ref + 0.5).astype(int))
    # structured: Nr = 10 + s/1e4 + z-offset term on a grid covering half the box
    s_ax, z_ax = np.linspace(0., 50e3, 6), np.linspace(R - 80e3, R, 5)
    S, Z = np.meshgrid(s_ax, z_ax, indexing="ij")
    from scipy.io import netcdf_file
    nc = netcdf_file(os.path.join(d, "nr.nc"), "w", version=2)
    nc.createDimension("ns", 6)
    nc.createDimension("nz", 5)
    for n, a, dim in (("structured_s", s_ax, "ns"), ("structured_z", z_ax, "nz")):
        v = nc.createVariable(n, "d", (dim,))
        v[:] = a
    v = nc.createVariable("structured_Nr", "d", ("ns", "nz"))
    v[:] = 10 + S / 1e4 + (R - Z) / 2e4
    nc.close()
    _set_nr(d, "type_Nr: STRUCTURED\nbound_Nr_by_inplane: false\nstructured:\n    nc_data_file: nr.nc\n"
               "    value_out_of_range: 3\n")
    nr = preloop._nr_field(mesh, Inparam(d), geo)
    s_, z_ = mesh.coords[:, 0], mesh.coords[:, 1]
    inside = s_ <= 50e3 + 1e-6
    assert np.all(nr[~inside] == 3)
    assert np.array_equal(nr[inside], np.floor(10 + s_[inside] / 1e4 + (R - z_[inside]) / 2e4 + 0.5).astype(int))
    # pointwise: control points on every mesh node carry 7 + node index % 5
    nc = netcdf_file(os.path.join(d, "pw.nc"), "w", version=2)
    nc.createDimension("dim_point", mesh.num_nodes)
    nc.createDimension("dim_sz", 2)
    v = nc.createVariable("pointwise_sz", "d", ("dim_point", "dim_sz"))
    v[:] = mesh.coords
    v = nc.createVariable("pointwise_Nr", "i", ("dim_point",))
    v[:] = 7 + np.arange(mesh.num_nodes) % 5
    nc.close()
    _set_nr(d, "type_Nr: POINTWISE\nbound_Nr_by_inplane: false\npointwise:\n    nc_data_file: pw.nc\n"
               "    multip_factor: 2.\n")
    nr = preloop._nr_field(mesh, Inparam(d), geo)
    assert np.array_equal(nr, 2 * (7 + np.arange(mesh.num_nodes) % 5))
