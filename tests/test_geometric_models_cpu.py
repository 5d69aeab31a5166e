"""CPU tests of the geometric and ocean-load 3-D models of the preloop, against closed forms:

  StructuredGridG3D   (models3D/geometric/StructuredGridG3D.cpp) a constant undulation A
                      between min < interface < max ramps linearly, so in a Cartesian box with
                      the three radii on element boundaries dZ/dz is A / (interface - min)
                      below the interface and -A / (max - interface) above it, exactly:
                      PRT X0 = 1, X1 = X2 = 0, X3 = 1 / (1 + dZ/dz), |J| = 1 + dZ/dz
                      (Undulation::createPRT), and the total mass is unchanged (the map
                      moves material inside [min, max] only; Undulation::getMassJacobian)
  StructuredGridO3D   (models3D/ocean_load/StructuredGridO3D.cpp) a constant sum(rho depth)
                      D gives MassOceanLoad1D masses summing to D times the top surface
                      integral (s ds per radian), the same measure as the solid masses
  Ellipticity         (models3D/geometric/Ellipticity.cpp) on the polar axis a point of
                      radius r moves to the semi-minor axis b = (1 - f(r))^(2/3) r
  undulatedToReference  (SE_Model.cpp:481-542) bisection back to the reference radius
"""
import math
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import exodus_fixture as fx  # noqa: E402
from test_gpu_preloop import _box, _shell  # noqa: E402

A, D = 500.0, 1000.0 * 4000.0


def _box_with(d, models):
    s = np.linspace(0, 200e3, 11)
    ph = np.linspace(0, 2 * np.pi, 9)
    fx.write_grid_v3d(os.path.join(d, "und.nc"), {"s": s, "phi": ph}, {"dz": np.full((11, 9), A)}, ["s", "phi"])
    fx.write_grid_v3d(os.path.join(d, "sea.nc"), {"s": s, "phi": ph}, {"srd": np.full((11, 9), D)}, ["s", "phi"])
    fx.add_3d_models(d, models)
    return d


def test_constant_undulation_box_prt_mass_and_ocean(built, tmp_path):
    from axisem3d_b200 import preloop
    plain = preloop.build(_box(str(tmp_path / "plain")), max_steps=10)
    d = _box_with(_box(str(tmp_path / "input")), [
        fx.geometric_yaml("moho", "und.nc", "DISTANCE_AZIMUTH", "RADIUS", ["s", "phi"], [0, 1], "dz",
                          6331e3, 6301e3, 6361e3),
        fx.ocean_yaml("sea", "sea.nc", "DISTANCE_AZIMUTH", ["s", "phi"], [0, 1], "srd")])
    sim = preloop.build(d, max_steps=10)
    m = sim.model
    p = m.prt
    assert len(p["element"]) == 80 and not p["is3d_prt"].any()
    x = p["x"].reshape(-1, 5, 25)
    assert np.allclose(x[:, 0], 1.0, rtol=0, atol=1e-14)
    assert np.abs(x[:, 1:3]).max() < 1e-12
    assert np.allclose(x[:, 4] * x[:, 3], 1.0, rtol=0, atol=1e-14)
    # dZ/dz per element from its centre height
    zc = np.array([plain.model.sp_coords[m.se_pts[e], 1].mean() for e in p["element"]])
    dzdz = np.where(zc < 6301e3, 0., np.where(zc < 6331e3, A / 30e3, np.where(zc < 6361e3, -A / 30e3, 0.)))
    assert np.allclose(1. / x[:, 3], 1. + dzdz[:, None], rtol=0, atol=1e-12)
    # mass: unchanged in total, moved inside the undulated layers
    assert m.sp_mass_nr is None
    assert abs(m.sp_mass.sum() - plain.model.sp_mass.sum()) <= 1e-12 * plain.model.sp_mass.sum()
    assert np.abs(m.sp_mass - plain.model.sp_mass).max() > 1e-3 * np.abs(plain.model.sp_mass).max()
    # ocean: MassOceanLoad1D on the 41 surface points, D * S^2 / 2 in total
    pts, mo, th = m.ocean_load
    assert len(pts) == 41 and m.ocean_load3d is None
    assert abs(mo.sum() - D * 100e3 ** 2 / 2.) <= 1e-12 * D * 100e3 ** 2
    assert np.allclose(th, 0.0)


def test_azimuthal_undulation_makes_3d_elements(built, tmp_path):
    """An undulation varying with phi: 3-D PRT on the elements it reaches, which become 3-D
    (per-slice operands), Mass3D on their points, MassOceanLoad3D under a phi-varying ocean."""
    from axisem3d_b200 import preloop
    d = _box(str(tmp_path / "input"))
    s, ph = np.linspace(0, 200e3, 11), np.linspace(0, 2 * np.pi, 9)
    fx.write_grid_v3d(os.path.join(d, "und.nc"), {"s": s, "phi": ph},
                      {"dz": 300.0 * np.cos(ph)[None, :] * np.ones((11, 1))}, ["s", "phi"])
    fx.write_grid_v3d(os.path.join(d, "sea.nc"), {"s": s, "phi": ph},
                      {"srd": D * (1 + 0.5 * np.sin(ph))[None, :] * np.ones((11, 1))}, ["s", "phi"])
    fx.add_3d_models(d, [fx.geometric_yaml("moho", "und.nc", "DISTANCE_AZIMUTH", "DEPTH", ["s", "phi"], [0, 1],
                                           "dz", 40e3, 10e3, 70e3),
                         fx.ocean_yaml("sea", "sea.nc", "DISTANCE_AZIMUTH", ["s", "phi"], [0, 1], "srd")])
    m = preloop.build(d, max_steps=10).model
    p = m.prt
    e3 = p["element"][p["is3d_prt"] == 1]
    assert len(e3) > 0 and np.all(m.se_is3d[e3] == 1)
    for k in np.nonzero(p["is3d_prt"])[0]:
        nr = int(m.se_nr[p["element"][k]])
        x = p["x"][p["offset"][k]:p["offset"][k] + 5 * nr * 25].reshape(5, nr, 25)
        assert np.ptp(x[4]) > 0 and np.all(x[4] > 0)
    assert m.sp_mass_nr is not None and (m.sp_mass_nr > 1).any()
    pts, off, mo, nrm = m.ocean_load3d
    assert len(pts) == 41 and np.allclose(np.linalg.norm(nrm, axis=1), 1.0)


def test_ellipticity_on_the_axis(built, tmp_path):
    from axisem3d_b200 import preloop
    d = _shell(str(tmp_path / "input"))
    fx.add_3d_models(d, [fx.ellipticity_yaml("ellipticity")])
    p = os.path.join(d, "inparam.model.yaml")
    with open(p) as f:
        txt = f.read()
    with open(p, "w") as f:
        f.write(txt.replace("flattening_on_surface: SPHERE", "flattening_on_surface: WGS84"))
    sim = preloop.build(d, max_steps=10)
    from axisem3d_b200.models3d import Ellipticity, element_spz
    from axisem3d_b200.preloop import Geodesy
    geo = Geodesy(sim.mesh, preloop.Inparam(d))
    f_s = geo.flattening(np.array([6371e3]))[0]
    assert abs(f_s - 1. / 298.257223563) < 1e-15
    r = 6371e3
    und, _ = Ellipticity("e").at(np.array([[0., 0., r]]), geo)
    assert abs(und[0] - ((1. - f_s) ** (2. / 3.) - 1.) * r) < 1e-6
    # the whole mesh is touched, solid and fluid
    assert len(sim.model.prt["element"]) == len(sim.model.se_nr)
    assert len(sim.model.prt_fluid["element"]) == len(sim.model.fe_nr)


def test_undulated_to_reference_bisection():
    """SE_Model::undulatedToReference with a linear ramp (undulation u(r) = c (r - r0) on
    [r0, r1]): the reference radius of an undulated radius R is r0 + (R - r0) / (1 + c)."""
    from axisem3d_b200.preloop import _Undulation

    class Ramp:
        def at(self, spz, geo):
            z = spz[:, 2]
            return np.where((z > 100.) & (z < 200.), 0.05 * (z - 100.), 0.), True

    class Geo:
        cartesian, inner_radius, outer_radius = True, 0., 300.

    und = _Undulation(None, True)
    ref = und.to_reference([Ramp()], np.array([1., 0., 150.]), Geo(), 1e-9)
    assert abs(ref[2] - (100. + 50. / 1.05)) < 1e-8
    assert und.to_reference([], np.array([1., 0., 150.]), Geo(), 1e-9)[2] == 150.


def test_geometric_model_errors(built, tmp_path):
    from axisem3d_b200 import preloop
    d = _box_with(_box(str(tmp_path / "input")), [
        fx.geometric_yaml("moho", "und.nc", "DISTANCE_AZIMUTH", "RADIUS", ["s", "phi"], [0, 1], "dz",
                          6301e3, 6301e3, 6361e3)])
    with pytest.raises(preloop.PreloopError, match="interface must lie within"):
        preloop.build(d, max_steps=10)
    d = _box_with(_box(str(tmp_path / "input2")), [fx.ellipticity_yaml("a"), fx.ellipticity_yaml("b")])
    with pytest.raises(preloop.PreloopError, match="cannot be added more than once"):
        preloop.build(d, max_steps=10)


def test_fluid_pressure_pattern_on_the_axis(built, tmp_path):
    """Mechanism::release (Mechanism.cpp:59-86) for a pressure on the axis: a monopole on
    the element's axis points, P w / (2 pi), in the fluid element that holds it."""
    from axisem3d_b200 import preloop
    from test_gpu_preloop import _pressure_source
    sim = preloop.build(_pressure_source(_shell(str(tmp_path / "input"))), max_steps=10)
    m = sim.model
    assert len(m.ps_elem) == 1 and len(m.ms_elem) == 0 and len(m.fs_elem) == 0
    e = int(m.ps_elem[0])
    assert m.fe_axial[e] == 1 and m.ps_nu[0] == 1
    pat = m.ps_pattern.reshape(1, 25)
    assert np.all(pat[0, 5:] == 0) and np.all(pat.imag == 0)
    assert abs(pat[0].real.sum() * 2. * math.pi / 1e12 - 1.) < 1e-9


def test_table_stf_parsing_and_errors(built, tmp_path):
    """STF::buildInparam for StreamSTF / NetCDF_STF: padding modes and the file checks."""
    from axisem3d_b200 import preloop
    from test_gpu_preloop import _table_stf
    d, t, v = _table_stf(_box(str(tmp_path / "a")), "StreamSTF", "[0.5, -0.25]")
    st = preloop.build(d, max_steps=5).model.ms_stf[0]
    assert (st.padding, st.left, st.right, st.pad_first) == (1, 0.5, -0.25, 0)
    assert np.array_equal(st.table[0], t) and np.allclose(st.table[1], v, rtol=0, atol=1e-15)
    d, t, v = _table_stf(_box(str(tmp_path / "b")), "NetCDF_STF", "NONE")
    st = preloop.build(d, max_steps=5).model.ms_stf[0]
    assert (st.padding, st.pad_first) == (0, 1)
    with open(os.path.join(str(tmp_path / "a"), "stf.txt"), "a") as f:
        f.write("1.0 2.0 3.0\n")
    with pytest.raises(preloop.PreloopError, match="two columns"):
        preloop.build(str(tmp_path / "a"), max_steps=5)
