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
        u = output.rotate_displacement(u, g.frame, g.theta, g.baz, g.phi, sim.cartesian)
        out[g.name] = (sim.t0 + steps * sim.dt, output.channel_data(u, g.channels))
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
