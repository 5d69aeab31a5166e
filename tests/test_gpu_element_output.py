"""GPU tests of element-wise output (list_of_element_groups): Exodus mesh + inparam files ->
preloop -> engine time loop with the element-record ring -> elements/<group>/
axisem3d_synthetics.nc.rank0, checked against a restatement written with plain loops on the
oracle's displacement at every record step:

  element fields  ElementOpSolid::record (core/output/element-wise/element/ElementOpSolid.cpp:
                  48-80) through SolidElement::getDisplField / getNablaField / getStrainField /
                  getCurlField (SolidElement.cpp:396-546): the RTZ frame as the rotation R(theta)
                  of each point (u' = R u, G' = R G R^T, strain and curl of G')
  rows            ElementOp::recordToElem (ElementOp.hpp:26-68): Fourier rows cut at na = nr, or
                  the series at each azimuth
  channels        ElementOp::dumpToIO (ElementOp.hpp:70-176), with its G_I1 (first three
                  gradient components) and E_J2 (shear products E23 E31 + E31 E12 + E12 E23)
  file            ElementIO_NetCDF::initialize / dumpToFile (ElementIO_NetCDF.cpp:14-249)

Tolerance (largest error over the largest value, per channel): FP64 1e-9, FP32 / mixed 1e-4.
"""
import math
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import exodus_fixture as fx  # noqa: E402
from test_gpu_preloop import _box, _element_displ_grad, _shell  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-9, "fp32": 1e-4, "mixed": 1e-4}
VOIGT = {"11": 0, "22": 1, "33": 2, "23": 3, "31": 4, "12": 5}


def _point_fields(U, g, ip, theta, rtz):
    """u [order, 3], G [order, 3, 3] (G[c, d] = d_d u_c) at GLL point ip, in the frame."""
    u = U[:, :, ip // 5, ip % 5]
    G = g[:, :, ip // 5, ip % 5].reshape(-1, 3, 3)
    if rtz:
        c, s = math.cos(theta), math.sin(theta)
        R = np.array([[c, 0., -s], [0., 1., 0.], [s, 0., c]])
        u = np.einsum("ij,aj->ai", R, u)
        G = np.einsum("ij,ajk,lk->ail", R, G, R)
    return u, G


def _rows(c, na, phis):
    """c [order, D] -> [na, D] real rows."""
    nu, D = c.shape
    if len(phis) == 0:
        rows = [c[0].real]
        for a in range(1, nu):
            rows += [c[a].real, c[a].imag]
        return np.array(rows)[:na]
    out = []
    for phi in phis:
        v = c[0].real.copy()
        for a in range(1, nu):
            v = v + (2. * np.exp(1j * a * phi) * c[a]).real
        out.append(v)
    return np.array(out)


def _channel(ch, u, G):
    """One channel of one row: u [3] and G [3, 3] real rows of the point."""
    E = np.array([G[0, 0], G[1, 1], G[2, 2], G[1, 2] + G[2, 1], G[0, 2] + G[2, 0], G[0, 1] + G[1, 0]])
    R = np.array([G[2, 1] - G[1, 2], G[0, 2] - G[2, 0], G[1, 0] - G[0, 1]])
    if ch == "U_NORM":
        return math.sqrt(float(np.sum(u * u)))
    if ch == "R_NORM":
        return math.sqrt(float(np.sum(R * R)))
    if ch == "G_I1":
        return G[0, 0] + G[0, 1] + G[0, 2]
    if ch == "E_I1":
        return E[0] + E[1] + E[2]
    if ch == "E_J2":
        i1 = E[0] + E[1] + E[2]
        return i1 * i1 / 3. - (E[0] * E[1] + E[1] * E[2] + E[2] * E[0]) + (E[3] * E[4] + E[4] * E[5] + E[5] * E[3])
    if ch[0] == "U":
        return u[int(ch[1]) - 1]
    if ch[0] == "G":
        return G[int(ch[1]) - 1, int(ch[2]) - 1]
    if ch[0] == "E":
        return E[VOIGT[ch[1:]]]
    return R[int(ch[1]) - 1]


def _expected(sim):
    """{group: (times, [element][na, point, channel, time])} from the oracle, with loops."""
    import oracle as O
    m = sim.model
    o = O.Oracle(m, "fp64")
    out = {g.name: ([], [[] for _ in g.elems]) for g in sim.element_groups}
    for t in range(sim.nsteps):
        time = sim.t0 + t * sim.dt
        groups = [g for g in sim.element_groups if t % g.interval == 0 and g.tmin <= time <= g.tmax]
        if groups:
            f = o.get_field("displ")
            cache = {}
            for g in groups:
                out[g.name][0].append(time)
                rtz = g.frame == "RTZ" and not sim.cartesian
                for k, e in enumerate(g.elems):
                    if e not in cache:
                        cache[e] = _element_displ_grad(m, f, int(e))
                    U, gr = cache[e]
                    blk = np.zeros((int(g.na[k]), g.npnts, len(g.channels)))
                    for j, ip in enumerate(g.ipnts[k]):
                        s, z = g.coords[k, j]
                        u, G = _point_fields(U, gr, int(ip), math.atan2(s, z), rtz)
                        ur = _rows(u, int(g.na[k]), g.phis)
                        Gr = _rows(G.reshape(-1, 9), int(g.na[k]), g.phis).reshape(-1, 3, 3)
                        for r in range(int(g.na[k])):
                            for c, ch in enumerate(g.channels):
                                blk[r, j, c] = _channel(ch, ur[r], Gr[r])
                    out[g.name][1][k].append(blk)
        o.run(1)
    o.close()
    return {k: (np.array(t), [np.stack(b, axis=-1) for b in v]) for k, (t, v) in out.items()}


def _read(path):
    from scipy.io import netcdf_file
    nc = netcdf_file(path, "r", mmap=False)
    out = {k: np.array(v.data) for k, v in nc.variables.items()}
    dims = {k: v.dimensions for k, v in nc.variables.items()}
    nc.close()
    return out, dims


def _check_group(g, path, exp, precision):
    v, dims = _read(path)
    times, blocks = exp
    assert np.allclose(v["data_time"], times, rtol=0, atol=1e-12 * max(1., np.abs(times).max()))
    assert [b"".join(r).decode() for r in v["list_channel"]] == g.channels
    assert v["list_na_grid"].tolist() == g.na_grid.tolist()
    assert np.array_equal(v["list_element_na"], g.elem_na)
    assert np.allclose(v["list_element_coords"], g.coords, rtol=0, atol=0)
    assert dims["list_element_coords"] == ("dim_element", "dim_GLL", "dim_2")
    nch = len(g.channels)
    got = [None] * len(g.elems)
    for nag in g.na_grid:
        w = v["data_wave__NaG=%d" % nag]
        tags = v["list_element__NaG=%d" % nag]
        assert dims["data_wave__NaG=%d" % nag] == ("dim_element__NaG=%d" % nag, "dim_na__NaG=%d" % nag, "dim_GLL",
                                                   "dim_channel", "dim_time")
        assert w.shape[2:] == (g.npnts, nch, len(times))
        for k in np.nonzero(g.elem_na[:, 2] == nag)[0]:
            i = int(g.elem_na[k, 3])
            assert tags[i] == g.tags[k]
            got[k] = w[i, :int(g.na[k])]
            assert not np.any(w[i, int(g.na[k]):])
    tol = TOL[precision]
    for c, ch in enumerate(g.channels):
        ref = np.concatenate([b[:, :, c].ravel() for b in blocks])
        val = np.concatenate([x[:, :, c].ravel() for x in got])
        scale = np.abs(ref).max()
        assert scale > 0, (g.name, ch)
        err = np.abs(val - ref).max() / scale
        assert err <= tol, (g.name, ch, err)


def _box_groups(d):
    fx.add_element_groups(d, [
        dict(name="whole_fourier", gll="[0, 2, 4]", channels="U, G, E_J2, R_NORM, G_I1, E_I1"),
        dict(name="surface_phis", edge_dim="VERTICAL", edge_pos=6371e3, phis="0.3, 2.0",
             channels="U_NORM, E, R", period="DTx3", window="[0.5, 3.0]", vmin=6300e3),
        dict(name="axis_side", edge_dim="HORIZONTAL", edge_pos=0.0, gll="[0, 1, 3]", channels="U, G_I1",
             buffer=7),
    ])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_box_element_groups_match_restatement(built, tmp_path, precision, monkeypatch):
    """Cartesian box, three groups (Fourier rows of all elements with gradient channels;
    top edge at two azimuths with a time window and every third step; the elements on the
    axis, edge points only). A ring of 4 records forces the chunked drain."""
    from axisem3d_b200 import preloop, simulation
    d = _box(str(tmp_path / "input"))
    _box_groups(d)
    sim = preloop.build(d, max_steps=30)
    assert [len(g.elems) for g in sim.element_groups] == [80, 10, 8]
    monkeypatch.setattr(simulation.ElementRecorder, "RING_BYTES", 1)
    res = simulation.run(d, str(tmp_path / "out"), precision=precision, max_steps=30)
    exp = _expected(res.sim)
    for g in res.sim.element_groups:
        _check_group(g, res.element_files[g.name], exp[g.name], precision)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_shell_element_groups_match_restatement(built, tmp_path, precision):
    """Spherical shell with a fluid layer and CG4 attenuation: RTZ groups in a theta / radius
    window at a latitude / longitude azimuth (strain channels) and on the surface edge with
    na_space 3 (Fourier rows, curl channels)."""
    from axisem3d_b200 import simulation
    d = _shell(str(tmp_path / "input"))
    fx.add_element_groups(d, [
        dict(name="slice", frame="RTZ", hmin=0.3, hmax=1.2, vmin=5000e3, latlon="[10.0, 20.0]", channels="U, E"),
        dict(name="top", edge_dim="VERTICAL", edge_pos=6371e3, frame="RTZ", na_space=3, channels="U, R",
             period="DTx2"),
    ])
    res = simulation.run(d, str(tmp_path / "out"), precision=precision, max_steps=24)
    exp = _expected(res.sim)
    assert [len(g.elems) for g in res.sim.element_groups] == [21, 24]
    for g in res.sim.element_groups:
        _check_group(g, res.element_files[g.name], exp[g.name], precision)


def test_element_record_ring_bounds(built, tmp_path):
    """Records that have left the ring, or are not recorded yet, are an argument error."""
    from axisem3d_b200 import preloop
    from axisem3d_b200.solver import EngineError, Solver
    d = _box(str(tmp_path / "input"))
    sim = preloop.build(d, max_steps=12)
    with Solver(sim.model, "fp32") as s:
        words = s.set_element_record([0, 5], [0, 12], [0, 1], 2, 3)
        nu = int(sim.model.se_nr[0]) // 2 + 1
        assert words == nu * 3 + (int(sim.model.se_nr[5]) // 2 + 1) * 9
        s.run(12)                                    # records 0 .. 5; ring holds 3 .. 5
        assert s.element_records(3, 3).shape == (3, words)
        for first, n in ((2, 1), (5, 2), (-1, 1)):
            with pytest.raises(EngineError):
                s.element_records(first, n)
