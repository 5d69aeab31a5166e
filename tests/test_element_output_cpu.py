"""CPU tests of element-wise output: the element groups of the preloop (ElementOutput::
buildInparam / release, preloop/output/ElementOutput.cpp:27-480, and the na grid of
ElementOpGroup::initialize, core/output/element-wise/element/ElementOpGroup.hpp:66-150), the
NetCDF writer, and the host side of the recorder (entry layout, record selection, frames,
rows, channels, file) driven by a stand-in for the engine that serves the oracle's
displacement and a numpy gradient as the engine's element records.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import exodus_fixture as fx  # noqa: E402
from test_gpu_element_output import _box_groups, _check_group, _expected  # noqa: E402
from test_gpu_preloop import _box, _element_displ_grad  # noqa: E402


def test_na_grid_spacing():
    from axisem3d_b200.preloop import _na_grid
    assert _na_grid([5, 5, 5], 1).tolist() == [5]
    assert _na_grid([3, 4, 5, 6, 7, 8, 20], 1).tolist() == [3, 4, 5, 6, 7, 8, 20]
    # from the largest down, keep a value only when it is na_space below the last kept one
    assert _na_grid([3, 4, 5, 6, 7, 8, 20], 3).tolist() == [5, 8, 20]
    assert _na_grid([], 2).tolist() == []


def test_element_group_selection(built, tmp_path):
    """Box of 10 x 8 quads: all elements, the top edge, the elements on the axis."""
    from axisem3d_b200 import preloop
    d = _box(str(tmp_path / "input"))
    _box_groups(d)
    sim = preloop.build(d, max_steps=30)
    whole, top, axis = sim.element_groups
    assert len(whole.elems) == 80 and whole.npnts == 9
    assert whole.ipnts[0].tolist() == [0, 2, 4, 10, 12, 14, 20, 22, 24]
    assert whole.na.tolist() == whole.nr.tolist() and whole.na_grid.tolist() == sorted(set(whole.nr.tolist()))
    assert len(top.elems) == 10 and top.npnts == 5
    assert np.allclose(top.coords[:, :, 1], 6371e3)
    assert top.na.tolist() == [2] * 10 and top.na_grid.tolist() == [2] and top.interval == 3
    assert len(axis.elems) == 8 and np.allclose(axis.coords[:, :, 0], 0.0)
    assert axis.ipnts[0].tolist() == [4, 3, 1]                 # edge 3 (4, 3, 2, 1, 0) at 0, 1, 3
    assert np.all(sim.model.se_axial[axis.elems] == 1)
    # list_element_na: tag, na, na-grid value, index in it, global index (one rank)
    assert np.array_equal(whole.elem_na[:, 3], whole.elem_na[:, 4])
    for g in sim.element_groups:
        for nag in g.na_grid:
            sel = g.elem_na[:, 2] == nag
            assert sorted(g.elem_na[sel, 3].tolist()) == list(range(int(sel.sum())))


@pytest.mark.parametrize("change, message", [
    (dict(gll="[]"), "cannot be empty"),
    (dict(gll="[0, 5]"), "ranged between"),
    (dict(window="[100.0, 200.0]"), "No time step to record"),
])
def test_element_group_errors(built, tmp_path, change, message):
    from axisem3d_b200 import preloop
    d = _box(str(tmp_path / "input"))
    fx.add_element_groups(d, [dict(dict(name="g"), **change)])
    with pytest.raises(preloop.PreloopError, match=message):
        preloop.build(d, max_steps=30)


def test_element_group_duplicate_name_and_fluid(built, tmp_path):
    from axisem3d_b200 import preloop
    d = _box(str(tmp_path / "input"))
    fx.add_element_groups(d, [dict(name="g"), dict(name="g")])
    with pytest.raises(preloop.PreloopError, match="must be unique"):
        preloop.build(d, max_steps=30)
    fx.add_element_groups(d, [dict(name="g", channels="S")])
    with pytest.raises(preloop.PreloopError, match="Stress channels"):
        preloop.build(d, max_steps=30)
    fx.add_element_groups(d, [dict(name="g")])
    p = os.path.join(d, "inparam.output.yaml")
    with open(p) as f:
        head, tail = f.read().rsplit("medium: SOLID", 1)        # the element group's medium
    with open(p, "w") as f:
        f.write(head + "medium: FLUID" + tail)
    with pytest.raises(preloop.PreloopError, match="Fluid element groups"):
        preloop.build(d, max_steps=30)


def test_nc3_writer_round_trip(tmp_path):
    from scipy.io import netcdf_file
    from axisem3d_b200.ncwrite import NC3File
    p = str(tmp_path / "f.nc")
    f = NC3File(p)
    f.add("data_time", [("dim_time", 5)], np.float64)
    f.add("data_wave__NaG=3", [("dim_element__NaG=3", 2), ("dim_na__NaG=3", 3), ("dim_GLL", 4),
                               ("dim_channel", 2), ("dim_time", 5)], np.float32)
    f.add("list_channel", [("dim_channel", 2), ("dim_channel_str_length", 6)], "S1")
    f.add("list_element_na", [("dim_element", 2), ("dim_5", 5)], np.int32)
    f.create()
    rng = np.random.default_rng(3)
    w = rng.standard_normal((2, 3, 4, 2, 5)).astype(np.float32)
    f.var("data_time")[:2] = [0.5, 1.0]
    f.var("data_wave__NaG=3")[..., :2] = w[..., :2]
    f.flush()
    f.var("data_time")[2:] = [1.5, 2.0, 2.5]
    f.var("data_wave__NaG=3")[..., 2:] = w[..., 2:]
    f.var("list_channel")[:] = np.array([list("U1\0\0\0\0"), list("U_NORM")], "S1")
    f.var("list_element_na")[:] = np.arange(10).reshape(2, 5)
    f.close()
    nc = netcdf_file(p, "r", mmap=False)
    assert np.array_equal(nc.variables["data_wave__NaG=3"].data, w)
    assert nc.variables["data_time"].data.tolist() == [0.5, 1.0, 1.5, 2.0, 2.5]
    assert nc.variables["list_element_na"].data.tolist() == np.arange(10).reshape(2, 5).tolist()
    assert nc.variables["data_wave__NaG=3"].dimensions[-1] == "dim_time"
    nc.close()


class _EngineStandIn:
    """What axg_set_element_record / axg_get_element_records return, computed on the CPU
    from the oracle's displacement at each step (gradient: the numpy computeGrad9)."""
    precision = "fp64"

    def __init__(self, model, fields):
        self.m, self.fields = model, fields

    def set_element_record(self, elem, gll, kind, interval, ring):
        self.entries = list(zip(elem, gll, kind))
        self.interval = interval
        return sum((int(self.m.se_nr[e]) // 2 + 1) * (9 if k else 3) for e, _, k in self.entries)

    def element_records(self, first, n):
        out = []
        for r in range(first, first + n):
            f = self.fields[r * self.interval]
            words, cache = [], {}
            for e, q, k in self.entries:
                if e not in cache:
                    cache[e] = _element_displ_grad(self.m, f, int(e))
                U, g = cache[e]
                words.append((g if k else U)[:, :, q // 5, q % 5].ravel())
            out.append(np.concatenate(words))
        return np.array(out)


def test_recorder_host_side_matches_restatement(built, tmp_path, monkeypatch):
    """The recorder's host side (entries, chunked drains through a 1-record ring, group
    steps and windows, frames, rows, channels, the NetCDF file) on records built from the
    oracle's fields, against the loop restatement of the GPU tests."""
    import oracle as O
    from axisem3d_b200 import preloop, simulation
    d = _box(str(tmp_path / "input"))
    _box_groups(d)
    sim = preloop.build(d, max_steps=30)
    o = O.Oracle(sim.model, "fp64")
    fields = {}
    for t in range(sim.nsteps):
        fields[t] = o.get_field("displ")
        o.run(1)
    o.close()
    eng = _EngineStandIn(sim.model, fields)
    monkeypatch.setattr(simulation.ElementRecorder, "RING_BYTES", 1)
    rec = simulation.ElementRecorder(eng, sim, str(tmp_path / "out"), np.float64)
    assert rec.interval == 1 and rec.ring == 1
    done = 0
    while done < sim.nsteps:
        done = min(sim.nsteps, done + rec.chunk_steps)
        rec.drain(done)
    rec.close()
    exp = _expected(sim)
    for g in sim.element_groups:
        path = os.path.join(str(tmp_path / "out"), "elements", g.name, "axisem3d_synthetics.nc.rank0")
        _check_group(g, path, exp[g.name], "fp64")
