"""Partitioned meshes on the CPU: the element partition, the sub-models, the exchange plan,
and whole partitioned runs over gloo (world size 2 and 3) with the oracle as each rank's
solver, against the single-domain run of the same model.

A partitioned run sums the stiffness of the points that ranks share once per step between
the boundary conditions before and after assembly (Messaging::commGatherSendRecv /
commWaitScatter, NewmarkTimeScheme.cpp:57-83). Every copy of a point then updates with the same
stiffness and mass, so the fields equal the single-domain run up to the order of the sums:
FP64 <= 1e-12 relative over every point mode.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _model(name):
    from axisem3d_b200 import meshgen
    if name == "box_abc":
        # axis, moment source on the axis, stations, Clayton edges (corner points with two
        # conditions) and a sponge layer
        m = meshgen.cartesian_model(nx=12, nz=10, nr=5, absorbing=True)
        return m
    if name == "microbench_3d":
        m = meshgen.microbench_model(n_elem=300, nr_max=24, seed=9)
        m.st_elem = np.zeros(0, np.int32)
        return m
    if name == "shell_fluid":
        return meshgen.spherical_model(n_theta=24, n_solid_layers=6, n_fluid_layers=2, nr_max=24)
    raise KeyError(name)


def test_partition_covers_balances_and_pins_coupling():
    from axisem3d_b200 import meshgen, partition as P
    m = meshgen.microbench_model(n_elem=4000, nr_max=64, seed=3)
    for nparts in (2, 3, 4, 8):
        se, fe = P.partition(m, nparts)
        assert set(np.unique(se)) == set(range(nparts))
        w = 25.0 * (m.se_nr // 2 + 1)
        loads = np.array([w[se == r].sum() for r in range(nparts)])
        assert loads.max() / loads.mean() < 1.05, loads
    sh = meshgen.spherical_model(n_theta=24, n_solid_layers=6, n_fluid_layers=2, nr_max=24)
    se, fe = P.partition(sh, 3)
    assert np.all(fe == 0)
    coupled = np.zeros(len(sh.sp_nr), bool)
    coupled[sh.sf_solid] = True
    assert np.all(se[coupled[sh.se_pts].any(axis=1)] == 0)


@pytest.mark.parametrize("name", ["box_abc", "shell_fluid"])
def test_split_assigns_everything_once(name):
    from axisem3d_b200 import partition as P
    m = _model(name)
    nparts = 3
    se, fe = P.partition(m, nparts)
    subs = [P.split(m, se, fe, r) for r in range(nparts)]
    assert sum(s.n_solid_elements for s in subs) == m.n_solid_elements
    assert sum(s.n_fluid_elements for s in subs) == m.n_fluid_elements
    assert sum(len(s.ms_elem) for s in subs) == len(m.ms_elem)
    assert sum(len(s.st_elem) for s in subs) == len(m.st_elem)
    if m.cl_solid:
        assert sum(len(s.cl_solid["point"]) if s.cl_solid else 0 for s in subs) == len(m.cl_solid["point"])
    # each sub-model's elements reference its own points, with the global masses
    for s in subs:
        g = s.meta["global"]["solid_points"]
        assert s.se_pts.max() < len(s.sp_nr)
        assert np.array_equal(s.sp_mass, m.sp_mass[g])
        assert np.array_equal(s.se_geom, m.se_geom[s.meta["global"]["solid_elements"]])
    # both sides of every shared boundary list the same number of slots
    plans = P.exchange_plan(m, se, fe, nparts)
    for a in range(nparts):
        for b, (ss, fs) in plans[a].items():
            assert len(plans[b][a][0]) == len(ss) and len(plans[b][a][1]) == len(fs)
            assert len(ss) % 3 == 0 and len(ss) > 0


def _rank_main(rank, world, port, name, nsteps, q, overlap=False):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]
    import torch.distributed as dist
    import oracle as O
    from axisem3d_b200 import partition as P
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = _model(name)
        run = P.PartitionedRun(m, lambda sub: O.Oracle(sub, "fp64"), overlap=overlap)
        if name == "microbench_3d":
            from axisem3d_b200 import meshgen
            run.set_global_field(meshgen.random_displacement(m, seed=4) * 1e-6, "displ")
        run.run(nsteps)
        solid = run.gather_field("displ", True)
        fluid = run.gather_field("displ", False) if len(m.fp_nr) else {}
        seis = run.solver.seismograms()
        q.put((rank, solid if rank == 0 else None, fluid if rank == 0 else None,
               run.sub.meta["global"]["stations"], seis))
    finally:
        dist.destroy_process_group()


def _whole(field, nr, ndim):
    nu = np.asarray(nr) // 2 + 1
    first = np.concatenate([[0], np.cumsum(nu)[:-1]])
    f = np.asarray(field).reshape(-1, ndim)
    return {p: f[first[p]:first[p] + nu[p]] for p in range(len(nr))}


@pytest.mark.parametrize("name,world,nsteps,overlap", [("box_abc", 2, 150, False), ("microbench_3d", 3, 20, False),
                                                       ("shell_fluid", 2, 60, False), ("box_abc", 2, 150, True),
                                                       ("microbench_3d", 3, 20, True), ("shell_fluid", 2, 60, True)])
def test_partitioned_run_equals_single_domain(built, name, world, nsteps, overlap):
    """gloo ranks, the oracle as every rank's solver, against one oracle holding the whole mesh
    (FP64 <= 1e-12). overlap: the elements at shared points first, the transfers posted before
    the others compute, the boundary conditions before assembly after the exchange (Clayton
    terms of shared points on every copy)."""
    import torch.multiprocessing as mp
    import oracle as O
    m = _model(name)
    if name == "microbench_3d":
        from axisem3d_b200 import meshgen
        u0 = meshgen.random_displacement(m, seed=4) * 1e-6
    o = O.Oracle(m, "fp64")
    if name == "microbench_3d":
        o.set_field(u0, "displ")
    o.run(nsteps)
    ref_s = _whole(o.get_field("displ"), m.sp_nr, 3)
    ref_f = _whole(o.get_field("displ", solid=False), m.fp_nr, 1) if len(m.fp_nr) else {}
    ref_seis = o.seismograms()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, name, nsteps, q, overlap)) for r in range(world)]
    for p in ps:
        p.start()
    out = [q.get(timeout=600) for _ in ps]
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    r0 = [x for x in out if x[0] == 0][0]
    solid, fluid = r0[1], r0[2]
    assert sorted(solid) == list(range(len(m.sp_nr)))
    a = np.concatenate([solid[p] for p in range(len(m.sp_nr))])
    b = np.concatenate([ref_s[p] for p in range(len(m.sp_nr))])
    assert np.abs(b).max() > 0
    assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-12
    if ref_f:
        af = np.concatenate([fluid[p] for p in range(len(m.fp_nr))])
        bf = np.concatenate([ref_f[p] for p in range(len(m.fp_nr))])
        assert np.linalg.norm(af - bf) / np.linalg.norm(bf) <= 1e-12
    # each station is recorded by the rank that holds its element
    if len(m.st_elem):
        got = np.zeros_like(ref_seis)
        for rank, _, _, st, seis in out:
            if len(st):
                got[:, st, :] = seis
        assert np.linalg.norm(got - ref_seis) / np.linalg.norm(ref_seis) <= 1e-12


def test_overlap_split_parts_and_clayton_copies():
    """split(overlap=True): part 0 = the elements touching a point another rank holds, part 1
    = the rest; the Clayton conditions of shared points on every copy (added after the
    exchange), the others unchanged."""
    from axisem3d_b200 import partition as P
    m = _model("box_abc")
    se, fe = P.partition(m, 2)
    holders = P._point_ranks(m.se_pts, se, len(m.sp_nr))
    plain = [P.split(m, se, fe, r) for r in range(2)]
    over = [P.split(m, se, fe, r, overlap=True) for r in range(2)]
    ncl_plain = ncl_over = 0
    for r in range(2):
        g = over[r].meta["global"]
        pts = np.asarray(m.se_pts)[g["solid_elements"]]
        shared = np.array([[len(holders[p]) > 1 for p in row] for row in pts])
        assert np.array_equal(np.asarray(over[r].se_part), np.where(shared.any(axis=1), 0, 1))
        ncl_plain += len(plain[r].cl_solid["point"]) if plain[r].cl_solid else 0
        ncl_over += len(over[r].cl_solid["point"]) if over[r].cl_solid else 0
        assert plain[r].se_part is None
    pt = np.asarray(m.cl_solid["point"])
    nshared = sum(len(holders[p]) - 1 for p in pt)
    assert nshared > 0
    assert ncl_plain == len(pt) and ncl_over == len(pt) + nshared
