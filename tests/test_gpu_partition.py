"""The boundary-stiffness exchange of a partitioned mesh on the GPU, through the C ABI.

Two ranks' sub-models live as two engine handles on one GPU, stepped in lockstep by one
process (no collective and no kernel waits on another: the host orders the launches). Between
the boundary conditions before and after assembly, each handle copies the stiffness of the
shared points into a device buffer (axg_gather_stiffness) and adds the other handle's buffer
(axg_scatter_add_stiffness): the data path of Messaging::commGatherSendRecv / commWaitScatter
(Messaging.hpp:26-47) with the transport left out. Against one handle holding the whole mesh:
FP64 <= 1e-12, mixed <= 1e-5 relative over every point mode (the sums run in another order).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "mixed": 1e-5}


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _model(name):
    from axisem3d_b200 import meshgen
    if name == "box_abc":
        return meshgen.cartesian_model(nx=12, nz=10, nr=5, absorbing=True), 150, None
    if name == "microbench_3d":
        m = meshgen.microbench_model(n_elem=400, nr_max=64, seed=9)
        return m, 10, meshgen.random_displacement(m, seed=4) * 1e-6
    return meshgen.spherical_model(n_theta=24, n_solid_layers=6, n_fluid_layers=2, nr_max=24), 60, None


def _global_slots(nr, points, ndim):
    nu = np.asarray(nr, np.int64) // 2 + 1
    first = np.concatenate([[0], np.cumsum(nu)[:-1]])
    return np.concatenate([first[p] * ndim + np.arange(nu[p] * ndim) for p in points])


def test_gather_and_scatter_add_match_numpy(built):
    import torch
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.microbench_model(n_elem=200, nr_max=32, seed=3)
    rng = np.random.default_rng(0)
    for precision in ("fp64", "mixed"):
        with Solver(m, precision) as s:
            f = meshgen.random_displacement(m, seed=8)
            s.set_field(f, "stiff")
            f = s.get_field("stiff")
            slots = np.sort(rng.choice(len(f), 500, replace=False)).astype(np.int64)
            dt = torch.complex128 if precision == "fp64" else torch.complex64
            sl = torch.from_numpy(slots).cuda()
            buf = torch.zeros(len(slots), dtype=dt, device="cuda")
            s.gather_stiffness(sl.data_ptr(), len(slots), buf.data_ptr())
            s.synchronize()
            assert np.allclose(buf.cpu().numpy(), f[slots], rtol=0, atol=0)
            add = torch.from_numpy((rng.normal(size=500) + 1j * rng.normal(size=500))).to(dt).cuda()
            s.scatter_add_stiffness(sl.data_ptr(), len(slots), add.data_ptr())
            g = s.get_field("stiff")
            want = f.copy()
            want[slots] += add.cpu().numpy()
            assert rel(g, want) <= (1e-15 if precision == "fp64" else 1e-7)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["box_abc", "microbench_3d", "shell_fluid"])
def test_two_subdomains_equal_one_domain(built, name, precision):
    import torch
    from axisem3d_b200 import partition as P
    from axisem3d_b200.solver import Solver
    m, nsteps, u0 = _model(name)
    se, fe = P.partition(m, 2)
    subs = [P.split(m, se, fe, r) for r in range(2)]
    plans = P.exchange_plan(m, se, fe, 2)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    solvers = [Solver(sub, precision) for sub in subs]
    try:
        if u0 is not None:
            for sub, s in zip(subs, solvers):
                s.set_field(u0[_global_slots(m.sp_nr, sub.meta["global"]["solid_points"], 3)], "displ")
        # device slots and buffers of every (rank, neighbour, medium)
        dev = {}
        for r in range(2):
            for other, (ss, fs) in plans[r].items():
                for solid, slots in ((True, ss), (False, fs)):
                    if len(slots):
                        dev[(r, other, solid)] = (torch.from_numpy(slots).cuda(),
                                                  torch.empty(len(slots), dtype=dt, device="cuda"))
        for t in range(nsteps):
            for s in solvers:
                s.apply_sources(t)
                s.compute_stiffness()
                s.apply_bc_before_assembly()
            for (r, other, solid), (sl, buf) in dev.items():
                solvers[r].gather_stiffness(sl.data_ptr(), len(sl), buf.data_ptr(), solid)
            for s in solvers:
                s.synchronize()
            for (r, other, solid), (sl, _) in dev.items():
                solvers[r].scatter_add_stiffness(sl.data_ptr(), len(sl), dev[(other, r, solid)][1].data_ptr(), solid)
            for s in solvers:
                s.synchronize()
                s.record_stations(t)
                s.apply_bc_after_assembly()
                s.stiff_to_accel()
                s.newmark_update()
        parts = [(sub.meta["global"], s.get_field("displ"),
                  s.get_field("displ", solid=False) if len(sub.fp_nr) else None)
                 for sub, s in zip(subs, solvers)]
    finally:
        for s in solvers:
            s.close()
    with Solver(m, precision) as s:
        if u0 is not None:
            s.set_field(u0, "displ")
        s.run(nsteps)
        ref = s.get_field("displ")
        ref_f = s.get_field("displ", solid=False) if len(m.fp_nr) else None
    got = np.zeros_like(ref)
    got_f = np.zeros_like(ref_f) if ref_f is not None else None
    for g, d, df in parts:
        got[_global_slots(m.sp_nr, g["solid_points"], 3)] = d
        if df is not None:
            got_f[_global_slots(m.fp_nr, g["fluid_points"], 1)] = df
    assert np.abs(ref).max() > 0
    assert rel(got, ref) <= TOL[precision], rel(got, ref)
    if ref_f is not None:
        assert rel(got_f, ref_f) <= TOL[precision], rel(got_f, ref_f)
