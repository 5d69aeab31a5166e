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


class _ThreadTransport:
    """The part of torch.distributed that PartitionedRun.exchange calls (P2POp, isend, irecv,
    batch_isend_irecv), for ranks that live as threads of one process on one GPU: a send
    waits for the sender's current stream and hands a copy of the buffer to the receiver
    through the host, a receive copies it into the buffer on the receiver's current stream.
    No kernel waits on another rank; the host orders everything."""

    def __init__(self, rank, box, cv, timeout=120.0):
        self.rank, self.box, self.cv, self.timeout = rank, box, cv, timeout
        self.isend, self.irecv = "isend", "irecv"

    @staticmethod
    def P2POp(op, tensor, peer):
        from types import SimpleNamespace
        return SimpleNamespace(op=op, tensor=tensor, peer=peer)

    def batch_isend_irecv(self, ops):
        import torch
        torch.cuda.current_stream().synchronize()
        with self.cv:
            for op in ops:
                if op.op == self.isend:
                    self.box.setdefault((self.rank, op.peer), []).append(op.tensor.cpu().clone())
            self.cv.notify_all()
        for op in ops:
            if op.op != self.irecv:
                continue
            key = (op.peer, self.rank)
            with self.cv:
                if not self.cv.wait_for(lambda: self.box.get(key), timeout=self.timeout):
                    raise TimeoutError("no message from rank %d" % op.peer)
                data = self.box[key].pop(0)
            op.tensor.copy_(data.to(op.tensor.device))

        class _Done:
            def wait(self):
                return True
        return [_Done()]


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("name", ["box_abc", "shell_fluid"])
def test_partitioned_run_device_path(built, name, overlap):
    """PartitionedRun's device path (the engine's gather / scatter-add on the run's own stream,
    buffers handed over by the transport between the boundary conditions before and after
    assembly) with two ranks as two threads of this process, against one handle holding the
    whole mesh: FP64 <= 1e-12. With overlap, the elements at shared points first, the transfer
    queued before the other elements (axg_compute_stiffness_part), the Clayton terms of shared
    points on every copy after the exchange. NCCL itself is not exercised (one GPU); the
    transport stands in for its point-to-point calls."""
    import threading
    import torch
    from axisem3d_b200 import partition as P
    from axisem3d_b200.solver import Solver
    m, nsteps, _ = _model(name)
    runs = [P.PartitionedRun(m, lambda sub: Solver(sub, "fp64"), rank=r, nparts=2, device="cuda",
                             overlap=overlap) for r in range(2)]
    if overlap:
        for run in runs:
            part = np.asarray(run.sub.se_part)
            assert 0 < int(part.sum()) < len(part)
    box, cv = {}, threading.Condition()
    for r, run in enumerate(runs):
        assert run.device_path
        run.dist = _ThreadTransport(r, box, cv)
    errors, parts = [None, None], [None, None]

    def rank_main(r):
        try:
            runs[r].run(nsteps)
            runs[r].stream.synchronize()
            sub, s = runs[r].sub, runs[r].solver
            parts[r] = (sub.meta["global"], s.get_field("displ"),
                        s.get_field("displ", solid=False) if len(sub.fp_nr) else None)
        except BaseException as exc:  # reported by the main thread
            errors[r] = exc

    try:
        threads = [threading.Thread(target=rank_main, args=(r,)) for r in range(2)]
        for t in threads:
            t.start()
        for t in threads:
            t.join(timeout=600)
        assert not any(t.is_alive() for t in threads), "rank thread did not finish"
        for e in errors:
            if e is not None:
                raise e
    finally:
        for run in runs:
            run.solver.close()
    with Solver(m, "fp64") as s:
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
    assert rel(got, ref) <= TOL["fp64"], rel(got, ref)
    if ref_f is not None:
        assert rel(got_f, ref_f) <= TOL["fp64"], rel(got_f, ref_f)
