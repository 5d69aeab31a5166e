"""Element partition of a mesh over ranks and the per-step boundary-stiffness exchange.

The reference runs one MPI rank per sub-mesh: the preloop partitions the elements (METIS,
weighted by nr or measured cost; LocalMesh.cpp), every rank builds the elements and GLL points
of its part, and points on a part boundary exist on each rank that touches them, with the
global mass (assembled over all ranks in the preloop). Once per step, between the boundary
conditions before assembly and those after it, the ranks sum the stiffness of their shared
points (NewmarkTimeScheme::solve, NewmarkTimeScheme.cpp:57-83 -> Domain::mpiGatherSendRecv /
mpiWaitScatter -> Messaging::commGatherSendRecv / commWaitScatter, Messaging.hpp:26-47 ->
MessageRank::gatherFromPoints / scatterToPoints, MessageRank.cpp:40-63, with
SolidPoint::feedComm / extractComm, SolidPoint.hpp:55-67). After that every copy of a shared
point holds the same stiffness and mass, so the point updates agree across ranks.

This module is the host side of that path for one process per GPU:

* ``partition``: recursive coordinate bisection of the element centroids, weighted by each
  element's cost 25 nu_e (the nr weighting of the reference's first partition); a stand-in for
  METIS that gives compact parts on the structured meshes here. Fluid elements, and solid
  elements that touch a solid-fluid point, all go to part 0, so that every coupling pair lives
  on one rank (the coupling mixes a point's own stiffness with the other medium's field).
* ``split``: one rank's sub-model (local point numbering, operand pools sliced, sources and
  stations of its elements, Clayton conditions on the lowest rank that holds their point:
  they add a velocity term to the stiffness before assembly, so one rank adds it).
* ``exchange_plan``: for each pair of ranks the shared points in global order, as complex
  slots of each side's stiffness field.
* ``PartitionedRun``: the step with the exchange between the two boundary-condition stages,
  over ``torch.distributed`` (NCCL between GPUs, gloo on CPU). Each rank's solver is the
  engine (``Solver``: device buffers, ``axg_gather_stiffness`` / ``axg_scatter_add_stiffness``)
  or any object with the same hooks and ``get_field`` / ``set_field`` (host buffers).

Models with PRT, ocean loads, 3-D absorbing boundaries, 3-D solid-fluid coupling, wavefield
scanning or batched wavefields are refused by ``split``.
"""
import copy

import numpy as np

_UNSUPPORTED = ("prt", "prt_fluid", "ocean_load", "ocean_load3d", "sf3", "cl3_solid", "cl3_fluid",
                "sponge3d_solid", "sponge3d_fluid", "scanning")


def _nmod(rheo):
    return {0: 2, 1: 5, 2: 21}[int(rheo)]


def _element_centroids(model):
    sc = np.asarray(model.sp_coords)[np.asarray(model.se_pts)].mean(axis=1)
    if model.n_fluid_elements:
        if model.fp_coords is not None:
            fc = np.asarray(model.fp_coords)[np.asarray(model.fe_pts)].mean(axis=1)
        else:
            fc = np.zeros((model.n_fluid_elements, 2))
    else:
        fc = np.zeros((0, 2))
    return sc, fc


def _rcb(xy, w, ids, nparts, first, out):
    """Recursive coordinate bisection: split `ids` along the longer extent at the weighted
    position that gives the lower half its share of the parts."""
    if nparts == 1 or len(ids) == 0:
        out[ids] = first
        return
    lo_parts = nparts // 2
    pts = xy[ids]
    ext = pts.max(axis=0) - pts.min(axis=0)
    axis = int(np.argmax(ext))
    order = ids[np.lexsort((ids, pts[:, axis]))]       # stable: ties by element id
    cw = np.cumsum(w[order])
    target = cw[-1] * lo_parts / nparts
    cut = int(np.searchsorted(cw, target, side="left")) + 1
    cut = min(max(cut, 1), len(order) - 1) if len(order) > 1 else len(order)
    _rcb(xy, w, order[:cut], lo_parts, first, out)
    _rcb(xy, w, order[cut:], nparts - lo_parts, first + lo_parts, out)


def partition(model, nparts):
    """Part of every solid and fluid element: (se_part, fe_part)."""
    ns, nf = model.n_solid_elements, model.n_fluid_elements
    se_part = np.zeros(ns, np.int32)
    fe_part = np.zeros(nf, np.int32)
    if nparts <= 1:
        return se_part, fe_part
    sc, _ = _element_centroids(model)
    w = 25.0 * (np.asarray(model.se_nr) // 2 + 1)
    pinned = np.zeros(ns, bool)
    if len(model.sf_solid):
        coupled = np.zeros(len(model.sp_nr), bool)
        coupled[np.asarray(model.sf_solid)] = True
        pinned = coupled[np.asarray(model.se_pts)].any(axis=1)
    free = np.nonzero(~pinned)[0]
    _rcb(sc, w, free, nparts, 0, se_part)
    se_part[pinned] = 0
    return se_part, fe_part


def _point_ranks(pts, part, npoints):
    """Sorted list of the ranks that hold each point."""
    holders = [set() for _ in range(npoints)]
    for e, row in enumerate(np.asarray(pts)):
        r = int(part[e])
        for p in row:
            holders[p].add(r)
    return [sorted(h) for h in holders]


def _slice_pool(pool, off, sizes, sel):
    parts, offs, o = [], [], 0
    for e in sel:
        n = int(sizes[e])
        parts.append(np.asarray(pool[int(off[e]):int(off[e]) + n]))
        offs.append(o)
        o += n
    return (np.concatenate(parts) if parts else np.zeros(0, np.asarray(pool).dtype)), np.array(offs, np.int64)


def split(model, se_part, fe_part, rank, overlap=False):
    """The sub-model of one rank, with the maps to the global numbering in `sub.meta['global']`
    (solid / fluid points, solid / fluid elements, stations).

    overlap: the sub-model of a rank that hides the exchange behind element work. Its elements
    carry parts (`se_part` / `fe_part`: 0 for the elements that touch a point another rank
    holds, 1 for the rest), and the Clayton conditions of a shared point sit on every copy,
    since they are then added after the exchange (each copy adds the whole term to the
    assembled sum) instead of once before it."""
    for key in _UNSUPPORTED:
        if getattr(model, key, None):
            raise NotImplementedError("partition.split || %s is not partitioned" % key)
    if int(getattr(model, "nwave", 1)) != 1:
        raise NotImplementedError("partition.split || batched wavefields are not partitioned")
    se = np.nonzero(np.asarray(se_part) == rank)[0]
    fe = np.nonzero(np.asarray(fe_part) == rank)[0]
    sub = copy.copy(model)
    sp_glob = np.unique(np.asarray(model.se_pts)[se]) if len(se) else np.zeros(0, np.int64)
    fp_glob = np.unique(np.asarray(model.fe_pts)[fe]) if len(fe) else np.zeros(0, np.int64)
    s_l = -np.ones(len(model.sp_nr), np.int64)
    s_l[sp_glob] = np.arange(len(sp_glob))
    f_l = -np.ones(len(model.fp_nr), np.int64)
    f_l[fp_glob] = np.arange(len(fp_glob))

    # points: global masses (assembled over every element), 1-D or per slice
    sub.sp_nr = np.asarray(model.sp_nr)[sp_glob].astype(np.int32)
    if model.sp_mass_nr is not None:
        sub.sp_mass_nr = np.asarray(model.sp_mass_nr)[sp_glob]
        sub.sp_mass, sub.sp_mass_off = _slice_pool(model.sp_mass, model.sp_mass_off, model.sp_mass_nr, sp_glob)
    else:
        sub.sp_mass = np.asarray(model.sp_mass)[sp_glob]
    for k in ("sp_axial", "sp_coords"):
        if getattr(model, k) is not None:
            setattr(sub, k, np.asarray(getattr(model, k))[sp_glob])
    sub.fp_nr = np.asarray(model.fp_nr)[fp_glob].astype(np.int32)
    if len(model.fp_nr):
        if model.fp_mass_nr is not None:
            sub.fp_mass_nr = np.asarray(model.fp_mass_nr)[fp_glob]
            sub.fp_mass, sub.fp_mass_off = _slice_pool(model.fp_mass, model.fp_mass_off, model.fp_mass_nr, fp_glob)
        else:
            sub.fp_mass = np.asarray(model.fp_mass)[fp_glob]
        for k in ("fp_axial", "fp_surface", "fp_coords"):
            if getattr(model, k) is not None:
                setattr(sub, k, np.asarray(getattr(model, k))[fp_glob])

    # solid elements and their operand pools
    nr = np.asarray(model.se_nr)
    nsl = np.where(np.asarray(model.se_is3d) != 0, nr, 1) if model.se_is3d is not None else np.ones_like(nr)
    sub.se_nr = nr[se]
    sub.se_pts = s_l[np.asarray(model.se_pts)[se]].astype(np.int32)
    for k in ("se_axial", "se_geom", "se_rheo", "se_is3d", "se_rtz", "se_theta", "se_att"):
        if getattr(model, k) is not None:
            setattr(sub, k, np.asarray(getattr(model, k))[se])
    msize = np.array([_nmod(r) for r in np.asarray(model.se_rheo)]) * nsl * 25
    sub.se_moduli, sub.se_mat_off = _slice_pool(model.se_moduli, model.se_mat_off, msize, se)
    if model.se_att is not None and model.se_att_moduli is not None:
        npa = np.where(np.asarray(model.se_att) == 2, 4, 25)
        asize = np.where(np.asarray(model.se_att) != 0, 2 * nsl * npa, 0)
        sub.se_att_moduli, sub.se_att_off = _slice_pool(model.se_att_moduli, model.se_att_off, asize, se)
    if getattr(model, "meta_rho", None) is not None:
        sub.meta_rho = np.asarray(model.meta_rho)[se]

    # fluid elements
    if model.n_fluid_elements:
        fnr = np.asarray(model.fe_nr)
        fnsl = np.where(np.asarray(model.fe_is3d) != 0, fnr, 1) if model.fe_is3d is not None else np.ones_like(fnr)
        sub.fe_nr = fnr[fe]
        sub.fe_pts = f_l[np.asarray(model.fe_pts)[fe]].astype(np.int32)
        for k in ("fe_axial", "fe_geom", "fe_is3d", "fe_theta"):
            if getattr(model, k) is not None:
                setattr(sub, k, np.asarray(getattr(model, k))[fe])
        sub.fe_moduli, sub.fe_mat_off = _slice_pool(model.fe_moduli, model.fe_mat_off, fnsl * 25, fe)

    # solid-fluid coupling pairs whose two points are both here (all of them on part 0)
    if len(model.sf_solid):
        keep = (s_l[np.asarray(model.sf_solid)] >= 0) & (f_l[np.asarray(model.sf_fluid)] >= 0)
        sub.sf_solid = s_l[np.asarray(model.sf_solid)[keep]].astype(np.int32)
        sub.sf_fluid = f_l[np.asarray(model.sf_fluid)[keep]].astype(np.int32)
        for k in ("sf_nsu", "sf_nzu", "sf_nsa", "sf_nza", "sf_mass_fluid"):
            setattr(sub, k, np.asarray(getattr(model, k))[keep])

    # sources on this rank's elements
    e_l = -np.ones(model.n_solid_elements, np.int64)
    e_l[se] = np.arange(len(se))
    fe_l = -np.ones(model.n_fluid_elements, np.int64)
    fe_l[fe] = np.arange(len(fe))
    for pre, emap in (("ms", e_l), ("fs", e_l), ("ps", fe_l)):
        elem = np.asarray(getattr(model, pre + "_elem"))
        if not len(elem):
            continue
        keep = np.nonzero(emap[elem] >= 0)[0]
        nu = np.asarray(getattr(model, pre + "_nu"))
        pat = np.asarray(getattr(model, pre + "_pattern"))
        off = np.asarray(getattr(model, pre + "_pat_off"))
        width = 150 if pre == "ms" else (75 if pre == "fs" else 25)
        pats, offs, o = [], [], 0
        for i in keep:
            n = int(nu[i]) * width
            pats.append(pat[int(off[i]):int(off[i]) + n])
            offs.append(o)
            o += n
        setattr(sub, pre + "_elem", emap[elem[keep]].astype(np.int32))
        setattr(sub, pre + "_nu", nu[keep].astype(np.int32))
        setattr(sub, pre + "_pat_off", np.array(offs, np.int64))
        setattr(sub, pre + "_pattern", np.concatenate(pats) if pats else np.zeros(0, np.complex128))
        setattr(sub, pre + "_stf", [getattr(model, pre + "_stf")[i] for i in keep])
        setattr(sub, pre + "_wave", None)

    # stations on this rank's elements
    st_keep = np.zeros(0, np.int64)
    if len(model.st_elem):
        st_keep = np.nonzero(e_l[np.asarray(model.st_elem)] >= 0)[0]
        sub.st_elem = e_l[np.asarray(model.st_elem)[st_keep]].astype(np.int32)
        sub.st_w = np.asarray(model.st_w)[st_keep]
        sub.st_phi = np.asarray(model.st_phi)[st_keep]

    # Clayton conditions: on the lowest rank that holds the point; sponges on every copy
    sranks = _point_ranks(model.se_pts, se_part, len(model.sp_nr))
    franks = _point_ranks(model.fe_pts, fe_part, len(model.fp_nr)) if len(model.fp_nr) else []
    for key, lmap, holders in (("cl_solid", s_l, sranks), ("cl_fluid", f_l, franks)):
        cl = getattr(model, key)
        if cl:
            pt = np.asarray(cl["point"])
            keep = np.array([lmap[p] >= 0 and (overlap or holders[p][0] == rank) for p in pt], bool)
            d = {k: np.asarray(v)[keep] for k, v in cl.items()}
            d["point"] = lmap[pt[keep]].astype(np.int32)
            setattr(sub, key, d if len(d["point"]) else None)
    for key, lmap in (("sponge_solid", s_l), ("sponge_fluid", f_l)):
        sg = getattr(model, key)
        if sg is not None:
            pt, g = np.asarray(sg[0]), np.asarray(sg[1])
            keep = lmap[pt] >= 0
            setattr(sub, key, (lmap[pt[keep]].astype(np.int32), g[keep]) if np.any(keep) else None)

    if overlap:
        shared_s = np.array([len(h) > 1 for h in sranks], bool)
        sub.se_part = np.where(shared_s[np.asarray(model.se_pts)[se]].any(axis=1), 0, 1).astype(np.uint8) \
            if len(se) else np.zeros(0, np.uint8)
        if model.n_fluid_elements:
            shared_f = np.array([len(h) > 1 for h in franks], bool)
            sub.fe_part = np.where(shared_f[np.asarray(model.fe_pts)[fe]].any(axis=1), 0, 1).astype(np.uint8) \
                if len(fe) else np.zeros(0, np.uint8)
    sub.meta = dict(model.meta, rank=int(rank),
                    **{"global": {"solid_points": sp_glob, "fluid_points": fp_glob, "solid_elements": se,
                                  "fluid_elements": fe, "stations": st_keep}})
    return sub


def _field_slots(nr, points, ndim):
    """Complex slots of the given local points in a [sum nu][ndim] field."""
    nu = np.asarray(nr, np.int64) // 2 + 1
    first = np.concatenate([[0], np.cumsum(nu)[:-1]])
    out = []
    for p in points:
        base = first[p] * ndim
        out.append(base + np.arange(nu[p] * ndim, dtype=np.int64))
    return np.concatenate(out) if out else np.zeros(0, np.int64)


def exchange_plan(model, se_part, fe_part, nparts):
    """For each rank: {other rank: (solid slots, fluid slots)}, the slots of the points both
    hold, in global point order on both sides (so the two buffers line up)."""
    plans = [dict() for _ in range(nparts)]
    locs = []
    for r in range(nparts):
        se = np.nonzero(np.asarray(se_part) == r)[0]
        fe = np.nonzero(np.asarray(fe_part) == r)[0]
        sp = np.unique(np.asarray(model.se_pts)[se]) if len(se) else np.zeros(0, np.int64)
        fp = np.unique(np.asarray(model.fe_pts)[fe]) if len(fe) else np.zeros(0, np.int64)
        locs.append((sp, fp))
    for a in range(nparts):
        for b in range(nparts):
            if a == b:
                continue
            sa, fa = locs[a]
            sb, fb = locs[b]
            ss = np.intersect1d(sa, sb)
            ff = np.intersect1d(fa, fb)
            if not len(ss) and not len(ff):
                continue
            s_slots = _field_slots(np.asarray(model.sp_nr)[sa], np.searchsorted(sa, ss), 3)
            f_slots = _field_slots(np.asarray(model.fp_nr)[fa], np.searchsorted(fa, ff), 1) if len(ff) else \
                np.zeros(0, np.int64)
            plans[a][b] = (s_slots, f_slots)
    return plans


class PartitionedRun:
    """One rank's share of a partitioned run: the rank's sub-model, its solver and the
    exchange with the neighbours, over an initialised torch.distributed process group.

    make_solver(sub_model) -> solver with the hooks apply_sources, compute_stiffness,
    apply_bc_before_assembly, record_stations, apply_bc_after_assembly, stiff_to_accel,
    newmark_update, and get_field / set_field; with gather_stiffness / scatter_add_stiffness
    (the engine) the buffers stay on the device."""

    def __init__(self, model, make_solver, rank=None, nparts=None, device=None, overlap=False):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.rank = dist.get_rank() if rank is None else rank
        self.nparts = dist.get_world_size() if nparts is None else nparts
        self.se_part, self.fe_part = partition(model, self.nparts)
        self.overlap = bool(overlap)
        self.sub = split(model, self.se_part, self.fe_part, self.rank, overlap=self.overlap)
        self._nr_global = (np.asarray(model.sp_nr), np.asarray(model.fp_nr))
        self.plan = exchange_plan(model, self.se_part, self.fe_part, self.nparts)[self.rank]
        self.solver = make_solver(self.sub)
        self.device_path = hasattr(self.solver, "gather_stiffness") and device is not None
        if self.overlap and not hasattr(self.solver, "compute_stiffness_part"):
            raise ValueError("PartitionedRun || overlap needs a solver with compute_stiffness_part")
        self.device = device
        self.torch = torch
        self._dev = {}
        if self.device_path:
            # The engine's hooks, its gather / scatter-add and the NCCL send / receive are
            # ordered on one stream of this run's own: ProcessGroupNCCL makes its stream wait on
            # the current torch stream when an operation is queued, and req.wait() makes the
            # current stream wait on it, so the exchange runs with that stream current and the
            # handle launches on it (the engine's own stream does not synchronise with others).
            self.stream = torch.cuda.Stream(device=device)
            if hasattr(self.solver, "set_stream"):
                self.solver.set_stream(self.stream.cuda_stream)
            cdt = torch.complex128 if self.solver.precision == "fp64" else torch.complex64
            for other, (ss, fs) in self.plan.items():
                ent = []
                for solid, slots in ((True, ss), (False, fs)):
                    sl = torch.from_numpy(np.ascontiguousarray(slots)).to(device)
                    ent.append((solid, sl, torch.empty(len(slots), dtype=cdt, device=device),
                                torch.empty(len(slots), dtype=cdt, device=device)))
                self._dev[other] = ent

    def exchange(self):
        """Domain::mpiGatherSendRecv + mpiWaitScatter: send this rank's stiffness at the shared
        points to each neighbour, receive theirs and add it."""
        dist, torch = self.dist, self.torch
        ops, recv = [], []
        if self.device_path:
            with torch.cuda.stream(self.stream):
                self._exchange_finish(*self._exchange_start())
            return
        fields = {}
        for solid in (True, False):
            if (solid and len(self.sub.sp_nr)) or (not solid and len(self.sub.fp_nr)):
                fields[solid] = self.solver.get_field("stiff", solid=solid)
        for other in sorted(self.plan):
            ss, fs = self.plan[other]
            for solid, slots in ((True, ss), (False, fs)):
                if not len(slots):
                    continue
                send = torch.view_as_real(torch.from_numpy(np.ascontiguousarray(fields[solid][slots])))
                rbuf = torch.zeros_like(send)
                ops.append(dist.P2POp(dist.isend, send, other))
                ops.append(dist.P2POp(dist.irecv, rbuf, other))
                recv.append((solid, slots, rbuf))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for solid, slots, rbuf in recv:
            fields[solid][slots] += torch.view_as_complex(rbuf).numpy()
        for solid, f in fields.items():
            self.solver.set_field(f, "stiff", solid=solid)

    def _exchange_start(self):
        """Gather the shared points' stiffness and queue the transfers (device path, with the
        run's stream current); returns what _exchange_finish waits on and adds."""
        dist, torch = self.dist, self.torch
        ops, recv = [], []
        for other in sorted(self.plan):
            for solid, sl, sbuf, rbuf in self._dev[other]:
                if len(sl) == 0:
                    continue
                self.solver.gather_stiffness(sl.data_ptr(), len(sl), sbuf.data_ptr(), solid)
                ops.append(dist.P2POp(dist.isend, torch.view_as_real(sbuf), other))
                ops.append(dist.P2POp(dist.irecv, torch.view_as_real(rbuf), other))
                recv.append((solid, sl, rbuf))
        reqs = dist.batch_isend_irecv(ops) if ops else []
        return reqs, recv

    def _host_exchange_start(self):
        """Host path: send the shared points' stiffness as it stands, post the receives."""
        dist, torch = self.dist, self.torch
        ops, recv = [], []
        for solid in (True, False):
            if not ((solid and len(self.sub.sp_nr)) or (not solid and len(self.sub.fp_nr))):
                continue
            f = self.solver.get_field("stiff", solid=solid)
            for other in sorted(self.plan):
                slots = self.plan[other][0 if solid else 1]
                if not len(slots):
                    continue
                send = torch.view_as_real(torch.from_numpy(np.ascontiguousarray(f[slots])))
                rbuf = torch.zeros_like(send)
                ops.append(dist.P2POp(dist.isend, send, other))
                ops.append(dist.P2POp(dist.irecv, rbuf, other))
                recv.append((solid, slots, rbuf))
        reqs = dist.batch_isend_irecv(ops) if ops else []
        return reqs, recv

    def _host_exchange_finish(self, reqs, recv):
        for req in reqs:
            req.wait()
        fields = {}
        for solid, slots, rbuf in recv:
            if solid not in fields:
                fields[solid] = self.solver.get_field("stiff", solid=solid)
            fields[solid][slots] += self.torch.view_as_complex(rbuf).numpy()
        for solid, f in fields.items():
            self.solver.set_field(f, "stiff", solid=solid)

    def _exchange_finish(self, reqs, recv):
        for req in reqs:
            req.wait()
        for solid, sl, rbuf in recv:
            self.solver.scatter_add_stiffness(sl.data_ptr(), len(sl), rbuf.data_ptr(), solid)

    def step(self, tstep):
        """One Newmark step in the order of NewmarkTimeScheme::solve. With overlap, the
        elements that touch a shared point go first, the transfers run while the others
        compute, and the boundary conditions before assembly follow the exchange (the
        solid-fluid pairs live on one rank; the Clayton terms of shared points are on every
        copy)."""
        s = self.solver
        if self.overlap and not self.device_path:
            # host transport: the shared points' values after part 0 travel while part 1
            # (which touches none of them) computes
            s.apply_sources(tstep)
            s.compute_stiffness_part(0)
            pending = self._host_exchange_start()
            s.compute_stiffness_part(1)
            self._host_exchange_finish(*pending)
            s.apply_bc_before_assembly()
            s.record_stations(tstep)
            s.apply_bc_after_assembly()
            s.stiff_to_accel()
            s.newmark_update()
            return
        if self.overlap:
            with self.torch.cuda.stream(self.stream):
                s.apply_sources(tstep)
                s.compute_stiffness_part(0)
                pending = self._exchange_start()
                s.compute_stiffness_part(1)
                self._exchange_finish(*pending)
                s.apply_bc_before_assembly()
            s.record_stations(tstep)
            s.apply_bc_after_assembly()
            s.stiff_to_accel()
            s.newmark_update()
            return
        s.apply_sources(tstep)
        s.compute_stiffness()
        s.apply_bc_before_assembly()
        self.exchange()
        s.record_stations(tstep)
        s.apply_bc_after_assembly()
        s.stiff_to_accel()
        s.newmark_update()

    def run(self, nsteps, first=0):
        for t in range(first, first + nsteps):
            self.step(t)

    def set_global_field(self, values, which="displ", solid=True):
        """Set a field given on the whole mesh ([sum nu][ndim] in the global point order) on
        this rank's points."""
        m = self.sub
        glob = m.meta["global"]["solid_points" if solid else "fluid_points"]
        nr_g = np.asarray(self._nr_global[0 if solid else 1])
        ndim = 3 if solid else 1
        slots = _field_slots(nr_g, glob, ndim)
        self.solver.set_field(np.asarray(values).ravel()[slots], which, solid=solid)

    def gather_field(self, which="displ", solid=True):
        """The whole mesh's field on every rank (for checks): each rank's points in the global
        numbering, shared points taken from the lowest rank."""
        dist, torch = self.dist, self.torch
        m = self.sub
        glob = m.meta["global"]["solid_points" if solid else "fluid_points"]
        nr_l = np.asarray(m.sp_nr if solid else m.fp_nr)
        ndim = 3 if solid else 1
        f = np.asarray(self.solver.get_field(which, solid=solid)).reshape(-1, ndim) if len(nr_l) else \
            np.zeros((0, ndim), np.complex128)
        payload = [(glob, nr_l, f)]
        out = [None] * self.nparts
        dist.all_gather_object(out, payload)
        pieces = {}
        for r in range(self.nparts):
            g, nrs, ff = out[r][0]
            nu = nrs // 2 + 1
            first = np.concatenate([[0], np.cumsum(nu)[:-1]]).astype(np.int64)
            for i, p in enumerate(g):
                if int(p) not in pieces:
                    pieces[int(p)] = ff[first[i]:first[i] + nu[i]]
        return pieces
