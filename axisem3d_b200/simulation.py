"""A whole simulation from the reference's inputs: preloop, time loop on the GPU, station
files. This is the path of the reference's `main` (SOLVER/src/main.cpp): the inputs
(inparam.*.yaml and the Exodus mesh they name) go through `preloop.build`, the Newmark loop
runs in the engine (one CUDA graph per step), and each station group is written in its
format (`output.write_group`).

    from axisem3d_b200 import simulation
    res = simulation.run("input", "output", precision="fp32")
"""
from __future__ import annotations

import os
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import output, preloop
from .solver import Solver


@dataclass
class Result:
    sim: "preloop.Simulation"
    traces: dict = field(default_factory=dict)     # group -> (times, [station, channel, time])
    seconds_preloop: float = 0.0
    seconds_loop: float = 0.0
    seconds_element_output: float = 0.0
    element_files: dict = field(default_factory=dict)   # element group -> file (None: no element)
    element_data: dict = field(default_factory=dict)    # element group -> [(times, per element)]


class ElementRecorder:
    """The element groups of one run (ElementOpGroup::record / dumpToFile, core/output/
    element-wise/element/ElementOpGroup.hpp:197-236): the engine keeps the Fourier
    coefficients of every group's points in a device ring (axg_set_element_record, one
    interval for all groups, the gcd of theirs); after each chunk of steps that fills the ring
    at most once, the host takes the chunk's records, keeps each group's own steps and time
    window, forms its channels and writes them to the group's file."""

    RING_BYTES = 256 << 20

    def __init__(self, solver, sim, out_dir, wave_dtype):
        self.s, self.sim = solver, sim
        self.groups = [g for g in sim.element_groups]
        nr = np.asarray(sim.model.se_nr, np.int64)
        elem, gll, kind = [], [], []
        self.layout = []            # per group: {kind: [element, point] entry numbers}
        for g in self.groups:
            need = {c[0] for c in g.channels}
            d = {}
            for kd, on in ((0, "U" in need), (1, bool(need & set("GER")))):
                if not on or len(g.elems) == 0:
                    continue
                idx = np.arange(len(elem), len(elem) + len(g.elems) * g.npnts).reshape(len(g.elems), g.npnts)
                elem += np.repeat(g.elems, g.npnts).tolist()
                gll += g.ipnts.ravel().tolist()
                kind += [kd] * (len(g.elems) * g.npnts)
                d[kd] = idx
            self.layout.append(d)
        elem, kind = np.array(elem, np.int64), np.array(kind, np.int64)
        width = (nr[elem] // 2 + 1) * np.where(kind == 1, 9, 3) if len(elem) else np.zeros(0, np.int64)
        self.off = np.concatenate([[0], np.cumsum(width)[:-1]]).astype(np.int64) if len(elem) else width
        words = int(width.sum())
        self.interval = int(np.gcd.reduce([g.interval for g in self.groups])) if self.groups else 1
        self.interval = max(1, min(self.interval, sim.nsteps))
        total = (sim.nsteps + self.interval - 1) // self.interval
        per = max(1, words) * max(1, int(sim.model.nwave)) * (16 if solver.precision == "fp64" else 8)
        self.ring = int(max(1, min(total, self.RING_BYTES // per)))
        self.active = len(elem) > 0
        if self.active:
            w = solver.set_element_record(elem, gll, kind, self.interval, self.ring)
            assert w == words
        self.chunk_steps = self.ring * self.interval
        self.next_rec = 0
        self.writers = [output.ElementGroupWriter(out_dir, g, wave_dtype) if out_dir is not None else None
                        for g in self.groups]
        self.data = [[] for _ in self.groups]      # kept when no output directory is given

    def _coeffs(self, recs, g, idx, D):
        """[element][record, point, order, D] complex coefficients of one kind."""
        out = []
        for k, e in enumerate(g.elems):
            nu = int(g.nr[k]) // 2 + 1
            cols = self.off[idx[k]][:, None] + np.arange(nu * D)[None, :]       # [point, nu * D]
            out.append(recs[:, cols].reshape(len(recs), g.npnts, nu, D))
        return out

    def drain(self, step):
        """Take the records of steps below `step` that are not taken yet."""
        if not self.active:
            return
        last = (step - 1) // self.interval
        if last < self.next_rec:
            return
        recs = self.s.element_records(self.next_rec, last - self.next_rec + 1)
        if recs.ndim == 3:
            recs = recs[:, 0]
        rec_ids = np.arange(self.next_rec, last + 1)
        self.next_rec = last + 1
        sim = self.sim
        for gi, g in enumerate(self.groups):
            if len(g.elems) == 0:
                continue
            steps = rec_ids * self.interval
            t = sim.t0 + steps * sim.dt
            keep = (steps % g.interval == 0) & (t >= g.tmin) & (t <= g.tmax)
            if not keep.any():
                continue
            r = recs[keep]
            need = {c[0] for c in g.channels}
            lay = self.layout[gi]
            us = self._coeffs(r, g, lay[0], 3) if 0 in lay else None
            gs = self._coeffs(r, g, lay[1], 9) if 1 in lay else None
            per_elem = []
            for k in range(len(g.elems)):
                th = np.broadcast_to(g.theta[k], (len(r), g.npnts)).reshape(-1)
                u = us[k].reshape(-1, *us[k].shape[2:]) if us is not None else None
                gg = gs[k].reshape(-1, *gs[k].shape[2:]) if gs is not None else None
                f = output.element_fields(u, gg, need, g.frame, th, sim.cartesian)
                rows = {key: output.fourier_rows(v, int(g.na[k]), g.phis).reshape(len(r), g.npnts, -1, v.shape[-1])
                        for key, v in f.items()}
                ch = output.element_channels(rows, g.channels)                  # [rec, point, na, channel]
                per_elem.append(np.transpose(ch, (2, 1, 3, 0)))                 # [na, point, channel, rec]
            if self.writers[gi] is not None:
                self.writers[gi].write(t[keep], per_elem)
            else:
                self.data[gi].append((t[keep], per_elem))

    def close(self):
        for w in self.writers:
            if w is not None:
                w.close()


def write_scanning(path, model, solid_nr, fluid_nr):
    """Domain::reportScanning (Domain.cpp:495-569): the scanned points' (s, z), their scanned
    Nr and their Nr during the run, solid points then fluid points; the file a later run
    reads as a POINTWISE Nr field."""
    from scipy.io import netcdf_file
    rows = []
    for nr_scan, nr0, crd in ((solid_nr, model.sp_nr, model.sp_coords), (fluid_nr, model.fp_nr, None)):
        for p in np.nonzero(np.asarray(nr_scan) != -1)[0]:
            c = crd[p] if crd is not None else model.fp_coords[p]
            rows.append((c[0], c[1], int(nr_scan[p]), int(nr0[p])))
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    nc = netcdf_file(path, "w", version=2)
    nc.createDimension("dim_point", len(rows))
    nc.createDimension("dim_sz", 2)
    v = nc.createVariable("pointwise_sz", "d", ("dim_point", "dim_sz"))
    v[:] = np.array([[r[0], r[1]] for r in rows]).reshape(-1, 2)
    v = nc.createVariable("pointwise_Nr", "i", ("dim_point",))
    v[:] = np.array([r[2] for r in rows], np.int32)
    v = nc.createVariable("starting_Nr_for_scanning", "i", ("dim_point",))
    v[:] = np.array([r[3] for r in rows], np.int32)
    nc.close()


def run(input_dir: str, output_dir: Optional[str] = None, precision: str = "fp32",
        max_steps: Optional[int] = None, device: int = 0, skip_unsupported_channels: bool = False,
        stability_interval: Optional[int] = None) -> Result:
    """Run one simulation; write the station groups under output_dir when it is given."""
    t = time.perf_counter()
    sim = preloop.build(input_dir, max_steps=max_steps, skip_unsupported_channels=skip_unsupported_channels)
    res = Result(sim=sim, seconds_preloop=time.perf_counter() - t)
    if stability_interval is None:
        stability_interval = sim.info["stability_interval"]
    wave_precision = 16 if precision == "fp64" else 8
    with Solver(sim.model, precision, device=device, stability_interval=stability_interval) as s:
        rec = None
        if sim.element_groups:
            rec = ElementRecorder(s, sim, output_dir, np.float64 if precision == "fp64" else np.float32)
        t = time.perf_counter()
        if rec is None or not rec.active:
            s.run(sim.nsteps)
            s.synchronize()
        else:
            done = 0
            while done < sim.nsteps:
                n = min(rec.chunk_steps, sim.nsteps - done)
                s.run(n)
                done += n
                t1 = time.perf_counter()
                rec.drain(done)
                res.seconds_element_output += time.perf_counter() - t1
        res.seconds_loop = time.perf_counter() - t - res.seconds_element_output
        if rec is not None:
            rec.close()
            for g, w in zip(rec.groups, rec.writers):
                res.element_files[g.name] = (os.path.join(output_dir, "elements", g.name, "axisem3d_synthetics.nc.rank0")
                                             if w is not None and len(g.elems) else None)
            res.element_data = {g.name: d for g, d in zip(rec.groups, rec.data)}
        seis = s.seismograms() if len(sim.model.st_elem) else np.zeros((0, 0, 3))
        scan = s.scanning_nr() if sim.model.scanning else None
        grad = s.station_gradients() if sim.model.st_gradient and len(sim.model.st_elem) else None
    if scan is not None and output_dir is not None and sim.info.get("scanning_file"):
        write_scanning(os.path.join(output_dir, sim.info["scanning_file"]), sim.model, *scan)
    for g in sim.groups:
        steps, rows = output.group_records(g, sim.nsteps, sim.t0, sim.dt, sim.model.st_interval)
        sl = slice(g.first, g.first + len(g.keys))
        u = np.transpose(seis[rows][:, sl, :], (1, 0, 2))          # [station, time, 3]
        gs = np.transpose(grad[rows][:, sl, :], (1, 0, 2)) if grad is not None else None
        data = output.group_channels(u, gs, g.channels, g.frame, g.theta, g.baz, g.phi, sim.cartesian)
        times = sim.t0 + steps * sim.dt
        res.traces[g.name] = (times, data)
        if output_dir is not None:
            output.write_group(output_dir, g, times, data, wave_precision)
    return res
