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
    with Solver(sim.model, precision, device=device, stability_interval=stability_interval) as s:
        t = time.perf_counter()
        s.run(sim.nsteps)
        s.synchronize()
        res.seconds_loop = time.perf_counter() - t
        seis = s.seismograms() if len(sim.model.st_elem) else np.zeros((0, 0, 3))
        scan = s.scanning_nr() if sim.model.scanning else None
        grad = s.station_gradients() if sim.model.st_gradient and len(sim.model.st_elem) else None
    if scan is not None and output_dir is not None and sim.info.get("scanning_file"):
        write_scanning(os.path.join(output_dir, sim.info["scanning_file"]), sim.model, *scan)
    wave_precision = 16 if precision == "fp64" else 8
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
