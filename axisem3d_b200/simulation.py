"""A whole simulation from the reference's inputs: preloop, time loop on the GPU, station
files. This is the path of the reference's `main` (SOLVER/src/main.cpp): the inputs
(inparam.*.yaml and the Exodus mesh they name) go through `preloop.build`, the Newmark loop
runs in the engine (one CUDA graph per step), and each station group is written in its
format (`output.write_group`).

    from axisem3d_b200 import simulation
    res = simulation.run("input", "output", precision="fp32")
"""
from __future__ import annotations

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
        grad = s.station_gradients() if sim.model.st_gradient and len(sim.model.st_elem) else None
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
