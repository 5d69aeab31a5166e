"""Benchmark: GLL-point x mode updates per second of the full time step.

Workload (stiffness microbenchmark, uneven batching): ~200k non-axial solid
quads with nPol = 4, per-element nr log-uniform on [1, 64], transversely
isotropic moduli at +-10 % around vp = 8, vs = 4.5 km/s, rho = 3.3 g/cc per
(element, slice, point) -- the 3-D (slice) path -- with 3 SLS attenuation
memory variables (Q_mu uniform in [80, 600]). Seeded synthetic data.

One step = the whole Newmark step on every element and point: fused solid
stiffness (gather, gradient, phi transform, TI stress, SLS attenuation,
inverse transform, quadrature, scatter-add), then boundary conditions, 1/M and
the Newmark update. Updates per step = sum_e 25 nu_e (nu = nr/2 + 1).

  value  device-timed with CUDA events on the engine's stream, state resident in
         HBM, one CUDA graph per step; inputs larger than L2 (the step streams
         ~20 GB)
  e2e    the same steps through the C ABI with the displacement field copied
         host -> device from pinned memory before every step and the updated
         displacement copied back after it (axg_set_field_raw / axg_run /
         axg_get_field_raw)
  roofline  the solid stiffness kernels: algorithmic bytes per evaluation /
         measured duration, against the measured HBM copy bandwidth
  cpu_baseline  the C++ CPU restatement (oracle, FP32 like the reference's
         default build) on all host cores: full steps of the whole workload,
         built with the oracle's own operands, as many as fit the time bound

--impl reference times the same restatement on the same workload and config
(W warm-up and K timed full steps, a stated prefix of them if K steps would
run over five minutes).

Run with N GPUs (torchrun): every rank advances its own replica of the
workload (weak scaling, no exchange); value = all ranks' updates / max time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GLL-pt*mode updates/s"
UNIT = "updates/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="mixed", choices=["mixed", "fp32", "fp64"])
    p.add_argument("--elements", type=int, default=200000)
    p.add_argument("--nr-max", type=int, default=64)
    p.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison runs")
    p.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward timing")
    p.add_argument("--adjoint-steps", type=int, default=4000)
    p.add_argument("--ensemble", type=int, default=64, help="sources of the ensemble leg (0 = skip)")
    p.add_argument("--no-oned", action="store_true", help="skip the 1-D (in-Fourier) leg")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--shell-steps", type=int, default=100,
                   help="steps of the spherical-shell leg in each precision (0 = skip; the full run is 5000)")
    p.add_argument("--shell-theta", type=int, default=1200, help="quads along theta of the shell leg")
    return p.parse_args()


# ----------------------------------------------------------------- helpers ---
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def dist_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), float(f[3]), f[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        load = [r for r in rows if r[2] > 250.0] or rows
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in load:
            for n, v in zip(names, r[3]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(r[0] for r in load), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": sorted(reasons), "samples": len(load)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """dram bytes per stiffness evaluation from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "stiffness_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def build_model(args, seed=1, builder=None):
    """The workload, built with the engine's operand builder or with `builder` (the oracle's
    own restatement, so that the CPU legs map no library of the engine)."""
    import contextlib
    from axisem3d_b200 import meshgen
    with (meshgen.operands(builder) if builder is not None else contextlib.nullcontext()):
        return meshgen.microbench_model(n_elem=args.elements, nr_max=args.nr_max, seed=seed)


def oracle_workload(args, seed=1):
    """The oracle module and the workload built through the oracle's operands."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O, build_model(args, seed, O.OracleOperands())


def workload_config(args, m):
    """The workload's description; the same dictionary on both arms."""
    return {"workload": "stiffness microbenchmark, uneven nr: %d solid quads nPol=4, nr log-uniform "
                        "[1,%d], TI 3-D slices, 3 SLS FULL, full Newmark step" % (m.n_solid_elements, args.nr_max),
            "elements": int(m.n_solid_elements), "updates_per_step": int(m.updates_per_step()),
            "l2": "inputs larger than L2 (the step streams >10 GB)"}


# --------------------------------------------------------------- CPU legs ---
def cpu_timed_steps(o, steps):
    t0 = time.perf_counter()
    o.run(steps)
    return time.perf_counter() - t0


def cpu_baseline(args, seconds):
    """The oracle (FP32, the reference's default precision) on all host cores, on the full
    workload built through the oracle's own operands: one untimed step, then whole steps
    for about `seconds`."""
    from axisem3d_b200 import meshgen
    O, m = oracle_workload(args, seed=1)
    cores = os.cpu_count() or 1
    o = O.Oracle(m, "fp32", threads=cores)
    o.set_field(meshgen.random_displacement(m, seed=2) * 1e-6, "displ")
    t1 = cpu_timed_steps(o, 1)
    steps = max(1, min(20, int(seconds / max(t1, 1e-3))))
    dt = cpu_timed_steps(o, steps)
    U = m.updates_per_step()
    return {"value": U * steps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "%d full steps of the whole %d-element workload in %.1f s (FP32 oracle, model built "
                      "with the oracle's operands)" % (steps, m.n_solid_elements, dt)}


# --------------------------------------------------------------------- arms ---
def run_reference(args, world, rank):
    """The reference's CPU path (the oracle port: the reference cannot be built here) on the
    whole workload, FP32 like the reference's default build, all host threads: W untimed
    steps, then K timed steps (a prefix of them, stated in `sample`, should K steps take
    longer than about five minutes)."""
    if rank != 0:
        return
    from axisem3d_b200 import meshgen
    O, m = oracle_workload(args, seed=1)
    cores = os.cpu_count() or 1
    o = O.Oracle(m, "fp32", threads=cores)
    o.set_field(meshgen.random_displacement(m, seed=2) * 1e-6, "displ")
    tw = cpu_timed_steps(o, max(1, args.warmup))
    per = tw / max(1, args.warmup)
    steps = max(1, args.steps)
    timed = max(1, min(steps, int(300.0 / max(per, 1e-3))))
    t = cpu_timed_steps(o, timed)
    U = m.updates_per_step()
    v = U * timed / t
    sample = ("%d of %d full steps of the whole %d-element workload in %.1f s after %d warm-up steps "
              "(FP32 oracle port on %d threads, model built with the oracle's operands)"
              % (timed, steps, m.n_solid_elements, t, max(1, args.warmup), cores))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": t / timed * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args, m),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def time_steps(solver, steps, stream, graph=True):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    solver.run(steps, graph=graph)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3


def log(msg):
    sys.stderr.write("[bench %.1fs] %s\n" % (time.time() - T_START, msg))
    sys.stderr.flush()


T_START = time.time()


def run_ours(args, world, rank, local):
    import torch
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    log("building model")
    m = build_model(args, seed=1 + rank)
    U = m.updates_per_step()
    log("model: %d elements, %d updates/step" % (m.n_solid_elements, U))
    s = Solver(m, args.precision, device=local)
    log("solver finalized")
    s.set_stream(stream.cuda_stream)
    u0 = meshgen.random_displacement(m, seed=2 + rank) * 1e-6
    s.set_field(u0, "displ")
    clocks = ClockSampler(local)
    with clocks:
        log("warmup")
        s.run(max(3, args.warmup), graph=True)
        s.synchronize()
        log("timed run")
        barrier(world)
        torch.cuda.synchronize()
        n0 = s.launch_count()
        t = time_steps(s, args.steps, stream)
        launches = s.launch_count() - n0
        t = dist_max(t, world)
        log("stiffness timing")
        # stiffness kernels alone: per-step events around the solid stiffness launches
        s.set_timing(True)
        s.run(5, graph=False)
        kms, kn = s.stiffness_time()
        s.set_timing(False)
        log("e2e")
        # end to end through the C ABI with host buffers
        nb = s.field_raw_bytes("displ")
        host = torch.empty(nb, dtype=torch.uint8, pin_memory=True)
        s.get_field_raw(host.data_ptr(), nb, "displ")
        torch.cuda.synchronize()
        ke = max(3, min(args.steps, 10))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier(world)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        e0.record(stream)
        for _ in range(ke):
            s.set_field_raw(host.data_ptr(), nb, "displ")
            s.run(1, graph=True)
            s.get_field_raw(host.data_ptr(), nb, "displ")
        e1.record(stream)
        torch.cuda.synchronize()
        te = max(e0.elapsed_time(e1) / 1e3, time.perf_counter() - w0)
        te = dist_max(te, world)
    bytes_, flops = s.stiffness_cost()
    pbytes = s.point_cost()
    s.close()
    value = U * args.steps * world / t
    out = {"value": value, "t": t, "launches": launches, "kms": kms / max(kn, 1), "bytes": bytes_,
           "flops": flops, "pbytes": pbytes, "U": U, "e2e": U * ke * world / te, "e2e_bytes": nb,
           "clocks": clocks.summary(), "model": m}
    # FP64 runs of the same workload: the plain method (one team per element, one
    # launch per kernel, no graph) and the fused batched path in FP64
    if not args.no_fp64 and args.precision != "fp64":
        for key, kw in (("value_fp64_plain", dict(plain=True)), ("value_fp64", {})):
            log("fp64 run " + key)
            s64 = Solver(m, "fp64", device=local, **kw)
            s64.set_stream(stream.cuda_stream)
            s64.set_field(u0, "displ")
            s64.run(2, graph=not kw)
            k64 = max(3, args.steps // 5)
            t64 = dist_max(time_steps(s64, k64, stream, graph=not kw), world)
            out[key] = U * k64 * world / t64
            s64.close()
        log("trace error")
        out["trace"] = trace_error(args, local)
    if not args.no_adjoint:
        log("adjoint")
        out["adjoint"] = adjoint_timing(args, local, stream, world)
    if args.ensemble > 0:
        log("ensemble")
        out["ensemble"] = ensemble_timing(args, local, stream, world)
    if not args.no_oned:
        log("1-D leg")
        out["oned"] = oned_timing(args, local, stream, world)
    if not args.no_fp64 and args.precision != "fp32":
        log("fp32 run")
        with Solver(m, "fp32", device=local) as s32:
            s32.set_stream(stream.cuda_stream)
            s32.set_field(u0, "displ")
            s32.run(3)
            t32 = dist_max(time_steps(s32, max(3, args.steps // 2), stream), world)
            out["value_fp32"] = U * max(3, args.steps // 2) * world / t32
    if args.shell_steps > 0:
        log("shell leg")
        out["shell"] = shell_timing(args, local, stream, world)
    return out


def shell_timing(args, local, stream, world):
    """Spherical-shell workload: a half annulus r 3480-6371 km of --shell-theta x 250 quads
    (10 fluid layers 3480-3600 km, FluidElement, then 240 solid layers), spherical mapping, a
    seeded piecewise-linear 1-D background with a 2 % Gaussian random field dlnVs (200 km
    correlation) sampled on every element's slices, per-element nr from the field's azimuthal
    bandwidth in [3, 128], CG4 attenuation with Q_mu = 300, a moment tensor with a Ricker
    wavelet of 20 s period, 20 surface stations. From rest, --shell-steps steps in the bench
    precision and in FP64: updates/s of each (the first 3 steps, which capture the step graph,
    untimed), the solid stiffness kernels against the HBM roofline, and the seismograms of the
    bench precision against FP64 (relative L2)."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.spherical_model(n_theta=args.shell_theta, n_solid_layers=240, n_fluid_layers=10)
    U = m.updates_per_step()
    n = max(4, args.shell_steps)
    peak, kind = measured_peaks()
    out = {"workload": "spherical shell %d solid + %d fluid quads, nr %d..%d (mean %.1f) from the dlnVs field, "
                       "iso 3-D slices, CG4 Q=300, Ricker 20 s, %d steps from rest"
                       % (m.n_solid_elements, len(m.fe_nr), int(m.se_nr.min()), int(m.se_nr.max()),
                          float(np.mean(m.se_nr)), n),
           "updates_per_step": int(U), "dt": m.dt}
    seis = {}
    for prec in (args.precision, "fp64"):
        with Solver(m, prec, device=local) as s:
            s.set_stream(stream.cuda_stream)
            s.run(3)
            t = dist_max(time_steps(s, n - 3, stream), world)
            seis[prec] = s.seismograms()
            out["value_" + prec] = U * (n - 3) * world / t
            out["ms_per_step_" + prec] = t / (n - 3) * 1e3
            if prec == args.precision:
                s.set_timing(True)
                s.run(3, graph=False)
                kms, kn = s.stiffness_time()
                s.set_timing(False)
                b, _ = s.stiffness_cost()
                kms /= max(kn, 1)
                out["stiffness_ms"] = kms
                out["stiffness_GBps"] = b / (kms / 1e3) / 1e9
                out["stiffness_frac_of_" + kind + "_hbm"] = out["stiffness_GBps"] / peak
        log("shell %s done" % prec)
    ref = seis["fp64"]
    if n >= 2000:
        out["trace_rel_l2_vs_fp64"] = float(np.linalg.norm(seis[args.precision] - ref) / np.linalg.norm(ref))
    else:
        # before ~2000 steps the waves have not reached the stations: both precisions record
        # values at the underflow level, and their difference says nothing
        out["trace_rel_l2_vs_fp64"] = None
        out["trace_note"] = "seismograms are compared on the full run (--shell-steps 5000)"
    out[args.precision + "_over_fp64"] = out["value_" + args.precision] / out["value_fp64"]
    return out


def oned_timing(args, local, stream, world):
    """The same microbenchmark with per-(element, point) moduli: every element takes the 1-D
    path (stress and SLS attenuation in Fourier space, no phi transforms), in the bench
    precision; step rate and the stiffness kernels against the HBM roofline."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.microbench_model(n_elem=args.elements, nr_max=args.nr_max, seed=5, is3d=False)
    U = m.updates_per_step()
    k = max(10, args.steps)
    with Solver(m, args.precision, device=local) as s:
        s.set_stream(stream.cuda_stream)
        s.set_field(meshgen.random_displacement(m, seed=6) * 1e-6, "displ")
        s.run(3)
        t = dist_max(time_steps(s, k, stream), world)
        s.set_timing(True)
        s.run(5, graph=False)
        kms, kn = s.stiffness_time()
        s.set_timing(False)
        b, _ = s.stiffness_cost()
    kms = kms / max(kn, 1)
    peak, kind = measured_peaks()
    gbs = b / (kms / 1e3) / 1e9
    return {"workload": "stiffness microbenchmark, 1-D moduli (Fourier-space path): %d quads, nr "
                        "log-uniform [1,%d], TI, 3 SLS FULL" % (m.n_solid_elements, args.nr_max),
            "updates_per_step": int(U), "value": U * k * world / t, "ms_per_step": t / k * 1e3,
            "stiffness_ms": kms, "stiffness_bytes": b, "stiffness_GBps": gbs,
            "stiffness_frac_of_" + kind + "_hbm": gbs / peak}


def ensemble_timing(args, local, stream, world):
    """Batched ensemble: `--ensemble` moment-tensor sources (Ricker, periods 10-40 s) with
    full 21-Cij on a spherical-shell mesh (8000 solid + 400 fluid quads, r 3480-6371 km,
    fluid 3480-3600 km, nr 3..100 from a 2 % dlnVs random field, elastic, RTZ frame),
    all advanced as one wavefield batch per launch, one CUDA graph per step, autotuned
    team sizes, in the bench precision; against the plain FP64 method (one bucket per
    material kind, eager launches) advancing one of the sources on the same mesh."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    base = meshgen.spherical_model(n_theta=200, n_solid_layers=40, n_fluid_layers=2, rheology="aniso",
                                   attenuation=None)
    ens = meshgen.ensemble_model(base, nsrc=args.ensemble, seed=21)
    U = base.updates_per_step()
    k = 20
    with Solver(ens, args.precision, device=local, autotune=True) as s:
        s.set_stream(stream.cuda_stream)
        s.run(3)
        t_b = dist_max(time_steps(s, k, stream), world)
    with Solver(meshgen.single_source(ens, 0), "fp64", device=local, plain=True) as s1:
        s1.set_stream(stream.cuda_stream)
        s1.run(3, graph=False)
        t_p = dist_max(time_steps(s1, k, stream, graph=False), world)
    vb = ens.nwave * U * k * world / t_b
    vp = U * k * world / t_p
    return {"workload": "spherical shell 8000+400 quads, 21-Cij RTZ, nr 3..100, %d sources"
                        % ens.nwave, "updates_per_step_per_source": int(U),
            "value_batched": vb, "ms_per_step_batched": t_b / k * 1e3,
            "value_fp64_plain_one_source": vp, "ms_per_step_fp64_plain": t_p / k * 1e3,
            "batched_over_fp64_plain": vb / vp}


def trace_error(args, local):
    """Seismograms of the plain forward case (40 x 40 quads, nr = 5, 2000 steps) in the
    bench precision against the FP64 engine: relative L2 over all traces."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = meshgen.cartesian_model(nx=40, nz=40, nr=5)
    seis = {}
    for prec in (args.precision, "fp64"):
        with Solver(m, prec, device=local) as s:
            s.run(2000)
            seis[prec] = s.seismograms()
    ref = seis["fp64"]
    return {"workload": "cartesian 40x40 quads, nr=5, 20 stations, 2000 steps",
            "rel_l2": float(np.linalg.norm(seis[args.precision] - ref) / np.linalg.norm(ref))}


def adjoint_timing(args, local, stream, world):
    """Adjoint sensitivity workload: 200 x 200 quads, uniform nr = 9, 5 % Gaussian blob in
    mu and rho, 50 surface receivers, checkpoint every 100 steps. Ratio = time of the
    adjoint sweep (recompute from checkpoints + time-reversed adjoint steps) over the time
    of a plain forward solve of the same steps, both in FP64 (the adjoint's precision)."""
    import torch
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    base = meshgen.cartesian_model(nx=200, nz=200, nr=9, nstations=50, nr_aware_dt=True)
    m = meshgen.blob_model(base, amp=0.05, seed=3)
    n = args.adjoint_steps

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return r, max(e0.elapsed_time(e1) / 1e3, time.perf_counter() - w0)

    # the adjoint is an FP64 path: forward and adjoint are both timed in FP64
    with Solver(m, "fp64", device=local) as f:
        f.set_stream(stream.cuda_stream)
        _, t_fwd = timed(lambda: (f.run(n), f.synchronize()))
    with Solver(m, "fp64", device=local) as s:
        s.set_stream(stream.cuda_stream)
        _, t_ck = timed(lambda: (s.forward_checkpointed(n, 100), s.synchronize()))
        seis = s.seismograms()
        _, t_adj = timed(lambda: s.adjoint(seis))
    t_fwd, t_ck, t_adj = (dist_max(x, world) for x in (t_fwd, t_ck, t_adj))
    return {"workload": "cartesian 200x200 quads, nr=9, mu/rho blob, 50 receivers, %d steps, "
                        "checkpoint every 100" % n,
            "forward_s": t_fwd, "forward_checkpointed_s": t_ck, "adjoint_s": t_adj,
            "adjoint_over_forward": t_adj / t_fwd}


def main():
    import faulthandler
    faulthandler.enable()
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    r = run_ours(args, world, rank, local)
    if rank == 0:
        m = r["model"]
        peak, peak_kind = measured_peaks()
        achieved = r["bytes"] / (r["kms"] / 1e3) / 1e9
        trafficd = profiled_traffic()
        traffic = None
        if trafficd and trafficd.get("elements") == m.n_solid_elements:
            traffic = trafficd.get("dram_bytes_per_launch_group")
        log("cpu baseline")
        cb = cpu_baseline(args, args.cpu_seconds)
        line = {
            "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["t"] / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"mixed": "f32 (f64 Newmark d/v and SLS state)", "fp32": "f32", "fp64": "f64"}[args.precision],
            "data": "synthetic", "config": workload_config(args, m),
            "precision": args.precision, "graph": "one CUDA graph per step",
            "gpu_launches": int(r["launches"]),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "solid stiffness (fused), %.3f ms per evaluation, %.2f GB algorithmic"
                                   % (r["kms"], r["bytes"] / 1e9),
                         "peak_kind": peak_kind + " HBM copy bandwidth"},
            "cpu_baseline": cb,
            "e2e": {"value": r["e2e"], "unit": UNIT, "h2d_bytes_per_step": int(r["e2e_bytes"]),
                    "d2h_bytes_per_step": int(r["e2e_bytes"])},
            "clocks": r["clocks"],
            "stiffness_flops_per_step": r["flops"],
            "point_update_bytes_per_step": r["pbytes"],
        }
        if "value_fp64" in r:
            line["value_fp64_plain"] = r["value_fp64_plain"]
            line["value_fp64"] = r["value_fp64"]
            line["fp32_over_fp64_plain"] = r["value"] / r["value_fp64_plain"]
            line["fp32_over_fp64"] = r["value"] / r["value_fp64"]
            line["trace"] = r["trace"]
        if "adjoint" in r:
            line["adjoint"] = r["adjoint"]
        if "ensemble" in r:
            line["ensemble"] = r["ensemble"]
        if "oned" in r:
            line["oned"] = r["oned"]
        if "value_fp32" in r:
            line["value_fp32"] = r["value_fp32"]
            if "value_fp64_plain" in r:
                line["fp32_only_over_fp64_plain"] = r["value_fp32"] / r["value_fp64_plain"]
        if "shell" in r:
            line["shell"] = r["shell"]
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
