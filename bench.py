"""Benchmark of the PDP3 per-timestep PIC loop on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|fp32]
                    [--workload wake|thermal|large|ensemble|adjoint|diag]

Workload (default): the beam-plasma wake case, 256 x 2048 cells over
r in [0, 0.1] m, z in [0, 0.8] m, electrons and protons at 64 macroparticles
per cell and 1e17 m^-3 (67,108,864 plasma particles), 1 eV electrons, a
gamma = 5 electron bunch (r 5 mm, length 2 cm, 5e16 m^-3, 64 macroparticles
per bunch cell) injected at z = 0, 10-cell absorbing layer, Courant 0.5,
relativistic Boris.  Seeded synthetic inputs (no dataset is involved).

A "step" is one full pass of the loop body: bunch injection, H update, J
clear, push + deposition of every species, E update.  value is
particle-steps/s (alive macroparticles x steps / s) over all ranks, with the
state resident in HBM, of the FP32 cell-local form (int cell + FP32 offsets
and momenta, FP64 grids); the FP64 plain form runs the same workload beside
it, and both report the Gauss-law residual and energies after the run
("forms").  Multi-GPU runs are independent replicas (the path
does not shard: no collective in the data path).  Particle arrays (~3 GB)
are far larger than L2, so no L2 flush is needed between steps.

--impl reference times the upstream OpenMP CPU step (oracle/_ref, the
unmodified upstream sources) on a bounded sample of the same workload.

--workload diag times the upstream's diagnostics and initial-field solve
through their C-ABI calls (charge density, temperature, density, a full
probe frame on the wake case; the Dirichlet Poisson solve on a 257 x 2047
grid) beside the upstream CPU code, one JSON line with one entry per call.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "particle-steps/s & cell-updates/s: FP32 vs FP64 GPU form at fixed Gauss error"
UNIT = "particle-steps/s"
BYTES_PER_PARTICLE = {"fp64": 88, "fp32": 52}
# Yee E + H update per node: H reads E 3 + H 3, writes H 3 + H_half 3 (96 B);
# E reads E 3 + H 3 + J 3 + sigma, writes E 3 (104 B); the FP32 form also
# writes the FP32 copies of E and the half-step H (24 B)
BYTES_PER_NODE = {"fp64": 200, "fp32": 224}
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return dict(PEAKS_FALLBACK), "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_workload(name, seed, ppc=None):
    from pdp3_b200 import workloads as W
    if name == "wake":
        return W.wake_config(seed=seed, steps=1000, ppc=ppc or 64)
    if name == "thermal":
        return W.thermal_config(seed=seed, steps=200, ppc=ppc or 32)
    if name == "large":
        return W.large_config(ppc=ppc or 64)
    raise ValueError(name)


def plasma_species_count(wl):
    return len(wl.species) + (2 if wl.device_plasma is not None else 0)


def species_bytes(sim, wl, precision):
    """Algorithmic bytes of one pass of the particle phase."""
    b = BYTES_PER_PARTICLE[precision]
    total = 0
    for sid in range(plasma_species_count(wl)):
        total += sim.species_size(sid) * b
    if wl.beam is not None:
        n_b = wl.beam.number_macro * wl.beam.number_bunches
        total += n_b * 2  # alive flag read (every slot) and written
    return total


def alive_count(sim, wl):
    n_pl = plasma_species_count(wl)
    n = sum(sim.species_size(sid) for sid in range(n_pl))
    for sid in range(n_pl, n_pl + (wl.beam.number_bunches if wl.beam is not None else 0)):
        n += int(sim.species(sid)["alive"].sum())
    return n


# ------------------------------------------------------------ CPU reference


def cpu_sample_run(wl, steps, warmup, fraction, threads):
    """Times the upstream CPU step (oracle/_ref) or, if it is not built, the
    oracle restatement, on the workload's grid with `fraction` of its plasma
    particles (a seeded subset) and the full bunch.  Returns (rate, kind,
    cores, sample text)."""
    from oracle import refsim
    rng = np.random.default_rng(12345)
    sub = []
    species = wl.species
    if wl.device_plasma is not None:
        # plasma generated on the GPU: the sample is the same grid and density
        # profile at round(ppc * fraction) particles per cell, built on the host
        from pdp3_b200 import workloads as W
        dp = wl.device_plasma
        k_ppc = max(1, int(round(dp.ppc * fraction)))
        fraction = k_ppc / dp.ppc
        dens = ((lambda zc: dp.n_max * np.minimum(zc / dp.z_ramp, 1.0)) if dp.z_ramp > 0
                else (lambda zc: np.full_like(zc, dp.n_max)))
        species = W.thermal_plasma(np.random.default_rng(dp.seed), dp.r_size, dp.z_size,
                                   dp.n_grid_r, dp.n_grid_z, k_ppc, dens, dp.t_ev, dp.ion_mass_me)
        sub = [(s, np.arange(s.n)) for s in species]
    for s in ([] if sub else species):
        k = max(1, int(s.n * fraction))
        idx = np.sort(rng.choice(s.n, size=k, replace=False))
        sub.append((s, idx))
    if refsim.available(wl.pusher if wl.pusher != "boris_classic" else "boris"):
        kind = "reference"
        sim = refsim.RefSim(wl.r_size, wl.z_size, wl.n_grid_r, wl.n_grid_z, wl.dt, end_time=1.0,
                            pml=wl.pml, pusher=wl.pusher)
        sim.L.ref_set_threads(threads)
        for s, idx in sub:
            sim.add_species(s.name, s.charge_e, s.mass_me, s.r[idx], s.z[idx], s.vr[idx],
                            s.vphi[idx], s.vz[idx], s.w[idx])
        if wl.beam is not None:
            b = wl.beam
            sim.set_beam(b.charge_e, b.mass_me, b.number_macro, b.bunch_length, b.radius,
                         b.density, b.velocity, b.number_bunches, b.bunches_distance)
        if warmup:
            sim.run(warmup)
        secs = sim.run(steps)
        n_alive = sum(len(idx) for _, idx in sub)
        if wl.beam is not None:
            for sid in range(len(sub), sim.n_species()):
                n_alive += int(sim.species(sid)["alive"].sum())
    else:
        kind = "port"
        from oracle.oracle import OracleSim
        os.environ["OMP_NUM_THREADS"] = str(threads)
        sim = OracleSim(wl.r_size, wl.z_size, wl.n_grid_r, wl.n_grid_z, wl.dt, pml=wl.pml,
                        pusher=wl.pusher)
        for s, idx in sub:
            sim.add_species(s.charge_e, s.mass_me, s.r[idx], s.z[idx], s.vr[idx], s.vphi[idx],
                            s.vz[idx], s.w[idx])
        if wl.beam is not None:
            b = wl.beam
            sim.add_bunch(b.charge_e, b.mass_me, b.number_macro, b.bunch_length / b.velocity,
                          b.radius, b.density, b.velocity, 0, b.bunches_distance / b.velocity)
        sim.run(warmup)
        t0 = time.perf_counter()
        sim.run(steps)
        secs = time.perf_counter() - t0
        n_alive = sum(len(idx) for _, idx in sub)
    rate = n_alive * steps / secs
    sample = ("%s grid (%dx%d nodes), %.4g of the plasma particles (%d) + bunch, %d steps "
              "after %d warm-up, %d OpenMP threads" % (wl.name, wl.n_grid_r, wl.n_grid_z,
                                                       fraction, sum(len(i) for _, i in sub),
                                                       steps, warmup, threads))
    return rate, kind, threads, sample, secs


def cpu_baseline(wl, steps, fraction, one_thread_fraction):
    """The upstream CPU step on all host cores, plus a 1-thread figure on a
    smaller sample of the same workload (the upstream sets its OpenMP thread
    count to all cores itself, src/loadInitParam.cpp:25-29)."""
    threads = os.cpu_count() or 1
    rate, kind, cores, sample, _ = cpu_sample_run(wl, steps, 1, fraction, threads)
    out = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
    if threads > 1 and one_thread_fraction > 0:
        r1, _, _, s1, _ = cpu_sample_run(wl, max(1, min(steps, 2)), 1, one_thread_fraction, 1)
        out["one_thread"] = {"value": r1, "unit": UNIT, "cores": 1, "sample": s1}
        out["threads_speedup"] = rate / r1
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    wl = make_workload(args.workload, 1002, args.ppc)
    threads = os.cpu_count() or 1
    fraction = args.cpu_fraction
    steps = max(1, args.steps)
    rate, kind, cores, sample, secs = cpu_sample_run(wl, steps, args.warmup, fraction, threads)
    one = None
    if threads > 1 and args.cpu_one_thread_fraction > 0:
        r1, _, _, s1, _ = cpu_sample_run(wl, 2, 1, args.cpu_one_thread_fraction, 1)
        one = {"value": r1, "unit": UNIT, "cores": 1, "sample": s1}
    line = {
        "metric": METRIC, "value": rate, "unit": UNIT, "impl": "reference", "n_gpus": 0,
        "steps": steps, "warmup": args.warmup, "ms_per_step": 1000.0 * secs / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": wl.name, "n_grid_r": wl.n_grid_r, "n_grid_z": wl.n_grid_z,
                   "particles": wl.n_particles, "pusher": wl.pusher, "sample": sample},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": sample, "one_thread": one},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------ GPU run


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32"],
                    help="the form reported as value (the other is measured beside it)")
    ap.add_argument("--workload", default="wake",
                    choices=["wake", "thermal", "large", "ensemble", "adjoint", "diag"])
    ap.add_argument("--adjoint-scale", type=int, default=1,
                    help="--workload adjoint: divide the grid's cells in r and z by this "
                         "(1: the 128x1024 case)")
    ap.add_argument("--adjoint-steps", type=int, default=500)
    ap.add_argument("--adjoint-interval", type=int, default=50)
    ap.add_argument("--adjoint-fd-params", default="near",
                    help="parameters checked by finite differences in --workload adjoint: "
                         "'near' (the 4 density bumps nearest the probe, gamma, radius), "
                         "'all', or 'none'")
    ap.add_argument("--ensemble-runs", type=int, default=64)
    ap.add_argument("--ensemble-scale", type=int, default=1,
                    help="divide every ensemble run's grid by this (smaller runs)")
    ap.add_argument("--ppc", type=int, default=None,
                    help="macroparticles per cell (profiling runs on a smaller case)")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="untimed FP32-vs-FP64 run of this many steps after the timing "
                         "(0: skip)")
    ap.add_argument("--cpu-fraction", type=float, default=1.0 / 32)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--cpu-one-thread-fraction", type=float, default=1.0 / 256,
                    help="plasma fraction of the 1-thread CPU figure (0: skip it)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "diag":
        return run_diag(args, rank, world)
    if args.workload in ("ensemble", "adjoint"):
        import torch
        dist = None
        if world > 1:
            import datetime
            import torch.distributed as dist
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local_rank))
        fn = run_ensemble if args.workload == "ensemble" else run_adjoint
        rc = fn(args, rank, world, local_rank, dist)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return rc

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    from pdp3_b200 import api

    assert args.warmup >= 3, "at least 3 warm-up steps"
    wl = make_workload(args.workload, 1002, args.ppc)
    clocks = ClockSampler(local_rank)

    def measure(precision, sample_clocks):
        """W warm-up + K timed steps of one form; timing with CUDA events on
        the library's stream, max over ranks."""
        sim = api.from_workload(wl, precision=precision, device=local_rank)
        sim.mark_initial_charge()
        stream = torch.cuda.ExternalStream(sim.stream_ptr,
                                           device=torch.device("cuda", local_rank))
        sim.step(args.warmup)
        sim.sync()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        alive0 = alive_count(sim, wl)
        sim.reset_timing()
        if sample_clocks:
            clocks.start()
            time.sleep(0.3)
        # the timed steps as a user runs them: one captured graph per step
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        sim.step(args.steps)
        ev1.record(stream)
        sim.sync()
        torch.cuda.synchronize()
        clk = clocks.stop() if sample_clocks else None
        ms = ev0.elapsed_time(ev1)
        launches = sim.timing()["launches"]
        alive1 = alive_count(sim, wl)
        # the per-phase breakdown (kernel_ms, the roofline's particle-phase
        # time) from as many further steps, launched one by one with events
        # between the phases (the re-sort schedule counts steps from the
        # start, so these steps re-sort as often as the timed ones)
        sim.reset_timing()
        sim.set_timing(True)
        sim.step(args.steps)
        sim.sync()
        tm = sim.timing()
        tm["launches"] = launches
        sim.set_timing(False)
        particle_steps = 0.5 * (alive0 + alive1) * args.steps
        ms_max, total_ps = aggregate_ranks(dist, ms, particle_steps, "cuda")
        diag = sim.diagnostics()
        return sim, stream, {"ms": ms_max, "value": total_ps / (ms_max / 1000.0), "tm": tm,
                             "clk": clk, "diag": diag}

    # headline: the FP32 cell-local form; the FP64 plain form beside it
    head_prec = args.precision
    other_prec = "fp64" if head_prec == "fp32" else "fp32"
    sim_o, _, res_o = measure(other_prec, False)
    sim_o.close()
    del sim_o
    sim, stream, res = measure(head_prec, True)
    value, ms_max, tm, clk = res["value"], res["ms"], res["tm"], res["clk"]

    # roofline of the dominant kernel (the fused push + deposition)
    peaks, peak_src = load_peaks()
    bytes_particle_phase = species_bytes(sim, wl, head_prec)
    ms_part = tm["ms_particles"] / max(tm["steps"], 1)
    achieved = bytes_particle_phase / (ms_part / 1000.0) / 1e9
    n_nodes = wl.n_grid_r * wl.n_grid_z
    ms_fields = tm["ms_fields"] / max(tm["steps"], 1)

    def gauss_rel(d):
        return d["gauss_residual"] / d["gauss_norm"] if d["gauss_norm"] > 0 else None

    d32 = res["diag"] if head_prec == "fp32" else res_o["diag"]
    d64 = res_o["diag"] if head_prec == "fp32" else res["diag"]
    v32 = res["value"] if head_prec == "fp32" else res_o["value"]
    v64 = res_o["value"] if head_prec == "fp32" else res["value"]
    forms = {
        "fp32_cell_local": {"value": v32, "gauss_rel_residual": gauss_rel(d32),
                            "field_energy_J": d32["field_energy"],
                            "kinetic_energy_J": d32["kinetic_energy"]},
        "fp64_plain": {"value": v64, "gauss_rel_residual": gauss_rel(d64),
                       "field_energy_J": d64["field_energy"],
                       "kinetic_energy_J": d64["kinetic_energy"]},
        "fp32_over_fp64": v32 / v64,
        "field_energy_rel_diff": abs(d32["field_energy"] - d64["field_energy"]) /
        d64["field_energy"] if d64["field_energy"] > 0 else None,
        "after_steps": args.warmup + 2 * args.steps,
    }

    # end to end through the public API from pinned host buffers: every step
    # uploads the particle state, steps, and reads the state and E_z back.
    e2e = None
    if args.e2e_steps > 0 and wl.device_plasma is None:
        e2e = run_e2e(sim, wl, torch, stream, args.e2e_steps)
        # whole job: the particle-steps of all ranks over the slowest rank's time
        e2e_ms, e2e_work = aggregate_ranks(dist, 1000.0 * e2e.pop("_secs"), e2e.pop("_work"),
                                           "cuda")
        e2e["value"] = e2e_work / (e2e_ms / 1000.0)
        e2e["h2d_bytes_per_step"] *= world  # every rank copies its own replica
        e2e["d2h_bytes_per_step"] *= world
    elif wl.device_plasma is not None:
        e2e = {"value": None, "unit": UNIT, "h2d_bytes_per_step": None,
               "d2h_bytes_per_step": None,
               "note": "not measured: the full-state round trip of this case (~30 GB per "
                       "step in FP64 host arrays) exceeds the host memory budget"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(wl, args.cpu_steps, args.cpu_fraction,
                               args.cpu_one_thread_fraction)
            if wl.device_plasma is not None:
                cpu["full_size"] = (
                    "not run: memory and time (the upstream double** layout holds ~62 GB of "
                    "host memory for the %d particles, and one step takes ~%.0f s at the "
                    "rate above); the sample is the same grid, density ramp, bunch and "
                    "pusher at a reduced ppc" % (wl.n_particles, wl.n_particles / cpu["value"]))
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": None,
                   "sample": "failed: %s" % exc}

    # accuracy over a long run (untimed): both forms from the same initial
    # state, FP64 diagnostics of each every `every` steps
    accuracy = None
    if world == 1 and args.accuracy_steps > 0:
        sim.close()
        accuracy = run_accuracy(api, wl, local_rank, args.accuracy_steps,
                                max(1, args.accuracy_steps // 10))

    traffic = load_traffic(args.workload, head_prec, wl)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if head_prec == "fp64" else "f32+f64acc",
            "fp64_plain_value": v64, "fp32_over_fp64": v32 / v64,
            "data": "synthetic (seeded)",
            "config": {"workload": wl.name, "n_grid_r": wl.n_grid_r, "n_grid_z": wl.n_grid_z,
                       "particles": wl.n_particles, "pusher": wl.pusher,
                       "precision": head_prec, "parallelism": "replicas x%d" % world,
                       "l2": "inputs larger than L2 (particle state %.2f GB)"
                             % (bytes_particle_phase / 1e9)},
            "forms": forms,
            "cell_updates_per_s": n_nodes / (ms_fields / 1000.0) if ms_fields > 0 else None,
            "cell_updates_per_s_step": n_nodes * args.steps * world / (ms_max / 1000.0),
            "kernel_ms": {"particles": ms_part, "fields": ms_fields,
                          "sort": tm["ms_sort"] / max(tm["steps"], 1),
                          "other": tm["ms_other"] / max(tm["steps"], 1)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks.get("hbm_gbs"),
                         "unit": "GB/s", "frac": achieved / peaks.get("hbm_gbs"),
                         "traffic": traffic,
                         "kernel": "k_push_deposit_f%s (all species)" % head_prec[-2:],
                         "peak_source": peak_src,
                         "algorithmic_bytes_per_launch": bytes_particle_phase},
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gpu_launches": tm["launches"],
            "clocks": clk,
            "accuracy": accuracy,
        }
        print(json.dumps(line), flush=True)
    if accuracy is None:
        sim.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def aggregate_ranks(dist, ms, work, device):
    """Whole-job timing of replicas: the slowest rank's device time (max) and
    the work of all ranks (sum).  dist None: one process."""
    if dist is None:
        return ms, work
    import torch
    t = torch.tensor([ms, work], dtype=torch.float64, device=device)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(t[1])


def run_accuracy(api, wl, device, steps, every):
    """The FP32 cell-local form against the FP64 plain form over `steps`
    steps from identical inputs: Gauss-law relative residual of each form and
    the relative difference of their total field energies, every `every`
    steps."""
    sims = {p: api.from_workload(wl, precision=p, device=device) for p in ("fp32", "fp64")}
    for s_ in sims.values():
        s_.mark_initial_charge()
    rows = []
    done = 0
    first_status = {}
    while done < steps:
        k = min(every, steps - done)
        for s_ in sims.values():
            s_.step(k)
        done += k
        for p, s_ in sims.items():
            st = s_.status()   # device error flags (e.g. v >= c in the FP64 velocity form)
            if st != 0 and p not in first_status:
                first_status[p] = {"step": done, "status": st}
        d = {p: s_.diagnostics() for p, s_ in sims.items()}
        g = {p: d[p]["gauss_residual"] / d[p]["gauss_norm"] for p in d}
        fe = abs(d["fp32"]["field_energy"] - d["fp64"]["field_energy"]) / d["fp64"]["field_energy"]
        ke = abs(d["fp32"]["kinetic_energy"] - d["fp64"]["kinetic_energy"]) / \
            d["fp64"]["kinetic_energy"]
        rows.append({"step": done, "gauss_rel_fp32": g["fp32"], "gauss_rel_fp64": g["fp64"],
                     "field_energy_rel_diff": fe, "kinetic_energy_rel_diff": ke})
    for s_ in sims.values():
        s_.close()
    return {"steps": steps, "every": every, "status_events": first_status,
            "max_gauss_rel_fp32": max(r["gauss_rel_fp32"] for r in rows),
            "max_gauss_rel_fp64": max(r["gauss_rel_fp64"] for r in rows),
            "max_field_energy_rel_diff": max(r["field_energy_rel_diff"] for r in rows),
            "max_kinetic_energy_rel_diff": max(r["kinetic_energy_rel_diff"] for r in rows)}


def run_ensemble(args, rank, world, local_rank, dist=None):
    """Batched ensemble: independent FP32 runs of uneven grids advanced by one
    persistent kernel (pdp3g_ensemble_run), against the same runs stepped one
    after another with their own launches.  value = ensemble particle-steps/s."""
    import torch
    from pdp3_b200 import api
    from pdp3_b200 import workloads as W
    torch.cuda.set_device(local_rank)
    params = W.ensemble_params(seed=1005 + 100 * rank, n_runs=args.ensemble_runs,
                               scale=args.ensemble_scale)
    sims, n_slots = [], 0
    for p in params:
        wl = W.ensemble_run_workload(p, steps=500)
        sims.append(api.from_workload(wl, precision="fp32", device=local_rank))
        n_slots += wl.n_particles
    # sequential reference: every run on its own, its own launches
    for s_ in sims:
        s_.step(args.warmup)
        s_.sync()
    # each run stepped alone, one after another, as pdp3g_step runs it
    # (one captured graph per step): device time from the first to the last
    # launch of each run's K steps (CUDA events on its stream), summed; the
    # sum of its kernels' own times (K more steps launched one by one with
    # per-phase events) is reported beside it
    seq_ms = seq_kernel_ms = 0.0
    for s_ in sims:
        st_ = torch.cuda.ExternalStream(s_.stream_ptr, device=torch.device("cuda", local_rank))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st_)
        s_.step(args.steps)
        e1.record(st_)
        s_.sync()
        seq_ms += e0.elapsed_time(e1)
        s_.reset_timing()
        s_.set_timing(True)
        s_.step(args.steps)
        s_.sync()
        seq_kernel_ms += s_.timing()["ms_step_total"]
        s_.set_timing(False)
    ens = api.Ensemble(sims)
    bpsm = ens.autotune(2)
    chosen = "step_graph" if ens.info()["mode"] == 1 else "persistent"
    # both modes timed (every rank takes the same steps in the same order);
    # the autotuner's choice is the value
    modes = {}
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    for m in ([x for x in ("persistent", "step_graph") if x != chosen] + [chosen]):
        ens.set_mode(m)
        ens.run(args.warmup)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        ens.run(args.steps)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        inf = ens.info()
        modes[m] = {"ms_per_step": inf["last_ms"] / args.steps,
                    "cuda_graph": bool(inf["used_graph"])}
    clk = clocks.stop()
    info = ens.info()
    ms = info["last_ms"]
    alive = 0
    for s_ in sims:
        for sid in range(3):
            n = s_.species_size(sid)
            alive += n if sid < 2 else int(s_.species(sid)["alive"].sum())
    ms_max, alive_all = aggregate_ranks(dist, ms, float(alive), "cuda")
    seq_ms_max, _ = aggregate_ranks(dist, seq_ms, float(alive), "cuda")
    value = alive_all * args.steps / (ms_max / 1000.0)
    seq_value = alive_all * args.steps / (seq_ms_max / 1000.0)
    # roofline of the one persistent kernel: particle state and grid bytes of
    # a step of every run over the step time
    nodes = sum(s_.nr * s_.nz for s_ in sims)
    step_bytes = (n_slots * BYTES_PER_PARTICLE["fp32"] + nodes * BYTES_PER_NODE["fp32"]) * world
    peaks, peak_src = load_peaks()
    achieved = step_bytes / (ms_max / args.steps / 1000.0) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = ensemble_cpu_baseline(params, alive, args.steps, args.cpu_fraction / 2)
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": None,
                   "sample": "failed: %s" % exc}
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64acc", "data": "synthetic (seeded)",
            "config": {"workload": "ensemble_%druns%s" % (
                           len(sims), "" if args.ensemble_scale == 1 else
                           "_scale%d" % args.ensemble_scale),
                       "runs": len(sims),
                       "particle_slots": n_slots, "alive_particles": alive,
                       "grids": "r in {64,128,256} x z in {256,512,1024} cells / %d"
                                % args.ensemble_scale,
                       "parallelism": "replicas x%d" % world},
            "ensemble": {"mode": chosen, "blocks_per_sm": info["blocks_per_sm"],
                         "graph_blocks_per_sm": info["graph_blocks_per_sm"],
                         "blocks": info["blocks"], "cuda_graph": bool(info["used_graph"]),
                         "ms_per_step": ms / args.steps,
                         "modes": {m: dict(v, value=alive_all * args.steps /
                                           (v["ms_per_step"] * args.steps / 1000.0),
                                           over_sequential=(seq_ms_max / args.steps) /
                                           v["ms_per_step"])
                                   for m, v in modes.items()},
                         "autotuner": "persistent kernel at every feasible CTAs-per-SM "
                                      "count and the step graph with the runs' particle "
                                      "kernels at 2, 4 and 8 CTAs per SM, 2 steps each; "
                                      "the fastest is kept"},
            "sequential": {"value": seq_value, "ms_per_step": seq_ms_max / args.steps,
                           "kernel_ms_per_step": seq_kernel_ms / args.steps,
                           "note": "same runs, each stepped alone by pdp3g_step (one "
                                   "captured graph per step); ms_per_step spans each run's "
                                   "steps on its stream, kernel_ms_per_step sums the "
                                   "kernels alone (steps launched one by one)"},
            "ensemble_over_sequential": value / seq_value,
            "cell_updates_per_s": nodes * world * args.steps / (ms_max / 1000.0),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks.get("hbm_gbs"),
                         "unit": "GB/s", "frac": achieved / peaks.get("hbm_gbs"),
                         "traffic": None, "kernel": "k_ensemble (whole step)",
                         "peak_source": peak_src,
                         "algorithmic_bytes_per_step": step_bytes},
            "cpu_baseline": cpu,
            "clocks": clk}), flush=True)
    ens.close()
    for s_ in sims:
        s_.close()
    return 0


def ensemble_cpu_baseline(params, alive, steps, fraction, n_sample=4):
    """The upstream CPU step on a sample of the ensemble's runs (n_sample runs
    spread over the list, `fraction` of each one's plasma, 2 steps each, all
    host cores), extrapolated to every run for `steps` steps: the runs are
    independent, so the CPU would step them one after another at the sampled
    particle-steps rate."""
    from pdp3_b200 import workloads as W
    threads = os.cpu_count() or 1
    picks = sorted(set(int(round(x)) for x in np.linspace(0, len(params) - 1, n_sample)))
    work = secs = 0.0
    kind = None
    for j in picks:
        wl = W.ensemble_run_workload(params[j], steps=500)
        rate, kind, _, _, sec = cpu_sample_run(wl, 2, 1, fraction, threads)
        work += rate * sec
        secs += sec
    rate = work / secs
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": "runs %s of %d, %.4g of each run's plasma particles + bunch, 2 steps "
                      "after 1 warm-up each, %d OpenMP threads" % (picks, len(params), fraction,
                                                                    threads),
            "extrapolated_seconds": alive * steps / rate,
            "extrapolation": "%d runs x %d steps (%d alive particles) one after another at "
                             "the sampled rate" % (len(params), steps, alive)}


def fitted_fd_slope(api, W, fam, theta, j, steps, probe, hmax=0.02, npts=4):
    """dL/dtheta_j of the FP64 form from a cubic fitted to the loss at 2*npts
    relative steps in [-hmax, hmax] (the loss of a many-particle run is a
    staircase of small jumps, so a single central difference is noisy).
    Returns (slope, standard error)."""
    xs = np.concatenate([-np.arange(npts, 0, -1), np.arange(1, npts + 1)]) * (hmax / npts)
    ls = []
    for x in xs:
        t = theta.copy()
        t[j] = theta[j] * (1 + x)
        wl, _ = fam.workload(t)
        sim = api.from_workload(wl, precision="fp64")
        sim.step(steps)
        sim.sync()
        ls.append(W.probe_loss(sim.field("E_z"), wl.dr, wl.dz, probe))
        sim.close()
    X = np.vstack([np.ones_like(xs), xs, xs ** 2, xs ** 3]).T
    coef = np.linalg.lstsq(X, np.array(ls), rcond=None)[0]
    resid = np.array(ls) - X @ coef
    s2 = float(resid @ resid) / max(len(xs) - 4, 1)
    se = math.sqrt(s2 * np.linalg.inv(X.T @ X)[1, 1])
    return coef[1] / theta[j], se / abs(theta[j])


def run_adjoint(args, rank, world, local_rank, dist=None):
    """Differentiable window (128x1024 cells, 32 ppc per species, gamma=5
    bunch, 500 steps, checkpoints every 50): device time of the forward and
    backward window, and the gradient against FP64 finite differences.
    value = forward-window particle-steps/s."""
    import torch
    from pdp3_b200 import api
    from pdp3_b200 import workloads as W
    torch.cuda.set_device(local_rank)
    steps, interval = args.adjoint_steps, args.adjoint_interval
    sc = max(1, args.adjoint_scale)
    kw = {}
    probe = W.ADJOINT_PROBE
    if sc > 1:
        kw = dict(n_grid_r=128 // sc + 1, n_grid_z=1024 // sc + 1, r_size=0.1 / sc,
                  z_size=0.8 / sc)
        probe = (0, max(2, 16 // sc), 120 // sc, 184 // sc)
    theta = W.adjoint_theta()
    fam = W.AdjointFamily(theta, **kw)
    wl, aux = fam.workload(theta)
    # warm-up: one window on a separate context (a second forward on the
    # same context would start from the first window's end state)
    sim = api.from_workload(wl, precision="fp32", device=local_rank)
    adj = api.Adjoint(sim, steps, interval, probe)
    adj.forward()
    adj.backward()
    adj.close()
    sim.close()
    sim = api.from_workload(wl, precision="fp32", device=local_rank)
    adj = api.Adjoint(sim, steps, interval, probe)
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    loss = adj.forward()
    adj.backward()
    if dist is not None:
        dist.barrier()
    clk = clocks.stop()
    t = adj.timing()

    def grad(mean_field):
        return W.adjoint_gradient(wl, aux, [adj.species(0), adj.species(1)], adj.species(2),
                                  adj.bunch_velocity(2), mean_field=mean_field)
    g_mf = grad(True)
    # the mean-field terms beyond the default, for the record
    variants = {"gather_wall_cells": ("gather", "wall_cells"),
                "gather_walls_wall_cells": ("gather", "walls", "wall_cells")}
    g_var = {}
    for name, terms in variants.items():
        adj.set_jump_terms(*terms)
        adj.backward()
        g_var[name] = grad(True)
    # the jump densities: uniform inside each cell (face width 0) and a
    # narrower box kernel than the default 1/8 cell
    adj.set_mode("mean_field")
    for hw in (0.0, 0.0625):
        adj.set_face_width(hw)
        adj.backward()
        g_var["face_width_%g" % hw] = grad(True)
    adj.set_face_width(0.125)
    adj.set_mode("pathwise")
    adj.backward()
    g_pw = grad(False)
    n_alive_end = sum(sim.species_size(s) for s in (0, 1)) + int(sim.species(2)["alive"].sum())
    adj_bytes = adj.device_bytes()
    adj.close()
    sim.close()
    if args.adjoint_fd_params == "none":
        params = []
    elif args.adjoint_fd_params == "all":
        params = list(range(theta.size))
    else:
        zc = (np.arange(W.N_BUMPS) + 0.5) * wl.z_size / W.N_BUMPS
        zp = 0.5 * (probe[2] + probe[3]) * wl.dz
        params = sorted(np.argsort(np.abs(zc - zp))[:4].tolist()) + [W.N_BUMPS, W.N_BUMPS + 1]
    fd = {}
    for j in params:
        slope, se = fitted_fd_slope(api, W, fam, theta, j, steps, probe)
        fd[j] = {"fd": slope, "fd_se": se, "mean_field": g_mf[j], "pathwise": g_pw[j],
                 "rel_err_mean_field": (g_mf[j] - slope) / slope,
                 "rel_err_pathwise": (g_pw[j] - slope) / slope}
        for name, g in g_var.items():
            fd[j]["rel_err_" + name] = (g[j] - slope) / slope
        if j == W.N_BUMPS:
            # gamma: a second fit over +-1% with 16 points (the loss is a
            # staircase of small jumps; past about +-2% the injection's
            # ceil(duration / dt) changes the particles injected per step)
            s1, se1 = fitted_fd_slope(api, W, fam, theta, j, steps, probe, hmax=0.01, npts=8)
            fd[j]["fd_pm1pct_16pts"] = s1
            fd[j]["fd_pm1pct_16pts_se"] = se1
            fd[j]["rel_err_mean_field_vs_pm1pct"] = (g_mf[j] - s1) / s1
            for name, g in g_var.items():
                fd[j]["rel_err_%s_vs_pm1pct" % name] = (g[j] - s1) / s1
    dens = [j for j in params if j < W.N_BUMPS]
    summary = {}
    if dens:
        f = np.array([fd[j]["fd"] for j in dens])
        for mode, g in [("mean_field", g_mf), ("pathwise", g_pw)] + list(g_var.items()):
            a = np.array([g[j] for j in dens])
            summary["density_block_rel_err_" + mode] = float(np.linalg.norm(a - f) /
                                                             np.linalg.norm(f))
    fwd_max, particles_all = aggregate_ranks(dist, t["forward_ms"], float(wl.n_particles), "cuda")
    bwd_max, _ = aggregate_ranks(dist, t["backward_ms"], 0.0, "cuda")
    value = particles_all * steps / (fwd_max / 1000.0)
    # roofline of the forward window: particle state and grid bytes of each
    # step over the forward device time (the window also captures its inputs)
    nodes = wl.n_grid_r * wl.n_grid_z
    step_bytes = (wl.n_particles * BYTES_PER_PARTICLE["fp32"] +
                  nodes * BYTES_PER_NODE["fp32"]) * world
    peaks, peak_src = load_peaks()
    achieved = step_bytes / (fwd_max / steps / 1000.0) / 1e9
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": steps, "ms_per_step": fwd_max / steps,
            "cell_updates_per_s": nodes * world * steps / (fwd_max / 1000.0),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks.get("hbm_gbs"),
                         "unit": "GB/s", "frac": achieved / peaks.get("hbm_gbs"),
                         "traffic": None, "kernel": "forward window (whole step)",
                         "peak_source": peak_src,
                         "algorithmic_bytes_per_step": step_bytes},
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64acc", "data": "synthetic (seeded)",
            "config": {"workload": wl.name, "window_steps": steps,
                       "checkpoint_interval": interval, "probe_nodes": list(probe),
                       "particles": wl.n_particles, "alive_at_end": n_alive_end,
                       "parallelism": "replicas x%d" % world},
            "adjoint": {"loss": loss, "forward_ms": fwd_max,
                        "backward_ms": bwd_max,
                        "backward_over_forward": bwd_max / fwd_max,
                        "device_bytes": adj_bytes,
                        "fd": "FP64 form, cubic fit over 8 relative steps in [-2%, 2%]",
                        "params": {str(j): v for j, v in fd.items()}, "summary": summary},
            "clocks": clk}), flush=True)
    return 0


# ------------------------------------------------------ diagnostics (rows f1, f2, f4)

DIAG_POISSON_GRID = (257, 2047)  # the wake grid's size where 2 n_grid_z + 2 is a power of two


def diag_cpu_times(wl, fractions, threads):
    """The upstream CPU charge weighting, TemperatureClassic and
    ParticlesDensity (oracle/_ref) on the wake grid with seeded subsets of
    the plasma: milliseconds per call at each sample size, and a straight
    line through them in the particle count extrapolated to the full count
    (all plasma species for the charge density, the electrons for the
    per-species diagnostics)."""
    from oracle import refsim
    if not refsim.available("boris"):
        return None
    rng = np.random.default_rng(4321)
    rows = []
    for frac in fractions:
        sim = refsim.RefSim(wl.r_size, wl.z_size, wl.n_grid_r, wl.n_grid_z, wl.dt, end_time=1.0,
                            pml=wl.pml, pusher="boris")
        sim.L.ref_set_threads(threads)
        counts = []
        for s in wl.species:
            k = max(1, int(s.n * frac))
            idx = np.sort(rng.choice(s.n, size=k, replace=False))
            sim.add_species(s.name, s.charge_e, s.mass_me, s.r[idx], s.z[idx], s.vr[idx],
                            s.vphi[idx], s.vz[idx], s.w[idx])
            counts.append(k)
        t = {}
        for name, fn in (("charge_density", lambda: sim.charge_density()),
                         ("temperature_electrons", lambda: sim.temperature(0)),
                         ("density_electrons", lambda: sim.density(0))):
            fn()
            reps = []
            for _ in range(3):
                t0 = time.perf_counter()
                fn()
                reps.append(time.perf_counter() - t0)
            t[name] = 1e3 * statistics.median(reps)
        rows.append(({"charge_density": sum(counts), "temperature_electrons": counts[0],
                      "density_electrons": counts[0]}, t))
        sim.close()
    full = {"charge_density": sum(s.n for s in wl.species),
            "temperature_electrons": wl.species[0].n, "density_electrons": wl.species[0].n}
    out = {}
    (c0, t0), (c1, t1) = rows[0], rows[-1]
    for name in t0:
        slope = (t1[name] - t0[name]) / max(c1[name] - c0[name], 1)
        out[name] = {"ms_extrapolated": max(t1[name], t1[name] + slope * (full[name] - c1[name])),
                     "samples": [{"particles": c[name], "ms": tt[name]} for c, tt in rows]}
    return out


def diag_cpu_poisson(threads):
    from oracle import refsim
    if not refsim.available("boris"):
        return None
    nr, nz = DIAG_POISSON_GRID
    sim = refsim.RefSim(0.1, 0.8, nr, nz, 4.6e-13, end_time=1.0, pml=None, pusher="boris")
    sim.L.ref_set_threads(threads)
    rho = np.random.default_rng(5).normal(0.0, 1e-3, (nr, nz))
    sim.poisson_dirichlet(rho)
    reps = []
    for _ in range(3):
        t0 = time.perf_counter()
        sim.poisson_dirichlet(rho)
        reps.append(time.perf_counter() - t0)
    sim.close()
    return 1e3 * statistics.median(reps)


def run_diag(args, rank, world):
    """The upstream's diagnostics and initial-field solve on one GPU: charge
    density (Particles::charge_weighting), TemperatureClassic and
    ParticlesDensity of the electrons, a full-frame E_z probe read
    (ProbePlain frame) on the wake case, and PoissonDirichlet on a 257 x 2047
    grid, each through its C-ABI call with the result copied to host memory;
    device time with CUDA events on the context's stream, the upstream CPU
    code timed beside it."""
    if rank != 0:
        return 0
    import torch
    from pdp3_b200 import api
    peaks, peak_src = load_peaks()
    hbm = peaks["hbm_gbs"]
    wl = make_workload("wake", 1002, args.ppc)
    sim = api.from_workload(wl, precision=args.precision)
    sim.step(args.warmup)
    sim.sync()
    stream = torch.cuda.ExternalStream(sim.stream_ptr)
    n_all = sum(sim.species_size(s) for s in range(len(wl.species)))
    n_el = sim.species_size(0)
    ng = wl.n_grid_r * wl.n_grid_z
    part_b = 16 if args.precision == "fp32" else 24  # position (+ cell) and weight
    vel_b = 12 if args.precision == "fp32" else 24

    def timed(fn, reps=5):
        fn()
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return statistics.median(ms)

    items = {}

    def add(name, ms, nbytes, what):
        achieved = nbytes / (ms * 1e-3) / 1e9
        items[name] = {"ms": ms, "algorithmic_bytes": nbytes, "what": what,
                       "achieved_gbs": achieved, "frac": achieved / hbm}

    add("charge_density", timed(lambda: sim.charge_density()),
        n_all * part_b + ng * 8 * 2,
        "every plasma particle's position and weight read, the rho grid written and copied out")
    add("temperature_electrons", timed(lambda: sim.temperature(0)),
        n_el * (part_b + vel_b) + ng * 8 * 2,
        "the electrons' positions, velocities and weights read, the T grid written and copied out")
    add("density_electrons", timed(lambda: sim.density(0)),
        n_el * part_b + ng * 8 * 2,
        "the electrons' positions and weights read, the density grid written and copied out")
    add("probe_frame_E_z", timed(lambda: sim.probe("E_z", "frame", 0, 0, wl.n_grid_r,
                                                     wl.n_grid_z)),
        ng * 8 * 2, "the E_z grid read and its frame copied out")
    sim.close()
    nr, nz = DIAG_POISSON_GRID
    ps = api.Simulation(0.1, 0.8, nr, nz, 4.6e-13, precision=args.precision)
    rho = np.random.default_rng(5).normal(0.0, 1e-3, (nr, nz))
    ps_stream = torch.cuda.ExternalStream(ps.stream_ptr)
    stream = ps_stream
    add("poisson_dirichlet_257x2047", timed(lambda: ps.poisson_solve(rho)),
        nr * nz * 8 * 5, "rho copied in, phi, E_r, E_z written, phi copied out")
    ps.close()
    cpu = None if args.no_cpu_baseline else diag_cpu_times(
        wl, (1.0 / 64, 1.0 / 32), os.cpu_count() or 1)
    cpu_p = None if args.no_cpu_baseline else diag_cpu_poisson(os.cpu_count() or 1)
    if cpu:
        for name in ("charge_density", "temperature_electrons", "density_electrons"):
            items[name]["cpu_reference_ms"] = cpu[name]["ms_extrapolated"]
            items[name]["cpu_samples"] = cpu[name]["samples"]
            items[name]["speedup_vs_cpu"] = cpu[name]["ms_extrapolated"] / items[name]["ms"]
    if cpu_p is not None:
        items["poisson_dirichlet_257x2047"]["cpu_reference_ms"] = cpu_p
        items["poisson_dirichlet_257x2047"]["speedup_vs_cpu"] = (
            cpu_p / items["poisson_dirichlet_257x2047"]["ms"])
    total = sum(v["ms"] for v in items.values())
    print(json.dumps({
        "metric": "diagnostics and Poisson solve, device ms per C-ABI call (result copied out)",
        "value": total, "unit": "ms", "n_gpus": 1, "higher_is_better": False,
        "dtype": "f64 arithmetic on " + args.precision + " particle state",
        "data": "synthetic (seeded)",
        "config": {"workload": wl.name, "particles": n_all,
                   "poisson_grid": "%dx%d nodes" % DIAG_POISSON_GRID,
                   "cpu_reference": ("upstream code (oracle/_ref), %d threads, seeded plasma "
                                     "subsets of 1/64 and 1/32, linear in the particle count"
                                     % (os.cpu_count() or 1))},
        "items": items, "peak_gbs": hbm, "peak_source": peak_src}), flush=True)
    return 0


def load_traffic(workload, precision, wl):
    """DRAM bytes (read + write) of one pass of the particle phase, from the
    committed ncu summary of the same kernel on the small cases of this
    workload: a per-particle part scaled by the plasma particle count (the
    kernel streams each particle once) plus, where the summary gives one, a
    fixed part per species launch (the field data the launch reads, the same
    at every particle count).  None when no summary exists."""
    path = os.path.join(ROOT, "profiles", "push_deposit_%s_%s_ppc8.md" % (precision, workload))
    per = fixed = None
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_particle:"):
                    per = float(line.split(":")[1])
                elif line.startswith("dram_bytes_per_launch_fixed:"):
                    fixed = float(line.split(":")[1])
    except OSError:
        return None
    if per is None:
        return None
    n_plasma = wl.n_particles - (wl.beam.number_macro * wl.beam.number_bunches
                                 if wl.beam is not None else 0)
    return per * n_plasma + (fixed or 0.0) * len(wl.species)


def run_e2e(sim, wl, torch, stream, steps):
    """Same metric through the public C-ABI with host buffers: each step runs
    one step, copies every species' state to pinned host memory and from
    there back as the next step's input (pdp3g_exchange_all: both directions
    at once, all species in one pipeline), and copies the E_z grid back."""
    n_sp = len(wl.species) + (wl.beam.number_bunches if wl.beam is not None else 0)
    bufs = []
    for sid in range(n_sp):
        n = sim.species_size(sid)
        # the five arrays of a species in one pinned block: the exchange then
        # moves each chunk of all five with one 2-D copy per direction
        block = torch.empty(5 * n, dtype=torch.float64, pin_memory=True).numpy()
        arrs = {k: block[j * n:(j + 1) * n]
                for j, k in enumerate(("r", "z", "vr", "vphi", "vz"))}
        alive = torch.empty(n, dtype=torch.uint8, pin_memory=True).numpy()
        st = sim.species(sid)
        for k in arrs:
            arrs[k][:] = st[k]
        alive[:] = st["alive"]
        bufs.append((sid, arrs, alive, st["w"]))
    ez = torch.empty(wl.n_grid_r * wl.n_grid_z, dtype=torch.float64, pin_memory=True).numpy()
    import ctypes
    from pdp3_b200.api import _U8
    h2d = d2h = 0
    for sid, arrs, alive, _ in bufs:
        h2d += sum(a.nbytes for a in arrs.values()) + (alive.nbytes if sid >= len(wl.species)
                                                       else 0)
    d2h = h2d + ez.nbytes
    alive_total = 0
    P = ctypes.POINTER(ctypes.c_double)
    step_rates = []
    from pdp3_b200.api import ExchangeItem
    items = (ExchangeItem * len(bufs))()
    for j, (sid, arrs, alive, _w) in enumerate(bufs):
        it = items[j]
        it.id = sid
        for k in ("r", "z", "vr", "vphi", "vz"):
            setattr(it, "out_" + k, arrs[k].ctypes.data_as(P))
            setattr(it, "in_" + k, arrs[k].ctypes.data_as(P))
        al = alive.ctypes.data_as(_U8) if sid >= len(wl.species) else None
        it.out_alive = al
        it.in_alive = al
    # one untimed exchange: the first call allocates the staging and events
    sim._check(sim.L.pdp3g_exchange_all(sim.h, items, len(bufs)), "exchange_all")
    sim.sync()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        ts = time.perf_counter()
        sim.step(1)
        # this step's state out and, from the same host arrays, the next
        # step's input in, every species in one pipeline with both PCIe
        # directions busy (pdp3g_exchange_all)
        sim._check(sim.L.pdp3g_exchange_all(sim.h, items, len(bufs)), "exchange_all")
        sim._check(sim.L.pdp3g_get_field(sim.h, 2, ez.ctypes.data_as(P)), "get_field")
        te = time.perf_counter()
        n_step = sum(len(a["r"]) if sid < len(wl.species) else int(al.sum())
                     for sid, a, al, _ in bufs)
        alive_total += n_step
        step_rates.append(n_step / (te - ts))
    secs = time.perf_counter() - t0
    return {"value": alive_total / secs, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": steps, "_secs": secs, "_work": alive_total,
            "per_step": {"median": statistics.median(step_rates), "min": min(step_rates),
                         "max": max(step_rates)},
            "note": "per step, through the C ABI: one step, then every species' full state "
                    "D2H into pinned host arrays and from them H2D as the next step's input "
                    "(pdp3g_exchange_all: one pipeline over all species, both directions "
                    "concurrently), E_z D2H"}


if __name__ == "__main__":
    sys.exit(main())
