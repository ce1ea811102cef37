"""Benchmark of the nonbonded force path (cutoff + PME) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload: the 14,281-atom chain-in-water box (4,463 TIP3P waters + an
892-atom random-walk chain, 52.3 A cube), LJ C2 10 -> 12 A + Ewald real space
(Cutoff 12 A, alpha 0.32) as one NonbondedCutoff force, plus PME 64^3, order
4, reciprocal + correction.  One step = one full force evaluation (binning,
pair force, PME, energy and virial).  Synthetic seeded data.

`value`: mixed-precision force evaluations/s with positions already in HBM
(device API), timed per step with CUDA events on the library's stream; the
L2 is flushed (256 MB write) between timed steps, outside the events.
`e2e`: the same through pmgpu_evaluate with pinned host buffers (positions
H2D, forces + energies D2H inside the timed region), wall clock per call.
Under torchrun each rank evaluates its own replica (the path does not
shard); value = total evaluations/s over ranks from the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "force evals/s (cutoff+PME) mixed vs FP64 on one B200 at ≤1e-5 force error"
UNIT = "evals/s"
FP32_LANES_PER_SM = 128
N_SMS = 148
# DRAM bytes (read + write) of one pair-kernel launch on this workload, by
# layout: dram__bytes_read.sum + dram__bytes_write.sum of an ncu capture of
# the kernel on this bench command (L2 flushed before the evaluation)
PAIR_DRAM_BYTES_PER_LAUNCH = {"columns": 10_208_512, "cells": 4_994_304}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=20)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extra", action="store_true",
                   help="skip the batched (96 boxes) and 1,000,000-atom measurements")
    p.add_argument("--workload", default="chain14281", choices=["chain14281", "water1m"],
                   help="water1m: only the 1,000,000-atom box (one GPU; --steps evaluations)")
    return p.parse_args()


def dist_setup(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=None)
        pg = dist
    return rank, world, local, pg


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi takes a moment to start: the timed region begins
            # once it is sampling (at most 5 s)
            t0 = time.perf_counter()
            while not self.samples and time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def cpu_baseline(system, defs, evals):
    """The reference's own CPU force path (oracle/_ref/pmref_fast, built from
    the ProtoMol sources with its gcc preset), 1 core."""
    from oracle import oracle
    from protomol_b200 import forces as F
    specs = [F.parse_definition(d) for d in defs]
    fast = oracle.reference_available(fast=True)
    if fast or oracle.reference_available():
        r = oracle.run_reference(system, specs, repeat=evals, fast=fast, timeout=600)
        sec = r["seconds_per_eval"]
        kind = "reference"
    else:
        t0 = time.perf_counter()
        for _ in range(evals):
            oracle.evaluate(system, specs)
        sec = (time.perf_counter() - t0) / evals
        kind = "port"
    return {"value": 1.0 / sec, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{evals} full evaluations (after 1 warm-up) of the 14,281-atom cutoff+PME force, "
                      f"{'pmref_fast (reference sources, -O3 -ffast-math preset)' if kind == 'reference' else 'CPU port'}"}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_all_cores(system, defs, evals):
    """The reference's CPU force path on every host core: one pmref_fast
    process per core (the path is single-threaded), all at once; throughput
    = sum of the per-process evaluation rates."""
    from oracle import oracle
    from protomol_b200 import forces as F
    specs = [F.parse_definition(d) for d in defs]
    procs = host_cores()
    if oracle.reference_available(fast=True):
        secs = oracle.run_reference_parallel(system, specs, evals, procs, fast=True, timeout=900)
        return {"value": float(sum(1.0 / t for t in secs)), "unit": UNIT, "cores": procs, "kind": "reference",
                "sample": f"{procs} concurrent processes x {evals} full evaluations (after 1 warm-up each) of the "
                          "14,281-atom cutoff+PME force, pmref_fast (reference sources, -O3 -ffast-math preset); "
                          "value = sum of the per-process rates"}
    base = cpu_baseline(system, defs, evals)           # the oracle port, one core
    return base


def run_reference_arm(args, rank, world, pg):
    from protomol_b200 import workloads
    w = workloads.chain14281()
    if rank != 0:
        if pg:
            pg.barrier()
        return
    # at least two timed evaluations: the reference driver times repeats only
    evals = min(max(2, args.steps), 12)
    base = reference_all_cores(w.system, w.forces, evals)
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": world,
            "steps": evals, "warmup": 1, "ms_per_step": 1000.0 / base["value"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "chain14281 cutoff12 C2 + EwaldReal + PME 64^3 order 4",
                       "atoms": w.system.n_atoms, "parallelism": f"{base['cores']} host processes"},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()


def main():
    args = parse()
    rank, world, local, pg = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference_arm(args, rank, world, pg)
        if pg:
            pg.destroy_process_group()
        return

    import torch
    from protomol_b200 import _lib
    from protomol_b200 import forces as F
    from protomol_b200 import workloads
    if args.workload == "water1m":              # the large-system configuration alone
        torch.cuda.set_device(local)
        if rank == 0:
            m = measure_1m(local, torch, max(1, min(args.steps, 50)))
            print(json.dumps({"metric": "force evals/s (cutoff+PME), 1,000,000 atoms", "value": m["mixed"]["evals_per_s"],
                              "unit": "evals/s", "n_gpus": 1, "steps": max(1, min(args.steps, 50)),
                              "ms_per_step": m["mixed"]["ms_per_step"], "higher_is_better": True, "data": "synthetic",
                              "config": {"workload": m["workload"], "atoms": m["atoms"]}, "scale_1m": m}), flush=True)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return

    torch.cuda.set_device(local)
    lib = _lib.load()
    w = workloads.chain14281()
    s = w.system
    n = s.n_atoms
    topo = F.Topology(s, device=local)
    mixed = [F.ForceFactory.make(topo, d, "mixed") for d in w.forces]
    fp64 = [F.ForceFactory.make(topo, d, "fp64") for d in w.forces]
    # the project's autotuner picks the launch shapes for this system
    tuning = topo.autotune(mixed, s.positions, evals=50)
    stream = torch.cuda.ExternalStream(topo.stream)
    dpos = torch.tensor(s.positions, dtype=torch.float64, device=f"cuda:{local}")
    dfor = torch.zeros((n, 3), dtype=torch.float64, device=f"cuda:{local}")
    den = torch.zeros(11, dtype=torch.float64, device=f"cuda:{local}")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    VP = C.c_void_p

    def step(forces):
        arr = (VP * len(forces))(*[f.handle for f in forces])
        _lib.check(lib.pmgpu_evaluate_device(topo.handle, len(forces), arr, VP(dpos.data_ptr()),
                                             VP(dfor.data_ptr()), VP(den.data_ptr()), _lib.FLAG_VIRIAL), topo.handle)

    def timed(forces, steps, warmup, sampler=None):
        torch.cuda.synchronize()
        for _ in range(warmup):
            step(forces)
        _lib.check(lib.pmgpu_synchronize(topo.handle), topo.handle)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        launches0 = topo.launch_count()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for k in range(steps):
                flush.zero_()                      # L2 flush, outside the timed events
                evs[k][0].record(stream)
                step(forces)
                evs[k][1].record(stream)
        torch.cuda.synchronize()
        _lib.check(lib.pmgpu_synchronize(topo.handle), topo.handle)
        if pg:
            pg.barrier()
        ms = [a.elapsed_time(b) for a, b in evs]
        return ms, topo.launch_count() - launches0

    # accuracy of the mixed path against the FP64 kernels on this input
    fm = np.zeros((n, 3)); em = F.ScalarStructure()
    F.evaluate_group(topo, mixed, s.positions, fm, em)
    fd = np.zeros((n, 3)); ed = F.ScalarStructure()
    F.evaluate_group(topo, fp64, s.positions, fd, ed)
    force_err = float(np.sqrt(((fm - fd) ** 2).sum() / (fd ** 2).sum()))
    e_err = abs((em.lennard_jones + em.coulomb) - (ed.lennard_jones + ed.coulomb)) / (
        abs(ed.lennard_jones) + abs(ed.coulomb))

    # the clocks are sampled from the FP64 loop on, so that a short timed
    # region still has samples under the same load
    with ClockSampler(local) as clk:
        # FP64 kernels (the comparison point of the metric)
        ms64, _ = timed(fp64, max(20, args.steps // 10), args.warmup)
        # mixed precision (the value)
        ms_mixed, launches = timed(mixed, args.steps, args.warmup)
    # per-kernel profile of the dominant kernel: pair kernel timed alone
    t_local = float(np.mean(ms_mixed))
    t_fp64 = float(np.mean(ms64))
    if pg:
        t = torch.tensor([t_local, t_fp64], dtype=torch.float64, device=f"cuda:{local}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        t_local, t_fp64 = float(t[0]), float(t[1])

    # end to end through the host API with pinned buffers
    hpos = torch.tensor(s.positions, dtype=torch.float64).pin_memory()
    hfor = torch.zeros((n, 3), dtype=torch.float64).pin_memory()
    e = _lib.Energies()
    arr = (VP * len(mixed))(*[f.handle for f in mixed])
    for _ in range(args.warmup):
        _lib.check(lib.pmgpu_evaluate(topo.handle, len(mixed), arr, VP(hpos.data_ptr()), VP(hfor.data_ptr()),
                                      C.byref(e), _lib.FLAG_VIRIAL), topo.handle)
    e2e_steps = max(10, args.steps // 4)
    walls = []
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _lib.check(lib.pmgpu_evaluate(topo.handle, len(mixed), arr, VP(hpos.data_ptr()), VP(hfor.data_ptr()),
                                      C.byref(e), _lib.FLAG_VIRIAL), topo.handle)
        walls.append(time.perf_counter() - t0)
    t_e2e = float(np.mean(walls)) * 1000.0
    if pg:
        t = torch.tensor([t_e2e], dtype=torch.float64, device=f"cuda:{local}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        t_e2e = float(t[0])

    # the ProtoMol drop-in: the same two forces made by ProtoMol's own
    # ForceFactory and evaluated through SystemForce::evaluate into a
    # Vector3DBlock (the adapter's group of GPU forces runs as one call)
    e2e_adapter = measure_adapter(s, w.forces, max(20, min(args.steps, 400)))

    # per-phase device times (CUDA events on the library's stream) over a
    # profiled copy of the timed loop, for the rooflines
    phases = profile_phases(lib, topo, mixed, step, flush, stream, torch, max(50, min(args.steps, 400)))
    peaks, peak_src = measured_peaks()
    # within-cutoff pair set of this input, recorded by the pair kernel itself
    # (bit-exact with the oracle's, tests/test_gpu_parity.py)
    n_pairs = int(len(mixed[0].pairs(s.positions)))
    flops_per_pair = 95
    fp32_peak = N_SMS * FP32_LANES_PER_SM * 2 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6 / 1e12
    pair_ms = phases["pair"]
    achieved = n_pairs * flops_per_pair / (pair_ms * 1e-3) / 1e12
    layout = topo.pair_layout() or "cells"
    kname = {"columns": "k_pair_col", "cells": "k_pair_mixed"}.get(layout, "k_pair_fp64")
    roofline = {"bound": "fp32", "kernel": f"{kname}<LJ C2 + EwaldReal Cutoff>", "layout": layout,
                "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                "traffic": PAIR_DRAM_BYTES_PER_LAUNCH.get(layout), "traffic_unit": "B per launch (ncu)",
                "launch_ms": pair_ms,
                "peak_source": f"nominal FP32 CUDA-core rate at sm_max_mhz of MEASURED_PEAKS.json ({peak_src}): "
                               "148 SMs x 128 lanes x 2 flop",
                "algorithmic": f"{n_pairs} pairs x {flops_per_pair} flop per launch"}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    kx = 64
    kzh = kx // 2 + 1
    pme_bytes = pme_algorithmic_bytes(n, kx)
    pme_roof = {k: {"achieved_gbs": b / (phases[k] * 1e-3) / 1e9, "peak_gbs": hbm,
                    "frac": b / (phases[k] * 1e-3) / 1e9 / hbm, "bytes": b, "launch_ms": phases[k]}
                for k, b in pme_bytes.items() if phases.get(k)}

    extra = {}
    if not args.no_extra:
        extra["batched"] = measure_batched(local, rank, world, pg, torch, flush, max(20, min(args.steps // 10, 200)))
        if rank == 0:
            extra["scale_1m"] = measure_1m(local, torch, 10)
            extra["leapfrog"] = measure_leapfrog(local, torch)
            extra["table_potentials"] = measure_table(local, torch, flush, 200)
            extra["adjoint"] = measure_adjoint(local, s, w.forces)
    if rank == 0:
        value = world * 1000.0 / t_local
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_local, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+i64 fixed-point forces, f64 sums", "data": "synthetic",
            "config": {"workload": "chain14281 cutoff12 C2 + EwaldReal + PME 64^3 order 4", "atoms": n,
                       "parallelism": "replicas" if world > 1 else "single", "l2": "flushed between steps (256 MB)",
                       "tuning": tuning},
            "fp64": {"value": world * 1000.0 / t_fp64, "ms_per_step": t_fp64},
            "speedup_vs_fp64": t_fp64 / t_local,
            "accuracy_vs_fp64": {"force_rel_rms": force_err, "energy_rel": e_err},
            "e2e": {"value": world * 1000.0 / t_e2e, "unit": UNIT, "ms_per_step": t_e2e,
                    # positions, and the page-locked force accumulator the
                    # library adds to on the device; forces and energies back
                    "h2d_bytes_per_step": 24 * n + 24 * n, "d2h_bytes_per_step": 24 * n + 88},
            "e2e_adapter": e2e_adapter,
            "gpu_launches": int(launches),
            "pair_interactions_per_s": n_pairs * world * 1000.0 / t_local,
            "roofline": roofline,
            "phases_ms": phases,
            "pme_roofline_hbm": pme_roof,
            "clocks": clk.summary(),
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(s, w.forces, 12)
        if extra:
            line.update(extra)
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def measure_adapter(system, defs, repeat):
    """Evaluations/s through ProtoMol's own ForceFactory and SystemForce::
    evaluate (protomol_b200/adapter/_build/gpu_force_driver, built where the
    ProtoMol sources are): Vector3DBlock positions in, forces accumulated
    into a Vector3DBlock, energies into a ScalarStructure; the driver's wall
    clock per evaluation over ``repeat`` evaluations after one warm-up."""
    import tempfile
    driver = os.path.join(ROOT, "protomol_b200", "adapter", "_build", "gpu_force_driver")
    if not os.path.exists(driver):
        return {"unavailable": "the drop-in driver was not built (it links the ProtoMol sources)"}
    with tempfile.TemporaryDirectory() as td:
        sp, op = os.path.join(td, "s.bin"), os.path.join(td, "o.bin")
        system.save(sp)
        p = subprocess.run([driver, sp, op, str(repeat), *defs], capture_output=True, text=True, timeout=600,
                           env=dict(os.environ, PMGPU_PRECISION="mixed"))
        if p.returncode != 0:
            return {"unavailable": f"driver exit {p.returncode}"}
        sec = float(np.frombuffer(open(op, "rb").read(104), np.float64)[11])
    return {"value": 1.0 / sec, "unit": UNIT, "ms_per_step": sec * 1000.0, "evaluations": repeat,
            "path": "ForceFactory::make -> GpuNonbondedForce::evaluate (one pmgpu_evaluate per group) "
                    "-> Vector3DBlock / ScalarStructure, wall clock"}


def measure_batched(local, rank, world, pg, torch, flush, steps):
    """The 96 uneven water boxes (300-9,000 atoms, cutoff 9, PME ~1 A grid),
    sharded over the ranks by atom count; each rank evaluates its shard with
    one graph launch per step.  Compared with the same boxes evaluated one at
    a time (each box's own graph launch, waited for before the next)."""
    from protomol_b200 import forces as F
    from protomol_b200 import workloads
    from protomol_b200.batch import Batch, shard_by_atoms
    ws = workloads.batched96()
    mine = shard_by_atoms([w.system.n_atoms for w in ws], world)[rank]
    batch = Batch(local)
    keep = []
    for k in mine:
        w = ws[k]
        topo = F.Topology(w.system, device=local)
        fs = [F.ForceFactory.make(topo, d, "mixed") for d in w.forces]
        batch.add(topo, fs, w.system.positions)
        keep.append((topo, fs))
    atoms = sum(ws[k].system.n_atoms for k in mine)
    tuning = batch.autotune(evals=3)                  # one tuning for the rank's shard
    bstream = torch.cuda.ExternalStream(batch.stream)
    for _ in range(3):
        batch.evaluate()
    batch.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(bstream):
        for a, b in evs:
            flush.zero_()
            a.record(bstream)
            batch.evaluate()
            b.record(bstream)
    torch.cuda.synchronize()
    batch.synchronize()
    t_batch = float(np.mean([a.elapsed_time(b) for a, b in evs]))
    # one system at a time through the single-system device API
    lib = _lib_load()
    VP = C.c_void_p
    seq = []
    for (topo, fs), (_, _, pos, fout, energy, _) in zip(keep, batch.members):
        arr = (VP * len(fs))(*[f.handle for f in fs])
        seq.append((topo, arr, len(fs), pos, fout, energy))

    def one_by_one():
        for topo, arr, nfs, pos, fout, energy in seq:
            lib.pmgpu_evaluate_device(topo.handle, nfs, arr, VP(pos.data_ptr()), VP(fout.data_ptr()),
                                      VP(energy.data_ptr()), 1)
            lib.pmgpu_synchronize(topo.handle)
    one_by_one()
    reps = max(3, steps // 4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        one_by_one()
    t_seq = (time.perf_counter() - t0) * 1000.0 / reps
    if pg:
        t = torch.tensor([t_batch, t_seq], dtype=torch.float64, device=f"cuda:{local}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        t_batch, t_seq = float(t[0]), float(t[1])
    total_atoms = sum(w.system.n_atoms for w in ws)
    batch.close()
    # like for like: the largest box of the set (same forces, ~9,000 atoms)
    # evaluated alone as one system, CUDA events, L2 flushed between steps
    big = ws[int(np.argmax([w.system.n_atoms for w in ws]))]
    topo = F.Topology(big.system, device=local)
    fs = [F.ForceFactory.make(topo, d, "mixed") for d in big.forces]
    nb = big.system.n_atoms
    dpos = torch.tensor(big.system.positions, dtype=torch.float64, device=f"cuda:{local}")
    dfor = torch.zeros((nb, 3), dtype=torch.float64, device=f"cuda:{local}")
    den = torch.zeros(20, dtype=torch.float64, device=f"cuda:{local}")
    arr = (VP * len(fs))(*[f.handle for f in fs])
    sstream = torch.cuda.ExternalStream(topo.stream)

    def single():
        lib.pmgpu_evaluate_device(topo.handle, len(fs), arr, VP(dpos.data_ptr()), VP(dfor.data_ptr()),
                                  VP(den.data_ptr()), 1)
    for _ in range(5):
        single()
    lib.pmgpu_synchronize(topo.handle)
    sev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    with torch.cuda.stream(sstream):
        for a, b in sev:
            flush.zero_()
            a.record(sstream)
            single()
            b.record(sstream)
    torch.cuda.synchronize()
    lib.pmgpu_synchronize(topo.handle)
    t_single = float(np.mean([a.elapsed_time(b) for a, b in sev]))
    topo.close()
    single_rate = nb * 1000.0 / t_single
    return {"workload": "96 water boxes of 100-3,000 waters, cutoff 9 (C2 8->9), PME ~1 A grid, mixed",
            "single_box": {"atoms": nb, "ms_per_step": t_single, "atom_evals_per_s": single_rate,
                           "what": "the set's largest box with the same forces, evaluated alone"},
            "per_atom_vs_single_box": (total_atoms * 1000.0 / t_batch) / single_rate,
            "systems": len(ws), "atoms": total_atoms, "sharding": f"{world} rank(s), greedy by atom count",
            "ms_per_step": t_batch, "batch_evals_per_s": 1000.0 / t_batch,
            "atom_evals_per_s": total_atoms * 1000.0 / t_batch,
            "one_at_a_time_ms": t_seq, "one_at_a_time_atom_evals_per_s": total_atoms * 1000.0 / t_seq,
            "speedup_vs_one_at_a_time": t_seq / t_batch, "tuning": tuning,
            "timing": "CUDA events on the batch stream (batched, L2 flushed between steps); "
                      "wall clock for one at a time (each box synchronized)"}


def measure_adjoint(local, system, defs, repeat=10):
    """The backward pass (pmgpu_adjoint: dE/dq~, dE/d(LJ table) and the
    Hessian-vector product H v) on the metric system, FP64 and mixed: wall
    clock per call through the host API (positions and v copied in, the
    three gradients copied out), after one warm-up call."""
    from protomol_b200 import forces as F
    rng = np.random.default_rng(5)
    v = rng.normal(size=(system.n_atoms, 3))
    out = {"workload": "chain14281, the metric forces (cutoff pairs over the cell list, PME reciprocal "
                       "+ correction)", "outputs": "dE/dq, dE/dLJ, H v", "calls": repeat}
    for prec in ("fp64", "mixed"):
        topo = F.Topology(system, device=local)
        fs = [F.ForceFactory.make(topo, d, prec) for d in defs]
        F.adjoint(topo, fs, system.positions, v)
        t0 = time.perf_counter()
        for _ in range(repeat):
            F.adjoint(topo, fs, system.positions, v)
        out[prec] = {"ms_per_call": (time.perf_counter() - t0) * 1000.0 / repeat}
        topo.close()
    return out


def _leapfrog_leg(local, torch, s, defs, v, prec, steps, cons=None):
    """One timed Leapfrog run after the autotuner has picked the launch
    chain (on a few hundred atoms it may give the mixed forces the FP64 pair
    kernels, whose chain is shorter)."""
    from protomol_b200 import forces as F
    from protomol_b200 import integrate
    topo = F.Topology(s, device=local)
    fs = [F.ForceFactory.make(topo, d, prec) for d in defs]
    tuned = topo.autotune(fs, s.positions, evals=20, virial=False)
    lf = integrate.Leapfrog(topo, fs, s.positions, v, s.mass, 1.0, device=local, constraints=cons).initialize()
    lf.run(20)                                       # warm-up (graph capture)
    lf.synchronize()
    stream = torch.cuda.ExternalStream(topo.stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    lf.run(steps)
    b.record(stream)
    lf.synchronize()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    topo.close()
    return {"ms_per_step": ms / steps, "steps_per_s": steps * 1000.0 / ms,
            "fp64_pairs": int(tuned["fp64_pairs"])}


def measure_leapfrog(local, torch, steps=1000):
    """GPU-resident Leapfrog (pmgpu_leapfrog_run): one force evaluation plus
    ``steps`` steps of 1 fs on the 216-oxygen LJ fluid (cutoff 9, C2 8 -> 9),
    positions, velocities and forces staying in HBM; CUDA events around the
    run on the system's stream, after the autotuner's pick of each system's
    launch chain."""
    from protomol_b200 import integrate, workloads
    w = workloads.lj_fluid216()
    s = w.system
    v = integrate.maxwell_boltzmann(s.mass, 300.0, seed=216)
    out = {"workload": "216-oxygen LJ fluid (the 648-atom water box without hydrogens), cutoff 9 C2 8->9, "
                       "1 fs steps", "atoms": s.n_atoms, "steps": steps}
    for prec in ("fp64", "mixed"):
        out[prec] = _leapfrog_leg(local, torch, s, w.forces, v, prec, steps)
    # the configuration as stated: the 216 waters rigid (SHAKE after every
    # drift, RATTLE after every step, epsilon 1e-5, 30 sweeps)
    from protomol_b200 import systems
    w = workloads.water216()
    s = w.system
    v = integrate.maxwell_boltzmann(s.mass, 300.0, seed=648)
    atoms, rest = systems.rattle_shake_constraints(s)
    cons = {"atoms": atoms, "rest": rest, "shake": (1e-5, 30), "rattle": (1e-5, 30)}
    rigid = {"workload": "216 rigid TIP3P waters (648 atoms), LJ + Coulomb C2 8->9, SHAKE + RATTLE 1e-5, 1 fs",
             "atoms": s.n_atoms, "steps": steps}
    for prec in ("fp64", "mixed"):
        rigid[prec] = _leapfrog_leg(local, torch, s, w.forces, v, prec, steps, cons)
    out["rigid_water"] = rigid
    return out


def measure_table(local, torch, flush, steps):
    """The 14,281-atom system with the Ewald real part tabulated
    (LennardJones CoulombEwaldRealTable, the look-up table of
    CoulombEwaldRealTableForce) beside the analytic form, both with the PME
    reciprocal + correction force: evaluations/s per precision, L2 flushed
    between evaluations, CUDA events on the system's stream."""
    from protomol_b200 import forces as F
    from protomol_b200 import workloads
    lib = _lib_load()
    w = workloads.chain14281()
    s = w.system
    n = s.n_atoms
    table = ("LennardJones CoulombEwaldRealTable -switchingFunction C2 -algorithm NonbondedCutoff "
             "-switchon 10 -cutoff 12 -cutoff 12 -alpha 0.32 -cutoff 12")
    out = {"workload": "14,281-atom chain in water, LJ C2 10->12 + Ewald real 12 (analytic or tabulated) "
                       "+ PME 64^3", "atoms": n, "table_definition": table}
    dpos = torch.tensor(s.positions, dtype=torch.float64, device=f"cuda:{local}")
    dfor = torch.zeros((n, 3), dtype=torch.float64, device=f"cuda:{local}")
    den = torch.zeros(11, dtype=torch.float64, device=f"cuda:{local}")
    VP = C.c_void_p
    for form, cut in (("analytic", w.forces[0]), ("table", table)):
        for prec in ("mixed", "fp64"):
            topo = F.Topology(s, device=local)
            stream = torch.cuda.ExternalStream(topo.stream)
            fs = [F.ForceFactory.make(topo, d, prec) for d in (cut, w.forces[1])]
            arr = (VP * len(fs))(*[f.handle for f in fs])
            topo.autotune(fs, s.positions, evals=20)

            def step():
                lib.pmgpu_evaluate_device(topo.handle, len(fs), arr, VP(dpos.data_ptr()), VP(dfor.data_ptr()),
                                          VP(den.data_ptr()), 1)
            for _ in range(3):
                step()
            torch.cuda.synchronize()
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(steps)]
            with torch.cuda.stream(stream):
                for a, b in evs:
                    flush.zero_()                  # L2 flush, outside the timed events
                    a.record(stream)
                    step()
                    b.record(stream)
            torch.cuda.synchronize()
            ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
            out.setdefault(form, {})[prec] = {"ms_per_eval": ms, "evals_per_s": 1000.0 / ms}
            for f in fs:
                f.close()
            topo.close()
    return out


def measure_1m(local, torch, steps):
    """The 1,000,000-atom box (cutoff 12, PME 216^3): mixed and FP64
    evaluations/s, pair interactions/s and the PME kernels' HBM rates."""
    from protomol_b200 import forces as F
    from protomol_b200 import workloads
    lib = _lib_load()
    w = workloads.water1m()
    s = w.system
    n = s.n_atoms
    topo = F.Topology(s, device=local)
    stream = torch.cuda.ExternalStream(topo.stream)
    dpos = torch.tensor(s.positions, dtype=torch.float64, device=f"cuda:{local}")
    dfor = torch.zeros((n, 3), dtype=torch.float64, device=f"cuda:{local}")
    den = torch.zeros(11, dtype=torch.float64, device=f"cuda:{local}")
    VP = C.c_void_p
    out = {"workload": "333,333 TIP3P waters + Na+, 215.4 A, LJ C2 10->12 + Ewald real 12 + PME 216^3", "atoms": n}
    for prec in ("mixed", "fp64"):
        fs = [F.ForceFactory.make(topo, d, prec) for d in w.forces]
        arr = (VP * len(fs))(*[f.handle for f in fs])
        if prec == "mixed":
            out["tuning"] = topo.autotune(fs, s.positions, evals=3)

        def step():
            lib.pmgpu_evaluate_device(topo.handle, len(fs), arr, VP(dpos.data_ptr()), VP(dfor.data_ptr()),
                                      VP(den.data_ptr()), 1)
        for _ in range(2):
            step()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        with torch.cuda.stream(stream):
            for a, b in evs:
                a.record(stream)
                step()
                b.record(stream)
        torch.cuda.synchronize()
        ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
        out[prec] = {"ms_per_step": ms, "evals_per_s": 1000.0 / ms}
        if prec == "mixed":
            lib.pmgpu_set_profiling(topo.handle, 1)
            with torch.cuda.stream(stream):
                for _ in range(3):
                    step()
            from protomol_b200 import _lib
            msp = (C.c_double * len(_lib.PHASES))()
            cnt = C.c_longlong(0)
            lib.pmgpu_phase_times(topo.handle, msp, len(_lib.PHASES), C.byref(cnt))
            lib.pmgpu_set_profiling(topo.handle, 0)
            ph = {k: msp[i] / max(1, cnt.value) for i, k in enumerate(_lib.PHASES)}
            # count only (capacity 0: the call reports the count it would need)
            cnt = C.c_longlong(0)
            pos = np.ascontiguousarray(s.positions, np.float64)
            lib.pmgpu_get_pairs(topo.handle, fs[0].handle, pos.ctypes.data_as(VP), C.byref(cnt), None, 0)
            npairs = int(cnt.value)
            out["pairs_within_cutoff"] = npairs
            out["pair_interactions_per_s"] = npairs * 1000.0 / ms
            out["pair_kernel_ms"] = ph["pair"]
            kx = 216
            kzh = kx // 2 + 1
            b = pme_algorithmic_bytes(n, kx)
            out["pme_hbm_gbs"] = {k: v / (ph[k] * 1e-3) / 1e9 for k, v in b.items() if ph.get(k)}
            out["phases_ms"] = ph
            out["trajectory_100"] = measure_1m_trajectory(lib, topo, fs, dpos, dfor, den, stream, torch, npairs)
        for f in fs:
            f.close()
    out["speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    topo.close()
    return out


def measure_1m_trajectory(lib, topo, fs, dpos, dfor, den, stream, torch, npairs, evals=100, every=10, skin=1.0):
    """The large-system configuration as specified: 100 force evaluations of
    a moving configuration with the pair list rebuilt every 10 (a 1 A skin,
    the within-cutoff decision exact at every evaluation).  The positions
    drift along fixed per-molecule directions at up to 0.005 A per
    evaluation (a synthetic trajectory in HBM, updated between the timed
    events): each water moves as a whole, so the molecules keep their
    shape."""
    VP = C.c_void_p
    arr = (VP * len(fs))(*[f.handle for f in fs])
    g = torch.Generator(device=dpos.device).manual_seed(100)
    mol = torch.as_tensor(np.asarray(topo.system.molecule), dtype=torch.long, device=dpos.device)
    nm = int(mol.max().item()) + 1
    um = torch.randn((nm, 3), dtype=torch.float64, device=dpos.device, generator=g)
    um *= 0.005 * torch.rand((nm, 1), dtype=torch.float64, device=dpos.device, generator=g) / um.norm(dim=1,
                                                                                                  keepdim=True)
    u = um[mol]
    base = dpos.clone()
    topo.set_pair_list(skin, every)
    builds0 = topo.pair_list_builds()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(evals)]
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k, (a, b) in enumerate(evs):
            dpos.copy_(base + k * u)                 # between the timed events
            a.record(stream)
            lib.pmgpu_evaluate_device(topo.handle, len(fs), arr, VP(dpos.data_ptr()), VP(dfor.data_ptr()),
                                      VP(den.data_ptr()), 1)
            b.record(stream)
    torch.cuda.synchronize()
    st = lib.pmgpu_synchronize(topo.handle)
    ms = [a.elapsed_time(b) for a, b in evs]
    builds = topo.pair_list_builds() - builds0
    topo.set_pair_list(0.0, 1)
    dpos.copy_(base)
    total = float(np.sum(ms))
    return {"evaluations": evals, "rebuild_every": every, "skin_A": skin, "lists_built": int(builds),
            "status": int(st), "ms_total": total, "evals_per_s": evals * 1000.0 / total,
            "ms_build_evaluation_mean": float(np.mean(ms[::every])),
            "ms_reuse_evaluation_mean": float(np.mean([m for k, m in enumerate(ms) if k % every])),
            "pair_interactions_per_s": npairs * evals * 1000.0 / total}


def _lib_load():
    from protomol_b200 import _lib
    return _lib.load()


def pme_algorithmic_bytes(n, k):
    """Bytes each reciprocal phase must move once, for n atoms on a k^3 grid
    (half spectrum k * k * (k / 2 + 1)): spread reads positions and charges
    (32 B per atom) and writes the int64 charge grid (8 B per point); the FFT
    chain reads that grid, writes and reads the FP32 complex half spectrum
    twice (forward, inverse) and writes the FP32 real grid; the gather reads
    the real grid and the positions and charges and adds three int64 forces
    per atom; the FP64 energy transform reads the charge grid and passes the
    FP64 half spectrum three times."""
    half = k * k * (k // 2 + 1)
    return {"pme_spread": 32 * n + 8 * k ** 3,
            "pme_fft": 8 * k ** 3 + 2 * 2 * 8 * half + 4 * k ** 3,
            "pme_gather": 4 * k ** 3 + 32 * n + 24 * n,
            "pme_energy64": 8 * k ** 3 + 3 * 2 * 16 * half}


def profile_phases(lib, topo, forces, step, flush, stream, torch, steps):
    """Average device milliseconds per evaluation phase: the library records
    CUDA events around each phase on its own stream (profiling mode)."""
    from protomol_b200 import _lib
    _lib.check(lib.pmgpu_set_profiling(topo.handle, 1), topo.handle)
    with torch.cuda.stream(stream):
        for _ in range(steps):
            flush.zero_()
            step(forces)
    ms = (C.c_double * len(_lib.PHASES))()
    n = C.c_longlong(0)
    _lib.check(lib.pmgpu_phase_times(topo.handle, ms, len(_lib.PHASES), C.byref(n)), topo.handle)
    _lib.check(lib.pmgpu_set_profiling(topo.handle, 0), topo.handle)
    evals = max(int(n.value), 1)
    return {name: ms[k] / evals for k, name in enumerate(_lib.PHASES)}


if __name__ == "__main__":
    main()
