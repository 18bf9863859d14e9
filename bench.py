#!/usr/bin/env python
"""Benchmark of the nonbonded hot path: pair interactions per second on rigid SPC/E water
(98,304 atoms, 9^3 cells, cutoff 1.0 nm, 3 exclusions per molecule) by default; also LJ
argon (32,000 atoms), the 1,048,576-atom LJ slab and the 512-replica argon ensemble
(--workload argon|slab|replicas).

One step = one nonbonded force evaluation of the whole system (of every replica): sort every
cell along the 13 pair directions, sweep all cell-pair/self tasks, fixed-point force
accumulation, FP64 energy and virial.  The launch shape comes from the autotuner and every
evaluation replays a CUDA graph of its launches.

  value   device-resident: positions already in HBM, kernels only (CUDA events around each
          step on the launching stream; L2 flushed with a 256 MiB write before every step,
          outside the events).
  e2e     the C-ABI call engine_nonbond_cuda (engine_batch_nonbond for the replicas) with
          host buffers: packing the cells, one host->device copy of positions/ids/cell
          offsets, sort + sweep, one device->host copy of forces and energies, unpacking.
  plain   the plain form (one block per task) on the same protocol; for the replicas also
          the ensemble evaluated as 512 sequential single-engine plain runs.

Multi-GPU: the path is not partitioned here ("replicas only"): each rank evaluates its own
copy of the workload and value = ranks * pairs / max-over-ranks time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload W]
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mdcore-history_b200"))

METRIC = "pair interactions/s + ns/day, 1 B200: tuned vs plain at ≤1e-5 rel force err"
UNIT = "pair interactions/s"
FLOPS_PER_PAIR = 45          # per accepted pair, FMA = 2 (roofline)
DT_FS = 2.0


def ns_per_day(ms_per_step):
    return DT_FS * 1e-6 * 86400.0 / (ms_per_step * 1e-3)


WORKLOADS = {
    "water": ("rigid SPC/E water, 98,304 atoms (32,768 molecules) in a 9.9365 nm periodic box, 9x9x9 cells, "
              "cutoff 1.0 nm, 98,304 exclusions, seeded", lambda W: W.water_spce(32),
              "sweep_water98k_traffic.txt"),
    "slab": ("LJ liquid slab in vapour, 1,048,576 atoms (80/20 two types) in a 40x40x160 nm box, 40x40x160 cells, "
             "cutoff 1.0 nm, seeded", lambda W: W.lj_slab(), "sweep_slab1m_traffic.txt"),
    "argon": ("LJ argon, 32,000 atoms on a jittered FCC lattice in an 11.5074 nm box, 11^3 cells, cutoff 1.0 nm, "
              "seeded", lambda W: W.argon_fcc(20), "sweep_argon32k_traffic.txt"),
    "replicas": ("512 LJ argon replicas, N log-uniform 500-8,000 (1,451,403 atoms in all), density 18-24 "
                 "atoms/nm^3, cubic periodic boxes, cutoff 1.0 nm, seeded; one batch", lambda W: W.argon_replicas(),
                 "sweep_replicas512_traffic.txt"),
}
SELECTED = "water"


def build_system():
    import workloads as W
    return WORKLOADS[SELECTED][1](W)


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.out = None

    def start(self):
        try:
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.strip()]
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) >= 9:
                for k, n in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def run_reference_driver(sysm, threads, warmup, steps):
    import workloads as W
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    with tempfile.TemporaryDirectory() as tmp:
        sysf = os.path.join(tmp, "system.sys")
        W.write_sysfile(sysm, sysf)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_WAIT_POLICY="PASSIVE")
        r = subprocess.run([exe, "bench", sysf, str(threads), str(warmup), str(steps)], capture_output=True,
                           text=True, env=env, check=True)
    line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
    return json.loads(line)


def run_reference_md(threads, warmup, steps):
    """The reference's engine_step on rigid SPC/E water (P-SHAKE, dt = 2 fs), all runners."""
    import workloads as W
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    sysm = W.with_rigid_water(W.water_spce(32), 300.0, seed=1)
    with tempfile.TemporaryDirectory() as tmp:
        sysf, rigf = os.path.join(tmp, "water.sys"), os.path.join(tmp, "water.rig")
        W.write_sysfile(sysm, sysf)
        W.write_rigidfile(sysm, rigf, shake=False)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_WAIT_POLICY="PASSIVE")
        r = subprocess.run([exe, "mdbench", sysf, rigf, str(threads), str(warmup), str(steps)], capture_output=True,
                           text=True, env=env, check=True)
    d = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    return {"ms_per_step": d["ms_per_step"], "ns_per_day": ns_per_day(d["ms_per_step"]), "steps": steps,
            "cores": threads, "what": "reference engine_step of rigid SPC/E water (P-SHAKE), pthreads runners"}


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_sample(systems, threads, steps=5, every=16):
    """The reference's pthreads CPU runner on a bounded sample of the workload: the whole
    system, or every `every`-th replica of an ensemble; pairs per second over the sample."""
    sample = systems if len(systems) == 1 else systems[::every]
    try:
        ms = pairs = 0.0
        for s in sample:
            r = run_reference_driver(s, threads, 1, steps)
            ms += r["ms_per_step"]
            pairs += pair_count(s)
    except (FileNotFoundError, subprocess.CalledProcessError) as exc:
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {exc}"}
    what = ("the full system" if len(systems) == 1 else
            f"{len(sample)} of the {len(systems)} replicas (every {every}th, {int(sum(s.n for s in sample))} atoms)")
    return {"value": pairs / (ms * 1e-3), "unit": UNIT, "cores": threads, "kind": "reference",
            "ms_per_step": ms, "sample": f"{steps} engine_step calls (dt=0) of {what} on {threads} pthreads runners, "
                                        f"reference build in oracle/_ref"}


def reference_arm(args, rank):
    """The reference's own pthreads CPU runner (oracle/_ref, built from the reference
    sources) on the same workload, all host threads."""
    if rank != 0:
        return
    built = build_system()
    systems = built if isinstance(built, list) else [built]
    threads = host_threads()
    steps = max(1, min(args.steps, 20 if len(systems) == 1 else 3))
    cb = cpu_sample(systems, threads, steps=steps)
    if cb["value"] is None:
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build failed: {cb['sample']}"}))
        return
    ms = cb.pop("ms_per_step")
    v = cb["value"]
    pairs = sum(pair_count(s) for s in systems)
    md = None
    if SELECTED == "water":
        try:
            md = run_reference_md(threads, 2, max(2, min(args.steps, 10)))
        except (FileNotFoundError, subprocess.CalledProcessError) as exc:
            md = {"unavailable": str(exc)}
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": 1, "ms_per_step": pairs / v * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "ns_per_day": ns_per_day(pairs / v * 1e3),
        "config": {"workload": WORKLOADS[SELECTED][0], "pairs_per_step": pairs, "parallelism": "pthreads runners",
                   "sample_ms_per_step": ms},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        **({"md_step": md} if md is not None else {}),
    }))


_PAIRS = {}


def pair_count(sysm):
    """Pairs per step of the workload (the reference's pair set, counted by the oracle)."""
    if sysm.name not in _PAIRS:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import mdcore_b200 as M
        import oracle as O
        tables = [M.create_potential(p).contents.table() for p in sysm.pots]
        _PAIRS[sysm.name] = O.nonbond(sysm, tables)["pairs"]
    return _PAIRS[sysm.name]


def cell_counts(sysm, e):
    """Particles per cell of one engine (cells as space_init lays them out)."""
    import numpy as np
    cdim = np.floor(np.asarray(sysm.dim) / np.asarray(sysm.L)).astype(int)
    return np.bincount(e.cells(), minlength=int(np.prod(cdim)))


def transfer_bytes(systems, engines):
    """Bytes copied per host-buffer evaluation: positions+types and ids per padded slot and
    the cell offsets/counts up; float forces per slot, cell energies and virials and the
    counters down."""
    slots = ncells = 0
    for s, e in zip(systems, engines):
        c = cell_counts(s, e)
        slots += int((((c + 3) // 4) * 4).sum())
        ncells += len(c)
    return 20 * slots + 4 * (2 * ncells + 1), 12 * slots + 16 * ncells + 64, ncells, \
        any((cell_counts(s, e) == 0).any() for s, e in zip(systems, engines))


def timed_resident(tgt, stream, flush, steps, torch):
    """Mean device time (ms) of `steps` device-resident evaluations, L2 flushed before
    each (outside the events), and the mean sweep-kernel time."""
    tot = sweep = 0.0
    for _ in range(steps):
        flush.zero_()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        tgt.resident()
        ev1.record(stream)
        ev1.synchronize()
        tot += ev0.elapsed_time(ev1)
        sweep += tgt.kernel_times()[1]
    return tot / steps, sweep / steps


def ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import mdcore_b200 as M

    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    built = build_system()
    replicas = isinstance(built, list)
    systems = built if replicas else [built]
    if replicas:
        engines = [M.Engine.from_system(s, start=False) for s in systems]
        tgt = M.Batch(engines, device=local_rank)
    else:
        engines = [M.Engine.from_system(built, device=local_rank)]
        tgt = engines[0]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    tgt.set_stream(stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # warm-up (host-buffer path, which also uploads the particles)
    for _ in range(args.warmup):
        tgt.nonbond()
    st = tgt.stats()
    if st.status != 0:
        raise SystemExit(f"bench.py: device status {st.status}")
    pairs = int(st.pairs)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- launch shape by the autotuner (or --launch), then CUDA-graph replay of every evaluation
    tgt.load_parts()
    if args.launch:
        warps, layout, stages, occupancy = (int(v) for v in (args.launch + ",640").split(",")[:4])
        tgt.tune(warps)
        tgt.set_layout(layout, stages, occupancy)
        tune_ms = None
    else:
        warps, layout, stages, occupancy, tune_ms = tgt.autotune(reps=3)
    tgt.graph(True)
    for _ in range(3):                   # direct launch, capture, first replay
        tgt.resident()

    clocks = ClockSampler(local_rank)
    clocks.start()

    # ---- device-resident timed region
    barrier()
    ms, ms_sweep = timed_resident(tgt, stream, flush, args.steps, torch)
    barrier()
    tgt.unload_parts()
    if tgt.stats().status != 0:
        raise SystemExit("bench.py: device status after timed region")

    # ---- end-to-end timed region (host buffers through the C ABI, graph replay)
    barrier()
    e2e_ms = 0.0
    host = {"pack": 0.0, "device": 0.0, "unpack": 0.0}
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        tgt.nonbond()
        ev1.record(stream)
        ev1.synchronize()
        e2e_ms += ev0.elapsed_time(ev1)
        hs = tgt.stats()
        host["pack"] += hs.ms_pack / args.steps
        host["device"] += hs.ms_device / args.steps
        host["unpack"] += hs.ms_unpack / args.steps
    barrier()
    clk = clocks.stop()
    if tgt.stats().status != 0:
        raise SystemExit("bench.py: device status after e2e region")

    # ---- water: full MD steps (engine_step: rebin, forces, integration, P-SHAKE on the
    # device) of the rigid SPC/E system, dt = 2 fs
    md = None
    if SELECTED == "water":
        import workloads as W
        rig = M.Engine.from_system(W.with_rigid_water(W.water_spce(32), 300.0, seed=1), device=local_rank)
        rig.set_stream(stream.cuda_stream)
        rig.load_parts()
        rig.tune(warps)
        rig.set_layout(layout, stages, occupancy)
        rig.graph(True)
        for _ in range(max(args.warmup, 25)):        # past the 20 P-SHAKE refinement steps
            rig.step()
        barrier()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            rig.step()
        ev1.record(stream)
        ev1.synchronize()
        md_ms = ev0.elapsed_time(ev1) / args.steps
        itmax, bad = rig.rigid_stats()
        if rig.stats().status != 0 or bad != 0:
            raise SystemExit("bench.py: rigid water steps failed")
        md = {"ms_per_step": md_ms, "ns_per_day": ns_per_day(md_ms), "dt_fs": DT_FS,
              "what": "engine_step of rigid SPC/E water (32,768 molecules, 98,304 constraints): rebin, "
                      "forces with host buffers, symplectic Euler, P-SHAKE on the device (FP64)",
              "shake_max_iterations": itmax}
        # the same MD steps with the particles resident on the device: re-binning,
        # forces, integration and P-SHAKE as one CUDA graph per step, no host copies
        rig.resident_begin()
        rig.resident_steps(max(args.warmup, 3))
        barrier()
        ev0.record(stream)
        rig.resident_steps(args.steps)
        ev1.record(stream)
        ev1.synchronize()
        res_ms = ev0.elapsed_time(ev1) / args.steps
        rig.resident_sync()
        itmax, bad = rig.rigid_stats()
        if rig.stats().status != 0 or bad != 0:
            raise SystemExit("bench.py: resident rigid water steps failed")
        md["resident"] = {"ms_per_step": res_ms, "ns_per_day": ns_per_day(res_ms),
                          "what": "engine_cuda_resident_steps: the same steps with the particles resident "
                                  "in HBM, one CUDA graph per step",
                          "shake_max_iterations": itmax}
        rig.resident_end()
        rig.close()

    # ---- the plain form (one CTA per task, IEEE sqrt/div, no graph), same protocol
    tgt.graph(False)
    tgt.tune(0, plain=True)
    tgt.load_parts()
    tgt.resident()
    barrier()
    plain_ms, plain_sweep = timed_resident(tgt, stream, flush, args.steps, torch)
    barrier()
    tgt.tune(warps, plain=False)

    # ---- replicas: the same ensemble as sequential single-engine runs of the plain form
    seq = None
    if replicas:
        singles = [M.Engine.from_system(s, device=local_rank) for s in systems]
        for e in singles:
            e.set_stream(stream.cuda_stream)
            e.tune(0, plain=True)
            e.load_parts()
            e.resident()
        barrier()
        seq_ms = 0.0
        for _ in range(args.steps):
            flush.zero_()
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            for e in singles:
                e.resident()
            ev1.record(stream)
            ev1.synchronize()
            seq_ms += ev0.elapsed_time(ev1)
        barrier()
        seq_ms /= args.steps
        seq = {"value": world * pairs / (seq_ms * 1e-3), "ms_per_step": seq_ms,
               "what": f"{len(singles)} sequential single-engine evaluations of the plain form, device-resident"}
        for e in singles:
            e.close()

    if dist is not None:
        t = torch.tensor([ms, e2e_ms / args.steps, ms_sweep], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e, ms_sweep = [float(v) for v in t.tolist()]
    else:
        ms_e2e = e2e_ms / args.steps
    if rank == 0:
        h2d, d2h, ncells, compact = transfer_bytes(systems, engines)
        peak = M.fp32_peak_tflops(local_rank)
        achieved = FLOPS_PER_PAIR * pairs / (ms_sweep * 1e-3) / 1e12
        traffic = None
        prof = os.path.join(ROOT, "profiles", WORKLOADS[SELECTED][2])
        if os.path.exists(prof):       # dram read + write bytes of one sweep launch, from ncu
            for ln in open(prof):
                if ln.startswith("dram_bytes_per_launch"):
                    traffic = int(ln.split()[1])
        line = {
            "metric": METRIC, "value": world * pairs / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "ns_per_day": ns_per_day(ms),
            "config": {"workload": WORKLOADS[SELECTED][0], "atoms": int(sum(s.n for s in systems)),
                       "pairs_per_step": pairs, "candidates_per_step": int(st.candidates),
                       "tasks": tgt.ntasks(), "cells": ncells, "parallelism": f"replicas x{world}",
                       "launch": {"warps_per_block": warps, "lanes": "8i x 4j" if layout else "32i",
                                  "staging_buffers": stages, "threads_per_sm": occupancy, "autotune_ms": tune_ms,
                                  "cuda_graph": True},
                       "l2": "256 MiB write before every timed step (outside the timed events)"},
            "e2e": {"value": world * pairs / (ms_e2e * 1e-3), "unit": UNIT, "ms_per_step": ms_e2e,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "host_ms": {k: round(v, 4) for k, v in host.items()}},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "sweep_tiled" if layout else "sweep_tuned", "kernel_ms": ms_sweep,
                         "peak_source": "measured FP32 FMA loop on this GPU (engine_cuda_fp32_peak); "
                                        "MEASURED_PEAKS.json has no FP32 figure"},
            "plain": {"value": world * pairs / (plain_ms * 1e-3), "ms_per_step": plain_ms,
                      "sweep_ms": plain_sweep,
                      "what": "plain form: one block per task, IEEE sqrt/div, per-step warp reductions"},
            "gpu_launches": (2 + 3 * int(compact)) * args.steps,
            "clocks": clk,
        }
        if seq is not None:
            line["sequential_plain"] = seq
        if md is not None:
            line["md_step"] = md
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_sample(systems, host_threads())
            if md is not None:
                try:
                    line["cpu_baseline"]["md_step"] = run_reference_md(host_threads(), 2, 5)
                except (FileNotFoundError, subprocess.CalledProcessError) as exc:
                    line["cpu_baseline"]["md_step"] = {"unavailable": str(exc)}
        print(json.dumps(line))
    tgt.close()
    for e in engines:
        e.close()
    if dist is not None:
        dist.destroy_process_group()


def sched_ab(args, local_rank):
    """Makespan of the sweep with the count-product order, the learned order, a random order
    and the cell-major order tasks are generated in (same workload, autotuned launch shape,
    device-resident, CUDA events, L2 flushed before every step)."""
    import numpy as np
    import torch
    import mdcore_b200 as M
    torch.cuda.set_device(local_rank)
    sysm = build_system()
    if isinstance(sysm, list):
        raise SystemExit("bench.py: --sched-ab takes a single system (water, argon or slab)")
    e = M.Engine.from_system(sysm, device=local_rank)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    e.set_stream(stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        e.nonbond()
    e.load_parts()
    warps, layout, stages, occupancy, _ = e.autotune(reps=3)
    t0 = time.time()
    e.sched_record(args.record)
    X = e.sched_features()
    y = e.sched_targets()
    loss = e.sched_train(epochs=args.epochs, batch=512, lr=3e-3, seed=1)
    train_s = time.time() - t0
    pred = e.sched_predict()

    def timed(order_name):
        e.resident()
        torch.cuda.synchronize()
        sweeps = []
        for _ in range(args.steps):
            flush.zero_()
            e.resident()
            sweeps.append(e.kernel_times()[1])
        return float(np.median(sweeps))

    res = {}
    e.sched_apply(False)
    res["count_product"] = timed("heuristic")
    e.sched_apply(True)
    res["learned"] = timed("mlp")
    e.set_order(np.random.default_rng(0).permutation(e.ntasks()))
    res["random"] = timed("random")
    e.set_order(np.arange(e.ntasks()))           # tasks as generated: cell-major (L2 locality)
    res["cell_order"] = timed("cells")
    e.tune(0, plain=True)
    res["plain_form"] = timed("plain")
    nz = y > 0
    print(json.dumps({"sched_ab": WORKLOADS[SELECTED][0], "sweep_ms_median": res, "tasks": e.ntasks(),
                      "launch": {"warps_per_block": warps, "lanes": "8i x 4j" if layout else "32i",
                                 "staging_buffers": stages, "threads_per_sm": occupancy},
                      "record_steps": args.record, "epochs": args.epochs, "train_s": round(train_s, 3),
                      "train_mse": loss, "corr_pred_target": float(np.corrcoef(pred[nz], y[nz])[0, 1])}))
    e.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU reference sample")
    ap.add_argument("--workload", default="water", choices=sorted(WORKLOADS),
                    help="water (default: the headline configuration), argon, slab or replicas")
    ap.add_argument("--launch", default="",
                    help="fixed persistent launch shape warps,layout,stages[,threads per SM] (e.g. 4,1,1,640) "
                         "instead of the autotuner")
    ap.add_argument("--sched-ab", action="store_true",
                    help="train the task-cost model and compare sweep makespans of the queue orders")
    ap.add_argument("--record", type=int, default=4, help="--sched-ab: steps of task timings to train on")
    ap.add_argument("--epochs", type=int, default=150, help="--sched-ab: training epochs")
    args = ap.parse_args()
    global SELECTED
    SELECTED = args.workload
    if args.sched_ab:
        sched_ab(args, int(os.environ.get("LOCAL_RANK", 0)))
        return
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
