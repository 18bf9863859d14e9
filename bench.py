#!/usr/bin/env python
"""Benchmark of the nonbonded hot path inside the MD step: pair interactions per second and
ns/day.  The headline line is the largest single-GPU configuration, the 512-replica LJ argon
ensemble (1,451,403 atoms, N log-uniform 500-8,000 per replica, 80-140 K, dt 5 fs, one
batch); by default the same line carries the 1,048,576-atom LJ slab (90 K) and rigid SPC/E
water (98,304 atoms, 300 K, dt 2 fs) as sub-objects under "configs" (--sub), each measured
the same way.  --workload water|argon|slab|chains|replicas picks another headline.

One step = one engine_step of the whole system (of every replica): re-binning, sort of
every cell along the 13 pair directions, the cell-pair/self sweep with fixed-point force
accumulation and FP64 energy/virial, the symplectic Euler update, the rigid constraints
(P-SHAKE, FP64).  Pairs per step = accepted pairs within the cutoff (excluded pairs not
counted), counted on the device every step.  The sweep's launch shape comes from the
autotuner.

  value   device-resident steps (engine_cuda_resident_steps / engine_batch_resident_steps):
          particles in HBM, one CUDA graph per step; CUDA events recorded on the launching
          stream inside the graph around each step's launches, L2 flushed with a 256 MiB
          write before every step (outside the events).
  e2e     engine_step (engine_batch_step) through the C ABI with host buffers: every step
          the host cells' positions, velocities and ids go up, one device step runs, and
          positions, velocities, forces, ids, energies and statistics come back into the
          host cells.
  plain   the same resident steps with the plain sweep (one block per task, IEEE sqrt/div):
          "tuned vs plain".
  force_eval  the force evaluation alone (sort + sweep) on the same particles, resident
          and through engine_nonbond_cuda with host buffers.
  roofline    the sweep kernel inside the timed resident steps (its own CUDA events).
  force_error after the timed steps, one more force evaluation with the timed launch shape,
          checked against the FP64 oracle on the same particles (per-atom relative error
          distribution, max |dF|/F_rms, energy, exact pair counts); rank 0, one GPU.

Multi-GPU: a single system is not partitioned here ("replicas only"): each rank steps its
own copy of the workload and value = ranks * pairs / max-over-ranks time (weak scaling).
The replica ensemble (--workload replicas) is dealt round-robin over the ranks instead
(rank r steps replicas r, r + N, ...): value = the pairs of all ranks / max-over-ranks time
(strong scaling).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload W]
                  [--sub slab,water]
"""
import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mdcore-history_b200"))

METRIC = "pair interactions/s + ns/day, 1 B200: tuned vs plain at ≤1e-5 rel force err"
UNIT = "pair interactions/s"
FLOPS_PER_PAIR = 45          # FP32 flops per accepted pair (FMA = 2): dx and r^2 8, r 1, interval
                             # index 4, x 2, Horner value+derivative 18, f 2, forces 9, energy 1


def ns_per_day(ms_per_step, dt_fs):
    return dt_fs * 1e-6 * 86400.0 / (ms_per_step * 1e-3)


def _water(W):
    return W.with_rigid_water(W.water_spce(32), 300.0, seed=1)


def _argon(W):
    s = W.argon_fcc(20)
    s.v = W.maxwell_velocities(s, 100.0, seed=1)
    return s


def _slab(W):
    s = W.lj_slab()
    s.v = W.maxwell_velocities(s, 90.0, seed=1)
    return s


def _chains(W):
    return W.chains_water()


def _replicas(W):
    import numpy as np
    out = W.argon_replicas()
    temps = np.random.default_rng(7).uniform(80.0, 140.0, size=len(out))
    for k, s in enumerate(out):
        s.v = W.maxwell_velocities(s, float(temps[k]), seed=100 + k)
    return out


WORKLOADS = {
    "water": ("rigid SPC/E water, 98,304 atoms (32,768 molecules, 98,304 constraints, P-SHAKE) in a 9.9365 nm "
              "periodic box, 9x9x9 cells, cutoff 1.0 nm, 98,304 exclusions, 300 K, dt 2 fs, seeded", _water,
              "sweep_water98k_traffic.txt"),
    "slab": ("LJ liquid slab in vapour, 1,048,576 atoms (80/20 two types) in a 40x40x160 nm box, 40x40x160 cells, "
             "cutoff 1.0 nm, 90 K, dt 5 fs, seeded", _slab, "sweep_slab1m_traffic.txt"),
    "argon": ("LJ argon, 32,000 atoms on a jittered FCC lattice in an 11.5074 nm box, 11^3 cells, cutoff 1.0 nm, "
              "100 K, dt 5 fs, seeded", _argon, "sweep_argon32k_traffic.txt"),
    "replicas": ("512 LJ argon replicas, N log-uniform 500-8,000 (1,451,403 atoms in all), density 18-24 "
                 "atoms/nm^3, cubic periodic boxes, cutoff 1.0 nm, 80-140 K, dt 5 fs, seeded; one batch",
                 _replicas, "sweep_replicas512_traffic.txt"),
    "chains": ("solvated chains, 92,200 atoms: 220 chains of 100 beads (20 LJ types, Lorentz-Berthelot, "
               "charges N(0, 0.3) e neutralised per chain, 1-2 and 1-3 exclusions) and 23,400 3-site waters in "
               "a 10.8 x 10.8 x 7.8 nm box (9 x 9 x 6 cells), cutoff 1.2 nm, 253 type tables and explicit "
               "electrostatics, seeded; force evaluation only",
               _chains, "sweep_chains92k_traffic.txt"),
}
# workloads whose bench step is a force evaluation
FORCE_ONLY = {"chains"}
DEFAULT_WORKLOAD = "replicas"
DEFAULT_SUB = "slab,water"
L2_RULE = "GPU arm: 256 MiB write before every timed step (outside the timed events)"


def build_system(workload):
    import workloads as W
    return WORKLOADS[workload][1](W)


def config_of(workload, systems, pairs):
    """The workload's config object, identical in both arms: what it is, its atoms, and the
    accepted pairs of its initial configuration (the device's count in this arm, the
    oracle's in the reference arm; the two are equal by construction)."""
    return {"workload": WORKLOADS[workload][0], "atoms": int(sum(s.n for s in systems)),
            "pairs_per_step": int(pairs), "l2": L2_RULE}


def host_cpu():
    """lscpu model, sockets and physical cores of this host."""
    info = {"model": None, "sockets": None, "physical_cores": None, "logical_cpus": os.cpu_count()}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, check=True).stdout
        kv = {}
        for ln in out.splitlines():
            if ":" in ln:
                k, v = ln.split(":", 1)
                kv[k.strip()] = v.strip()
        info["model"] = kv.get("Model name")
        sockets = int(kv.get("Socket(s)", "0") or 0)
        cores = int(kv.get("Core(s) per socket", "0") or 0)
        info["sockets"] = sockets or None
        info["physical_cores"] = sockets * cores or None
    except (OSError, subprocess.CalledProcessError, ValueError):
        pass
    return info


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


# ---------------------------------------------------------------- the reference on the host

def run_reference_md(sysm, threads, warmup, steps):
    """The reference's engine_step (oracle/_ref/ref_driver mdbench: its pthreads runners,
    integration, P-SHAKE for rigid systems) on one system; ms per step."""
    import workloads as W
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    with tempfile.TemporaryDirectory() as tmp:
        sysf, rigf = os.path.join(tmp, "system.sys"), os.path.join(tmp, "system.rig")
        W.write_sysfile(sysm, sysf)
        W.write_rigidfile(sysm, rigf, shake=False)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_WAIT_POLICY="PASSIVE")
        r = subprocess.run([exe, "mdbench", sysf, rigf, str(threads), str(warmup), str(steps)], capture_output=True,
                           text=True, env=env, check=True)
    return json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])["ms_per_step"]


_PAIRS = {}


def pair_count(sysm):
    """Accepted pairs of the system's initial configuration (the reference's pair set,
    counted by the oracle)."""
    if sysm.name not in _PAIRS:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import mdcore_b200 as M
        import oracle as O
        tables = [M.create_potential(p).contents.table() for p in sysm.pots]
        _PAIRS[sysm.name] = O.nonbond(sysm, tables)["pairs"]
    return _PAIRS[sysm.name]


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_sample(systems, threads, steps=20, warmup=1, every=16):
    """The reference's engine_step with its pthreads runners on a bounded sample of the
    workload (the whole system, or every `every`-th replica of an ensemble): `warmup`
    untimed steps, then `steps` timed ones; pairs per second over the sample, pairs of the
    initial configurations."""
    sample = systems if len(systems) == 1 else systems[::every]
    try:
        ms = pairs = 0.0
        for s in sample:
            ms += run_reference_md(s, threads, warmup, steps)
            pairs += pair_count(s)
    except (FileNotFoundError, subprocess.CalledProcessError) as exc:
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {exc}"}
    what = ("the full system" if len(systems) == 1 else
            f"{len(sample)} of the {len(systems)} replicas (every {every}th, {int(sum(s.n for s in sample))} atoms)")
    return {"value": pairs / (ms * 1e-3), "unit": UNIT, "cores": threads, "kind": "reference",
            "ms_per_step": ms, "steps": steps, "warmup": warmup, "host": host_cpu(),
            "sample": f"{steps} timed engine_step calls after {warmup} warm-up of {what} on {threads} pthreads "
                      f"runners (reference build in oracle/_ref, P-SHAKE where the system is rigid)"}


def reference_arm(args, rank):
    """The reference's own engine_step with its pthreads CPU runners (oracle/_ref, built from
    the reference sources) on the same workload, all host threads, args.warmup untimed and
    args.steps timed steps of the sample."""
    if rank != 0:
        return
    if args.workload in FORCE_ONLY:
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no per-particle charges "
                          "(engine_setexplepot is stored but never evaluated), so it cannot run this system"}))
        return
    built = build_system(args.workload)
    systems = built if isinstance(built, list) else [built]
    threads = host_threads()
    cb = cpu_sample(systems, threads, steps=args.steps, warmup=args.warmup)
    if cb["value"] is None:
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build failed: {cb['sample']}"}))
        return
    sample_ms = cb.pop("ms_per_step")
    v = cb["value"]
    pairs = sum(pair_count(s) for s in systems)
    ms = pairs / v * 1e3
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "ns_per_day": ns_per_day(ms, systems[0].dt * 1e3),
        "config": config_of(args.workload, systems, pairs),
        "parallelism": f"pthreads runners x{threads}", "sample_ms_per_step": sample_ms,
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def checker_force_error(systems, engines, stats):
    """Checker (outside every timed region; rank 0, one GPU): the forces, energy and pair
    count of the engines' last force evaluation against the FP64 oracle on the same
    particles (cell-relative float positions and cells as the engines hold them)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mdcore_b200 as M
    import oracle as O
    fs, fo = [], []
    epot = pairs = excluded = eabs = 0.0
    t0 = time.time()
    for s, e in zip(systems, engines):
        x, _, _, c = e.parts()
        cdim = np.floor(np.asarray(s.dim) / np.asarray(s.L)).astype(np.int32)
        binned = dict(cdim=cdim, h=np.asarray(s.dim) / cdim, cell=c, xrel=x)
        specs = list(s.pots) + ([s.ep] if getattr(s, "ep", None) is not None else [])
        o = O.nonbond(s, [M.create_potential(p).contents.table() for p in specs], binned=binned)
        fs.append(e.forces())
        fo.append(o["f"])
        epot += o["epot"]
        eabs += o["epot_abs"]
        pairs += o["pairs"]
        excluded += o["excluded"]
    f, f_ref = np.concatenate(fs), np.concatenate(fo)
    d = np.linalg.norm(f - f_ref, axis=1)
    fn = np.linalg.norm(f_ref, axis=1)
    rel = d / np.maximum(fn, 1e-30)
    frms = np.sqrt((f_ref ** 2).sum(1).mean())
    return {"global_rel": float(np.linalg.norm(f - f_ref) / np.linalg.norm(f_ref)),
            "max_over_frms": float(d.max() / frms), "rel_max": float(rel.max()),
            "rel_p99": float(np.percentile(rel, 99)), "rel_median": float(np.median(rel)),
            "frac_over_1e-5": float((rel > 1e-5).mean()),
            "epot_rel": float(abs(stats.epot - epot) / max(abs(epot), 1e-30)),
            "epot_err_over_sum_abs": float(abs(stats.epot - epot) / max(eabs, 1e-30)),
            "pairs_exact": bool(int(stats.pairs) == int(pairs) and int(stats.excluded) == int(excluded)),
            "atoms": int(len(f)), "oracle_s": round(time.time() - t0, 2),
            "what": "after the timed steps: one force evaluation with the timed launch shape vs the FP64 "
                    "oracle (the same float tables, double arithmetic) on the same particles"}


# ---------------------------------------------------------------- this library on the GPU

def reduce_max(values, dist, device):
    """Every rank's timings -> their maxima over the ranks (the max-over-ranks rule for a
    multi-GPU number); values unchanged when there is one rank (dist None)."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def reduce_sum(values, dist, device):
    """Every rank's counts -> their sums over the ranks; unchanged with one rank."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]


def cell_counts(sysm, e):
    """Particles per cell of one engine (cells as space_init lays them out)."""
    import numpy as np
    cdim = np.floor(np.asarray(sysm.dim) / np.asarray(sysm.L)).astype(int)
    return np.bincount(e.cells(), minlength=int(np.prod(cdim)))


def transfer_bytes(systems, engines):
    """Bytes copied per engine_step (device step with the host cells as input and output):
    up, position+type and velocity+id (32 B) per particle, counts and offsets (8 B) per
    cell; down, the step's status and counters (24 B), counts (4 B) per cell, position+upload
    index (16 B), velocity and force (24 B) per particle, offsets up (4 B per cell), cell
    energies and virials (16 B per cell), the 64-byte accumulator block and the constraint
    statistics (8 B per rigid engine).  Also the cell count and whether any cell
    is empty (the queue-compaction launches run then)."""
    n = ncells = nrigid = 0
    empty = False
    for s, e in zip(systems, engines):
        c = cell_counts(s, e)
        n += int(c.sum())
        ncells += len(c)
        empty = empty or bool((c == 0).any())
        nrigid += int(s.rigid is not None and len(s.rigid) > 0)
    h2d = 32 * n + 8 * ncells + 4 + 4 * (ncells + 1)
    d2h = 24 + 4 * ncells + 40 * n + 16 * ncells + 64 + 8 * nrigid
    return h2d, d2h, ncells, empty


def timed_force_evals(tgt, stream, flush, steps, torch):
    """Mean device time (ms) of `steps` device-resident force evaluations (zeroing, sort,
    sweep: CUDA events recorded on the launching stream inside the evaluation's graph), L2
    flushed before each (outside the events), and the mean sweep-kernel time."""
    tot = sweep = 0.0
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        tgt.resident()
        t, s = tgt.kernel_times()
        tot += t
        sweep += s
    return tot / steps, sweep / steps


def timed_resident_steps(tgt, stream, flush, steps, torch):
    """`steps` device-resident MD steps, one call each, L2 flushed before each (outside the
    events): mean step time (ms, CUDA events recorded on the launching stream inside the
    step's graph, first to last launch), mean sweep-kernel time (the sweep's own events),
    accepted pairs summed over the steps."""
    p0 = tgt.resident_info().pairs
    tot = sweep = 0.0
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        tgt.resident_steps(1)
        t, s = tgt.kernel_times()
        tot += t
        sweep += s
    info = tgt.resident_info()
    if info.regrows:
        raise SystemExit("bench.py: device cells were re-blocked inside the timed region")
    return tot / steps, sweep / steps, info.pairs - p0


def read_traffic(workload):
    """dram read + write bytes of one sweep launch, from the committed ncu summary."""
    prof = os.path.join(ROOT, "profiles", WORKLOADS[workload][2])
    if os.path.exists(prof):
        for ln in open(prof):
            if ln.startswith("dram_bytes_per_launch"):
                return int(ln.split()[1])
    return None


def launch_obj(warps, layout, stages, occupancy, tune_ms):
    return {"warps_per_block": warps, "lanes": "8i x 4j" if layout else "32i", "staging_buffers": stages,
            "threads_per_sm": occupancy, "autotune_ms": tune_ms, "cuda_graph": True}


def roofline_obj(M, local_rank, pairs, sweep_ms, layout, workload):
    peak = M.fp32_peak_tflops(local_rank)
    achieved = FLOPS_PER_PAIR * pairs / (sweep_ms * 1e-3) / 1e12
    return {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": read_traffic(workload), "kernel": "sweep_tiled" if layout else "sweep_tuned",
            "kernel_ms": sweep_ms, "flops_per_pair": FLOPS_PER_PAIR,
            "peak_source": "measured FP32 FMA loop on this GPU (engine_cuda_fp32_peak); "
                           "MEASURED_PEAKS.json has no FP32 figure"}


def measure(workload, args, rank, world, local_rank, dist, with_cpu):
    """Everything measured for one workload on this rank; returns the JSON object on rank 0
    (None elsewhere)."""
    import numpy as np
    import torch
    import mdcore_b200 as M

    built = build_system(workload)
    replicas = isinstance(built, list)
    share = replicas and world > 1          # the ensemble dealt round-robin over the ranks
    systems = (built[rank::world] if share else built) if replicas else [built]
    all_systems = built if replicas else [built]
    dt_fs = systems[0].dt * 1e3
    rigid = any(s.rigid is not None and len(s.rigid) for s in systems)
    if replicas:
        engines = [M.Engine.from_system(s, flags=args.engine_flags, start=False) for s in systems]
        tgt = M.Batch(engines, device=local_rank)
    else:
        engines = [M.Engine.from_system(built, flags=args.engine_flags, device=local_rank)]
        tgt = engines[0]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    tgt.set_stream(stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    h2d, d2h, ncells, compact = transfer_bytes(systems, engines)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- warm-up of the host-buffer force evaluation (uploads the particles)
    for _ in range(args.warmup):
        tgt.nonbond()
    st = tgt.stats()
    if st.status != 0:
        raise SystemExit(f"bench.py: device status {st.status}")
    fe_pairs = int(st.pairs)               # accepted pairs of the initial configuration

    # ---- launch shape by the autotuner (or --launch), CUDA-graph replay from here on
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
    # ---- force evaluation alone (sort + sweep), resident and with host buffers
    barrier()
    fe_ms, fe_sweep = timed_force_evals(tgt, stream, flush, args.steps, torch)
    barrier()
    tgt.unload_parts()
    fe_e2e = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        tgt.nonbond()
        ev1.record(stream)
        ev1.synchronize()
        fe_e2e += ev0.elapsed_time(ev1) / args.steps
    barrier()

    force_only = workload in FORCE_ONLY
    pairs_all_init = reduce_sum([fe_pairs], dist, "cuda")[0] if share else fe_pairs
    shake = None
    if force_only:
        # the plain form of the same force evaluation
        tgt.graph(False)
        tgt.tune(0, plain=True)
        tgt.load_parts()
        tgt.resident()
        barrier()
        plain_ms, plain_sweep = timed_force_evals(tgt, stream, flush, args.steps, torch)
        barrier()
        tgt.tune(warps, plain=False)
        tgt.set_layout(layout, stages, occupancy)
        tgt.graph(True)
        clk = clocks.stop()
        if tgt.stats().status != 0:
            raise SystemExit("bench.py: device status after the plain evaluations")
        fe_ms, fe_e2e, fe_sweep, plain_ms = reduce_max([fe_ms, fe_e2e, fe_sweep, plain_ms], dist, "cuda")
        ms, ms_sweep, pairs = fe_ms, fe_sweep, fe_pairs
        pairs_all = world * pairs
        plain_all = pairs_all
    else:
        # ---- MD steps resident in HBM: the headline value
        tgt.resident_begin()
        tgt.resident_steps(max(args.warmup, 25 if rigid else 3))     # past the P-SHAKE refinement steps
        barrier()
        ms, ms_sweep, pairs_timed = timed_resident_steps(tgt, stream, flush, args.steps, torch)
        barrier()
        pairs = pairs_timed / args.steps
        tgt.resident_sync()
        if tgt.stats().status != 0:
            raise SystemExit("bench.py: device status after the resident steps")
        if rigid:
            itmax, bad = engines[0].rigid_stats()
            if bad:
                raise SystemExit("bench.py: rigid groups did not converge")
            shake = itmax

        # ---- the plain sweep in the same resident steps ("tuned vs plain")
        tgt.graph(False)
        tgt.tune(0, plain=True)
        tgt.resident_steps(2)
        barrier()
        plain_ms, plain_sweep, plain_pairs = timed_resident_steps(tgt, stream, flush, args.steps, torch)
        barrier()
        tgt.tune(warps, plain=False)
        tgt.set_layout(layout, stages, occupancy)
        tgt.graph(True)
        tgt.resident_end()

        # ---- engine_step with host buffers through the C ABI (e2e)
        for _ in range(2):
            tgt.step()
        barrier()
        e2e_ms = 0.0
        host = {"pack": 0.0, "device_and_copies": 0.0, "unpack": 0.0}
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            tgt.step()
            ev1.record(stream)
            ev1.synchronize()
            e2e_ms += ev0.elapsed_time(ev1) / args.steps
            hs = tgt.stats()
            host["pack"] += hs.ms_pack / args.steps
            host["device_and_copies"] += hs.ms_device / args.steps
            host["unpack"] += hs.ms_unpack / args.steps
        barrier()
        host_ms = 0.0                       # the host-threaded step, for comparison
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            tgt.step_host()
            ev1.record(stream)
            ev1.synchronize()
            host_ms += ev0.elapsed_time(ev1) / args.steps
        barrier()
        clk = clocks.stop()
        if tgt.stats().status != 0:
            raise SystemExit("bench.py: device status after the host-buffer steps")
        ms, e2e_ms, ms_sweep, plain_ms, fe_ms, fe_e2e, host_ms = reduce_max(
            [ms, e2e_ms, ms_sweep, plain_ms, fe_ms, fe_e2e, host_ms], dist, "cuda")
        if share:
            pairs_all, plain_all = reduce_sum([pairs, plain_pairs / args.steps], dist, "cuda")
        else:
            pairs_all, plain_all = world * pairs, world * (plain_pairs / args.steps)
    fe_all = pairs_all_init if share else world * fe_pairs

    line = None
    if rank == 0:
        config = config_of(workload, all_systems, pairs_all_init if share else fe_pairs)
        parallelism = (f"replicas round-robin over {world} GPUs ({len(systems)} on rank 0)" if share
                       else f"replicas x{world}")
        setup = {"tasks": tgt.ntasks(), "cells": ncells, "candidates_per_step": int(st.candidates),
                 "launch": launch_obj(warps, layout, stages, occupancy, tune_ms)}
        if force_only:
            slots = sum(int((((cell_counts(s, e) + 3) // 4) * 4).sum()) for s, e in zip(systems, engines))
            fe_h2d, fe_d2h = 20 * slots + 4 * (2 * ncells + 1), 12 * slots + 16 * ncells + 64
            line = {
                "metric": METRIC, "value": world * pairs / (fe_ms * 1e-3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": fe_ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "ns_per_day": None,
                "config": config, "parallelism": parallelism,
                "step": "one force evaluation: sort + sweep (engine_nonbond_cuda_resident)", "setup": setup,
                "e2e": {"value": world * pairs / (fe_e2e * 1e-3), "unit": UNIT, "ms_per_step": fe_e2e,
                        "h2d_bytes_per_step": fe_h2d, "d2h_bytes_per_step": fe_d2h,
                        "what": "engine_nonbond_cuda with host buffers: positions and ids up, forces and "
                                "energies down"},
                "roofline": roofline_obj(M, local_rank, pairs, fe_sweep, layout, workload),
                "plain": {"value": world * pairs / (plain_ms * 1e-3), "ms_per_step": plain_ms,
                          "sweep_ms": plain_sweep,
                          "what": "plain form: one block per task, IEEE sqrt/div, per-step warp reductions"},
                "gpu_launches": (2 + 3 * int(compact)) * args.steps,
                "clocks": clk,
            }
        else:
            # kernels of one resident step: re-binning (2), sort, queue compaction (3, systems
            # with empty cells), sweep, integration, constraints (rigid, one per engine)
            # (the update runs inside the constraint kernel when every particle of a single
            # system is in a rigid group)
            fused = (rigid and len(systems) == 1 and
                     len(set(np.asarray(systems[0].rigid)[:, :2].astype(int).ravel().tolist())) == systems[0].n)
            per_step = 2 + 1 + 3 * int(compact) + 1 + int(not fused) + int(rigid) * len(engines)
            line = {
                "metric": METRIC, "value": pairs_all / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "strong" if share else "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "ns_per_day": ns_per_day(ms, dt_fs),
                "config": config, "parallelism": parallelism,
                "pairs_per_step_timed": pairs_all,
                "step": "engine_step on the device: re-binning, sort, sweep, integration"
                        + (", P-SHAKE" if rigid else "") + "; one CUDA graph per step"
                        + ("; Verlet skin (re-binning and sort only on rebuild steps)" if args.verlet else ""),
                "setup": setup,
                "e2e": {"value": pairs_all / (e2e_ms * 1e-3), "unit": UNIT, "ms_per_step": e2e_ms,
                        "ns_per_day": ns_per_day(e2e_ms, dt_fs), "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "host_ms": {k: round(v, 4) for k, v in host.items()},
                        "what": "engine_step (engine_batch_step for the replicas) with the host cells as input "
                                "and output every step"},
                "roofline": roofline_obj(M, local_rank, pairs, ms_sweep, layout, workload),
                "plain": {"value": plain_all / (plain_ms * 1e-3), "ms_per_step": plain_ms,
                          "sweep_ms": plain_sweep,
                          "what": "the same resident steps with the plain sweep: one block per task, IEEE "
                                  "sqrt/div, per-step warp reductions, no graph"},
                "step_host": {"value": pairs_all / (host_ms * 1e-3), "ms_per_step": host_ms,
                              "what": "engine_step_host: re-binning and integration on the host threads, forces "
                                      "and constraints through host buffers"},
                "force_eval": {"value": fe_all / (fe_ms * 1e-3), "ms_per_step": fe_ms, "sweep_ms": fe_sweep,
                               "e2e": {"value": fe_all / (fe_e2e * 1e-3), "ms_per_step": fe_e2e},
                               "what": "sort + sweep alone at the initial positions (engine_nonbond_cuda_resident; "
                                       "e2e: engine_nonbond_cuda with host buffers)"},
                "gpu_launches": per_step * args.steps,
                "clocks": clk,
            }
            if shake is not None:
                line["shake_max_iterations"] = shake
        if with_cpu:
            # checker and CPU baseline, outside every timed region
            tgt.nonbond()
            line["force_error"] = checker_force_error(systems, engines, tgt.stats())
            if force_only:
                line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                        "host": host_cpu(),
                                        "sample": "not run: the reference has no per-particle charges "
                                                  "(engine_setexplepot is stored but never evaluated), so it "
                                                  "cannot run this system"}
            else:
                line["cpu_baseline"] = cpu_sample(systems, host_threads())
                if line["cpu_baseline"]["value"] is not None:     # the same sample on one runner
                    big = sum(s.n for s in systems) > 500_000
                    one = cpu_sample(systems, 1, steps=1 if big else 2, warmup=0 if big else 1)
                    line["cpu_baseline"]["one_core"] = {"value": one["value"], "ms_per_step": one.get("ms_per_step"),
                                                        "sample": one["sample"]}
    tgt.close()
    for e in engines:
        e.close()
    del flush
    torch.cuda.empty_cache()
    return line


def ours(args, rank, world, local_rank):
    import torch

    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    with_cpu = world == 1 and not args.no_cpu_baseline
    line = measure(args.workload, args, rank, world, local_rank, dist, with_cpu)
    # the other large configurations as sub-objects of the same line (one GPU only)
    subs = [w for w in args.sub.split(",") if w and w != args.workload] if world == 1 else []
    if subs:
        configs = {}
        for w in subs:
            sub = measure(w, args, rank, world, local_rank, dist, with_cpu)
            if sub is not None:
                for k in ("metric", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "vs_baseline",
                          "data", "dtype"):
                    sub.pop(k, None)
                configs[w] = sub
        if line is not None:
            line["configs"] = configs
    if line is not None:
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def drift(args, local_rank):
    """The solvated-chain system over args.drift_steps MD steps (dt 2 fs, NVE) from a state
    relaxed on the device (steepest descent, then Maxwell-Boltzmann velocities at 300 K):
    the plain FP32 arm (the plain form, forces accumulated with float atomics) and the
    fixed-point arm (the persistent sweep, 64-bit fixed-point accumulation), from the same
    state; per-atom force errors of each against the FP64 oracle at steps 0, 1,000 and the
    last, and the drift of the total energy."""
    import numpy as np
    import torch
    import workloads as W
    import mdcore_b200 as M
    torch.cuda.set_device(local_rank)
    sysm = build_system(args.workload)
    if isinstance(sysm, list):
        raise SystemExit("bench.py: --drift takes a single system")
    dt_ps = sysm.dt
    # ---- relaxation on the device: steepest descent (rigid water held by the constraints)
    t0 = time.time()
    e = M.Engine.from_system(sysm, device=local_rank)
    e.graph(True)
    e.energy_log(args.min_steps + 8)
    e.resident_begin()
    phases = [(args.min_steps // 4, 2e-6, 0.003), (args.min_steps - args.min_steps // 4, 1e-6, 0.001)]
    for nst, gamma, dmax in phases:
        e.minimize(gamma, dmax)
        e.resident_steps(nst)
    lg = e.energy_log_read(args.min_steps + 8)
    u_start, u_relaxed = float(lg[0, 1]), float(lg[-1, 1])
    e.minimize(0.0)
    e.resident_end()
    x, _, pid, _ = e.unload()
    xr = np.zeros_like(x)
    xr[pid] = x
    e.close()
    relaxed = dataclasses.replace(sysm, x=W.wrap_positions(xr, np.asarray(sysm.dim)))
    relaxed.v = W.maxwell_velocities(relaxed, 300.0, seed=11)
    relax_s = time.time() - t0

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    specs = list(sysm.pots) + ([sysm.ep] if getattr(sysm, "ep", None) is not None else [])
    tables = [M.create_potential(p).contents.table() for p in specs]
    cdim = np.floor(np.asarray(sysm.dim) / np.asarray(sysm.L)).astype(np.int32)

    def errors(eng):
        xrel, _, _, c = eng.parts()
        o = O.nonbond(relaxed, tables, binned=dict(cdim=cdim, h=np.asarray(sysm.dim) / cdim, cell=c, xrel=xrel))
        f, fo = eng.forces(), o["f"]
        d = np.linalg.norm(f - fo, axis=1)
        rel = d / np.maximum(np.linalg.norm(fo, axis=1), 1e-30)
        frms = np.sqrt((fo ** 2).sum(1).mean())
        st = eng.stats()
        return {"global_rel": float(np.linalg.norm(f - fo) / np.linalg.norm(fo)),
                "max_over_frms": float(d.max() / frms), "rel_max": float(rel.max()),
                "rel_p99": float(np.percentile(rel, 99)), "rel_median": float(np.median(rel)),
                "frac_over_1e-5": float((rel > 1e-5).mean()),
                "epot_rel": float(abs(st.epot - o["epot"]) / abs(o["epot"])),
                "pairs_exact": bool(int(st.pairs) == o["pairs"] and int(st.excluded) == o["excluded"])}

    checkpoints = sorted({0, min(1000, args.drift_steps), args.drift_steps})
    arms = {}
    nat = relaxed.n
    ndof = 3 * nat - (len(relaxed.rigid) if relaxed.rigid is not None else 0) - 3
    for arm in ("fp32", "fixed"):
        eng = M.Engine.from_system(relaxed, device=local_rank)
        if arm == "fp32":
            eng.tune(0, plain=True)
            eng.set_accum(True)
        eng.graph(True)
        cap = max(args.drift_steps, 2) + 8
        eng.energy_log(cap)
        logs, errs, done = [], {}, 0
        t_steps = 0.0
        for cp in checkpoints:
            if cp > done:
                eng.resident_begin()
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                ev0.record()
                eng.resident_steps(cp - done)
                ev1.record()
                ev1.synchronize()
                t_steps += ev0.elapsed_time(ev1)
                lg = eng.energy_log_read(cap)
                if len(lg) != cp - done:
                    raise SystemExit(f"bench.py: energy log holds {len(lg)} records, expected {cp - done}")
                lg[:, 0] += done
                logs.append(lg)
                eng.resident_end()
                done = cp
            eng.nonbond()                      # forces at the positions of step `cp`
            errs[str(cp)] = errors(eng)
            if cp > 0:
                itmax, bad = eng.rigid_stats()
                errs[str(cp)]["shake_max_iterations"] = itmax
                errs[str(cp)]["shake_unconverged"] = bad
        log = np.concatenate(logs)
        E, t_ns, slope = M.leapfrog_energy(log, dt_ps)
        K = log[:, 2]
        arms[arm] = {
            "force_error": errs,
            "energy": {"E_first": float(E[0]), "E_last": float(E[-1]), "E_mean": float(E.mean()),
                       "E_std": float(E.std()), "drift_kJ_mol_ns": slope,
                       "drift_per_atom_kJ_mol_ns": slope / nat,
                       "drift_rel_to_K_per_ns": slope / float(abs(K.mean())),
                       "T_mean_K": float(2.0 * K.mean() / (ndof * W.KB)),
                       "U_first": float(log[0, 1]), "U_last": float(log[-1, 1])},
            "ms_per_step": t_steps / max(1, args.drift_steps),
            "what": ("plain form, FP32 float-atomic force accumulation, FP64 energy sums" if arm == "fp32" else
                     "persistent sweep, 64-bit fixed-point force accumulation, FP64 energy sums"),
        }
        eng.close()
    # time-step scan of the fixed-point arm: the drift of a leap-frog integrator limited by
    # its stiffest modes falls as dt^2
    scan = []
    nscan = min(2000, args.drift_steps)
    for dt_fs in [float(v) for v in args.drift_dts.split(",") if v]:
        eng = M.Engine.from_system(dataclasses.replace(relaxed, dt=dt_fs * 1e-3), device=local_rank)
        eng.graph(True)
        eng.energy_log(nscan + 8)
        eng.resident_begin()
        eng.resident_steps(nscan)
        lg = eng.energy_log_read(nscan + 8)
        eng.resident_end()
        itmax, bad = eng.rigid_stats()
        eng.close()
        _, _, sl = M.leapfrog_energy(lg, dt_fs * 1e-3)
        scan.append({"dt_fs": dt_fs, "steps": nscan, "drift_per_atom_kJ_mol_ns": sl / nat,
                     "T_mean_K": float(2.0 * lg[:, 2].mean() / (ndof * W.KB)),
                     "shake_max_iterations": itmax, "shake_unconverged": bad})
    # run-to-run reproducibility: each arm twice over the same steps from the same state
    nrep = min(1000, args.drift_steps)
    for arm in ("fp32", "fixed"):
        runs = []
        for _ in range(2):
            eng = M.Engine.from_system(relaxed, device=local_rank)
            if arm == "fp32":
                eng.tune(0, plain=True)
                eng.set_accum(True)
            eng.graph(True)
            eng.resident_begin()
            eng.resident_steps(nrep)
            eng.resident_end()
            xx, _, pp, _ = eng.unload()
            xs = np.zeros_like(xx)
            xs[pp] = xx
            runs.append(xs)
            eng.close()
        d = runs[1] - runs[0]
        d -= np.round(d / np.asarray(sysm.dim)) * np.asarray(sysm.dim)
        arms[arm]["repeat"] = {"steps": nrep, "bit_identical": bool(np.array_equal(runs[0], runs[1])),
                               "max_dx_nm": float(np.abs(d).max())}
    print(json.dumps({
        "drift": WORKLOADS[args.workload][0].replace("; force evaluation only", ""), "atoms": nat, "dof": ndof, "steps": args.drift_steps,
        "dt_fs": dt_ps * 1e3, "ensemble": "NVE after relaxation",
        "relaxation": {"steepest_descent_steps": args.min_steps, "phases": phases, "U_first": u_start,
                       "U_relaxed": u_relaxed,
                       "velocities": "Maxwell-Boltzmann 300 K (seed 11), net momentum removed", "s": round(relax_s, 2)},
        "checkpoints": checkpoints, "arms": arms, "dt_scan_fixed_point": scan,
        "oracle": "FP64 restatement on the same float tables and positions (the checker)",
    }))


def sched_ab(args, local_rank):
    """The learned scheduler's protocol on one system (default: the slab): clock64 task
    timings recorded over the first args.record device-resident MD steps, the cost network
    trained on them (its own GPU kernels), then args.sched_steps MD steps from the same state
    with each queue order -- the count-product heuristic longest-first (the reference's), the network's
    longest-first order, both orders in locality tiles (cost classes, cell-major within a
    class), and the cell-major order tasks are generated in -- and, for scale, the plain form.
    Makespan = device time of the steps (CUDA events around the whole run) / steps."""
    import numpy as np
    import torch
    import mdcore_b200 as M
    torch.cuda.set_device(local_rank)
    sysm = build_system(args.workload)
    if isinstance(sysm, list):
        raise SystemExit("bench.py: --sched-ab takes a single system (water, argon or slab)")
    e = M.Engine.from_system(sysm, flags=args.engine_flags, device=local_rank)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    e.set_stream(stream.cuda_stream)
    for _ in range(args.warmup):
        e.nonbond()
    e.load_parts()
    warps, layout, stages, occupancy, _ = e.autotune(reps=3)
    e.graph(True)
    e.resident_begin()
    t0 = time.time()
    e.sched_record(args.record)                  # the first MD steps, timed per task
    X = e.sched_features()
    y = e.sched_targets()
    t1 = time.time()
    loss = e.sched_train(epochs=args.epochs, batch=512, lr=3e-3, seed=1)
    train_s = time.time() - t1
    pred = e.sched_predict()
    # every order starts from the state after the recorded steps (host copy, re-uploaded)
    e.resident_sync()
    ntasks = e.ntasks()
    # every order computed now, from the state after the recorded steps
    orders = []
    for name, make in [("count_product", lambda: e.sched_apply(False)),
                       ("learned", lambda: e.sched_apply(True)),
                       ("learned_tiled", lambda: e.sched_order(1, 0)),
                       ("count_product_tiled", lambda: e.sched_order(0, 0)),
                       ("cell_major", lambda: e.set_order(np.arange(ntasks)))]:
        make()
        orders.append((name, e.get_order()))
    res = {}

    def run(nsteps):
        e.resident_begin()
        e.resident_steps(3)                      # direct launch, capture, replay
        p0 = e.resident_info().pairs
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        e.resident_steps(nsteps)
        ev1.record(stream)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1) / nsteps
        pairs = (e.resident_info().pairs - p0) / nsteps
        if e.stats().status != 0:
            raise SystemExit("bench.py: device status in the scheduled steps")
        return {"ms_per_step": ms, "pairs_per_s": pairs / (ms * 1e-3)}

    clocks = ClockSampler(local_rank)
    clocks.start()
    for name, order in orders:
        e.set_order(order)
        res[name] = run(args.sched_steps)
    e.sched_apply(False)
    e.tune(0, plain=True)
    res["plain_form"] = run(max(1, args.sched_steps // 10))
    clk = clocks.stop()
    e.resident_end()
    nz = y > 0
    best = min((k for k in res if k != "plain_form"), key=lambda k: res[k]["ms_per_step"])
    print(json.dumps({"sched_ab": WORKLOADS[args.workload][0], "tasks": ntasks,
                      "protocol": {"record_md_steps": args.record, "scheduled_md_steps": args.sched_steps,
                                   "plain_form_steps": max(1, args.sched_steps // 10),
                                   "start": "every order from the state after the recorded steps"},
                      "makespan": res, "fastest": best,
                      "learned_vs_count_product": res["count_product"]["ms_per_step"] / res["learned_tiled"]["ms_per_step"],
                      "learned_tiled_vs_cell_major": res["cell_major"]["ms_per_step"] / res["learned_tiled"]["ms_per_step"],
                      "launch": {"warps_per_block": warps, "lanes": "8i x 4j" if layout else "32i",
                                 "staging_buffers": stages, "threads_per_sm": occupancy},
                      "epochs": args.epochs, "train_s": round(train_s, 3), "record_s": round(t1 - t0, 3),
                      "train_mse": loss, "corr_pred_target": float(np.corrcoef(pred[nz], y[nz])[0, 1]),
                      "clocks": clk}))
    e.close()


def profile_steps(args):
    """--profile-steps K: the workload's device-resident steps alone (upload, K steps,
    download), so that an ncu launch list or a capture of one kernel sees only the step's
    kernels."""
    import mdcore_b200 as M
    built = build_system(args.workload)
    systems = built if isinstance(built, list) else [built]
    if isinstance(built, list):
        engines = [M.Engine.from_system(s, flags=args.engine_flags, start=False) for s in systems]
        tgt = M.Batch(engines, device=0)
    else:
        engines = [M.Engine.from_system(built, flags=args.engine_flags, device=0)]
        tgt = engines[0]
    warps, layout, stages, occupancy = (int(v) for v in ((args.launch or "8,1,1") + ",1024").split(",")[:4])
    tgt.tune(warps)
    tgt.set_layout(layout, stages, occupancy)
    tgt.graph(True)
    tgt.resident_begin()
    tgt.resident_steps(args.profile_steps)
    tgt.resident_sync()
    status = tgt.stats().status
    tgt.resident_end()
    if status != 0:
        raise SystemExit(f"bench.py: device status {status}")
    print(json.dumps({"profile_steps": args.profile_steps, "workload": args.workload,
                      "launch": [warps, layout, stages, occupancy], "status": status}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU reference sample")
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS),
                    help="headline workload: replicas (default, the largest single-GPU configuration), slab, "
                         "water, argon or chains")
    ap.add_argument("--sub", default=None,
                    help="comma-separated workloads measured as sub-objects of the same line (one GPU only); "
                         f"default {DEFAULT_SUB} with the default workload, none otherwise")
    ap.add_argument("--launch", default="",
                    help="fixed persistent launch shape warps,layout,stages[,threads per SM] (e.g. 4,1,1,640) "
                         "instead of the autotuner")
    ap.add_argument("--sched-ab", action="store_true",
                    help="train the task-cost model and compare sweep makespans of the queue orders")
    ap.add_argument("--record", type=int, default=200, help="--sched-ab: MD steps of task timings to train on")
    ap.add_argument("--sched-steps", type=int, default=5000, help="--sched-ab: MD steps timed per queue order")
    ap.add_argument("--epochs", type=int, default=150, help="--sched-ab: training epochs")
    ap.add_argument("--drift", action="store_true",
                    help="energy drift and force errors over an MD trajectory of --workload (default chains): "
                         "plain FP32 accumulation vs fixed point, against the FP64 oracle")
    ap.add_argument("--drift-steps", type=int, default=10000, help="--drift: MD steps")
    ap.add_argument("--min-steps", type=int, default=2000, help="--drift: steepest-descent steps first")
    ap.add_argument("--drift-dts", default="2,1,0.5", help="--drift: time steps (fs) of the fixed-point dt scan")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="only K device-resident steps of --workload with the --launch shape (default "
                         "8,1,1,1024), nothing timed: the command for ncu captures of the step's kernels")
    ap.add_argument("--verlet", action="store_true",
                    help="engine_flag_verlet_pseudo: the resident steps re-bin and sort only when the largest "
                         "displacement exceeds half the skin (min h - cutoff)")
    args = ap.parse_args()
    import mdcore_b200 as M
    args.engine_flags = M.engine_flag_cuda | (M.engine_flag_verlet_pseudo if args.verlet else 0)
    if args.sub is None:
        args.sub = DEFAULT_SUB if args.workload == DEFAULT_WORKLOAD else ""
    if args.sched_ab:
        if "--workload" not in sys.argv:
            args.workload = "slab"
        sched_ab(args, int(os.environ.get("LOCAL_RANK", 0)))
        return
    if args.drift:
        if "--workload" not in sys.argv:
            args.workload = "chains"
        drift(args, int(os.environ.get("LOCAL_RANK", 0)))
        return
    if args.profile_steps > 0:
        profile_steps(args)
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
