"""Throughput of the DSMC time step on B200, and the reference's CPU arm.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--spinup S]
                    [--impl ours|reference] [--wall diffuse|cll]
                    [--precision fp32|fp64]

Workload: the HBM-roofline case - 1000x1000 cells on [-20, 20]^2 m, NPCFree 20
(~2e7 particles), angle of attack 10 deg, diffuse walls at Tw 300 K (or CLL
0.8/0.8), Dt 1e-6 s, FP32 particle state with FP64 hit times, inflow counts and
moment accumulators, sampling every step.  Particles and cells are
generated by the engine's own cold start (seeded Philox), so the data is
synthetic by construction.  A "step" is one full DSMC time step: move + wall
scattering, inflow, removal, cell sort, NTC collisions and moment sampling.

The run first spins the flow up for S steps (default 10000, the step the
case's sampling starts at: the box's shock, wake and wall layers have
formed), through
the public API with host buffers - context creation, cold start, the S steps
with every step's counters copied to a pinned host ring, the field read back
into host memory - and that whole run, timed on the host clock, is the `e2e`
number.  Then W warm-up steps and the K timed steps (CUDA events on the
context's stream; every one samples) give `value`.

Metric: particle-steps/s = sum over timed steps of the particle count / time.
With --gpus N each rank runs an independent replica (its own Philox key): per-
GPU work is fixed (weak scaling); the replicas' FP64 moments are summed with
one NCCL all-reduce after the timed region, as replica statistics are.
--ensemble C instead times C cases of the batched-ensemble generator, case i
on rank i mod N (total work fixed: strong scaling), no exchange between ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/s on 1 B200"
UNIT = "particle-steps/s"

# Algorithmic bytes per particle (and per cell) of the step's kernels, FP32
# state (x, y, vx, vy, vz = 20 B) / FP64 state (40 B); the 4-byte key is the
# cell index the sort needs from the move.
#   k_move     reads x, y, vx, vy; writes x, y and the key
#   k_scatter  reads the key and the state, writes the state once
#   k_sample   reads vx, vy, vz; read-modify-write of the 13 FP64 moments of
#              every cell plus its start offset
ALGO = {
    "k_move": {"fp32": 28, "fp64": 52},
    "k_scatter": {"fp32": 44, "fp64": 84},
    "k_sample": {"fp32": 12, "fp64": 24},
}
CELL_BYTES = {"k_sample": 2 * 13 * 8 + 4}

# DRAM bytes per particle (read + write) of each kernel from one ncu capture
# of the same kernels on the 640x640 case (8.1e6 particles, FP32), scaled by
# the particles of a launch (profiles/*_640_case_ncu.md).  Below the
# algorithmic bytes because part of the written state is still in the 126 MB
# L2 when the kernel ends.
NCU_TRAFFIC_PER_PARTICLE = {"k_scatter": 37.7, "k_move": 22.2, "k_sample": 19.4}


def peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().splitlines() if r.strip()]
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]),
                "power_w_max": max(float(r[3]) for r in rows), "samples": len(rows),
                "reasons": reasons}


def _mem_available_gb() -> float:
    try:
        for line in Path("/proc/meminfo").read_text().splitlines():
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) / 2**20
    except OSError:
        pass
    return 0.0


# Resident memory of one reference copy at 1000x1000 (static arrays sized by
# the raised capacities: particles, cell lists, cells), with a margin.
REF_LARGE_COPY_GB = 2.0


def cpu_baseline(steps: int, cores: int, wall: str, warmup: int = 1) -> dict:
    """The reference solver - its own sources, its MWC generator, the
    single-rank MPI stub - run as concurrent single-rank processes with
    distinct seeds on this host's cores (MPI is not installed, so the
    copies stand in for ranks; their summed throughput bounds an MPI run
    from above), on the benchmarked case: 1000x1000 cells, NPCFree 20,
    angle 10, Dt 1e-6, sampling every timed step.  That grid exceeds the
    reference's static capacities, so it runs the build whose capacities
    are raised (oracle/Makefile, ref-large; routines unchanged); without it,
    the largest grid the stock build allows (200x200).  Each copy runs
    `warmup` + `steps` steps from its cold start; only the steps are timed
    (around the reference's own loop).  Returns the summed particle-steps/s
    and what ran."""
    big = ROOT / "oracle" / "_ref" / "dsmc_ref_baseline_1000"
    small = ROOT / "oracle" / "_ref" / "dsmc_ref_baseline"
    if big.exists():
        exe, grid = big, 1000
        copies = max(1, min(cores, int(_mem_available_gb() / REF_LARGE_COPY_GB)))
    elif small.exists():
        exe, grid, copies = small, 200, cores
    else:
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref/dsmc_ref_baseline not built"}
    wall_id = {"diffuse": 0, "specular": 1, "cll": 2}[wall]
    procs = []
    for i in range(copies):
        cmd = [str(exe), str(grid), str(grid), "20", str(warmup), str(steps), str(wall_id),
               "0.8", "0.8", "10", "1e-6", str(1000 + i), "0"]
        procs.append(subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    rates, np_ = [], []
    for pr in procs:
        out, err = pr.communicate()
        line = out.strip().splitlines()[-1] if out.strip() else "{}"
        r = json.loads(line)
        if r.get("seconds"):
            rates.append(r["particle_steps"] / r["seconds"])
            np_.append(r["np"])
    total = sum(rates)
    n_mean = int(statistics.mean(np_)) if np_ else 0
    build = ("the reference's sources with raised static capacities" if grid == 1000 else
             "the stock reference at its largest grid (200x200: static capacities)")
    return {"value": total, "unit": UNIT, "cores": len(rates), "kind": "reference",
            "per_core": total / max(1, len(rates)), "grid": [grid, grid],
            "particles_per_copy": n_mean, "host_cores": cores,
            "sample": f"{len(rates)} concurrent single-rank copies of {build}, own MWC RNG, "
                      f"distinct seeds; {grid}x{grid} cells, NPCFree 20 (~{n_mean} particles "
                      f"each), {wall} walls, angle 10, Dt 1e-6; {steps} timed steps after "
                      f"{warmup} from the cold start, sampling every step"}


def reference_config(args, r: dict) -> dict:
    """The reference arm's config: what the CPU run above actually ran."""
    g = r.get("grid", [1000, 1000])[0]
    c = workload_config(args, grid=g)
    c["workload"] = (f"{g}x{g} cells, NPCFree 20 (~{r.get('particles_per_copy', 0):.2e} "
                     f"particles per copy), angle 10 deg, {args.wall} walls, Dt 1e-6 s, FP64 "
                     f"(the reference's precision); {r['cores']} concurrent single-rank copies "
                     "on the host cores, timed from their cold start")
    c["precision"] = "fp64"
    c["parallelism"] = f"{r['cores']} independent CPU processes"
    c["spinup"] = 0
    return c


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    # One step of the 1000x1000 case takes seconds per copy: at most 30
    # timed steps after at most 5 warm-up steps keep the run to minutes.
    steps = max(1, min(args.steps, 30))
    warmup = max(1, min(args.warmup, 5))
    r = cpu_baseline(steps, cores, args.wall, warmup=warmup)
    wall_s = time.perf_counter() - t0
    if r["value"] is None:
        print(json.dumps({"impl": "reference", "unavailable": r["sample"]}))
        return
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": steps, "warmup": warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": reference_config(args, r),
            "cpu_baseline": r,
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "wall_s": wall_s}
    print(json.dumps(line))


def workload_config(args, grid: int | None = None) -> dict:
    g = grid or getattr(args, "grid", 1000)
    return {"workload": f"{g}x{g} cells, NPCFree 20 (~{20 * g * g:.1e} particles), angle 10 "
                        f"deg, {args.wall} walls, Dt 1e-6 s, {args.precision} state with FP64 "
                        f"accumulators, timed after a {args.spinup}-step spin-up to developed "
                        "flow",
            "grid": [g, g], "npc_free": 20, "attack_angle": 10, "wall": args.wall,
            "dt": 1e-6, "precision": args.precision, "spinup": args.spinup,
            "sampling": "every step (spin-up and timed), as in the CPU arm",
            "l2": "inputs larger than L2 (particle state ~400 MB)",
            "parallelism": f"replicas x{args.gpus}"}


def kernel_table(kt: dict, key: str, np_mean: float, ncell: int) -> dict:
    kernels = {}
    for name, (kms, launches) in kt.items():
        if launches == 0:
            continue
        avg = kms / launches
        ent = {"ms_avg": avg, "launches": launches}
        if name in ALGO:
            b = ALGO[name][key] * np_mean + CELL_BYTES.get(name, 0) * ncell
            ent["algo_bytes"] = b
            ent["gbs"] = b / (avg / 1e3) / 1e9
        kernels[name] = ent
    return kernels


def run_ensemble(args, torch, dist, rank, world, local):
    """--ensemble C: C cases of the batched-ensemble generator (grid side
    U[64, 400], ...), case i on rank i mod N, each rank's share in one
    context; W warm-up then K timed steps, max time over ranks."""
    from dsmc_erlend_b200 import Engine
    from dsmc_erlend_b200.abi import FP32, FP64
    from dsmc_erlend_b200.ensemble import ensemble_cases, shard

    prec = FP32 if args.precision == "fp32" else FP64
    cases = ensemble_cases(args.ensemble, 2024, precision=prec)
    mine = [p for _, p in shard(cases, rank, world)]
    for p in mine:
        p.first_sampling_step = 0
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        eng = Engine(mine, stream=stream.cuda_stream)
        eng.InitialConditions()
        eng.step(args.spinup_ensemble + args.warmup)
        eng.synchronize()
        c0 = sum(eng.counters(i)["particle_steps"] for i in range(len(mine)))
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.step(args.steps)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        ms = e0.elapsed_time(e1)
        ps = sum(eng.counters(i)["particle_steps"] for i in range(len(mine))) - c0
        status = eng.synchronize()
        eng.close()
    if dist is not None:
        t = torch.tensor([ms, float(ps)], dtype=torch.float64, device="cuda")
        tm = t.clone()
        dist.all_reduce(tm[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        ms, ps = float(tm[0].item()), float(t[1].item())
    if rank == 0:
        print(json.dumps({
            "metric": METRIC + " (batched ensemble)", "value": ps / (ms / 1e3), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32" if prec == FP32 else "f64",
            "data": "synthetic", "status": status,
            "config": {"workload": f"{args.ensemble} cases of the ensemble generator (seed "
                                   "2024: grid side U[64,400], Ma U[2,8], angle U[-30,30], n "
                                   "log-U[1e16,1e18], box U[2,6], walls S/D/CLL, NPCFree "
                                   "U[5,20]), case i on rank i mod N",
                       "precision": args.precision, "sampling": "every timed step",
                       "parallelism": f"ensemble shards x{world}"}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--spinup", type=int, default=10000,
                    help="steps from the cold start to developed flow before the warm-up")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--wall", default="diffuse", choices=["diffuse", "cll", "specular"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true",
                    help="spin up without the host-clocked end-to-end measurement")
    ap.add_argument("--profile-steps", type=int, default=10)
    ap.add_argument("--grid", type=int, default=1000,
                    help="cells per side; smaller grids are for profiler captures only")
    ap.add_argument("--ensemble", type=int, default=0,
                    help="time this many ensemble cases sharded over the ranks instead")
    ap.add_argument("--spinup-ensemble", type=int, default=100)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        run_reference(args)
        return

    import ctypes as C

    import torch

    from dsmc_erlend_b200 import Engine
    from dsmc_erlend_b200.abi import FP32, FP64, WALL_CLL, WALL_DIFFUSE, WALL_SPECULAR, Counters
    from dsmc_erlend_b200.abi import Params, large_case

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    if args.ensemble > 0:
        run_ensemble(args, torch, dist, rank, world, local)
        if dist is not None:
            dist.destroy_process_group()
        return

    wall = {"diffuse": WALL_DIFFUSE, "cll": WALL_CLL, "specular": WALL_SPECULAR}[args.wall]
    prec = FP32 if args.precision == "fp32" else FP64
    p = large_case(wall_model=wall, precision=prec, seed=20251 + rank)
    p.nx = p.ny = args.grid
    # Every step samples, the spin-up's too: the case's heaviest step, and the
    # step the CPU arm times (the field statistics, not the dynamics, depend
    # on where sampling starts).
    p.first_sampling_step = 0
    stream = torch.cuda.Stream()

    def barrier():
        if dist is not None:
            dist.barrier()

    # End to end through the public API with host buffers: the spin-up run -
    # context, cold start, every step's counters read back to a pinned host
    # ring, the field read back into host memory - on the host clock.
    e2e = None
    field_out = torch.empty((p.nx * p.ny, 17), dtype=torch.float64, pin_memory=True).numpy()
    n_spin = max(args.spinup, 1)
    ring = torch.zeros(n_spin * C.sizeof(Counters), dtype=torch.uint8, pin_memory=True)
    torch.cuda.synchronize()
    barrier()
    with torch.cuda.stream(stream):
        t = time.perf_counter()
        marks = [t]
        sim = Engine(p, stream=stream.cuda_stream)
        marks.append(time.perf_counter())
        sim.InitialConditions()
        if args.no_e2e:
            sim.step(args.spinup)
            sim.synchronize()
        else:
            sim.step_read(n_spin, ring.data_ptr())
            marks.append(time.perf_counter())
            f = sim.GatherGlobalField(out=field_out)
            status_e2e = sim.synchronize()
            wall_s = time.perf_counter() - t
            marks.append(t + wall_s)
            last = (Counters * n_spin).from_address(ring.data_ptr())[-1]
            if last.step != n_spin:
                raise RuntimeError(f"e2e: the last step record says step {last.step}, not {n_spin}")
            e2e_ps = sim.counters()["particle_steps"]
            d2h = n_spin * C.sizeof(Counters) + f.nbytes
            phases = {k: round((marks[i + 1] - marks[i]) * 1e3, 2)
                      for i, k in enumerate(("create_ms", "cold_start_and_enqueue_ms",
                                             "steps_and_fields_ms"))}
            e2e = {"value": e2e_ps / wall_s * world, "unit": UNIT,
                   "h2d_bytes_per_step": C.sizeof(Params) / n_spin,
                   "d2h_bytes_per_step": d2h / n_spin,
                   "includes": f"a {n_spin}-step run through the C ABI: context creation, "
                               "cold start (the particles are generated on the device from "
                               "the parameters, the run's only input), every step's counters "
                               "read back asynchronously into a pinned host ring, the field "
                               "read back into a pinned host buffer",
                   "steps": n_spin, "wall_s": wall_s, "status": status_e2e, "phases": phases}

        sim.step(args.warmup)
        sim.synchronize()
        barrier()
        torch.cuda.synchronize()
        c0 = sim.counters()
        clocks = ClockSampler(local)
        clocks.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.step(args.steps)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier()
        clk = clocks.stop()
        status = sim.synchronize()
        ms = e0.elapsed_time(e1)
        c1 = sim.counters()
        ps = c1["particle_steps"] - c0["particle_steps"]
        np_mean = ps / args.steps

        # Replica statistics: one all-reduce of the FP64 moments.
        reduce_ms = None
        if dist is not None:
            ncell = p.nx * p.ny
            buf = torch.empty(ncell * 17, dtype=torch.float64, device="cuda")
            sim.fields_to_device(0, buf.data_ptr())
            torch.cuda.synchronize()
            t = time.perf_counter()
            dist.all_reduce(buf)
            torch.cuda.synchronize()
            reduce_ms = (time.perf_counter() - t) * 1e3
            sim.fields_from_device(0, buf.data_ptr(), c1["sample_step"] * world)
            del buf

        if dist is not None:
            t_all = torch.tensor([ms], dtype=torch.float64, device="cuda")
            ps_all = torch.tensor([ps], dtype=torch.float64, device="cuda")
            dist.all_reduce(t_all, op=dist.ReduceOp.MAX)
            dist.all_reduce(ps_all)
            ms_max, ps_total = float(t_all.item()), float(ps_all.item())
        else:
            ms_max, ps_total = ms, float(ps)

        # Per-kernel device time over profiled steps (events around each kernel).
        sim.set_profiling(True)
        sim.step(args.profile_steps)
        sim.synchronize()
        kt = sim.kernel_times()
        sim.set_profiling(False)
        sim.close()

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    value = ps_total / (ms_max / 1e3)
    peak, peak_kind = peaks()
    key = "fp32" if prec == FP32 else "fp64"
    ncell = p.nx * p.ny
    kernels = kernel_table(kt, key, np_mean, ncell)
    tops = sorted(kernels.items(), key=lambda kv: -kv[1]["ms_avg"] * kv[1]["launches"])
    dom = next((n for n, _ in tops if n in ALGO), None)
    roof = None
    if dom:
        ach = kernels[dom]["gbs"]
        roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": peak,
                "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind,
                "traffic": (NCU_TRAFFIC_PER_PARTICLE[dom] * np_mean
                            if key == "fp32" and dom in NCU_TRAFFIC_PER_PARTICLE else None),
                "algo_bytes_per_launch": kernels[dom]["algo_bytes"],
                "units_per_launch": np_mean}
    # Launches of this library's kernels per step (all launches of the
    # profiled steps, which run the same sequence as the graph of a step).
    step_kernels = sum(v["launches"] for v in kernels.values()) / max(1, args.profile_steps)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if prec == FP32 else "f64", "data": "synthetic",
            "config": workload_config(args), "particles_mean": np_mean,
            "status": status, "roofline": roof, "kernels": kernels,
            "gpu_launches": int(round(step_kernels * args.steps)), "clocks": clk, "e2e": e2e}
    if reduce_ms is not None:
        line["replica_allreduce_ms"] = reduce_ms
    if world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(3, os.cpu_count() or 1, args.wall, warmup=1)
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
