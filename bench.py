"""Throughput of the DSMC time step on B200, and the reference's CPU arm.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--wall diffuse|cll] [--precision fp32|fp64]

Workload: the HBM-roofline case - 1000x1000 cells on [-20, 20]^2 m, NPCFree 20
(~2e7 particles), angle of attack 10 deg, diffuse walls at Tw 300 K (or CLL
0.8/0.8), Dt 1e-6 s, FP32 particle state with FP64 hit times, inflow counts and
moment accumulators.  Particles and cells are generated by the engine's own
cold start (seeded Philox), so the data is synthetic by construction.  A
"step" is one full DSMC time step: move + wall scattering, inflow, removal,
cell sort, NTC collisions and moment sampling (every timed step samples).

Metric: particle-steps/s = sum over timed steps of the particle count / time.
With --gpus N each rank runs an independent replica (its own Philox key): per-
GPU work is fixed (weak scaling); the replicas' FP64 moments are summed with
one NCCL all-reduce after the timed region, as replica statistics are.
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


def cpu_baseline(steps: int, cores: int, wall: str, seconds_hint: float = 15.0) -> dict:
    """The reference solver (its own sources, MWC RNG, single-rank MPI stub)
    run as `cores` concurrent processes with distinct seeds on this host, on
    the largest grid its static capacities allow (200x200 cells, NPCFree 20,
    ~8e5 particles), everything else as the benchmarked case.  Returns the
    summed particle-steps/s."""
    exe = ROOT / "oracle" / "_ref" / "dsmc_ref_baseline"
    if not exe.exists():
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref/dsmc_ref_baseline not built"}
    wall_id = {"diffuse": 0, "specular": 1, "cll": 2}[wall]
    procs = []
    for i in range(cores):
        cmd = [str(exe), "200", "200", "20", "3", str(steps), str(wall_id), "0.8", "0.8", "10",
               "1e-6", str(1000 + i), "0"]
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
    return {"value": total, "unit": UNIT, "cores": len(rates), "kind": "reference",
            "per_core": total / max(1, len(rates)),
            "sample": f"{len(rates)} concurrent single-rank copies of the reference (own RNG), "
                      f"200x200 cells, NPCFree 20 (~{int(statistics.mean(np_)) if np_ else 0} "
                      f"particles each, its capacity limit), {wall} walls, angle 10, Dt 1e-6, "
                      f"{steps} timed steps after 3 warm-up, sampling every step"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    steps = max(args.steps, 1)
    r = cpu_baseline(steps, cores, args.wall)
    wall_s = time.perf_counter() - t0
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args),
            "cpu_baseline": r,
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "wall_s": wall_s}
    if r["value"] is None:
        line = {"impl": "reference", "unavailable": r["sample"]}
    print(json.dumps(line))


def workload_config(args) -> dict:
    g = getattr(args, "grid", 1000)
    return {"workload": f"{g}x{g} cells, NPCFree 20 (~{20 * g * g:.1e} particles), angle 10 "
                        f"deg, {args.wall} walls, Dt 1e-6 s, {args.precision} state with FP64 "
                        "accumulators",
            "grid": [g, g], "npc_free": 20, "attack_angle": 10, "wall": args.wall,
            "dt": 1e-6, "precision": args.precision, "sampling": "every timed step",
            "l2": "inputs larger than L2 (particle state ~400 MB)",
            "parallelism": f"replicas x{args.gpus}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--wall", default="diffuse", choices=["diffuse", "cll", "specular"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=10)
    ap.add_argument("--grid", type=int, default=1000,
                    help="cells per side; smaller grids are for profiler captures only")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        run_reference(args)
        return

    import torch

    from dsmc_erlend_b200 import Engine
    from dsmc_erlend_b200.abi import FP32, FP64, WALL_CLL, WALL_DIFFUSE, WALL_SPECULAR, large_case

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

    wall = {"diffuse": WALL_DIFFUSE, "cll": WALL_CLL, "specular": WALL_SPECULAR}[args.wall]
    prec = FP32 if args.precision == "fp32" else FP64
    p = large_case(wall_model=wall, precision=prec, seed=20251 + rank)
    p.nx = p.ny = args.grid
    p.first_sampling_step = 0  # every timed step samples
    stream = torch.cuda.Stream()

    def barrier():
        if dist is not None:
            dist.barrier()

    with torch.cuda.stream(stream):
        sim = Engine(p, stream=stream.cuda_stream)
        sim.InitialConditions()
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

    # End to end through the public API with host buffers: context, cold
    # start, steps with a host read of the counters after each, and the field
    # read back into host memory.
    e2e = None
    if not args.no_e2e:
        import ctypes as C

        from dsmc_erlend_b200.abi import Counters, Params

        sim.close()
        del sim
        torch.cuda.synchronize()
        barrier()
        n_e2e = args.warmup + args.steps
        # The host buffer of the field read-back, pinned like the inputs of
        # the contract, is allocated before the timed region.
        field_out = torch.empty((p.nx * p.ny, 17), dtype=torch.float64,
                                pin_memory=True).numpy()
        # ... and so is the ring that receives every step's counters.
        ring = torch.zeros(n_e2e * C.sizeof(Counters), dtype=torch.uint8, pin_memory=True)
        t = time.perf_counter()
        marks = [t]
        with torch.cuda.stream(stream):
            s2 = Engine(p, stream=stream.cuda_stream)
            marks.append(time.perf_counter())
            s2.InitialConditions()
            # Every step's counters are read back to the host, asynchronously:
            # the device runs the steps back to back.
            s2.step_read(n_e2e, ring.data_ptr())
            d2h = n_e2e * C.sizeof(Counters)
            marks.append(time.perf_counter())
            f = s2.GatherGlobalField(out=field_out)
            d2h += f.nbytes
            status2 = s2.synchronize()
        wall_s = time.perf_counter() - t
        marks.append(t + wall_s)
        last = (Counters * n_e2e).from_address(ring.data_ptr())[-1]
        if last.step != n_e2e:
            raise RuntimeError(f"e2e: the last step record says step {last.step}, not {n_e2e}")
        phases = {k: round((marks[i + 1] - marks[i]) * 1e3, 2)
                  for i, k in enumerate(("create_ms", "init_and_enqueue_ms", "steps_and_fields_ms"))}
        e2e_ps = s2.counters()["particle_steps"]
        s2.close()
        e2e = {"value": e2e_ps / wall_s * world, "unit": UNIT,
               "h2d_bytes_per_step": C.sizeof(Params) / n_e2e,
               "d2h_bytes_per_step": d2h / n_e2e,
               "includes": "context creation, cold start, steps with an asynchronous "
                           "device-to-host read of every step's counters into a pinned ring, "
                           "field download into a pinned host buffer", "wall_s": wall_s,
               "phases": phases}
    else:
        sim.close()

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    value = ps_total / (ms_max / 1e3)
    peak, peak_kind = peaks()
    key = "fp32" if prec == FP32 else "fp64"
    ncell = p.nx * p.ny
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
        line["cpu_baseline"] = cpu_baseline(150, os.cpu_count() or 1, args.wall)
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
