"""Benchmark of the tracking path (ringpass! on the GPU).

Metric: particle*element*turns/s in FP64 (alive-at-start particles x lattice
entries x turns per second).  Workload (default): the DBA storage ring, 3 GeV
electrons, 401 elements (20 cells + RF), 1,048,576 Gaussian particles plus a
512 x 512 dynamic-aperture grid, rectangular aperture 0.02 m.  One step is
ringpass! over STEP_TURNS turns of that whole beam, restarted from the input
distribution.  Synthetic, seeded inputs (Philox); no dataset is involved.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload dba|fodo|batched]

Under torchrun each rank tracks its own beam of the same size (weak scaling,
no collective on the data path); time is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STEP_TURNS = 10
L2_FLUSH_BYTES = 256 << 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="dba", choices=["dba", "fodo", "batched"])
    p.add_argument("--n-gauss", type=int, default=1 << 20)
    p.add_argument("--grid", type=int, default=512)
    p.add_argument("--contract", action="store_true", help="kernels built with FMA contraction")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def workload(args, rank):
    import trackpad_b200.workloads as W
    if args.workload == "fodo":
        lat, beam = W.fodo_ring(), W.fodo_beam()
        coords = W.gaussian(10000, seed=rank)
        return dict(name="FODO ring, 8 cells (32 elements), 1 GeV e-, 10,000 Gaussian particles, aperture 0.05 m",
                    lat=lat, beam=beam, coords=coords, aperture=0.05, turns=STEP_TURNS)
    lat, beam = W.dba_ring(), W.dba_beam()
    coords = W.dba_particles(args.n_gauss, args.grid, seed=rank)
    return dict(name=(f"DBA ring, 20 cells + RF (401 elements), 3 GeV e-, {args.n_gauss:,} Gaussian + "
                      f"{args.grid}x{args.grid} DA grid, aperture 0.02 m"),
                lat=lat, beam=beam, coords=coords, aperture=0.02, turns=STEP_TURNS)


def cpu_baseline(w, target_s=10.0, chunk=1024, threads=0):
    """The oracle (C++ restatement of the reference loop order: elements outer,
    particles inner, OpenMP over particles) on the host cores, on successive
    chunks of the workload's own beam, each tracked over the step's turns, until
    about `target_s` seconds."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ref
    import trackpad_b200 as tp
    lat, beam = w["lat"], w["beam"]
    nthreads = threads or oracle_ref.lib().orc_max_threads()
    n = w["coords"].shape[0]
    rng = np.random.Generator(np.random.Philox(1234))
    units, dt, chunks = 0.0, 0.0, 0
    while dt < target_s and chunks < 4096:
        idx = rng.integers(0, n, chunk)
        c = np.asfortranarray(w["coords"][idx])
        lost = np.zeros(len(c), np.int64)
        t0 = time.perf_counter()
        oracle_ref.ringpass(lat, c, lost, tp.beti(beam), w["turns"], aperture=w["aperture"], nthreads=nthreads)
        dt += time.perf_counter() - t0
        units += float(len(c)) * len(lat) * w["turns"]
        chunks += 1
    return {"value": units / dt, "unit": "particle*element*turns/s", "cores": nthreads, "kind": "port",
            "sample": f"{chunks} x {chunk} particles drawn from the workload's beam, {w['turns']} turns each "
                      f"(one step), OpenMP over particles, {dt:.1f} s"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import __graft_entry__
    __graft_entry__.load_package()
    w = workload(args, 0)
    # Each step is a bounded sample of the workload: ~4 s of CPU work.
    vals = []
    base = None
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(w, target_s=4.0 if i >= args.warmup else 0.5)
        if i >= args.warmup:
            vals.append(r["value"])
        base = r
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": "particle*element*turns/s FP64", "value": v,
            "unit": "particle*element*turns/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 4000.0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Philox Gaussian beam + DA grid)",
            "config": {"workload": w["name"], "step": f"about 4 s of {w['turns']}-turn chunks of the beam per step"},
            "cpu_baseline": {"value": v, "unit": base["unit"], "cores": base["cores"], "kind": "port",
                             "sample": base["sample"]},
            "e2e": {"value": v, "unit": "particle*element*turns/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# DRAM bytes per particle of one tracking launch: ncu capture of track_single on
# the DBA ring, 69,632 particles x 10 turns (5.425 MB read + written).  Traffic
# grows with the particle count (the table lives in shared memory).
DRAM_BYTES_PER_PARTICLE = 5.425152e6 / 69632


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank, world, local = dist_env()
    import torch
    import __graft_entry__
    tp = __graft_entry__.load_package()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    w = workload(args, rank)
    lat, beam, aperture, turns = w["lat"], w["beam"], w["aperture"], w["turns"]
    n = w["coords"].shape[0]
    dev = torch.device("cuda", local)
    # Inputs resident in HBM: the (6, N) tensor is the N x 6 column-major matrix.
    init = torch.from_numpy(np.ascontiguousarray(w["coords"].T)).to(dev)
    coords = torch.empty_like(init)
    lost = torch.zeros(n, dtype=torch.int64, device=dev)
    lost_turn = torch.full((n,), -1, dtype=torch.int32, device=dev)
    lost_elem = torch.full((n,), -1, dtype=torch.int32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream

    def step():
        coords.copy_(init)
        lost.zero_()
        tp.ringpass_(coords.T, lat, beam, lost, turns, aperture=aperture, lost_turn=lost_turn, lost_elem=lost_elem,
                     contract=args.contract, stream=sptr)
        st = tp.last_stats(local)
        flush.fill_(1)  # L2 flush between timed iterations
        return st

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    kernel_ms, flops, units, launches = [], 0.0, 0.0, 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        st = step()
        kernel_ms.append(st["kernel_ms"])
        flops += st["flops"]
        units += st["units"]
        launches += st["launches"]
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    elapsed = e0.elapsed_time(e1) / 1e3
    t = torch.tensor([elapsed, units], dtype=torch.float64, device=dev)
    if dist:
        tt = t.clone()
        dist.all_reduce(tt[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(tt[1:2], op=dist.ReduceOp.SUM)
        elapsed, units_all = float(tt[0]), float(tt[1])
    else:
        units_all = units
    value = units_all / elapsed

    # Roofline of the tracking kernel: algorithmic FP64 FLOPs per launch / its
    # event-timed duration, against the measured FP64 FMA peak of this device.
    peak = tp.probe_fp64_peak(local)
    k_ms = float(np.mean(kernel_ms))
    achieved = (flops / args.steps) / (k_ms * 1e-3) / 1e12

    e2e = None
    if not args.no_e2e:
        # Same metric through the public API with pinned host buffers: the
        # host->device copy of the input and the device->host copy of the
        # result are inside the timed region of every step.
        hbuf = torch.empty((6, n), dtype=torch.float64).pin_memory()
        hl = torch.empty(n, dtype=torch.int64).pin_memory().numpy()
        src = np.asfortranarray(w["coords"])
        hc_f = hbuf.numpy().T  # (N, 6) column-major view of pinned memory
        e2e_units, t_e2e = 0.0, 0.0
        for i in range(max(2, args.steps // 2) + 1):
            hc_f[...] = src
            hl[...] = 0
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tp.ringpass_(hc_f, lat, beam, hl, turns, aperture=aperture)
            t1 = time.perf_counter()
            stt = tp.last_stats(local)
            if i > 0:
                t_e2e += t1 - t0
                e2e_units += stt["units"]
        e2e = {"value": e2e_units / t_e2e * world, "unit": "particle*element*turns/s",
               "h2d_bytes_per_step": int(stt["h2d_bytes"]), "d2h_bytes_per_step": int(stt["d2h_bytes"])}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w)

    if rank == 0:
        line = {
            "metric": "particle*element*turns/s FP64", "value": value, "unit": "particle*element*turns/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Philox Gaussian beam + DA grid)",
            "config": {"workload": w["name"], "turns_per_step": turns, "particles_per_gpu": n,
                       "elements": len(lat), "l2": "flushed between timed steps (256 MiB write)",
                       "fp": "FMA contraction" if args.contract else "no FMA contraction (reference operation order)"},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": DRAM_BYTES_PER_PARTICLE * n,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch on "
                                           "69,632 particles x 10 turns, scaled by particles",
                         "peak_source": "measured FP64 FMA throughput of this device (tp_probe_fp64_peak)",
                         "flops_per_launch": flops / args.steps, "kernel_ms": k_ms},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
