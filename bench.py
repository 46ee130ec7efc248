"""Benchmark of the tracking path (ringpass! on the GPU).

Metric: particle*element*turns/s in FP64 (alive-at-start particles x lattice
entries x turns per second).  Workload (default): the DBA storage ring, 3 GeV
electrons, 401 elements (20 cells + RF), 1,048,576 Gaussian particles plus a
512 x 512 dynamic-aperture grid, rectangular aperture 0.02 m.  One step is
ringpass! over STEP_TURNS turns of that whole beam, restarted from the input
distribution.  Synthetic, seeded inputs (Philox); no dataset is involved.  The
default line also carries, under the same clock: the adjoint/forward time
ratio of the gradient workload (65,536 particles, 256 turns, 120 k1 + 80 k2;
key "adjoint"), the batched forward workload (256 variants, 100-turn steps,
its roofline fraction and its speed-up over the plain tracker run lattice by
lattice; key "batched") and the batched time-dependent adjoint / batched
forward time ratio (64 variants, 50-turn steps; key "batched_adjoint").

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload dba|fodo|batched|adjoint|batched_adjoint]

  batched          256 DBA variants (4..20 cells, strengths +-2%), 4,096 x U[0.25, 1]
                   particles each, one CUDA-graph launch per step
  adjoint          loss + gradient on the DBA ring: 65,536 particles, 256 turns
  batched_adjoint  64 time-dependent DBA variants (Q1 ramp +1%, RF voltage 5% at a
                   200-turn period), 16,384 particles each, gradients of every variant

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
SIGMA_LOSS = 1e-4      # sigma_x of the beam-size loss
LOST_WEIGHT = 1e3

# DRAM bytes per particle of one tracking launch, by the kernel instance's
# resident blocks per SM: ncu captures of track_single on the DBA ring, 135,168
# particles x 10 turns, dram__bytes.sum.per_second x gpu__time_duration (8
# blocks, 64 registers: 2.420 GB; 7 blocks, 72 registers: 1.324 GB, captured
# with the multipole integrator out of line), almost all of it the write-back of
# spilled stack lines.  Scaled by the launch's particle count; instances without
# a capture report no traffic.
DRAM_BYTES_PER_PARTICLE_BY_MINB = {7: 1.3236e9 / 135168, 8: 2.4199e9 / 135168}


def dram_traffic(min_blocks, n):
    per = DRAM_BYTES_PER_PARTICLE_BY_MINB.get(int(min_blocks))
    return None if per is None else per * n


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="dba", choices=["dba", "fodo", "batched", "adjoint", "batched_adjoint",
                                                         "tpsa"])
    p.add_argument("--order", type=int, default=4, help="tpsa workload: series order")
    p.add_argument("--maps", type=int, default=0, help="tpsa workload: maps per step (0: default)")
    p.add_argument("--n-gauss", type=int, default=1 << 20)
    p.add_argument("--grid", type=int, default=512)
    p.add_argument("--turns", type=int, default=0, help="turns per step (0: the workload's default)")
    p.add_argument("--nvar", type=int, default=0, help="variants of the batched workloads (0: default)")
    p.add_argument("--contract", action="store_true", help="kernels built with FMA contraction")
    p.add_argument("--min-blocks", type=int, default=0,
                   help="dba/fodo workloads: kernel instance sized for 8, 7, 6 or 5 resident blocks per SM "
                        "(0: chosen by the launch tuner)")
    p.add_argument("--table-smem", action="store_true",
                   help="stage element tables into shared memory (default: read through the L1 cache)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-adjoint", action="store_true", help="default workload: skip the adjoint ratio")
    p.add_argument("--no-full-length", action="store_true",
                   help="default workload: skip the one 1000-turn track of the whole beam")
    p.add_argument("--no-batched", action="store_true",
                   help="default workload: skip the batched forward and batched adjoint summaries")
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


# ---------------------------------------------------------------------------
# Workloads
# ---------------------------------------------------------------------------
def workload(args, rank):
    import trackpad_b200.workloads as W
    if args.workload == "fodo":
        lat, beam = W.fodo_ring(), W.fodo_beam()
        coords = W.gaussian(10000, seed=rank)
        return dict(name="FODO ring, 8 cells (32 elements), 1 GeV e-, 10,000 Gaussian particles, aperture 0.05 m",
                    lat=lat, beam=beam, coords=coords, aperture=0.05, turns=args.turns or STEP_TURNS)
    lat, beam = W.dba_ring(), W.dba_beam()
    coords = W.dba_particles(args.n_gauss, args.grid, seed=rank)
    return dict(name=(f"DBA ring, 20 cells + RF (401 elements), 3 GeV e-, {args.n_gauss:,} Gaussian + "
                      f"{args.grid}x{args.grid} DA grid, aperture 0.02 m"),
                lat=lat, beam=beam, coords=coords, aperture=0.02, turns=args.turns or STEP_TURNS)


def batched_workload(args, rank, time_dependent=False):
    import trackpad_b200.workloads as W
    if time_dependent:
        nvar = args.nvar or 64
        turns = args.turns or 50
        run_turns = 500  # the ramp and the modulation are defined over the full 500-turn run
        variants = [(W.time_dependent(v, run_turns), 16384)
                    for v, _ in W.dba_variants(nvar=nvar, seed=11 + rank, n_base=16384)]
        name = (f"{nvar} time-dependent DBA variants (4..20 cells, strengths +-2%, Q1 k1 ramp +1% over 500 turns, "
                f"RF voltage 5% at a 200-turn period), 16,384 Gaussian particles each, aperture 0.02 m")
    else:
        nvar = args.nvar or 256
        turns = args.turns or 100
        variants = W.dba_variants(nvar=nvar, seed=1 + rank, n_base=4096)
        name = (f"{nvar} DBA variants (4..20 cells, strengths +-2%), 4,096 x U[0.25, 1] Gaussian particles each, "
                f"aperture 0.02 m, one CUDA-graph launch")
    counts = [n for _, n in variants]
    poff = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    coords = np.asfortranarray(np.concatenate([W.gaussian(n, seed=1000 * rank + i) for i, n in enumerate(counts)]))
    return dict(name=name, lats=[v for v, _ in variants], counts=counts, poff=poff, coords=coords,
                beam=W.dba_beam(), aperture=0.02, turns=turns)


def cpu_baselines(w):
    """The all-core figure (OpenMP over particles) and, beside it, one host
    thread: the reference's own ringpass! is single-threaded."""
    allc = cpu_baseline(w)
    one = cpu_baseline(w, target_s=5.0, chunk=128, threads=1)
    allc["single_thread"] = {"value": one["value"], "unit": one["unit"], "cores": 1, "sample": one["sample"]}
    return allc


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
    turns = min(w["turns"], STEP_TURNS)
    units, dt, chunks = 0.0, 0.0, 0
    while dt < target_s and chunks < 4096:
        idx = rng.integers(0, n, chunk)
        c = np.asfortranarray(w["coords"][idx])
        lost = np.zeros(len(c), np.int64)
        t0 = time.perf_counter()
        oracle_ref.ringpass(lat, c, lost, tp.beti(beam), turns, aperture=w["aperture"], nthreads=nthreads)
        dt += time.perf_counter() - t0
        units += float(len(c)) * len(lat) * turns
        chunks += 1
    return {"value": units / dt, "unit": "particle*element*turns/s", "cores": nthreads, "kind": "port",
            "sample": f"{chunks} x {chunk} particles drawn from the workload's beam, {turns} turns each, "
                      f"OpenMP over particles, {dt:.1f} s"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import __graft_entry__
    __graft_entry__.load_package()
    w = workload(args, 0)
    # Each step is a bounded sample of the workload: ~4 s of CPU work.
    vals, step_ms = [], []
    base = None
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        r = cpu_baseline(w, target_s=4.0 if i >= args.warmup else 0.5)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            vals.append(r["value"])
            step_ms.append(dt * 1e3)
        base = r
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": "particle*element*turns/s FP64", "value": v,
            "unit": "particle*element*turns/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": float(np.mean(step_ms)), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Philox Gaussian beam + DA grid)",
            "config": {"workload": w["name"], "step": f"about 4 s of {w['turns']}-turn chunks of the beam per step"},
            "cpu_baseline": {"value": v, "unit": base["unit"], "cores": base["cores"], "kind": "port",
                             "sample": base["sample"]},
            "e2e": {"value": v, "unit": "particle*element*turns/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# Adjoint / forward ratio on the gradient workload
# ---------------------------------------------------------------------------
def adjoint_ratio(tp, local, turns=256, n=65536, warmup=6, steps=1):
    """Loss and gradient with respect to the 120 quadrupole k1 and 80 sextupole
    k2 of the DBA ring, 65,536 Gaussian particles, `turns` turns, against
    ringpass! of the same beam; device times from the library's CUDA events."""
    import torch
    import trackpad_b200.workloads as W
    lat, beam = W.dba_ring(), W.dba_beam()
    params = W.magnet_indices(lat)
    dev = torch.device("cuda", local)
    init = torch.from_numpy(np.ascontiguousarray(W.gaussian(n, seed=0).T)).to(dev)
    coords = torch.empty_like(init)
    lost = torch.zeros(n, dtype=torch.int64, device=dev)
    fwd, adj, rev, st = [], [], [], None
    loss = None
    for i in range(warmup + steps):
        coords.copy_(init)
        lost.zero_()
        tp.ringpass_(coords.T, lat, beam, lost, turns, aperture=0.02)
        f = tp.last_stats(local)["kernel_ms"]
        loss, _ = tp.ringpass_adjoint(init.T, lat, beam, None, turns, params, sigma=SIGMA_LOSS,
                                      lost_weight=LOST_WEIGHT, aperture=0.02)
        st = tp.adjoint_stats()
        if i >= warmup:
            fwd.append(f)
            adj.append(st["forward_ms"] + st["reverse_ms"])
            rev.append(st["reverse_ms"])
    f, a = float(np.median(fwd)), float(np.median(adj))
    return {"metric": "adjoint/forward time ratio", "value": a / f, "unit": "x", "higher_is_better": False,
            "config": f"DBA ring (401 elements), {n:,} Gaussian particles, {turns} turns, gradient w.r.t. "
                      f"{sum(1 for e in params if lat.elements[e].kind == 'QUADRUPOLE')} k1 + "
                      f"{sum(1 for e in params if lat.elements[e].kind == 'SEXTUPOLE')} k2, loss = mean "
                      f"(x^2+y^2)/sigma^2 + 1e3 lost fraction, sigma = 1e-4 m",
            "forward_ms": f, "adjoint_ms": a, "adjoint_forward_pass_ms": a - float(np.median(rev)),
            "adjoint_reverse_ms": float(np.median(rev)), "checkpoint_every": st["checkpoint_every"],
            "checkpoint_every_source": {0: "given", 1: "autotuner trial", 2: "autotuned by timing"}[st["k_tuning"]],
            "checkpoint_bytes": st["checkpoint_bytes"], "reconstruction_error": st["reconstruction_error"],
            "loss": loss, "target": "<= 3"}


# ---------------------------------------------------------------------------
# Single-lattice tracking (default)
# ---------------------------------------------------------------------------
def full_length_track(tp, torch, w, init, coords, lost, lost_turn, lost_elem, st_last, local, sptr, peak,
                      turns=1000):
    """The DBA configuration at its own length: one ringpass! of the whole beam over 1000 turns, device
    resident, with the launch configuration the tuner settled on for the 10-turn steps (no new trials)."""
    coords.copy_(init)
    lost.zero_()
    torch.cuda.synchronize()
    tp.ringpass_(coords.T, w["lat"], w["beam"], lost, turns, aperture=w["aperture"], lost_turn=lost_turn,
                 lost_elem=lost_elem, schedule=st_last["schedule"], min_blocks=st_last["min_blocks"], stream=sptr)
    st = tp.last_stats(local)
    achieved = st["flops"] / (st["kernel_ms"] * 1e-3) / 1e12
    return {"metric": "particle*element*turns/s FP64 (1000 turns)", "value": st["units"] / (st["kernel_ms"] * 1e-3),
            "unit": "particle*element*turns/s", "turns": turns, "kernel_ms": st["kernel_ms"],
            "survivors": st["survivors"], "particles": st["particles"],
            "maps_evaluated_per_s": st["element_passes"] / (st["kernel_ms"] * 1e-3),
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak},
            "schedule": st["schedule"], "min_blocks": st["min_blocks"]}


def main_track(args, tp, torch, rank, world, local, dist):
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
                     contract=args.contract, min_blocks=args.min_blocks, stream=sptr)
        st = tp.last_stats(local)
        flush.fill_(1)  # L2 flush between timed iterations
        return st

    # at least 5 warm-up steps: the launch tuner's trials (2 schedules at 7
    # blocks, then 8, 6 and 5 blocks) run on the first five calls
    n_warm = max(5, args.warmup)
    for _ in range(n_warm):
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
    passes = 0.0
    for _ in range(args.steps):
        st = step()
        kernel_ms.append(st["kernel_ms"])
        flops += st["flops"]
        units += st["units"]
        passes += st["element_passes"]
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
            tp.ringpass_(hc_f, lat, beam, hl, turns, aperture=aperture, min_blocks=args.min_blocks)
            t1 = time.perf_counter()
            stt = tp.last_stats(local)
            if i > 0:
                t_e2e += t1 - t0
                e2e_units += stt["units"]
        e2e = {"value": e2e_units / t_e2e * world, "unit": "particle*element*turns/s",
               "h2d_bytes_per_step": int(stt["h2d_bytes"]), "d2h_bytes_per_step": int(stt["d2h_bytes"])}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baselines(w)
    adj = bat = bat_adj = None
    if args.workload == "dba" and world == 1 and not args.no_adjoint:
        adj = adjoint_ratio(tp, local)
    full = None
    if args.workload == "dba" and world == 1 and not args.no_full_length:
        full = full_length_track(tp, torch, w, init, coords, lost, lost_turn, lost_elem, st, local, sptr, peak)
    if args.workload == "dba" and world == 1 and not args.no_batched:
        # the batched forward (256 variants, 100-turn steps) and the batched
        # time-dependent adjoint ratio, under the same clock as the headline
        bat = batched_summary(args, tp, torch, local)
        bat_adj = batched_adjoint_summary(args, tp, torch, local)

    if rank == 0:
        line = {
            "metric": "particle*element*turns/s FP64", "value": value, "unit": "particle*element*turns/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Philox Gaussian beam + DA grid)",
            "config": {"workload": w["name"], "turns_per_step": turns, "particles_per_gpu": n,
                       "elements": len(lat), "warmup_steps_run": n_warm,
                       "l2": "flushed between timed steps (256 MiB write)",
                       "fp": "FMA contraction" if args.contract else "no FMA contraction (reference operation order)",
                       "element_table": "shared memory (TMA bulk copy)" if args.table_smem else "L1 cache"},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": dram_traffic(st["min_blocks"], n),
                         "traffic_source": f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of the "
                                           f"{st['min_blocks']}-block instance on 135,168 particles x 10 turns, "
                                           f"scaled by particles; almost all of it is the write-back of spilled "
                                           f"stack lines",
                         "min_blocks": st["min_blocks"], "schedule": st["schedule"],
                         "peak_source": "measured FP64 FMA throughput of this device (tp_probe_fp64_peak)",
                         "flops_per_launch": flops / args.steps, "kernel_ms": k_ms},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk,
            # the maps actually evaluated (a lost particle's remaining turns are in the unit, not here)
            "maps_evaluated_per_s": passes / elapsed if world == 1 else None,
        }
        if adj is not None:
            line["adjoint"] = adj
        if full is not None:
            line["full_length"] = full
        if bat is not None:
            line["batched"] = bat
        if bat_adj is not None:
            line["batched_adjoint"] = bat_adj
        print(json.dumps(line))


# ---------------------------------------------------------------------------
# Batched forward tracking
# ---------------------------------------------------------------------------
def batched_measure(w, tp, torch, local, steps, warmup, dist=None):
    """Device-timed batched forward steps of workload `w` (inputs resident in
    HBM, one CUDA-graph launch per step, L2 flushed between steps)."""
    dev = torch.device("cuda", local)
    n = w["coords"].shape[0]
    batch = tp.Batch(w["lats"], device=local)
    betis = np.full(len(w["lats"]), tp.beti(w["beam"]))
    init = torch.from_numpy(np.ascontiguousarray(w["coords"].T)).to(dev)
    coords = torch.empty_like(init)
    lost = torch.zeros(n, dtype=torch.int64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream
    turns = w["turns"]

    def step():
        coords.copy_(init)
        lost.zero_()
        batch.ringpass_(coords.T, w["poff"], betis, lost, turns, aperture=w["aperture"], use_graph=True,
                        stream=sptr)
        st = tp.last_stats(local)
        flush.fill_(1)
        return st

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    kernel_ms, flops, units, launches = [], 0.0, 0.0, 0
    e0.record(stream)
    for _ in range(steps):
        st = step()
        kernel_ms.append(st["kernel_ms"])
        flops += st["flops"]
        units += st["units"]
        launches += st["launches"]
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    elapsed = e0.elapsed_time(e1) / 1e3
    return dict(batch=batch, betis=betis, init=init, sptr=sptr, elapsed=elapsed, units=units, flops=flops,
                kernel_ms=float(np.mean(kernel_ms)), launches=launches, st=st, clocks=clk)


def lattice_by_lattice(w, m, tp, torch, local, nsample=16):
    """The plain tracker run lattice by lattice on the same beams (a sample of
    variants, same turns): what batching replaces."""
    dev = torch.device("cuda", local)
    u, tms = 0.0, 0.0
    nsample = min(nsample, len(w["lats"]))
    for v in range(nsample):
        s = slice(int(w["poff"][v]), int(w["poff"][v + 1]))
        c = m["init"][:, s].contiguous()
        l = torch.zeros(c.shape[1], dtype=torch.int64, device=dev)
        for _rep in range(2):
            c.copy_(m["init"][:, s])
            l.zero_()
            tp.ringpass_(c.T, w["lats"][v], w["beam"], l, w["turns"], aperture=w["aperture"], stream=m["sptr"])
            stv = tp.last_stats(local)
        u += stv["units"]
        tms += stv["kernel_ms"]
    return {"value": u / (tms * 1e-3), "unit": "particle*element*turns/s",
            "sample": f"the first {nsample} variants, one ringpass! launch each, device time"}


def batched_summary(args, tp, torch, local):
    """The batched forward workload (256 DBA variants, 100-turn steps) as an
    object of the default line."""
    w = batched_workload(argparse.Namespace(nvar=0, turns=0), 0)
    m = batched_measure(w, tp, torch, local, steps=3, warmup=7)
    peak = tp.probe_fp64_peak(local)
    achieved = (m["flops"] / 3) / (m["kernel_ms"] * 1e-3) / 1e12
    value = m["units"] / m["elapsed"]
    lbl = lattice_by_lattice(w, m, tp, torch, local)
    return {"metric": "particle*element*turns/s FP64 (batched)", "value": value, "unit": "particle*element*turns/s",
            "steps": 3, "warmup": 7, "ms_per_step": m["elapsed"] / 3 * 1e3,
            "config": {"workload": w["name"], "turns_per_step": w["turns"],
                       "particles": int(w["coords"].shape[0]),
                       "schedule": {1: "static tiles", 2: "pooled refill"}.get(m["st"]["schedule"]),
                       "min_blocks": m["st"]["min_blocks"], "refill_fold": m["st"]["refill_fold"],
                       "survivors": m["st"]["survivors"], "l2": "flushed between timed steps (256 MiB write)"},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "kernel_ms": m["kernel_ms"],
                         "peak_source": "measured FP64 FMA throughput of this device (tp_probe_fp64_peak)"},
            "lattice_by_lattice": lbl, "speedup_vs_lattice_by_lattice": value / lbl["value"],
            "target": ">= 0.5 of the FP64 peak", "clocks": m["clocks"]}


def main_batched(args, tp, torch, rank, world, local, dist):
    w = batched_workload(args, rank)
    n = w["coords"].shape[0]
    # at least 7 warm-up steps: the launch tuner's trials (2 schedules at 7 blocks,
    # then 8, 6 and 5 blocks, then 2 refill folds if refill won) run on the first seven calls
    m = batched_measure(w, tp, torch, local, args.steps, max(7, args.warmup), dist)
    t = torch.tensor([m["elapsed"], m["units"]], dtype=torch.float64, device=torch.device("cuda", local))
    if dist:
        dist.all_reduce(t[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:2], op=dist.ReduceOp.SUM)
    elapsed, units_all = float(t[0]), float(t[1])
    peak = tp.probe_fp64_peak(local)
    achieved = (m["flops"] / args.steps) / (m["kernel_ms"] * 1e-3) / 1e12
    st = m["st"]
    lbl = lattice_by_lattice(w, m, tp, torch, local) if rank == 0 else None
    batch, betis, turns = m["batch"], m["betis"], w["turns"]

    e2e = None
    if not args.no_e2e:
        hbuf = torch.empty((6, n), dtype=torch.float64).pin_memory()
        hl = torch.empty(n, dtype=torch.int64).pin_memory().numpy()
        hc = hbuf.numpy().T
        e2e_units, t_e2e = 0.0, 0.0
        for i in range(3):
            hc[...] = w["coords"]
            hl[...] = 0
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            batch.ringpass_(hc, w["poff"], betis, hl, turns, aperture=w["aperture"], use_graph=True)
            t1 = time.perf_counter()
            stt = tp.last_stats(local)
            if i > 0:
                t_e2e += t1 - t0
                e2e_units += stt["units"]
        e2e = {"value": e2e_units / t_e2e * world, "unit": "particle*element*turns/s",
               "h2d_bytes_per_step": int(stt["h2d_bytes"]), "d2h_bytes_per_step": int(stt["d2h_bytes"])}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(dict(lat=w["lats"][0], beam=w["beam"], coords=w["coords"][:w["counts"][0]],
                                aperture=w["aperture"], turns=turns))
        cpu["sample"] = "variant 0: " + cpu["sample"]
    if rank == 0:
        line = {
            "metric": "particle*element*turns/s FP64", "value": units_all / elapsed,
            "unit": "particle*element*turns/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Philox variants and Gaussian beams)",
            "config": {"workload": w["name"], "turns_per_step": turns, "particles_per_gpu": n,
                       "variants": len(w["lats"]), "elements": [int(min(len(x) for x in w["lats"])),
                                                                int(max(len(x) for x in w["lats"]))],
                       "schedule": {1: "static tiles", 2: "pooled refill"}.get(st["schedule"], st["schedule"]),
                       "survivors": st["survivors"],
                       "l2": "flushed between timed steps (256 MiB write)",
                       "fp": "no FMA contraction (reference operation order)"},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": dram_traffic(st["min_blocks"], n),
                         "traffic_source": "per-particle DRAM bytes of the single-lattice capture of the same "
                                           "instance, scaled",
                         "peak_source": "measured FP64 FMA throughput of this device (tp_probe_fp64_peak)",
                         "flops_per_launch": m["flops"] / args.steps, "kernel_ms": m["kernel_ms"]},
            "lattice_by_lattice": lbl, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": m["launches"],
            "clocks": m["clocks"],
        }
        print(json.dumps(line))


# ---------------------------------------------------------------------------
# Gradients
# ---------------------------------------------------------------------------
def main_adjoint(args, tp, torch, rank, world, local, dist):
    import trackpad_b200.workloads as W
    turns = args.turns or 256
    clocks = Clocks(local)
    r = adjoint_ratio(tp, local, turns=turns, warmup=max(6, args.warmup), steps=args.steps)
    clk = clocks.stop()
    # end to end through the public API with host arrays (inputs staged every call)
    lat, beam = W.dba_ring(), W.dba_beam()
    c0 = W.gaussian(65536, seed=0)
    params = W.magnet_indices(lat)
    t0 = time.perf_counter()
    tp.ringpass_adjoint(c0, lat, beam, None, turns, params, sigma=SIGMA_LOSS, lost_weight=LOST_WEIGHT, aperture=0.02)
    t_adj = time.perf_counter() - t0
    c = c0.copy(order="F")
    l = np.zeros(len(c), np.int64)
    t0 = time.perf_counter()
    tp.ringpass_(c, lat, beam, l, turns, aperture=0.02)
    t_fwd = time.perf_counter() - t0
    if rank == 0:
        line = {"metric": r["metric"], "value": r["value"], "unit": "x", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["adjoint_ms"], "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Philox beam)",
                "config": {"workload": r["config"]}, "detail": r,
                "e2e": {"value": t_adj / t_fwd, "unit": "x", "h2d_bytes_per_step": 65536 * 48,
                        "d2h_bytes_per_step": 8 * (1 + len(params))},
                "gpu_launches": 3 * args.steps, "clocks": clk}
        print(json.dumps(line))


def batched_adjoint_measure(w, tp, torch, local, steps, warmup):
    """Per step: the batched forward (CUDA graph) and the batched adjoint
    (loss and gradients of every variant) on the same beams; device times."""
    import trackpad_b200.workloads as W
    dev = torch.device("cuda", local)
    n = w["coords"].shape[0]
    batch = tp.Batch(w["lats"], device=local)
    betis = np.full(len(w["lats"]), tp.beti(w["beam"]))
    params = [W.magnet_indices(l) for l in w["lats"]]
    init = torch.from_numpy(np.ascontiguousarray(w["coords"].T)).to(dev)
    coords = torch.empty_like(init)
    lost = torch.zeros(n, dtype=torch.int64, device=dev)
    turns = w["turns"]
    stream = torch.cuda.current_stream(dev)
    clocks = Clocks(local)
    fwd, adj, rev = [], [], []
    st = None
    for i in range(warmup + steps):
        coords.copy_(init)
        lost.zero_()
        batch.ringpass_(coords.T, w["poff"], betis, lost, turns, aperture=w["aperture"], use_graph=True,
                        stream=stream.cuda_stream)
        f = tp.last_stats(local)["kernel_ms"]
        batch.ringpass_adjoint(init.T, w["poff"], betis, None, turns, params, sigma=SIGMA_LOSS,
                               lost_weight=LOST_WEIGHT, aperture=w["aperture"])
        st = tp.adjoint_stats()
        if i >= warmup:
            fwd.append(f)
            adj.append(st["forward_ms"] + st["reverse_ms"])
            rev.append(st["reverse_ms"])
    clk = clocks.stop()
    f, a = float(np.median(fwd)), float(np.median(adj))
    return dict(f=f, a=a, rev=float(np.median(rev)), st=st, clocks=clk, params=int(sum(len(p) for p in params)))


def batched_adjoint_summary(args, tp, torch, local):
    """The batched time-dependent adjoint / batched forward time ratio (64
    variants, 16,384 particles each, 50-turn steps) as an object of the
    default line."""
    w = batched_workload(argparse.Namespace(nvar=0, turns=0), 0, time_dependent=True)
    m = batched_adjoint_measure(w, tp, torch, local, steps=2, warmup=7)
    return {"metric": "batched adjoint/forward time ratio", "value": m["a"] / m["f"], "unit": "x",
            "higher_is_better": False, "steps": 2, "warmup": 7,
            "config": {"workload": w["name"], "turns_per_step": w["turns"], "parameters": m["params"]},
            "batched_forward_ms": m["f"], "batched_adjoint_ms": m["a"], "reverse_ms": m["rev"],
            "checkpoint_every": m["st"]["checkpoint_every"], "checkpoint_bytes": m["st"]["checkpoint_bytes"],
            "reconstruction_error": m["st"]["reconstruction_error"], "target": "<= 3", "clocks": m["clocks"]}


def main_batched_adjoint(args, tp, torch, rank, world, local, dist):
    w = batched_workload(args, rank, time_dependent=True)
    m = batched_adjoint_measure(w, tp, torch, local, args.steps, max(7, args.warmup))
    st = m["st"]
    if rank == 0:
        line = {"metric": "adjoint/forward time ratio", "value": m["a"] / m["f"], "unit": "x", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["a"], "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded Philox variants and beams)",
                "config": {"workload": w["name"], "turns_per_step": w["turns"], "parameters": m["params"]},
                "detail": {"batched_forward_ms": m["f"], "batched_adjoint_ms": m["a"], "reverse_ms": m["rev"],
                           "checkpoint_every": st["checkpoint_every"], "checkpoint_bytes": st["checkpoint_bytes"],
                           "reconstruction_error": st["reconstruction_error"],
                           "forward_rate": st["units"] / (m["f"] * 1e-3), "target": "<= 3"},
                "gpu_launches": 3 * args.steps, "clocks": m["clocks"]}
        print(json.dumps(line))


# ---------------------------------------------------------------------------
# Truncated power series maps
# ---------------------------------------------------------------------------
def main_tpsa(args, tp, torch, rank, world, local, dist):
    """TPSA maps (ext/TrackPadPolySeriesExt.jl) of the FODO ring about seeded
    reference orbits: each step tracks `maps` series maps of order `order`
    through `turns` turns with host arrays in and out (tp_tpsa_ringpass)."""
    import trackpad_b200.workloads as W
    lat, beam = W.fodo_ring(), W.fodo_beam()
    nmaps = args.maps or 2048
    order = args.order
    turns = args.turns or 1
    refs = W.gaussian(nmaps, seed=100 + rank, sigma=(1e-4, 1e-5, 1e-4, 1e-5, 1e-3, 1e-4))
    base = np.ascontiguousarray(np.stack([tp.polyseries_variables(r, order).coef for r in refs]))
    m = base.shape[2]
    for _ in range(args.warmup):
        tp.tpsa.ringpass(lat, base, beam, turns, order=order)
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    k_ms, wall, flops, smul = [], [], 0.0, 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        out = tp.tpsa.ringpass(lat, base, beam, turns, order=order)
        wall.append(time.perf_counter() - t0)
        st = tp.tpsa.last_stats()
        k_ms.append(st["kernel_ms"])
        flops += st["flops"]
        smul += st["series_mul"]
    clk = clocks.stop()
    units = float(nmaps) * len(lat) * turns
    t = torch.tensor([float(np.sum(k_ms)) * 1e-3, float(np.sum(wall))], dtype=torch.float64,
                     device=torch.device("cuda", local))
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    kern_s, wall_s = float(t[0]), float(t[1])
    peak = tp.probe_fp64_peak(local)
    achieved = flops / kern_s / 1e12
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_ref
        nsamp, dt = 0, 0.0
        while dt < 10.0 and nsamp < nmaps:
            k = min(8, nmaps - nsamp)
            arr = np.ascontiguousarray(base[nsamp:nsamp + k])
            t0 = time.perf_counter()
            oracle_ref.tpsa_ringpass(lat, arr, tp.beti(beam), order, nturns=turns)
            dt += time.perf_counter() - t0
            nsamp += k
        cpu = {"value": nsamp * len(lat) * turns / dt, "unit": "map*element*turns/s", "cores": 1, "kind": "port",
               "sample": f"{nsamp} of the step's maps through the oracle's series algebra, one thread, {dt:.1f} s"}
    if rank == 0:
        line = {
            "metric": f"TPSA map*element*turns/s (order {order})", "value": units * world * args.steps / kern_s,
            "unit": "map*element*turns/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": kern_s / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Philox reference orbits)",
            "config": {"workload": f"FODO ring, 8 cells (32 elements), 1 GeV e-, {nmaps} maps of order {order} "
                                   f"({m} coefficients per series), {turns} turn(s) per step",
                       "maps_per_gpu": nmaps, "order": order, "coefficients": m,
                       "series_products_per_step": smul / args.steps,
                       "launch": {"grid": st["grid"], "block": st["block"], "shared_pool": st["shared_pool"],
                                  "slots": st["slots"], "slots_used": st["slots_used"]},
                       "l2": "inputs and outputs cross PCIe every step (host arrays)"},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None,
                         "flops_per_launch": flops / args.steps, "kernel_ms": kern_s / args.steps * 1e3,
                         "peak_source": "measured FP64 FMA throughput of this device (tp_probe_fp64_peak)"},
            "cpu_baseline": cpu,
            "e2e": {"value": units * world * args.steps / wall_s, "unit": "map*element*turns/s",
                    "h2d_bytes_per_step": int(base.nbytes), "d2h_bytes_per_step": int(base.nbytes)},
            "gpu_launches": args.steps, "clocks": clk,
        }
        print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank, world, local = dist_env()
    import torch
    import __graft_entry__
    tp = __graft_entry__.load_package()
    tp.tracking.TABLE_IN_SMEM = bool(args.table_smem)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    fn = {"dba": main_track, "fodo": main_track, "batched": main_batched, "adjoint": main_adjoint,
          "batched_adjoint": main_batched_adjoint, "tpsa": main_tpsa}[args.workload]
    fn(args, tp, torch, rank, world, local, dist)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
