"""Benchmark of the bit-exact flip dynamics on the a=b=c=500 hexagon.

Workload (both arms): lozenge tilings of the a=b=c=500 hexagon
(LozengeTiler::AlmostHexDomain(500, 0) -> MinTiling: a 1008 x 1008 tiling,
338,688 flip attempts per colour step), started from the minimal tiling,
TinyMT streams, uniform weights (int8 storage).  One bench step is one Walk
call of 3,000 reference colour steps (1,000 sweeps) with seed 42 + k,
continuing from the previous call's tiling; 20 steps are the 20,000-sweep
walk.  After the warm-up steps the chain restarts from the minimal tiling, so
the timed steps are always the same walk.

  value : attempts/s with the lattice resident on the device (rt_upload before
          the timed steps; rt_run per step), CUDA events on the library's
          stream, L2 flushed (256 MiB write) before every step;
  e2e   : the same steps through rt_walk (the reference's Walk contract: host
          int32 tiling in pinned memory, H2D + split + walk + merge + D2H
          every step), wall clock around the synchronous call.

Beside the headline the line carries the q = 0.99 int32 walk, the fast and
bit-plane modes, the Aztec diamond of order 2000, the batched workload of 4,096
mixed chains (per kernel family), a short CFTP run, the six-vertex model and
the warm vs cold start comparison (sweeps to 0.5 % mean-height error), each in
its own key.

`--impl reference` runs the same steps with the reference's own CPU code (its
kernels and LozengeTiler::Walk built through oracle/shim: oracle/_ref, OpenMP
over work items on every host core), or the oracle's C restatement where
oracle/_ref is absent.

Multi-GPU: one walk is a single lattice, which this path does not split, so
--gpus N runs N independent replicas (seeds 42 + rank), value = total
attempts / max over ranks of the device time.

Other workloads (their own JSON line, not the headline): --workload cftp
(coupling from the past on an Aztec diamond, optionally with two-periodic
domino weights), --workload extremal (extremal tilings of large domains, host
flood vs device), --legs (single legs for profiling captures).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "flip attempts/s & HBM GB/s vs peak; sweeps-to-0.5% height error, warm vs cold"
HEX_SIDE = 500
SEGMENT = 3000  # reference colour steps per bench step (1,000 sweeps of the three colours)
SEED = 42
L2_FLUSH_BYTES = 256 << 20
FALLBACK_HBM_GBS = 6650.0


def workload_config(world: int = 1) -> dict:
    """The workload of both arms (identical dicts)."""
    return {
        "workload": "lozenge hexagon a=b=c=500 (1008x1008 tiling, 338688 attempts per colour step), minimal "
                    "tiling start, TinyMT bit-exact mode, uniform weights; one step = one Walk call of 3000 colour "
                    "steps (1000 sweeps), seed 42+k, continuing the chain; 20 steps = the 20000-sweep walk",
        "domain": "LozengeTiler::AlmostHexDomain(500,0)",
        "tiling_side": 1008,
        "attempts_per_colour_step": 1008 * 336,
        "colour_steps_per_step": SEGMENT,
        "seed": SEED,
        "weights": "uniform (int8 lattice)",
        "l2": "flushed (256 MiB write) before every timed step",
        "parallelism": f"replicas{world}",
    }


def peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def start_tiling():
    import randomtilings_b200 as rt

    d = rt.LozengeTiler.AlmostHexDomain(HEX_SIDE, 0)
    return np.asarray(rt.LozengeTiler.MinTiling(d), dtype=np.int32)


def algorithmic_bytes_per_step(n: int, elem: int, rng_state: bool = True) -> int:
    """Bytes a colour step would move through HBM: every colour-array site read
    and written once, plus the TinyMT state (s0..s3 read + write, 32 B) of
    every attempt (none in the counter-based modes)."""
    sites = n * n
    attempts = n * (n // 3)
    return 2 * sites * elem + (attempts * 32 if rng_state else 0)


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while timing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        under_load = [x for x in sm if x > 500] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(under_load) if under_load else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons, "samples": len(rows)}


def dist_setup(ngpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        return rank, world, local, dist
    return 0, 1, 0, None


def _reduce_device(dist) -> str:
    # NCCL reduces CUDA tensors; the gloo backend (the CPU tests of this code) host ones
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def all_max(dist, x: float) -> float:
    """The largest x over the ranks (device times: the job is as slow as its slowest GPU)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def all_sum(dist, xs: list[float]) -> list[float]:
    """Element-wise sums over the ranks (attempts, bytes)."""
    if dist is None:
        return list(xs)
    import torch

    t = torch.tensor(xs, dtype=torch.float64, device=_reduce_device(dist))
    dist.all_reduce(t)
    return [float(v) for v in t.tolist()]


def shard(count: int, rank: int, world: int) -> range:
    """Independent units (batch chains, CFTP seeds) dealt round-robin to the ranks."""
    return range(rank, count, world)


def replica_seed(rank: int) -> int:
    """Seed of rank r's replica walk (the ranks walk independent replicas)."""
    return SEED + rank


def barrier(dist):
    if dist is not None:
        dist.barrier()


def time_device_steps(tiler, t0: np.ndarray, steps: int, warmup: int, seed: int, flush,
                      colour_steps: int = SEGMENT) -> tuple[list[float], np.ndarray]:
    """Device milliseconds of `steps` bench steps (CUDA events on the library's
    stream), after `warmup` untimed ones; the chain restarts from t0 before the
    timed steps.  Returns the times and the final tiling."""
    import torch

    s = torch.cuda.ExternalStream(tiler.stream)
    tiler.upload(t0)
    for w in range(warmup):
        tiler.run(colour_steps, seed + w)
    tiler.synchronize()
    tiler.upload(t0)
    out = []
    for k in range(steps):
        flush()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        tiler.run(colour_steps, seed + k)
        e1.record(s)
        tiler.synchronize()
        out.append(e0.elapsed_time(e1))
    final = np.empty_like(t0)
    tiler.download(final)
    return out, final


def time_e2e_steps(tiler_cls, kwargs, t0: np.ndarray, steps: int, warmup: int, seed: int,
                   flush) -> tuple[list[float], np.ndarray]:
    """The same steps through rt_walk with a host tiling in pinned memory: wall
    time of each synchronous call (H2D, split, walk, merge, D2H)."""
    import torch

    tl = tiler_cls(**kwargs)
    host = torch.empty(t0.size, dtype=torch.int32).pin_memory().numpy()
    host[:] = t0.reshape(-1)
    for w in range(warmup):
        tl.Walk(host, SEGMENT, seed + w)
    host[:] = t0.reshape(-1)
    out = []
    for k in range(steps):
        flush()
        torch.cuda.synchronize()
        a = time.perf_counter()
        tl.Walk(host, SEGMENT, seed + k)
        out.append((time.perf_counter() - a) * 1e3)
    tl.close()
    return out, host.copy()


def golden_digest(steps: int) -> str | None:
    """The reference's own result after `steps` bench steps from seed 42
    (tests/golden/bench_parity.json), when that fixture covers them."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "bench_parity.json")) as f:
            return json.load(f).get(f"hex500/uniform/segment{steps - 1}")
    except OSError:
        return None


def digest(a: np.ndarray) -> str:
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(a, dtype="<i4").tobytes()).hexdigest()


def leg(ms: list[float], attempts: int, world: int, dist, extra: dict | None = None) -> dict:
    total = all_max(dist, sum(ms))
    out = {"value": attempts * SEGMENT * len(ms) * world / (total / 1e3), "unit": "attempts/s",
           "ms_per_step": total / len(ms), "us_per_colour_step": total / len(ms) / SEGMENT * 1e3}
    out.update(extra or {})
    return out


def side_leg(fn, *a):
    """A leg beside the headline: its figures, or the error that stopped it
    (the headline line is printed either way)."""
    try:
        return fn(*a)
    except Exception as e:  # reported in the JSON line, not swallowed
        print(f"{fn.__name__} failed: {e!r}", file=sys.stderr, flush=True)
        return {"error": repr(e)}


def run_b200(args) -> None:
    import torch

    rank, world, local, dist = dist_setup(args.gpus)
    import randomtilings_b200 as rt

    rt.load(build_if_missing=False)
    t0 = start_tiling()
    n = int(round(t0.size ** 0.5))
    attempts = n * (n // 3)
    seed = replica_seed(rank)
    flush_buf = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def flush():
        flush_buf.fill_(1.0)

    tl = rt.LozengeTiler(device=local)
    tq = rt.LozengeTiler(device=local, kernel=rt.RT_KERNEL_QWEIGHT, q=0.99, qcmp=rt.RT_QCMP_FLOAT32)
    tf = rt.LozengeTiler(device=local, rng=rt.RT_RNG_PHILOX)
    tp = rt.LozengeTiler(device=local, rng=rt.RT_RNG_PLANES)

    barrier(dist)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        wall0 = time.perf_counter()
        ms, final = time_device_steps(tl, t0, args.steps, args.warmup, seed, flush)
        wall = time.perf_counter() - wall0
        torch.cuda.synchronize()
        barrier(dist)
        phases, launches = tl.last_run_info()
        e2e_ms, e2e_final = time_e2e_steps(rt.LozengeTiler, {"device": local}, t0, args.steps, args.warmup, seed,
                                           flush)
        ms_q, _ = time_device_steps(tq, t0, args.steps, args.warmup, seed, flush)
        ms_f, _ = time_device_steps(tf, t0, args.steps, args.warmup, seed, flush)
        ms_p, _ = time_device_steps(tp, t0, args.steps, args.warmup, seed, flush)
    clocks = clk.summary()
    for t in (tl, tq, tf, tp):
        t.close()

    total_ms = all_max(dist, sum(ms))
    total_e2e = all_max(dist, sum(e2e_ms))
    value = attempts * SEGMENT * args.steps * world / (total_ms / 1e3)
    per_launch_ms = sum(ms) / len(ms)
    peak, peak_kind = peaks()
    algo = algorithmic_bytes_per_step(n, 1) * SEGMENT
    achieved = algo / (per_launch_ms / 1e3) / 1e9
    want = golden_digest(args.steps) if seed == SEED else None
    parity = {"final_tiling_sha256": digest(final), "e2e_equal": bool(np.array_equal(final, e2e_final)),
              "reference_sha256": want, "equal_to_reference": None if want is None else digest(final) == want}

    aztec = side_leg(measure_aztec2000, args, local, seed, flush)
    sixv = side_leg(measure_sixv, args, local)
    batched = None if args.no_batch else side_leg(measure_batch, args, rank, world, dist, peak)
    cftp = None if args.no_cftp else side_leg(measure_cftp_small, args, rank, world, dist)
    warm = side_leg(measure_warm_cold, args, local) if (rank == 0 and not args.no_warm) else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(segments=args.cpu_segments)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "attempts/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "int8",
            "data": "synthetic (the reference's own domain builder; no dataset)",
            "config": workload_config(world),
            "impl": "b200",
            "us_per_colour_step": per_launch_ms / SEGMENT * 1e3,
            "sweeps_per_s": value / attempts / 3,
            "parity": parity,
            "e2e": {
                "value": attempts * SEGMENT * args.steps * world / (total_e2e / 1e3),
                "unit": "attempts/s",
                "h2d_bytes_per_step": n * n * 4,
                "d2h_bytes_per_step": n * n * 4,
                "ms_per_step": total_e2e / args.steps,
                "host_buffer": "pinned",
            },
            "roofline": {
                "bound": "hbm",
                "achieved": achieved,
                "peak": peak,
                "unit": "GB/s",
                "frac": achieved / peak,
                "peak_kind": peak_kind,
                "traffic": args.traffic,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one 600-colour-step "
                                  "launch of this kernel on this workload (a capture, not this run); a launch "
                                  "reads the lattice in and writes it back once whatever its step count",
                "dram_gbs": args.traffic / (per_launch_ms / 1e3) / 1e9,
                "limiter": "phase latency: the lattice and the TinyMT states stay on chip for the whole launch, "
                           "so a colour step costs the latency of one word's update plus the exchange of edge "
                           "rows between neighbouring CTAs, not DRAM bandwidth",
                "kernel": "rtb::word_kernel<FAM_LOZENGE8, 1, bit-exact> (one cooperative launch per step)",
                "algorithmic_bytes_per_launch": algo,
                "launch_ms": per_launch_ms,
            },
            "q_weighted": leg(ms_q, attempts, world, dist, {
                "q": 0.99, "compare": "float32", "dtype": "int8",
                "kernel": "rtb::word_kernel<FAM_LOZENGE8, 1, bit-exact, q> (add below thr[2], remove in [2^22, thr[3]))",
                "hbm_gbs_algorithmic": algorithmic_bytes_per_step(n, 1) * SEGMENT / (sum(ms_q) / len(ms_q) / 1e3) / 1e9}),
            "fast_mode": leg(ms_f, attempts, world, dist, {
                "rng": "Philox4x32-10 keyed by (position quad, step, chain), cyclic colours", "dtype": "int8"}),
            "bit_planes": leg(ms_p, attempts, world, dist, {
                "rng": "one Philox4x32-10 bit per site, heat-bath rule, lattice as bit planes, cyclic colours"}),
            "aztec2000": aztec,
            "six_vertex": sixv,
            "batched": batched,
            "cftp": cftp,
            "warm_vs_cold": warm,
            "gpu_launches": int(launches) * args.steps,
            "phases_per_launch": int(phases),
            "clocks": clocks,
            "wall_s_timed_region": wall,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def measure_aztec2000(args, device: int, seed: int, flush) -> dict:
    """The large lattice of the warm-start evaluation (Aztec diamond of order
    2000, 4006 x 4006 tiling, 8,012,004 attempts per colour step): fast mode and
    bit-plane mode, walks of 4,000 colour steps."""
    import randomtilings_b200 as rt

    d = rt.DominoTiler.AztecDiamond(2000)
    t0 = np.asarray(rt.DominoTiler.MinTiling(d), dtype=np.int32)
    n = int(round(t0.size ** 0.5))
    att = (n - 2) * (n // 2 - 2)
    steps = 4000
    out = {"workload": "Aztec diamond n=2000 (4006x4006), minimal tiling, walks of 4000 colour steps",
           "attempts_per_colour_step": att, "unit": "attempts/s"}
    for name, rng in (("fast_mode", rt.RT_RNG_PHILOX), ("bit_planes", rt.RT_RNG_PLANES)):
        tl = rt.DominoTiler(device=device, rng=rng)
        ms, _ = time_device_steps(tl, t0, 2, 3, seed, flush, colour_steps=steps)
        tl.close()
        out[name] = att * steps / (sum(ms) / len(ms) / 1e3)
    return out


def measure_sixv(args, device: int) -> dict:
    """The six-vertex model (domain-wall boundary, n = 1000, uniform weights):
    attempts/s of a walk of 400 sweeps from the minimal heights, wall clock
    around the synchronous call after one warm-up walk."""
    import randomtilings_b200 as rt

    n, sweeps = 1000, 400
    tl = rt.SixVertexTiler(device=device)
    h = rt.SixVertexTiler.MinHeights(n)
    tl.Walk(h.copy(), 20, 1)
    a = time.perf_counter()
    tl.Walk(h, sweeps, 2)
    dt = time.perf_counter() - a
    tl.close()
    return {"workload": f"six-vertex, domain-wall boundary n={n}, {sweeps} sweeps (4 colour steps each), "
                        "uniform weights, heat bath", "value": (n - 1) ** 2 * sweeps / dt, "unit": "attempts/s",
            "wall_s": dt, "valid": bool(rt.SixVertexTiler.IsValid(h))}


def measure_cftp_small(args, rank: int, world: int, dist) -> dict:
    """Coupling from the past in the default run (the 32-seed run at order
    500 is --workload cftp): an Aztec diamond of order
    args.cftp_small_order, bit-plane heat bath, coupled maximal and minimal
    chains in one launch, doubling from 1,024 colour steps, master seeds
    0..args.cftp_small_seeds-1 dealt to the ranks."""
    import randomtilings_b200 as rt

    d = rt.DominoTiler.AztecDiamond(args.cftp_small_order)
    tmax, tmin = rt.DominoTiler.MaxTiling(d), rt.DominoTiler.MinTiling(d)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    runs = []
    for s in shard(args.cftp_small_seeds, rank, world):
        tl = rt.DominoTiler(device=local, kernel=rt.RT_KERNEL_CFTP, rng=rt.RT_RNG_PLANES)
        a = time.perf_counter()
        _, st = tl.CFTP(tmax, tmin, first_steps=1024, master_seed=s, max_trials=24)
        st["wall_s"] = time.perf_counter() - a
        tl.close()
        runs.append(st)
    steps = [r["total_steps"] for r in runs]
    co = all_sum(dist, [float(sum(r["coalesced"] for r in runs)), float(len(runs))])
    wall = all_max(dist, sum(r["wall_s"] for r in runs))
    return {"workload": f"Aztec diamond n={args.cftp_small_order}, domino heat bath (bit planes), coupled max/min "
                        "chains, doubling from 1024 colour steps",
            "seeds": int(co[1]), "coalesced": int(co[0]),
            "median_colour_steps_rank0": statistics.median(steps) if steps else None,
            "max_colour_steps_rank0": max(steps) if steps else None,
            "device_ms_rank0": sum(r["device_ms"] for r in runs), "wall_s": wall}


def measure_warm_cold(args, device: int) -> dict:
    """Sweeps to a mean-height error of 0.5 % of the side, warm start vs cold
    start, at reduced size: the coordinate MLP is trained in the run on its own
    kernels from the mean heights of plain chains (Aztec diamonds of orders
    args.warm_train_aztec, hexagons of sides args.warm_train_hexagon), then
    judged on an Aztec diamond of order args.warm_aztec and an
    a=b=c=args.warm_hexagon hexagon against the long-chain mean, the max / min
    sandwich certifying convergence."""
    from randomtilings_b200 import warmstart as ws

    t0 = time.perf_counter()
    specs = ws.training_specs(args.warm_domains, seed=0, aztec=tuple(args.warm_train_aztec),
                              hexagon=tuple(args.warm_train_hexagon), q=(0.98, 1.0))
    x, y, _ = ws.generate_dataset(specs, device=device, samples=8)
    t_data = time.perf_counter() - t0
    w = ws.WarmStart(device=device, seed=0)
    t1 = time.perf_counter()
    losses = w.fit(x, y, steps=args.warm_train_steps, batch=8192, lr=3e-3)
    t_train = time.perf_counter() - t1
    out = {"threshold": 0.005, "train_domains": len(specs), "train_rows": int(x.shape[0]),
           "dataset_s": round(t_data, 2), "train_s": round(t_train, 2), "final_loss": float(losses[-1]), "eval": []}
    for kind, size in (("aztec", (args.warm_aztec,)), ("hexagon", (args.warm_hexagon,) * 3)):
        spec = ws.DomainSpec(kind, size)
        p = ws.prepare(spec, device)
        tw, st = w.warm_tiling(p)
        r = ws.relax(p, {"cold": p.tmin, "warm": tw}, int(1.5 * ws.burn_sweeps(spec)), points=40,
                     replicas=args.warm_replicas, device=device, threshold=0.005)
        s = r["sweeps_to_threshold"]
        out["eval"].append({
            "domain": spec.label(), "sweeps_to_0.5pct": s, "speedup": ws.speedup(r),
            "error_at_sweep0": {k: round(v[0], 5) for k, v in r["curves"].items()},
            "final_sandwich_gap": round(r["sandwich_gap"][-1], 5), "replicas": args.warm_replicas,
            "sweeps_run": r["sweeps"][-1], "device_ms": round(r["device_ms"], 1)})
    out["wall_s"] = round(time.perf_counter() - t0, 2)
    return out


def run_legs(args) -> None:
    """Profiling runs: only the walks named in args.legs (no JSON contract
    line, no timing claims), each `args.steps` walks after `args.warmup`."""
    import randomtilings_b200 as rt
    from randomtilings_b200 import workloads

    rt.load(build_if_missing=False)
    legs = set(args.legs.split(","))
    t0 = start_tiling()
    kinds = {"headline": {}, "q": {"kernel": rt.RT_KERNEL_QWEIGHT, "q": 0.99, "qcmp": 0},
             "fast": {"rng": rt.RT_RNG_PHILOX}, "planes": {"rng": rt.RT_RNG_PLANES}}
    for name, kw in kinds.items():
        if name not in legs:
            continue
        tl = rt.LozengeTiler(**kw)
        tl.upload(t0)
        for k in range(args.warmup + args.steps):
            tl.run(args.walk_steps, SEED + k)
        tl.synchronize()
        tl.close()
        print(f"{name}: {args.warmup + args.steps} walks of {args.walk_steps} colour steps", flush=True)
    if "sixv" in legs:
        # the six-vertex model at n = 1000, walks of walk_steps / 4 sweeps
        tl = rt.SixVertexTiler()
        h = rt.SixVertexTiler.MinHeights(1000)
        sweeps = max(1, args.walk_steps // 4)
        for k in range(args.warmup + args.steps):
            tl.Walk(h, sweeps, k + 1)
        tl.close()
        print(f"sixv: {args.warmup + args.steps} walks of {sweeps} sweeps", flush=True)
    if "batch" in legs:
        bt = rt.Batch()
        models = None if args.batch_models == "all" else {int(m) for m in args.batch_models.split(",")}
        n = 0
        for seed in range(args.batch_chains):
            model, spec = workloads.mixed_chain_spec(seed)
            if models is not None and model not in models:
                continue
            bt.add(model, workloads.start_tiling(model, spec), key=seed, chain=seed)
            n += 1
        if args.batch_plan:
            cl, block = (int(v) for v in args.batch_plan.split(","))
            bt.set_tuning(False, cl, block)
        bt.run(2)
        bt.run(args.batch_sweeps)
        print(f"batch: {n} chains, {args.batch_sweeps} sweeps, {bt.info()}", flush=True)
        bt.close()


def run_cftp(args) -> None:
    """CFTP on an Aztec diamond (order args.cftp_order), coupled
    chains from the maximal and minimal tilings, doubling from 1,024 colour
    steps, one run per master seed 0..args.cftp_seeds-1."""
    import randomtilings_b200 as rt

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    d = rt.DominoTiler.AztecDiamond(args.cftp_order)
    tmax, tmin = rt.DominoTiler.MaxTiling(d), rt.DominoTiler.MinTiling(d)
    rng = {"tinymt": rt.RT_RNG_TINYMT, "philox": rt.RT_RNG_PHILOX, "planes": rt.RT_RNG_PLANES}[args.cftp_rng]
    weights = [float(v) for v in args.cftp_weights.split(",")] if args.cftp_weights else None
    runs = []
    for s in shard(args.cftp_seeds, rank, world):
        tl = rt.DominoTiler(device=local, kernel=rt.RT_KERNEL_CFTP, rng=rng)
        if weights:
            tl.SetWeights(*rt.DominoTiler.TwoPeriodicWeights(*weights))
        a = time.perf_counter()
        _, st = tl.CFTP(tmax, tmin, first_steps=1024, master_seed=s, max_trials=24)
        st["wall_s"] = time.perf_counter() - a
        st["seed"] = s
        tl.close()
        runs.append(st)
        print(json.dumps(st), file=sys.stderr, flush=True)
    if rank == 0:
        steps = [r["total_steps"] for r in runs]
        print(json.dumps({
            "metric": "CFTP coalescence (colour steps from the past) and wall time",
            "workload": f"Aztec diamond n={args.cftp_order}, domino heat bath"
                        + (f", two-periodic weights a,b = {args.cftp_weights}" if weights else "")
                        + ", doubling from 1024 steps",
            "rng": args.cftp_rng, "seeds": len(runs), "coalesced": sum(r["coalesced"] for r in runs),
            "median_steps": statistics.median(steps), "max_steps": max(steps),
            "median_sweeps": statistics.median(steps) / 2,
            "total_wall_s": sum(r["wall_s"] for r in runs), "total_device_ms": sum(r["device_ms"] for r in runs),
            "runs": runs}), flush=True)


def run_extremal(args) -> None:
    """Set-up of a large domain: MinTiling, MaxTiling and the TilingToHeightfunc
    of both, on the host (the reference's flood) and on the device
    (rt_extremal_tilings into host arrays; rt_extremal_tilings_device into
    device buffers), on an Aztec diamond of order args.extremal_order and an
    a=b=c hexagon of side args.extremal_side; results compared.  The
    device-buffer leg runs after every host-output leg (its torch buffers stay
    cached in the process)."""
    import numpy as np

    import randomtilings_b200 as rt
    from randomtilings_b200 import builders

    if int(os.environ.get("RANK", "0")) != 0:
        return
    builders.extremal_tilings(rt.RT_DOMINO, rt.DominoTiler.AztecDiamond(4))  # context and module load
    out, kept = [], []
    for model, cls, d, name in (
            (rt.RT_DOMINO, rt.DominoTiler, rt.DominoTiler.AztecDiamond(args.extremal_order),
             f"Aztec diamond n={args.extremal_order}"),
            (rt.RT_LOZENGE, rt.LozengeTiler, rt.LozengeTiler.Hexagon(*[args.extremal_side] * 3),
             f"hexagon a=b=c={args.extremal_side}")):
        a = time.perf_counter()
        tmin, tmax = cls.MinTiling(d), cls.MaxTiling(d)
        hmin, hmax = cls.TilingToHeightfunc(tmin, d), cls.TilingToHeightfunc(tmax, d)
        host_s = time.perf_counter() - a
        walls, st, phases = [], None, []
        for _ in range(args.steps):
            a = time.perf_counter()
            dev, st = builders.extremal_tilings(model, d)
            walls.append(time.perf_counter() - a)
            phases.append({k: round(st[k], 2) for k in ("walk_ms", "alloc_ms", "upload_ms", "device_ms",
                                                        "download_ms")})
        equal = all(np.array_equal(dev[k], np.asarray(v)) for k, v in
                    (("tmin", tmin), ("tmax", tmax), ("hmin", hmin), ("hmax", hmax)))
        out.append({"domain": name, "n": st["n"], "equal_to_host": equal, "host_s": round(host_s, 4),
                    "device_call_s": round(statistics.median(walls), 4), "first_call_s": round(walls[0], 4),
                    "phases_ms": phases, "device_ms": round(st["device_ms"], 3),
                    "passes": st["passes"], "tile_updates": st["tile_updates"], "boundary": st["boundary"],
                    "speedup_call": round(host_s / statistics.median(walls), 1)})
        kept.append((model, d, dev))
    # the same into device buffers (rt_extremal_tilings_device): no copies back
    import torch

    for r, (model, d, dev) in zip(out, kept):
        bufs = {k: torch.empty(dev[k].size, dtype=torch.int32, device="cuda:0") for k in dev}
        dwalls = []
        for _ in range(args.steps):
            a = time.perf_counter()
            builders.extremal_tilings_device(model, d, **{k: v.data_ptr() for k, v in bufs.items()})
            dwalls.append(time.perf_counter() - a)
        r["equal_to_host"] = r["equal_to_host"] and all(np.array_equal(bufs[k].cpu().numpy(), dev[k]) for k in dev)
        r["device_outputs_call_s"] = round(statistics.median(dwalls), 4)
        r["speedup_device_outputs"] = round(r["host_s"] / statistics.median(dwalls), 1)
        print(json.dumps(r), file=sys.stderr, flush=True)
    print(json.dumps({"metric": "extremal tilings + heights set-up time (host flood vs device relaxation)",
                      "unit": "s", "higher_is_better": False, "runs": out}), flush=True)


FAMILY_NAMES = {0: "domino", 1: "lozenge", 2: "rect_triangle", 3: "triangle_dimer"}
STEPS_PER_SWEEP = {0: 2, 1: 3, 2: 3, 3: 30}


def chain_costs(model: int, n: int) -> tuple[int, int, int]:
    """(attempts, bytes at the batched kernels' stored widths, bytes at the
    reference's storage widths) of one sweep of a chain of tiling side n:
    every colour step reads and writes each colour-array site once.  Stored
    widths: dominoes and lozenges 1 B; rectangle-triangles 4 B; triangle
    dimers 51 bit planes (6.375 B for the 8 arrays' sites, against 32 B as
    the reference's int arrays)."""
    steps = STEPS_PER_SWEEP[model]
    if model == 0:
        att, stored, ref = (n - 2) * (n // 2 - 2), n * n, n * n
    elif model in (1, 2):
        att = n * (n // 3)
        stored = ref = n * n * (1 if model == 1 else 4)
    else:
        m = n // 2
        att, stored, ref = m * m, 51 * m * m / 8, 32 * m * m
    return att * steps, 2 * stored * steps, 2 * ref * steps


def measure_batch(args, rank: int, world: int, dist, peak: float) -> dict:
    """The batched pattern: args.batch_chains chains of the mixed workload
    (chain seed s: domain type s mod 4, sizes from std::mt19937(s)), minimal
    tilings (bibone hexagons: their canonical start), args.batch_sweeps sweeps
    each in fast mode, as one graph of persistent cluster launches per kernel
    family; then each family alone for a shorter run.  Ranks take seeds
    round-robin (no communication); value = all ranks' attempts / max device
    time.  Bytes are counted at the widths the kernels store (the lattices stay
    in shared memory, so they are what a streaming walk would move)."""
    import randomtilings_b200 as rt
    from randomtilings_b200 import workloads

    local = int(os.environ.get("LOCAL_RANK", "0"))
    chains = []
    for seed in shard(args.batch_chains, rank, world):
        model, t = workloads.mixed_chain(seed)
        chains.append((seed, model, t))
    per_fam = {}
    for seed, model, t in chains:
        n = int(round(np.asarray(t).size ** 0.5))
        a, b_st, b_ref = chain_costs(model, n)
        f = per_fam.setdefault(model, {"chains": 0, "attempts_per_sweep": 0, "stored_bytes_per_sweep": 0,
                                       "ref_bytes_per_sweep": 0})
        f["chains"] += 1
        f["attempts_per_sweep"] += a
        f["stored_bytes_per_sweep"] += b_st
        f["ref_bytes_per_sweep"] += b_ref

    bt = rt.Batch(device=local)
    for seed, model, t in chains:
        bt.add(model, t, key=seed, chain=seed)
    bt.run(2)  # autotuner (on a scratch copy) + graph build; then a short warm-up run
    bt.run(2)
    barrier(dist)
    bt.run(args.batch_sweeps)
    info = bt.info()
    bt.close()
    ms = all_max(dist, info["run_ms"])
    att = sum(f["attempts_per_sweep"] for f in per_fam.values()) * args.batch_sweeps
    stored = sum(f["stored_bytes_per_sweep"] for f in per_fam.values()) * args.batch_sweeps
    ref = sum(f["ref_bytes_per_sweep"] for f in per_fam.values()) * args.batch_sweeps
    tot_att, tot_stored, tot_ref = all_sum(dist, [float(att), float(stored), float(ref)])
    achieved = tot_stored / world / (ms / 1e3) / 1e9  # per GPU

    families = {}
    sweeps_f = max(1, min(args.batch_sweeps, args.batch_family_sweeps))
    for model, f in sorted(per_fam.items()):
        bf = rt.Batch(device=local)
        for seed, m_, t in chains:
            if m_ == model:
                bf.add(m_, t, key=seed, chain=seed)
        bf.run(2)
        bf.run(sweeps_f)
        fi = bf.info()
        bf.close()
        fms = fi["run_ms"]
        gbs = f["stored_bytes_per_sweep"] * sweeps_f / (fms / 1e3) / 1e9
        families[FAMILY_NAMES[model]] = {
            "chains_rank0": f["chains"], "sweeps": sweeps_f, "ms": fms,
            "attempts_per_s": f["attempts_per_sweep"] * sweeps_f / (fms / 1e3),
            "stored_gbs": gbs, "frac_stored": gbs / peak,
            "ref_width_gbs": f["ref_bytes_per_sweep"] * sweeps_f / (fms / 1e3) / 1e9,
            "plan": next(iter(fi["plans"].values()), None)}
    return {
        "workload": f"{args.batch_chains} chains of the mixed workload (seed s: s mod 4 -> Aztec diamond n in "
                    "[16,256] / hexagon a,b,c in [8,128] / bibone (triangle-dimer) hexagon side 64 / "
                    f"rectangle-triangle hexagon 64; sizes from std::mt19937(s)), minimal tilings, {args.batch_sweeps} "
                    "sweeps, fast mode (Philox), one CUDA graph",
        "value": tot_att / (ms / 1e3),
        "unit": "attempts/s",
        "ms": ms,
        "hbm_gbs_stored_widths": achieved,
        "frac": achieved / peak,
        "hbm_gbs_reference_widths": tot_ref / world / (ms / 1e3) / 1e9,
        "bytes_note": "frac counts every colour step reading and writing each site at the width the batched "
                      "kernels store it; the lattices stay in shared memory, so DRAM traffic is the load and "
                      "store of each chain once per launch",
        "families": families,
        "plans_rank0": info["plans"],
        "tune_ms_rank0": info["tune_ms"],
        "graph_launches": 1,
    }


def reference_walker(threads: int):
    """(start tiling, step function, kind, cores) of the reference's own CPU
    code: oracle/_ref's LozengeTiler::Walk over its kernels with OpenMP over
    work items, its own AlmostHexDomain / MinTiling for the start; else the
    oracle's C restatement (one core) on the library's builders."""
    from oracle import pyoracle as po

    if po.have_ref():
        d = po.ref_build("lozenge_almost_hex", p0=HEX_SIDE, p1=0)
        t0 = po.ref_build("lozenge_min", d).astype(np.int32)
        tiler = po.RefTiler("lozenge", t0.size, threads=threads)
        return t0, (lambda t, s: tiler.walk(t, SEGMENT, s)), "reference", threads
    t0 = start_tiling()
    return t0, (lambda t, s: po.lozenge_walk(t, SEGMENT, s)), "port", 1


def cpu_baseline(segments: int = 2) -> dict:
    """A bounded sample of the workload on the host cores: the first
    `segments` bench steps from the minimal tiling, wall clock."""
    threads = os.cpu_count() or 1
    t0, step, kind, cores = reference_walker(threads)
    attempts = t0.size // 3
    a = t0.copy()
    t = time.perf_counter()
    for k in range(segments):
        a = step(a, SEED + k)
    dt = time.perf_counter() - t
    return {"value": attempts * SEGMENT * segments / dt, "unit": "attempts/s", "cores": cores, "kind": kind,
            "sample": f"the first {segments} steps ({segments * SEGMENT} colour steps) of the hexagon walk from the "
                      f"minimal tiling, seed {SEED}, {dt:.1f} s"}


def run_reference(args) -> None:
    """The reference arm: the same steps (one Walk of 3,000 colour steps each,
    seeds 42 + k, continuing the chain) with the reference's own code on every
    host core; rank 0 alone under torchrun."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    threads = os.cpu_count() or 1
    t0, step, kind, cores = reference_walker(threads)
    attempts = t0.size // 3
    a = t0.copy()
    for w in range(args.warmup):
        a = step(a, SEED + w)
    a = t0.copy()
    times = []
    for k in range(args.steps):
        t = time.perf_counter()
        a = step(a, SEED + k)
        times.append((time.perf_counter() - t) * 1e3)
    value = attempts * SEGMENT * args.steps / (sum(times) / 1e3)
    want = golden_digest(args.steps)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "attempts/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": sum(times) / len(times),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int8",
        "data": "synthetic (the reference's own domain builder; no dataset)",
        "config": workload_config(world),
        "impl": "reference",
        "parity": {"final_tiling_sha256": digest(a), "reference_sha256": want,
                   "equal_to_reference": None if want is None else digest(a) == want},
        "cpu_baseline": {"value": value, "unit": "attempts/s", "cores": cores, "kind": kind,
                         "sample": f"the full timed run: {args.steps} steps of {SEGMENT} colour steps"},
        "e2e": {"value": value, "unit": "attempts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--cpu-segments", type=int, default=2, help="steps timed for cpu_baseline (about 10 s)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # dram__bytes_read.sum + dram__bytes_write.sum of one word_kernel launch on this workload (ncu
    # --set full of a 600-colour-step launch of this build: 1,160,960 B read, 0 written).  The
    # lattice stays on chip, so a launch of any number of colour steps moves the same bytes; a
    # timed run cannot read DRAM counters, so the figure comes from that capture.
    ap.add_argument("--traffic", type=float, default=1160960.0,
                    help="dram bytes per walk launch from an ncu capture (reported in roofline.traffic)")
    ap.add_argument("--batch-chains", type=int, default=4096)
    ap.add_argument("--batch-sweeps", type=int, default=5000)
    ap.add_argument("--batch-family-sweeps", type=int, default=500,
                    help="sweeps of each kernel family run alone (per-family figures)")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-cftp", action="store_true")
    ap.add_argument("--cftp-small-order", type=int, default=100)
    ap.add_argument("--cftp-small-seeds", type=int, default=8)
    ap.add_argument("--no-warm", action="store_true")
    ap.add_argument("--warm-domains", type=int, default=384)
    ap.add_argument("--warm-aztec", type=int, default=200)
    ap.add_argument("--warm-hexagon", type=int, default=100)
    ap.add_argument("--warm-replicas", type=int, default=16)
    ap.add_argument("--warm-train-aztec", type=int, nargs=2, default=(16, 160))
    ap.add_argument("--warm-train-hexagon", type=int, nargs=2, default=(8, 100))
    ap.add_argument("--warm-train-steps", type=int, default=3000)
    ap.add_argument("--legs", default="all",
                    help="profiling runs: comma-separated subset of headline,q,fast,planes,batch,sixv (no JSON line)")
    ap.add_argument("--batch-models", default="all",
                    help="with --legs batch: comma-separated rt_model values of the mixed workload to keep")
    ap.add_argument("--batch-plan", default="",
                    help="with --legs batch: 'cluster,block' instead of the autotuner (one launch per run)")
    ap.add_argument("--workload", choices=["walk", "cftp", "extremal"], default="walk",
                    help="walk: the headline line (default); cftp: CFTP runs on an Aztec diamond; "
                         "extremal: host vs device extremal tilings of large domains")
    ap.add_argument("--extremal-order", type=int, default=2000)
    ap.add_argument("--extremal-side", type=int, default=1000)
    ap.add_argument("--cftp-order", type=int, default=500)
    ap.add_argument("--cftp-seeds", type=int, default=32)
    ap.add_argument("--cftp-rng", choices=["tinymt", "philox", "planes"], default="planes")
    ap.add_argument("--cftp-weights", default="",
                    help="'a,b': two-periodic domino weights (TinyMT or Philox draws)")
    ap.add_argument("--walk-steps", type=int, default=SEGMENT, help="with --legs: colour steps per walk")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.workload == "cftp":
        run_cftp(args)
    elif args.workload == "extremal":
        run_extremal(args)
    elif args.legs != "all":
        run_legs(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
