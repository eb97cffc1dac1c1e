"""Benchmark of the bit-exact flip dynamics on the a=b=c=500 hexagon.

Workload: lozenge tilings of the a=b=c=500 hexagon (LozengeTiler::AlmostHexDomain
(500, 0) -> MinTiling, 1008 x 1008 tiling, 338,688 flip attempts per colour
step), started from the minimal tiling, 20,000 sweeps = 60,000 reference colour
steps per walk, TinyMT streams seeded from 42.  One bench "step" is one such
walk.  Uniform weights (int8 storage) are the headline; the q = 0.99 int32
walk (float32 comparison) is reported beside it.

  value : attempts/s with the lattice already resident on the device
          (rt_upload outside the timed region; rt_run inside), CUDA events on
          the library's stream, L2 flushed between walks;
  e2e   : the same metric through rt_walk (the reference's Walk contract:
          host int32 tiling in, host tiling out, H2D + split + walk + merge +
          D2H every walk).

`--impl reference` times the reference's own CPU code (its kernels and
LozengeTiler::Walk built through oracle/shim: oracle/_ref) on the host cores,
or the oracle's C restatement where oracle/_ref is absent.

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
STEPS_PER_WALK = 60000  # reference colour steps = 20,000 sweeps of the three colours
SEED = 42
L2_FLUSH_BYTES = 256 << 20


def workload_config() -> dict:
    return {
        "workload": "lozenge hexagon a=b=c=500 (1008x1008 tiling), minimal tiling start, "
                    "20000 sweeps = 60000 colour steps per walk, TinyMT bit-exact mode",
        "domain": "LozengeTiler::AlmostHexDomain(500,0)",
        "tiling_side": 1008,
        "attempts_per_step": 1008 * 336,
        "steps_per_walk": STEPS_PER_WALK,
        "seed": SEED,
        "weights": "uniform (int8 lattice); q=0.99 int32 in `q_weighted`",
        "l2": "flushed (256 MiB write) between timed walks",
    }


def peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def start_tiling():
    import randomtilings_b200 as rt

    d = rt.LozengeTiler.AlmostHexDomain(HEX_SIDE, 0)
    return rt.LozengeTiler.MinTiling(d)


def algorithmic_bytes_per_step(n: int, elem: int, rng_state: bool = True) -> int:
    """Lattice read + write of every colour-array site, plus the TinyMT state
    (s0..s3 read + write, 32 B) of every attempt (none in fast mode)."""
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
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
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


def time_device_walks(tiler, steps: int, warmup: int, seed: int, flush) -> list[float]:
    """Per-walk device milliseconds (events on the library's stream)."""
    import torch

    s = torch.cuda.ExternalStream(tiler.stream)
    for w in range(warmup):
        tiler.run(STEPS_PER_WALK, seed + 1000 + w)
    tiler.synchronize()
    out = []
    for k in range(steps):
        flush()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        tiler.run(STEPS_PER_WALK, seed + k)
        e1.record(s)
        tiler.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def time_e2e_walks(tiler_cls, kwargs, t0: np.ndarray, steps: int, warmup: int, seed: int, flush) -> list[float]:
    """rt_walk with a host tiling: wall time per walk (the call is synchronous)."""
    import torch

    tl = tiler_cls(**kwargs)
    host = np.array(t0, dtype=np.int32)
    for w in range(warmup):
        host[:] = t0
        tl.Walk(host, STEPS_PER_WALK, seed + 1000 + w)
    out = []
    for k in range(steps):
        host[:] = t0
        flush()
        torch.cuda.synchronize()
        a = time.perf_counter()
        tl.Walk(host, STEPS_PER_WALK, seed + k)
        out.append((time.perf_counter() - a) * 1e3)
    tl.close()
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
            tl.run(STEPS_PER_WALK, SEED + k)
        tl.synchronize()
        tl.close()
        print(f"{name}: {args.warmup + args.steps} walks of {STEPS_PER_WALK} colour steps", flush=True)
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
    tl.upload(t0)
    tq = rt.LozengeTiler(device=local, kernel=2, q=0.99, qcmp=0)
    tq.upload(t0)
    tf = rt.LozengeTiler(device=local, rng=rt.RT_RNG_PHILOX)
    tf.upload(t0)
    tp = rt.LozengeTiler(device=local, rng=rt.RT_RNG_PLANES)
    tp.upload(t0)

    barrier(dist)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        wall0 = time.perf_counter()
        ms = time_device_walks(tl, args.steps, args.warmup, seed, flush)
        wall = time.perf_counter() - wall0
    torch.cuda.synchronize()
    barrier(dist)
    clocks = clk.summary()
    ms_q = time_device_walks(tq, args.steps, args.warmup, seed, flush)
    ms_f = time_device_walks(tf, args.steps, args.warmup, seed, flush)
    ms_p = time_device_walks(tp, args.steps, args.warmup, seed, flush)
    aztec = measure_aztec2000(args, local, seed, flush)
    e2e_ms = time_e2e_walks(rt.LozengeTiler, {"device": local}, t0, args.steps, min(args.warmup, 3), seed, flush)
    phases, launches = tl.last_run_info()

    total_ms = all_max(dist, sum(ms))
    total_q = all_max(dist, sum(ms_q))
    total_f = all_max(dist, sum(ms_f))
    total_p = all_max(dist, sum(ms_p))
    total_e2e = all_max(dist, sum(e2e_ms))
    work = attempts * STEPS_PER_WALK * args.steps * world
    value = work / (total_ms / 1e3)
    per_launch_ms = sum(ms) / len(ms)
    algo = algorithmic_bytes_per_step(n, 1) * STEPS_PER_WALK
    peak, peak_kind = peaks()
    achieved = algo / (per_launch_ms / 1e3) / 1e9
    algo_q = algorithmic_bytes_per_step(n, 4) * STEPS_PER_WALK
    achieved_q = algo_q / (sum(ms_q) / len(ms_q) / 1e3) / 1e9
    algo_f = algorithmic_bytes_per_step(n, 1, rng_state=False) * STEPS_PER_WALK
    achieved_f = algo_f / (sum(ms_f) / len(ms_f) / 1e3) / 1e9

    batched = None if args.no_batch else measure_batch(args, rank, world, dist, peaks()[0])

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(t0, seconds=args.cpu_seconds)

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
            "config": workload_config() | {"parallelism": f"replicas{world}"},
            "impl": "b200",
            "hbm_gbs_algorithmic": achieved,
            "sweeps_per_s": value / attempts / 3,
            "e2e": {
                "value": attempts * STEPS_PER_WALK * args.steps * world / (total_e2e / 1e3),
                "unit": "attempts/s",
                "h2d_bytes_per_step": n * n * 4,
                "d2h_bytes_per_step": n * n * 4,
                "ms_per_step": total_e2e / args.steps,
            },
            "roofline": {
                "bound": "hbm",
                "achieved": achieved,
                "peak": peak,
                "unit": "GB/s",
                "frac": achieved / peak,
                "peak_kind": peak_kind,
                "traffic": args.traffic,
                "kernel": "rtb::walk_kernel (one cooperative launch per walk)",
                "algorithmic_bytes_per_launch": algo,
                "launch_ms": per_launch_ms,
            },
            "q_weighted": {
                "q": 0.99, "compare": "float32", "dtype": "int32",
                "value": attempts * STEPS_PER_WALK * args.steps * world / (total_q / 1e3),
                "unit": "attempts/s",
                "ms_per_step": total_q / args.steps,
                "hbm_gbs_algorithmic": achieved_q,
                "frac": achieved_q / peak,
            },
            "fast_mode": {
                "rng": "Philox4x32-10 keyed by (position quad, step, chain), cyclic colours", "dtype": "int8",
                "value": attempts * STEPS_PER_WALK * args.steps * world / (total_f / 1e3),
                "unit": "attempts/s",
                "ms_per_step": total_f / args.steps,
                "hbm_gbs_algorithmic": achieved_f,
                "frac": achieved_f / peak,
            },
            "bit_planes": {
                "rng": "one Philox4x32-10 bit per site, heat-bath rule, lattice as bit planes, cyclic colours",
                "value": attempts * STEPS_PER_WALK * args.steps * world / (total_p / 1e3),
                "unit": "attempts/s",
                "ms_per_step": total_p / args.steps,
            },
            "aztec2000": aztec,
            "batched": batched,
            "gpu_launches": int(launches) * args.steps,
            "phases_per_launch": int(phases),
            "clocks": clocks,
            "wall_s_timed_region": wall,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    tl.close()
    tq.close()
    tf.close()
    tp.close()
    if dist is not None:
        dist.destroy_process_group()


def measure_aztec2000(args, device: int, seed: int, flush) -> dict:
    """The large lattice of the warm-start evaluation (Aztec diamond of order
    2000, 4006 x 4006 tiling, 8,016,008 attempts per colour step): fast mode and
    bit-plane mode, 4,000 colour steps per walk."""
    import randomtilings_b200 as rt

    d = rt.DominoTiler.AztecDiamond(2000)
    t0 = rt.DominoTiler.MinTiling(d)
    n = int(round(t0.size ** 0.5))
    att = (n - 2) * (n // 2 - 2)
    steps = 4000
    out = {"workload": "Aztec diamond n=2000 (4006x4006), minimal tiling, 4000 colour steps per walk",
           "attempts_per_step": att, "unit": "attempts/s"}
    global STEPS_PER_WALK
    saved = STEPS_PER_WALK
    STEPS_PER_WALK = steps
    try:
        for name, rng in (("fast_mode", rt.RT_RNG_PHILOX), ("bit_planes", rt.RT_RNG_PLANES)):
            tl = rt.DominoTiler(device=device, rng=rng)
            tl.upload(t0)
            ms = time_device_walks(tl, max(1, args.steps), args.warmup, seed, flush)
            tl.close()
            out[name] = att * steps / (sum(ms) / len(ms) / 1e3)
    finally:
        STEPS_PER_WALK = saved
    return out


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


def measure_batch(args, rank: int, world: int, dist, peak: float) -> dict:
    """The batched pattern: args.batch_chains chains of the mixed workload
    (chain seed s: domain type s mod 4, sizes from std::mt19937(s)), minimal
    tilings, args.batch_sweeps sweeps each in fast mode, as one graph of one
    persistent cluster launch per kernel family.  Ranks take seeds round-robin
    (no communication); value = all ranks' attempts / max device time."""
    import randomtilings_b200 as rt
    from randomtilings_b200 import workloads

    bt = rt.Batch(device=int(os.environ.get("LOCAL_RANK", "0")))
    kinds = {}
    for seed in shard(args.batch_chains, rank, world):
        model, t = workloads.mixed_chain(seed)
        bt.add(model, t, key=seed, chain=seed)
        kinds[model] = kinds.get(model, 0) + 1
    bt.run(2)  # autotuner (on a scratch copy) + graph build; then a short warm-up run
    bt.run(2)
    barrier(dist)
    bt.run(args.batch_sweeps)
    info = bt.info()
    bt.close()
    ms = all_max(dist, info["run_ms"])
    total_attempts, total_bytes = all_sum(dist, [float(info["attempts"]), float(info["algorithmic_bytes"])])
    achieved = total_bytes / world / (ms / 1e3) / 1e9  # per GPU
    return {
        "workload": f"{args.batch_chains} chains of the mixed workload (seed s: s mod 4 -> Aztec diamond n in "
                    "[16,256] / hexagon a,b,c in [8,128] / triangle-dimer IceCreamCone(64,1) / rectangle-triangle "
                    f"hexagon 64; sizes from std::mt19937(s)), minimal tilings, {args.batch_sweeps} sweeps, "
                    "fast mode (Philox), one CUDA graph",
        "chains_per_model_rank0": {str(k): v for k, v in sorted(kinds.items())},
        "value": total_attempts / (ms / 1e3),
        "unit": "attempts/s",
        "ms": ms,
        "hbm_gbs_algorithmic": achieved,
        "frac": achieved / peak,
        "plans_rank0": info["plans"],
        "tune_ms_rank0": info["tune_ms"],
        "graph_launches": 1,
    }


def cpu_baseline(t0: np.ndarray, seconds: float = 15.0, threads: int | None = None) -> dict:
    """The reference's own kernels + LozengeTiler::Walk on the host cores
    (oracle/_ref), else the oracle's C restatement; a bounded sample of the
    same walk (same domain, start and seed), timed with a wall clock."""
    from oracle import pyoracle as po

    n = int(round(t0.size ** 0.5))
    attempts = n * (n // 3)
    threads = threads or os.cpu_count() or 1
    if po.have_ref():
        rt = po.RefTiler("lozenge", attempts, threads=threads)
        run = lambda s: rt.walk(t0, s, SEED)  # noqa: E731
        kind, cores = "reference", threads
    else:
        run = lambda s: po.lozenge_walk(t0, s, SEED)  # noqa: E731
        kind, cores = "port", 1
    probe = 20
    a = time.perf_counter()
    run(probe)
    dt = time.perf_counter() - a
    steps = max(probe, int(probe * seconds / max(dt, 1e-6)))
    a = time.perf_counter()
    run(steps)
    dt = time.perf_counter() - a
    return {
        "value": attempts * steps / dt,
        "unit": "attempts/s",
        "cores": cores,
        "kind": kind,
        "sample": f"hex a=b=c=500 walk, first {steps} colour steps (of 60000), seed {SEED}, {dt:.1f} s",
    }


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import randomtilings_b200 as rt  # builders only (host C++)

    t0 = start_tiling()
    n = int(round(t0.size ** 0.5))
    attempts = n * (n // 3)
    per_step_s = max(1.0, args.cpu_seconds / max(args.steps, 1))
    for _ in range(args.warmup):
        cpu_baseline(t0, seconds=0.5)
    vals = [cpu_baseline(t0, seconds=per_step_s) for _ in range(args.steps)]
    value = statistics.median(v["value"] for v in vals)
    ms_per_step = attempts * STEPS_PER_WALK / value * 1e3
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "attempts/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int8",
        "data": "synthetic (the reference's own domain builder; no dataset)",
        "config": workload_config() | {"parallelism": "cpu"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "attempts/s", "cores": vals[0]["cores"], "kind": vals[0]["kind"],
                         "sample": vals[0]["sample"]},
        "e2e": {"value": value, "unit": "attempts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    del rt
    print(json.dumps(line), flush=True)


def main() -> None:
    global STEPS_PER_WALK
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # dram__bytes_read.sum + dram__bytes_write.sum of one word_kernel launch (ncu, 600-step capture,
    # profiles/word_kernel_hex500.md): 1.146 MB + 3.1 KB; the lattice stays on chip, so a launch of
    # any number of colour steps moves the same bytes.
    ap.add_argument("--traffic", type=float, default=1149184.0,
                    help="dram bytes per walk launch from an ncu capture (reported in roofline.traffic)")
    ap.add_argument("--batch-chains", type=int, default=4096)
    ap.add_argument("--batch-sweeps", type=int, default=5000)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--legs", default="all",
                    help="profiling runs: comma-separated subset of headline,q,fast,planes,batch (no JSON line)")
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
    ap.add_argument("--walk-steps", type=int, default=STEPS_PER_WALK,
                    help="colour steps per walk (default 60000 = 20000 sweeps; smaller only for profiling captures)")
    args = ap.parse_args()
    STEPS_PER_WALK = args.walk_steps
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
