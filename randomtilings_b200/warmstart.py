"""Learned warm start of the flip dynamics (no reference counterpart).

A coordinate MLP (include/rt_b200_mlp.h) learns the mean height surface of
dominoes on Aztec diamonds and lozenges on a x b x c hexagons (volume weight
q) from the chains themselves:

1. dataset: plain fast-mode chains from the minimal tiling, run as batches
   (include/rt_b200_batch.h) -- chains too large for one cluster's shared
   memory one at a time on a single-lattice walk over the whole GPU -- for a
   burn-in proportional to the side squared, then sampled; their heights are
   summed on the device
   (include/rt_b200_height.h) and the mean surface becomes training rows
   (features of a vertex -> where its mean height sits between the extremal
   height functions, a fraction in [0, 1]);
2. training: Adam on the MLP's own BF16 / FP32 kernels;
3. warm start: prediction -> exact integer Lipschitz projection
   (include/rt_b200_project.h) -> HeightfuncToTiling -> a valid tiling that
   the unchanged flip dynamics then evolve;
4. judgement: coupled chains from the warm start, from the minimal tiling
   (cold) and from the maximal tiling (top of the monotone sandwich) run
   side by side; the error of a start after t sweeps is the mean over domain
   vertices of |mean height - reference| / side, the reference being the
   long-chain mean of all chains over the last part of the run, and the
   sandwich gap (mean |top - bottom| / side) certifying that the chains have
   met the equilibrium.  Optionally the reference is the mean of CFTP exact
   samples (small domains).

Features of a vertex (8): its position u, v in [-1, 1] within the domain's
bounding box of vertices, +1 for Aztec diamonds / -1 for hexagons, then for
Aztec diamonds +1 / -1 for even / odd order (slots 4-5 zero) and for hexagons
the side ratios 3a/(a+b+c) - 1, 3b/(a+b+c) - 1, 3c/(a+b+c) - 1, then the
volume-weight strength -side ln q, and 16 / side.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import math
import os
import time
from dataclasses import dataclass

import numpy as np

from . import _capi, builders
from .batch import Batch
from .heights import HeightPlan
from .mlp import CoordinateMLP
from .project import project_heights
from .tilers import DominoTiler, LozengeTiler

AZTEC, HEXAGON = "aztec", "hexagon"
INF = np.iinfo(np.int32).max

# Tiling sides (square root of the tiling's length) up to which a dataset
# chain runs in the batched kernels: Aztec diamonds to order 470, hexagons to
# sides 192 x 192 x 192, the sizes their cluster plans have held.  A larger
# chain runs alone on a single-lattice walk: dominoes and uniform lozenges on
# the bit-plane kernel, volume-weighted lozenges on the int32 kernel with
# Philox draws.
BATCH_MAX_SIDE = {AZTEC: 945, HEXAGON: 560}


@dataclass(frozen=True)
class DomainSpec:
    kind: str                  # "aztec" (dominoes) or "hexagon" (lozenges)
    size: tuple                # (n,) or (a, b, c)
    q: float = 1.0             # lozenge volume weight

    @property
    def model(self) -> int:
        return _capi.RT_DOMINO if self.kind == AZTEC else _capi.RT_LOZENGE

    @property
    def tiler(self):
        return DominoTiler if self.kind == AZTEC else LozengeTiler

    @property
    def side(self) -> float:
        return float(self.size[0]) if self.kind == AZTEC else float(sum(self.size)) / 3.0

    @property
    def steps_per_sweep(self) -> int:
        return 2 if self.kind == AZTEC else 3

    def domain(self) -> np.ndarray:
        if self.kind == AZTEC:
            return DominoTiler.AztecDiamond(int(self.size[0]))
        a, b, c = (int(x) for x in self.size)
        return LozengeTiler.Hexagon(a, b, c)

    def label(self) -> str:
        s = "x".join(str(int(x)) for x in self.size)
        return f"{self.kind}{s}" + (f"_q{self.q:.4f}" if self.q != 1.0 else "")


@dataclass
class Prepared:
    spec: DomainSpec
    domain: np.ndarray
    n: int
    tmin: np.ndarray
    tmax: np.ndarray
    hmin: np.ndarray
    hmax: np.ndarray
    idx: np.ndarray            # flat indices of the domain's vertices


def prepare(spec: DomainSpec, device: int | None = None) -> Prepared:
    """Extremal tilings and heights of the domain: on the host (the
    reference's flood), or on `device` (rt_extremal_tilings, the same arrays)."""
    cls = spec.tiler
    d = spec.domain()
    if device is None:
        tmin = np.asarray(cls.MinTiling(d), dtype=np.int32)
        tmax = np.asarray(cls.MaxTiling(d), dtype=np.int32)
        a = np.asarray(cls.TilingToHeightfunc(tmin, d), dtype=np.int32)
        b = np.asarray(cls.TilingToHeightfunc(tmax, d), dtype=np.int32)
    else:
        ext, _ = builders.extremal_tilings(spec.model, d, device)
        tmin, tmax, a, b = ext["tmin"], ext["tmax"], ext["hmin"], ext["hmax"]
    n = int(round(tmin.size ** 0.5))
    idx = np.flatnonzero(a != INF)
    return Prepared(spec, d, n, tmin, tmax, np.minimum(a, b), np.maximum(a, b), idx)


def features(p: Prepared) -> np.ndarray:
    s = p.spec
    ii, jj = np.divmod(p.idx, p.n)
    i0, i1, j0, j1 = ii.min(), ii.max(), jj.min(), jj.max()
    x = np.zeros((p.idx.size, _capi.RT_MLP_IN), dtype=np.float32)
    x[:, 0] = 2.0 * (jj - j0) / max(1, j1 - j0) - 1.0
    x[:, 1] = 2.0 * (ii - i0) / max(1, i1 - i0) - 1.0
    x[:, 2] = 1.0 if s.kind == AZTEC else -1.0
    if s.kind == AZTEC:
        # the extremal height functions of even and odd orders differ in
        # pattern, so the mean surface's place between them depends on n mod 2
        x[:, 3] = 1.0 if int(s.size[0]) % 2 == 0 else -1.0
    else:
        tot = float(sum(s.size))
        for k in range(3):
            x[:, 3 + k] = 3.0 * s.size[k] / tot - 1.0
    x[:, 6] = -s.side * math.log(s.q) if s.q < 1.0 else 0.0
    x[:, 7] = 16.0 / s.side
    return x


def fraction(p: Prepared, hmean: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(fraction of the way from h_min to h_max at each domain vertex, mask of
    the vertices where h_max > h_min)."""
    lo = p.hmin[p.idx].astype(np.float64)
    hi = p.hmax[p.idx].astype(np.float64)
    span = hi - lo
    live = span > 0
    f = np.where(live, (hmean[p.idx] - lo) / np.where(live, span, 1.0), 0.5)
    return np.clip(f, 0.0, 1.0).astype(np.float32), live


def heights_from_fraction(p: Prepared, f: np.ndarray) -> np.ndarray:
    t = np.zeros(p.n * p.n, dtype=np.float32)
    lo = p.hmin[p.idx].astype(np.float64)
    hi = p.hmax[p.idx].astype(np.float64)
    t[p.idx] = (lo + np.clip(f, 0.0, 1.0) * (hi - lo)).astype(np.float32)
    return t


def burn_sweeps(spec: DomainSpec, factor: float = 1.0) -> int:
    """Sweeps after which a chain from the minimal tiling has met its
    equilibrium on the scale that matters here (measured: the max / min
    sandwich closes to its fluctuation floor after ~1.2 n^2 sweeps on Aztec
    diamonds of order n and ~6 s^2 on hexagons of side s)."""
    c = 1.5 if spec.kind == AZTEC else 7.0
    return max(16, int(factor * c * spec.side ** 2))


def training_specs(count: int, seed: int = 0, aztec=(32, 384), hexagon=(16, 192), q=(0.98, 1.0)) -> list[DomainSpec]:
    """`count` domains, half Aztec diamonds with order uniform in `aztec`, half
    hexagons with each side uniform in `hexagon` and q uniform in `q`."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        if k % 2 == 0:
            out.append(DomainSpec(AZTEC, (int(rng.integers(aztec[0], aztec[1] + 1)),)))
        else:
            abc = tuple(int(x) for x in rng.integers(hexagon[0], hexagon[1] + 1, size=3))
            qq = float(np.float32(rng.uniform(q[0], q[1]))) if q[1] > q[0] else float(q[0])
            out.append(DomainSpec(HEXAGON, abc, min(1.0, qq)))
    return out


def _prepare_all(specs, threads: int | None = None) -> list[Prepared]:
    # the builders are C++ behind ctypes, which releases the GIL: threads run them in parallel
    with cf.ThreadPoolExecutor(max_workers=threads or min(32, os.cpu_count() or 1)) as ex:
        return list(ex.map(prepare, specs))


def _single_tiler(p: Prepared, device: int):
    if p.spec.kind == AZTEC:
        return DominoTiler(device=device, rng=_capi.RT_RNG_PLANES)
    if p.spec.q < 1.0:
        return LozengeTiler(device=device, kernel=_capi.RT_KERNEL_QWEIGHT, q=p.spec.q, rng=_capi.RT_RNG_PHILOX)
    return LozengeTiler(device=device, rng=_capi.RT_RNG_PLANES)


def single_chain_mean(p: Prepared, key: int, burn: int, gap: int, samples: int, device: int = 0):
    """Mean height function of one chain run alone on the whole GPU: `burn`
    sweeps from the minimal tiling, then `samples` samples `gap` sweeps apart,
    summed on the device on the walk's own stream.  Returns (mean heights,
    device milliseconds of the walk)."""
    import torch

    tl = _single_tiler(p, device)
    plan = HeightPlan(p.spec.model, p.domain, device)
    try:
        sums = torch.zeros(p.n ** 2, dtype=torch.int64, device=f"cuda:{device}")
        tl.upload(p.tmin)
        stream = tl.stream
        s = torch.cuda.ExternalStream(stream)
        ms = 0.0
        for seg, sweeps in enumerate([burn] + [gap] * samples):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            tl.run(sweeps * p.spec.steps_per_sweep, (key * 0x9E3779B1 + seg) & 0x7FFFFFFFFFFF)
            e1.record(s)
            if seg > 0:
                plan.accumulate(tl.device_tiling(), sums.data_ptr(), stream)
            tl.synchronize()
            ms += e0.elapsed_time(e1)
        return sums.cpu().numpy().astype(np.float64) / samples, ms
    finally:
        plan.close()
        tl.close()


def generate_dataset(specs, device: int = 0, samples: int = 8, burn_factor: float = 1.0, gap_factor: float = 0.05,
                     rows_per_domain: int = 4096, group_ratio: float = 2.0, seed: int = 0, log=None):
    """Training rows (X, y) from plain chains on `specs`, and per-domain stats."""
    import torch

    rng = np.random.default_rng(seed + 1)
    xs, ys, stats = [], [], []

    def add_rows(p: Prepared, k: int, hmean: np.ndarray, sweeps: int, alone: bool) -> None:
        f, live = fraction(p, hmean)
        x = features(p)
        sel = np.flatnonzero(live)
        if sel.size > rows_per_domain:
            sel = rng.choice(sel, rows_per_domain, replace=False)
        xs.append(x[sel])
        ys.append(f[sel])
        stats.append({"domain": p.spec.label(), "sweeps": sweeps, "rows": int(sel.size), "alone": alone})

    def side(spec: DomainSpec) -> int:
        return int(round(np.asarray(spec.domain()).size ** 0.5))

    alone = [k for k in range(len(specs)) if side(specs[k]) > BATCH_MAX_SIDE[specs[k].kind]]
    for k in alone:
        t0 = time.perf_counter()
        p = prepare(specs[k], device)
        burn = burn_sweeps(specs[k], burn_factor)
        gap = max(1, int(gap_factor * burn))
        hmean, ms = single_chain_mean(p, seed * 1_000_003 + k, burn, gap, samples, device)
        add_rows(p, k, hmean, burn + samples * gap, True)
        if log:
            log(f"dataset chain {p.spec.label()} alone, {burn + samples * gap} sweeps, device {ms:.0f} ms, "
                f"wall {time.perf_counter() - t0:.1f} s")
    specs_b = [k for k in range(len(specs)) if k not in set(alone)]

    order = sorted(specs_b, key=lambda k: burn_sweeps(specs[k], burn_factor))
    groups, cur = [], []
    for k in order:
        if cur and burn_sweeps(specs[k], burn_factor) > group_ratio * burn_sweeps(specs[cur[0]], burn_factor):
            groups.append(cur)
            cur = []
        cur.append(k)
    if cur:
        groups.append(cur)
    for g in groups:
        t0 = time.perf_counter()
        prep = dict(zip(g, _prepare_all([specs[k] for k in g])))
        bt = Batch(device)
        for c, k in enumerate(g):
            p = prep[k]
            bt.add(p.spec.model, p.tmin, key=seed * 1_000_003 + k, chain=c, q=p.spec.q if p.spec.q < 1 else 0.0)
        burn = max(burn_sweeps(specs[k], burn_factor) for k in g)
        gap = max(1, int(gap_factor * burn))
        with cf.ThreadPoolExecutor(max_workers=min(32, os.cpu_count() or 1)) as ex:
            plans = list(ex.map(lambda k: HeightPlan(prep[k].spec.model, prep[k].domain, device), g))
        sums = [torch.zeros(prep[k].n ** 2, dtype=torch.int64, device=f"cuda:{device}") for k in g]
        buf = torch.empty(max(prep[k].n for k in g) ** 2, dtype=torch.int32, device=f"cuda:{device}")
        bt.run(burn)
        ms = bt.info()["run_ms"]
        for _ in range(samples):
            bt.run(gap)
            ms += bt.info()["run_ms"]
            for c in range(len(g)):
                bt.device_tiling(c, buf.data_ptr())
                plans[c].accumulate(buf.data_ptr(), sums[c].data_ptr())
        torch.cuda.synchronize(device)
        for c, k in enumerate(g):
            add_rows(prep[k], k, sums[c].cpu().numpy().astype(np.float64) / samples, burn + samples * gap, False)
            plans[c].close()
        bt.close()
        if log:
            log(f"dataset group of {len(g)} chains, {burn + samples * gap} sweeps, device {ms:.0f} ms, "
                f"wall {time.perf_counter() - t0:.1f} s")
    return np.concatenate(xs), np.concatenate(ys), stats


class WarmStart:
    """The trained coordinate MLP and the warm-start tiling it gives."""

    def __init__(self, device: int = 0, seed: int = 0):
        self.device = device
        self.mlp = CoordinateMLP(device, seed)

    def fit(self, x, y, steps: int = 3000, batch: int = 16384, lr: float = 2e-3, seed: int = 0) -> list[float]:
        """Adam on (x, y) with the learning rate divided by 3 at one and two thirds of the steps."""
        self.mlp.set_data(x, y)
        losses = []
        for k, scale in enumerate((1.0, 1.0 / 3.0, 1.0 / 10.0)):
            losses.append(self.mlp.train(max(1, steps // 3), batch=batch, lr=lr * scale, seed=seed + k))
        return losses

    def predict_fraction(self, p: Prepared) -> np.ndarray:
        return np.clip(self.mlp.predict(features(p)), 0.0, 1.0)

    def warm_tiling(self, p: Prepared) -> tuple[np.ndarray, dict]:
        t = heights_from_fraction(p, self.predict_fraction(p))
        h, st = project_heights(p.spec.model, p.domain, p.hmin, p.hmax, t, self.device)
        tiling = np.asarray(p.spec.tiler.HeightfuncToTiling(h, p.domain), dtype=np.int32)
        st["target_l1_per_side"] = float(np.abs(h[p.idx].astype(np.float64) - t[p.idx]).mean() / p.spec.side)
        return tiling, st

    def save(self, path: str) -> None:
        np.save(path, self.mlp.params)

    def load(self, path: str) -> None:
        self.mlp.params = np.load(path)


class _Chains:
    """Chains that advance together: a Batch (fast mode) where the domain is
    small, else one bit-plane Tiler (RT_RNG_PLANES) per chain, which uses the
    whole GPU for one lattice.  Chains given the same key share their draws."""

    def __init__(self, p: Prepared, starts: list[np.ndarray], keys: list[int], device: int, use_batch: bool,
                 heat_bath: bool = False):
        self.p, self.device, self.keys = p, device, keys
        # the reference's own rules (dominokernel.cl, lozengekernel.cl); heat_bath: the domino CFTP rule
        kernel = _capi.RT_KERNEL_CFTP if (heat_bath and p.spec.kind == AZTEC) else _capi.RT_KERNEL_DEFAULT
        self.batch = None
        self.tilers = []
        self.chunk = 0
        if use_batch:
            self.batch = Batch(device)
            for t, k in zip(starts, keys):
                self.batch.add(p.spec.model, t, key=k, chain=0, kernel=kernel,
                               q=p.spec.q if p.spec.q < 1 else 0.0)
        else:
            if p.spec.q < 1.0:
                raise ValueError("volume-weighted chains run in batches")
            for t in starts:
                tl = p.spec.tiler(device=device, kernel=kernel, rng=_capi.RT_RNG_PLANES)
                tl.upload(t)
                self.tilers.append(tl)
        self.device_ms = 0.0

    def advance(self, sweeps: int) -> None:
        if sweeps <= 0:
            return
        if self.batch is not None:
            self.batch.run(sweeps)
            self.device_ms += self.batch.info()["run_ms"]
            return
        import torch

        steps = sweeps * self.p.spec.steps_per_sweep
        for tl, k in zip(self.tilers, self.keys):
            s = torch.cuda.ExternalStream(tl.stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            tl.run(steps, (k * 0x9E3779B1 + self.chunk) & 0x7FFFFFFFFFFF)
            e1.record(s)
            tl.synchronize()
            self.device_ms += e0.elapsed_time(e1)
        self.chunk += 1

    def tiling_ptr(self, c: int, buf) -> int:
        if self.batch is not None:
            self.batch.device_tiling(c, buf.data_ptr())
            return buf.data_ptr()
        ptr = self.tilers[c].device_tiling()
        self.tilers[c].synchronize()
        return ptr

    def close(self) -> None:
        if self.batch is not None:
            self.batch.close()
        for tl in self.tilers:
            tl.close()


def relax(p: Prepared, starts: dict, sweeps: int, points: int = 40, replicas: int = 1, seed: int = 0,
          device: int = 0, use_batch: bool | None = None, ref_tail: float = 0.25, threshold: float = 0.005,
          cftp_ref: np.ndarray | None = None, heat_bath: bool = False, log=None) -> dict:
    """Error curves of the named starting tilings (e.g. {"cold": tmin, "warm": tw}).

    Every start runs `replicas` independent chains (own Philox keys); as many
    more start from the maximal tiling ("top"): their mean height approaches
    the equilibrium from above as the cold start's does from below, and the
    sandwich gap is the mean over vertices of |top mean - cold mean| / side.
    At `points` checkpoints (geometric in sweeps up to `sweeps`) the mean
    height of each start's replicas is recorded on the device.  The reference
    surface is `cftp_ref` when given, else the mean of all chains over the
    checkpoints in the last `ref_tail` of the run (eight evenly spaced ones
    are added there to the geometric grid)."""
    import torch

    dev = f"cuda:{device}"
    side = p.spec.side
    names = list(starts)
    if use_batch is None:
        # small domains: many chains per launch; large ones: the whole GPU per chain
        use_batch = p.n <= 300 or (replicas > 1 and p.n <= 900)
    tilings, keys, owner = [], [], []
    for x, name in enumerate(names + ["top"]):
        for r in range(replicas):
            tilings.append(np.asarray(starts[name] if name != "top" else p.tmax, dtype=np.int32))
            keys.append((seed * 1_000_003 + x) * 7919 + r)
            owner.append(name)
    chains = _Chains(p, tilings, keys, device, use_batch, heat_bath)
    plan = HeightPlan(p.spec.model, p.domain, device)
    buf = torch.empty(p.n * p.n, dtype=torch.int32, device=dev)
    idx = torch.from_numpy(p.idx).to(dev)
    marks = sorted({0} | {int(round(x)) for x in np.geomspace(1, sweeps, points)} |
                   {int(round(x)) for x in np.linspace((1.0 - ref_tail) * sweeps, sweeps, 8)})
    saved = {name: [] for name in names + ["top"]}
    gap = []
    done = 0
    t0 = time.perf_counter()
    for m in marks:
        chains.advance(m - done)
        done = m
        sums = {name: torch.zeros(p.n * p.n, dtype=torch.int64, device=dev) for name in saved}
        for c, name in enumerate(owner):
            plan.accumulate(chains.tiling_ptr(c, buf), sums[name].data_ptr())
        for name in saved:
            saved[name].append((sums[name].index_select(0, idx).double() / replicas).float())
        if "cold" in saved:
            gap.append(float((saved["top"][-1] - saved["cold"][-1]).abs().double().mean() / side))
        if log and len(saved[names[0]]) % 10 == 0:
            log(f"  {p.spec.label()}: {m} sweeps, wall {time.perf_counter() - t0:.0f} s")
    if cftp_ref is not None:
        ref = torch.from_numpy(np.asarray(cftp_ref, dtype=np.float32)[p.idx]).to(dev)
        ref_kind = "cftp"
    else:
        tail = [k for k, m in enumerate(marks) if m >= (1.0 - ref_tail) * sweeps] or [len(marks) - 1]
        acc = torch.zeros(p.idx.size, dtype=torch.float64, device=dev)
        for k in tail:
            for name in saved:
                acc += saved[name][k].double()
        ref = (acc / (len(tail) * len(saved))).float()
        ref_kind = f"long-chain mean over the last {ref_tail:.0%} of the run"
    curves = {name: [float((h - ref).abs().double().mean() / side) for h in saved[name]] for name in saved}
    out = {"domain": p.spec.label(), "side": side, "sweeps": marks, "reference": ref_kind, "replicas": replicas,
           "curves": curves, "sandwich_gap": gap, "device_ms": chains.device_ms,
           "wall_s": time.perf_counter() - t0, "threshold": threshold}
    out["sweeps_to_threshold"] = {name: next((m for m, e in zip(marks, curves[name]) if e <= threshold), None)
                                  for name in names}
    chains.close()
    plan.close()
    return out


def speedup(result: dict, warm: str = "warm", cold: str = "cold") -> float | None:
    s = result["sweeps_to_threshold"]
    if s.get(cold) is None or s.get(warm) is None:
        return None
    return s[cold] / max(1, s[warm])


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description="learned warm start: dataset, training, warm vs cold")
    ap.add_argument("--domains", type=int, default=2000)
    ap.add_argument("--aztec", type=int, nargs=2, default=(32, 384))
    ap.add_argument("--hexagon", type=int, nargs=2, default=(16, 192))
    ap.add_argument("--q", type=float, nargs=2, default=(0.98, 1.0))
    ap.add_argument("--samples", type=int, default=8)
    ap.add_argument("--burn-factor", type=float, default=1.0)
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--eval", nargs="+", default=["aztec:2000", "hexagon:1000"])
    ap.add_argument("--eval-sweeps", type=float, default=2.0,
                    help="length of the comparison, in units of the cold start's burn-in")
    ap.add_argument("--points", type=int, default=40)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--params", default=None, help="save the trained parameters here (.npy)")
    a = ap.parse_args(argv)

    def log(msg):
        print(msg, flush=True)

    res = {"config": vars(a)}
    t0 = time.perf_counter()
    specs = training_specs(a.domains, a.seed, tuple(a.aztec), tuple(a.hexagon), tuple(a.q))
    x, y, stats = generate_dataset(specs, samples=a.samples, burn_factor=a.burn_factor, seed=a.seed, log=log)
    res["dataset"] = {"domains": len(specs), "rows": int(x.shape[0]), "wall_s": time.perf_counter() - t0}
    log(f"dataset: {x.shape[0]} rows from {len(specs)} chains in {res['dataset']['wall_s']:.0f} s")
    ws = WarmStart(seed=a.seed)
    t1 = time.perf_counter()
    res["train_loss"] = ws.fit(x, y, steps=a.train_steps, seed=a.seed)
    res["train_wall_s"] = time.perf_counter() - t1
    log(f"training: losses {res['train_loss']} in {res['train_wall_s']:.0f} s")
    if a.params:
        ws.save(a.params)
    res["eval"] = []
    for e in a.eval:
        kind, size = e.split(":")
        sz = tuple(int(v) for v in size.split("x"))
        spec = DomainSpec(kind, sz if kind == AZTEC or len(sz) == 3 else sz * 3)
        p = prepare(spec, ws.device)
        tw, st = ws.warm_tiling(p)
        r = relax(p, {"cold": p.tmin, "warm": tw}, int(a.eval_sweeps * burn_sweeps(spec)), points=a.points,
                  seed=a.seed + 1, log=log)
        r["projection"] = st
        r["speedup"] = speedup(r)
        log(f"{spec.label()}: sweeps to {r['threshold']:.1%}: {r['sweeps_to_threshold']}, speed-up {r['speedup']}, "
            f"final sandwich gap {r['sandwich_gap'][-1]:.4f}")
        res["eval"].append(r)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f)


if __name__ == "__main__":
    main()
