"""Regenerates the golden fixtures in this directory from the reference itself.

Run from the repository root, on a machine that has built oracle/_ref/libref.so
from the reference source tree (`make -C oracle ref REF=<reference tree>`), with
REF naming that tree for the example-output digests:

    REF=<reference tree> python tests/golden/make_golden.py [--only part,part]

Parts: builders, walks, aztec100, svg, examples (the original fixtures),
qf32 (q-lozenge walks on which the float32 and double comparisons of
qlozengekernel.cl part, from the reference kernel compiled both ways:
qlozenge_f32.npz) and bench (SHA-256 digests of the bench workloads run by
the reference and the oracle at their full sizes: bench_parity.json).

Everything here comes out of the reference's own code (its Tiler classes and
OpenCL kernels compiled for the CPU through oracle/shim): domains, extremal
tilings, height functions, and walk results for fixed seeds.  The reference's
deterministic example outputs (Examples/ExampleOuts) are checked against the
same code and recorded by SHA-256.  The GPU tests read only the .npz/.json
files written here; nothing reads the reference tree at test time.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)
from oracle import pyoracle as po  # noqa: E402

REF = os.environ.get("REF", "")
OUT = os.path.dirname(os.path.abspath(__file__))


def side(a) -> int:
    return int(round(np.asarray(a).size ** 0.5))


def digest(a) -> str:
    """SHA-256 of an int32 array's little-endian bytes (the tests hash the same way)."""
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<i4").tobytes()).hexdigest()


def q_divergence(t, seed: int, max_steps: int) -> int:
    """The smallest step count <= max_steps after which the q = 0.99 walk of
    tiling t (seed) differs between the float32 and the double comparison
    (the oracle's finder; 0 when none)."""
    return po.lozenge_q_divergence(t, seed, max_steps, 0.99)


def builders() -> dict:
    b = po.ref_build
    out = {}
    for n in (1, 2, 3, 5, 8, 13, 100):
        d = b("domino_aztec", p0=n)
        tmin, tmax = b("domino_min", d), b("domino_max", d)
        out[f"domino/aztec{n}/domain"] = d
        out[f"domino/aztec{n}/min"] = tmin
        out[f"domino/aztec{n}/max"] = tmax
        if n <= 13:
            out[f"domino/aztec{n}/vertices"] = b("domino_vertices", d)
            out[f"domino/aztec{n}/hmin"] = b("domino_t2h", tmin, d)
            out[f"domino/aztec{n}/hmax"] = b("domino_t2h", tmax, d)
            out[f"domino/aztec{n}/tiling_to_domain"] = b("domino_tiling_to_domain", tmin)
    for (m, n) in ((2, 2), (4, 6), (5, 8), (7, 7)):
        d = b("domino_rectangle", p0=m, p1=n)
        out[f"domino/rect{m}x{n}/domain"] = d
        out[f"domino/rect{m}x{n}/min"] = b("domino_min", d)
        out[f"domino/rect{m}x{n}/max"] = b("domino_max", d)
    for (n, rem) in ((4, (1,)), (6, (0, 2)), (7, (1, 3, 5))):
        d = b("domino_aztec_rectangle", np.array(rem, dtype=np.int32), p0=n)
        out[f"domino/aztecrect{n}_{'_'.join(map(str, rem))}/domain"] = d
    for (n, m) in ((2, 0), (4, 0), (4, 1), (10, 2), (13, 5), (20, 0)):
        d = b("lozenge_almost_hex", p0=n, p1=m)
        tmin, tmax = b("lozenge_min", d), b("lozenge_max", d)
        out[f"lozenge/hex{n}_{m}/domain"] = d
        out[f"lozenge/hex{n}_{m}/min"] = tmin
        out[f"lozenge/hex{n}_{m}/max"] = tmax
        out[f"lozenge/hex{n}_{m}/vertices"] = b("lozenge_vertices", d)
        out[f"lozenge/hex{n}_{m}/hmin"] = b("lozenge_t2h", tmin, d)
        out[f"lozenge/hex{n}_{m}/hmax"] = b("lozenge_t2h", tmax, d)
        out[f"lozenge/hex{n}_{m}/tiling_to_domain"] = b("lozenge_tiling_to_domain", tmin)
        out[f"lozenge/hex{n}_{m}/recttri"] = b("recttri_from_lozenge", tmin, d)
    for n in (1, 2, 3, 5, 6, 9, 20):
        for kind in ("max_hex", "min_hex", "slope_hex"):
            out[f"recttri/{kind}{n}"] = b(f"recttri_{kind}", p0=n)
    for (n, m) in ((6, 0), (5, 0), (8, 2), (10, 3), (12, 0)):
        t = b("tridimer_ice_cream_cone", p0=n, p1=m)
        out[f"tridimer/cone{n}_{m}/tiling"] = t
        out[f"tridimer/cone{n}_{m}/triangle_flips"] = b("tridimer_triangle_flips", t)
        out[f"tridimer/cone{n}_{m}/butterfly_flips"] = b("tridimer_butterfly_flips", t)
        out[f"tridimer/cone{n}_{m}/vertices"] = b("tridimer_vertices", t)
        out[f"tridimer/cone{n}_{m}/domain"] = b("tridimer_domain", t)
        for c in range(3):
            out[f"tridimer/cone{n}_{m}/dimer{c}"] = b("tridimer_dimer_indicator", t, p0=c)
    for k in range(3):
        out[f"tridimer/butterfly{k}"] = b("tridimer_test_butterfly", p0=k)
    return out


def walks(start: dict) -> dict:
    out = {}
    cases = []
    for n in (5, 13):
        t = start[f"domino/aztec{n}/min"]
        for cftp in (0, 1):
            for seed in (42, 34893, -7):
                cases.append(("domino_cftp" if cftp else "domino", f"domino{'_cftp' if cftp else ''}/aztec{n}/s{seed}",
                              t, 300, seed))
    for key in ("lozenge/hex4_1", "lozenge/hex10_2", "lozenge/hex13_5"):
        t = start[f"{key}/min"]
        for model in ("lozenge", "qlozenge"):
            for seed in (42, 5):
                cases.append((model, f"{model}/{key.split('/')[1]}/s{seed}", t, 700, seed))
    for n in (2, 5, 9):
        for kind in ("min_hex", "max_hex", "slope_hex"):
            t = start[f"recttri/{kind}{n}"]
            for seed in (42, 1234):
                cases.append(("recttri", f"recttri/{kind}{n}/s{seed}", t, 500, seed))
    for key in ("tridimer/cone6_0", "tridimer/cone8_2", "tridimer/cone10_3"):
        t = start[f"{key}/tiling"]
        for seed in (42, 7):
            cases.append(("tridimer", f"tridimer/{key.split('/')[1]}/s{seed}", t, 400, seed))
    for model, key, t, steps, seed in cases:
        rt = po.RefTiler(model, side(t) ** 2)
        out[f"{key}/start"] = t
        out[f"{key}/steps"] = np.array([steps])
        out[f"{key}/seed"] = np.array([seed])
        out[f"{key}/end"] = rt.walk(t, steps, seed)
        rt.close()
    # multi-epoch CFTP walks (DominoTiler.cpp:58-107)
    for n in (5, 13):
        for which in ("min", "max"):
            t = start[f"domino/aztec{n}/{which}"]
            st, se = np.array([256, 128], dtype=np.int64), np.array([2718281, 345903], dtype=np.int64)
            rt = po.RefTiler("domino_cftp", side(t) ** 2 // 2)
            key = f"domino_epochs/aztec{n}/{which}"
            out[f"{key}/start"] = t
            out[f"{key}/steps"] = st
            out[f"{key}/seeds"] = se
            out[f"{key}/end"] = rt.walk_epochs(t, st, se)
            rt.close()
    return out


def aztec100(start: dict) -> dict:
    """Aztec diamond n=100 from the minimal tiling, seed 42: the reference's walk."""
    out = {}
    t = start["domino/aztec100/min"]
    d = start["domino/aztec100/domain"]
    rt = po.RefTiler("domino", side(t) ** 2 // 2, threads=os.cpu_count() or 1)
    for steps in (10000, 20000):
        t0 = time.time()
        end = rt.walk(t, steps, 42)
        print(f"  cfg0 {steps} steps: {time.time() - t0:.1f}s", flush=True)
        out[f"cfg0/s{steps}/end"] = end
        out[f"cfg0/s{steps}/height"] = po.ref_build("domino_t2h", end, d)
    rt.close()
    return out


def qlozenge_f32(start: dict) -> dict:
    """q = 0.99 walks from qlozengekernel.cl compiled with single-precision
    arithmetic (an fp32-only OpenCL device), beside the double build: the
    seeds of the small hexagons, and walks of an a=b=c=40 hexagon stopped
    right after a draw at which the two comparisons part (the chains are
    monotone and heal such a difference within a few sweeps, so the step
    count matters).  Seeds 10000 m keep the work-item streams of different
    seeds apart (seed + id)."""
    out = {}
    cases = []
    for key in ("lozenge/hex4_1", "lozenge/hex10_2", "lozenge/hex13_5"):
        for seed in (42, 5):
            cases.append((f"qlozenge_f32/{key.split('/')[1]}/s{seed}", start[f"{key}/min"], 700, seed))
    d = po.ref_build("lozenge_almost_hex", p0=40, p1=0)
    t40 = po.ref_build("lozenge_min", d)
    found = 0
    for m in range(1, 400):
        steps = q_divergence(t40, 10000 * m, 3000)
        if steps:
            cases.append((f"qlozenge_f32/hex40_0/s{10000 * m}", t40, steps, 10000 * m))
            found += 1
            if found == 3:
                break
    for key, t, steps, seed in cases:
        f32 = po.RefTiler("qlozenge_f32", side(t) ** 2)
        dbl = po.RefTiler("qlozenge", side(t) ** 2)
        out[f"{key}/start"] = t
        out[f"{key}/steps"] = np.array([steps])
        out[f"{key}/seed"] = np.array([seed])
        out[f"{key}/end"] = f32.walk(t, steps, seed)
        out[f"{key}/end_double"] = dbl.walk(t, steps, seed)
        f32.close()
        dbl.close()
    return out


BENCH_SEGMENT = 3000  # colour steps per bench step (1,000 sweeps of the three colours)


def bench_parity() -> dict:
    """Digests of the bench's own workloads at their full sizes.

    hex500: LozengeTiler::AlmostHexDomain(500, 0) -> MinTiling (1008 x 1008),
    walked as the bench walks it -- 20 Walk calls of 3,000 colour steps with
    seeds 42..61, each continuing from the last (20,000 sweeps) -- by the
    reference's LozengeTiler::Walk and kernels (OpenMP over work items); the
    q = 0.99 int32 walk (qlozengekernel.cl, float32 and double comparisons);
    the fast and bit-plane modes (no reference counterpart: the oracle's
    replay).  The q walk starts from the uniform walk's final tiling (a minimal
    tiling has too few flippable sites for the comparisons to part within a
    test's walk) and runs, with the first seed from 42 on that gives one, to
    the step after which float32 and double differ.  aztec2000:
    AztecDiamond(2000) -> MinTiling (4006 x 4006), fast and bit-plane walks
    (the oracle's replay)."""
    threads = os.cpu_count() or 1
    out = {}
    t0 = time.time()
    d = po.ref_build("lozenge_almost_hex", p0=500, p1=0)
    t = po.ref_build("lozenge_min", d)
    out["hex500/start"] = digest(t)
    rt = po.RefTiler("lozenge", side(t) ** 2, threads=threads)
    a = t.copy()
    for k in range(20):
        a = rt.walk(a, BENCH_SEGMENT, 42 + k)
        out[f"hex500/uniform/segment{k}"] = digest(a)
        print(f"  hex500 segment {k}: {time.time() - t0:.0f}s", flush=True)
    out["hex500/uniform/s42/600"] = digest(rt.walk(t, 600, 42))
    rt.close()
    qseed, qsteps = 0, 0
    for qseed in range(42, 142):
        qsteps = q_divergence(a, qseed, 1000)
        if qsteps:
            break
    assert qsteps, "no float32/double divergence"
    out["hex500/q/start"] = "hex500/uniform/segment19"
    out["hex500/q/seed"] = qseed
    out["hex500/q/steps"] = qsteps
    print(f"  hex500 q: seed {qseed}, parts after {qsteps} steps: {time.time() - t0:.0f}s", flush=True)
    for name, model in (("qf32", "qlozenge_f32"), ("qdouble", "qlozenge")):
        rt = po.RefTiler(model, side(t) ** 2, threads=threads)
        out[f"hex500/{name}"] = digest(rt.walk(a, qsteps, qseed))
        rt.close()
    assert out["hex500/qf32"] != out["hex500/qdouble"]
    out["hex500/fast/k42/600"] = digest(po.walk_fast("lozenge", t, 600, 42))
    out["hex500/planes/k42/600"] = digest(po.walk_planes("lozenge", t, 600, 42))
    print(f"  hex500 done: {time.time() - t0:.0f}s", flush=True)
    d = po.ref_build("domino_aztec", p0=2000)
    t = po.ref_build("domino_min", d)
    out["aztec2000/start"] = digest(t)
    out["aztec2000/fast/k42/100"] = digest(po.walk_fast("domino", t, 100, 42))
    out["aztec2000/planes/k42/100"] = digest(po.walk_planes("domino", t, 100, 42))
    out["aztec2000/planes_hb/k42/100"] = digest(po.walk_planes("domino_cftp", t, 100, 42))
    print(f"  aztec2000 done: {time.time() - t0:.0f}s", flush=True)
    return out


def example_outputs() -> dict:
    """SHA-256 of the deterministic Examples/ExampleOuts files, each checked
    against the reference's code run here."""
    ex = os.path.join(REF, "Examples", "ExampleOuts")
    rec = {}
    b = po.ref_build
    for n, name in ((5, "MaxTiling"), (5, "MinTiling"), (5, "SlopeTiling")):
        kind = {"MaxTiling": "max_hex", "MinTiling": "min_hex", "SlopeTiling": "slope_hex"}[name]
        t = b(f"recttri_{kind}", p0=n)
        got = np.loadtxt(os.path.join(ex, "RectTriangle", f"{name}.txt"), dtype=np.int64).reshape(-1)
        assert (got == t).all(), name
        for ext in ("txt", "svg"):
            p = os.path.join(ex, "RectTriangle", f"{name}.{ext}")
            rec[f"RectTriangle/{name}.{ext}"] = hashlib.sha256(open(p, "rb").read()).hexdigest()
    t = b("tridimer_ice_cream_cone", p0=6, p1=0)
    d = b("tridimer_domain", t)
    assert (np.loadtxt(os.path.join(ex, "TriangleDimer", "DimerStart.txt"), dtype=np.int64).reshape(-1) == t).all()
    # SaveMatrix writes sqrt(size) x sqrt(size) entries (common.cpp:169-171); the
    # (M-1) x 2(M-1) domain is therefore saved truncated to its first k*k values.
    saved = np.loadtxt(os.path.join(ex, "TriangleDimer", "Domain.txt"), dtype=np.int64).reshape(-1)
    assert (saved == d[: saved.size]).all()
    for f in ("DimerStart.txt", "Domain.txt", "Domain.svg", "DimerStart.svg", "TilingStart.svg"):
        rec[f"TriangleDimer/{f}"] = hashlib.sha256(open(os.path.join(ex, "TriangleDimer", f), "rb").read()).hexdigest()
    for f in ("domainAlmostHex.svg", "tilingStartAlmostHex.svg"):
        rec[f"MinimalLozenge/{f}"] = hashlib.sha256(open(os.path.join(ex, "MinimalLozenge", f), "rb").read()).hexdigest()
    rec["MinimalDomino/StartTiling.svg"] = hashlib.sha256(
        open(os.path.join(ex, "MinimalDomino", "StartTiling.svg"), "rb").read()).hexdigest()
    return rec


SVG_CASES = [
    # (writer, builders.npz / walks.npz key of the first array, key of the second or None)
    ("domino_domain", "b:domino/aztec5/domain", None),
    ("domino_domain", "b:domino/rect5x8/domain", None),
    ("domino_tiling", "b:domino/aztec5/min", None),
    ("domino_tiling", "w:domino/aztec13/s42/end", None),
    ("domino_maya", "b:domino/aztec8/max", None),
    ("domino_dimer", "b:domino/aztec5/min", None),
    ("domino_dimer", "w:domino_cftp/aztec13/s-7/end", None),
    ("domino_dimer_d", "b:domino/aztec8/min", "b:domino/aztec8/domain"),
    ("lozenge_domain", "b:lozenge/hex10_2/domain", None),
    ("lozenge_tiling", "b:lozenge/hex10_2/max", None),
    ("lozenge_tiling", "w:lozenge/hex13_5/s42/end", None),
    ("lozenge_dimer", "b:lozenge/hex4_1/min", None),
    ("lozenge_dimer", "w:qlozenge/hex10_2/s5/end", None),
    ("lozenge_dimer_d", "b:lozenge/hex10_2/min", "b:lozenge/hex10_2/domain"),
    ("lozenge_print_domain", "b:lozenge/hex4_1/domain", None),
    ("recttri_tiling", "b:recttri/max_hex5", None),
    ("recttri_tiling", "b:recttri/min_hex5", None),
    ("recttri_tiling", "b:recttri/slope_hex5", None),
    ("recttri_tiling", "w:recttri/slope_hex9/s42/end", None),
    ("tridimer_domain", "b:tridimer/cone6_0/domain", None),
    ("tridimer_tiling", "b:tridimer/cone6_0/tiling", None),
    ("tridimer_tiling", "w:tridimer/cone10_3/s7/end", None),
    ("tridimer_dimer", "b:tridimer/cone6_0/tiling", None),
    ("tridimer_dimer", "w:tridimer/cone8_2/s42/end", None),
    ("tridimer_dimer_d", "b:tridimer/cone10_3/tiling", "b:tridimer/cone10_3/domain"),
    ("save_matrix", "b:recttri/max_hex5", None),
    ("save_matrix", "b:tridimer/cone6_0/domain", None),
]


def svg_digests(b: dict, w: dict) -> dict:
    """SHA-256 of the reference's writers on the cases above."""
    import tempfile

    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for k, (writer, ka, kb) in enumerate(SVG_CASES):
            get = lambda key: (b if key[0] == "b" else w)[key[2:]]  # noqa: E731
            path = os.path.join(tmp, f"{k}.out")
            po.ref_write(writer, path, get(ka), None if kb is None else get(kb))
            out[f"{k}:{writer}:{ka}:{kb}"] = hashlib.sha256(open(path, "rb").read()).hexdigest()
    return out


PARTS = ("builders", "walks", "aztec100", "svg", "examples", "qf32", "bench")


def main() -> None:
    ap = argparse.ArgumentParser(description="regenerate the golden fixtures from the reference")
    ap.add_argument("--only", default=",".join(PARTS), help="comma-separated subset of " + ",".join(PARTS))
    parts = set(ap.parse_args().only.split(","))
    if not po.have_ref():
        sys.exit("oracle/_ref/libref.so is missing: run `make -C oracle ref REF=<reference tree>`")
    t0 = time.time()
    start = builders()
    print(f"builders: {len(start)} arrays", flush=True)
    if "builders" in parts:
        np.savez_compressed(os.path.join(OUT, "builders.npz"), **start)
    w = None
    if parts & {"walks", "svg"}:
        w = walks(start)
        print(f"walks: {len(w)} arrays", flush=True)
    if "walks" in parts:
        np.savez_compressed(os.path.join(OUT, "walks.npz"), **w)
    if "aztec100" in parts:
        c0 = aztec100(start)
        np.savez_compressed(os.path.join(OUT, "aztec100.npz"), **c0)
    if "svg" in parts:
        with open(os.path.join(OUT, "svg_digests.json"), "w") as f:
            json.dump(svg_digests(start, w), f, indent=1)
    if "examples" in parts and REF and os.path.isdir(os.path.join(REF, "Examples")):
        with open(os.path.join(OUT, "example_outputs.json"), "w") as f:
            json.dump(example_outputs(), f, indent=1, sort_keys=True)
    if "qf32" in parts:
        q = qlozenge_f32(start)
        print(f"qf32: {len(q)} arrays", flush=True)
        np.savez_compressed(os.path.join(OUT, "qlozenge_f32.npz"), **q)
    if "bench" in parts:
        res = bench_parity()
        with open(os.path.join(OUT, "bench_parity.json"), "w") as f:
            json.dump(res, f, indent=1, sort_keys=True)
    print(f"done in {time.time() - t0:.1f}s")

if __name__ == "__main__":
    main()
