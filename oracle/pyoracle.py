"""ctypes access to the CPU oracle (TEST INFRASTRUCTURE ONLY).

Two libraries, both built by oracle/Makefile:
  _build/liboracle.so -- the C restatement (rt_oracle.c), always available;
  _ref/libref.so      -- the reference's own sources compiled through the
                         OpenCL shim; only where the reference tree was present
                         at build time.
Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline load this.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")

TINYMT32J = (0x8F7011EE, 0xFC78FF1F, 0x3793FDFF)

_P, _I32, _I64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64


def build_oracle() -> str:
    """Builds the C restatement if it is missing (gcc only)."""
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < max(
        os.path.getmtime(os.path.join(HERE, f)) for f in ("rt_oracle.c", "rt_oracle.h", "sixv_oracle.c")
    ):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return ORACLE_SO


_orc = None
_ref = None


def oracle() -> ctypes.CDLL:
    global _orc
    if _orc is None:
        lib = ctypes.CDLL(build_oracle())
        lib.orc_domino_walk.argtypes = [_P, ctypes.c_int, _I64, _I64, _P, _I64, ctypes.c_int]
        lib.orc_domino_walk_epochs.argtypes = [_P, ctypes.c_int, _P, _P, ctypes.c_int, _P, _I64, ctypes.c_int]
        lib.orc_lozenge_walk.argtypes = [_P, ctypes.c_int, _I64, _I64, _P, _I64, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_int]
        lib.orc_recttri_walk.argtypes = [_P, ctypes.c_int, _I64, _I64, _P, _I64, _P]
        lib.orc_tridimer_walk.argtypes = [_P, ctypes.c_int, _I64, _I64, _P, _I64]
        lib.orc_mt19937_stream.argtypes = [_I64, _I64, _P]
        lib.orc_minstd_raw_stream.argtypes = [_I64, _I64, _P]
        lib.orc_minstd_uniform_stream.argtypes = [_I64, _I64, _P, ctypes.c_int, _P]
        lib.orc_domino_colours.argtypes = [_I64, _I64, ctypes.c_int, _P]
        lib.orc_lozenge_colours.argtypes = [_I64, _I64, _P]
        lib.orc_lozenge_walk_epochs.argtypes = [_P, ctypes.c_int, _P, _P, ctypes.c_int, _P, _I64, ctypes.c_int,
                                                ctypes.c_double, ctypes.c_int]
        lib.orc_philox4x32_10.argtypes = [_P, _P, _P]
        lib.orc_domino_walk_fast.argtypes = [_P, ctypes.c_int, _P, _P, ctypes.c_int, ctypes.c_uint32, ctypes.c_int]
        lib.orc_domino_walk_weighted.argtypes = [_P, ctypes.c_int, _P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_uint32, _P, _I64, ctypes.c_int, _P, _P]
        lib.orc_lozenge_walk_weighted.argtypes = [_P, ctypes.c_int, _P, _P, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_uint32, _P, _I64, ctypes.c_int, _P, _P, _P]
        lib.orc_domino_walk_planes.argtypes = [_P, ctypes.c_int, _P, _P, ctypes.c_int, ctypes.c_uint32, ctypes.c_int]
        lib.orc_lozenge_walk_planes.argtypes = [_P, ctypes.c_int, _P, _P, ctypes.c_int, ctypes.c_uint32]
        lib.orc_lozenge_walk_fast.argtypes = [_P, ctypes.c_int, _P, _P, ctypes.c_int, ctypes.c_uint32, ctypes.c_int,
                                              ctypes.c_double, ctypes.c_int]
        lib.orc_recttri_walk_fast.argtypes = [_P, ctypes.c_int, _I64, _I64, ctypes.c_uint32, _P]
        lib.orc_tridimer_walk_fast.argtypes = [_P, ctypes.c_int, _I64, _I64, ctypes.c_uint32]
        lib.orc_tridimer_arrays.argtypes = [_P, ctypes.c_int, _P]
        lib.orc_project_heights.argtypes = [ctypes.c_int, _P, _I64, _P, _P, _P, _P, ctypes.c_int, _P]
        lib.orc_lozenge_q_divergence.argtypes = [_P, ctypes.c_int, _I64, _I64, ctypes.c_double]
        lib.orc_lozenge_q_divergence.restype = _I64
        lib.orc_sixv_dwbc.argtypes = [ctypes.c_int, _P, _P]
        lib.orc_sixv_vertex_type.argtypes = [ctypes.c_int] * 4
        lib.orc_sixv_thresholds.argtypes = [_P, _P]
        lib.orc_sixv_walk.argtypes = [_P, ctypes.c_int, _P, _P, ctypes.c_int, ctypes.c_uint32, _P]
        lib.orc_sixv_step_rows.argtypes = [_P, ctypes.c_int, ctypes.c_int64, ctypes.c_uint64, ctypes.c_uint32, _P,
                                           ctypes.c_int, ctypes.c_int]
        lib.orc_tinymt_init.argtypes = [_P, ctypes.c_uint32]
        lib.orc_tinymt_bits12.argtypes = [_P]
        lib.orc_tinymt_bits12.restype = ctypes.c_uint32
        _orc = lib
    return _orc


def have_ref() -> bool:
    return os.path.exists(REF_SO)


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        if not have_ref():
            raise FileNotFoundError(REF_SO)
        lib = ctypes.CDLL(REF_SO)
        lib.ref_set_threads.argtypes = [ctypes.c_int]
        lib.ref_write_params.argtypes = [ctypes.c_char_p, ctypes.c_long, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint]
        lib.ref_tiler_create.restype = _P
        lib.ref_tiler_create.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_long]
        lib.ref_tiler_destroy.argtypes = [_P]
        lib.ref_tiler_walk.argtypes = [_P, _P, ctypes.c_long, ctypes.c_long, ctypes.c_long]
        lib.ref_tiler_walk_epochs.argtypes = [_P, _P, ctypes.c_long, _P, _P, ctypes.c_int]
        lib.ref_build.restype = ctypes.c_long
        lib.ref_build.argtypes = [ctypes.c_int, _P, ctypes.c_long, _P, ctypes.c_long, ctypes.c_int, ctypes.c_int, _P,
                                  ctypes.c_long]
        lib.ref_write.argtypes = [ctypes.c_int, _P, ctypes.c_long, _P, ctypes.c_long, ctypes.c_char_p]
        _ref = lib
    return _ref


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what} failed with {rc}")


def _tiling(t) -> tuple[np.ndarray, int]:
    a = np.array(t, dtype=np.int32).reshape(-1).copy()
    n = int(round(a.size ** 0.5))
    assert n * n == a.size
    return a, n


def _table(params):
    if params is None:
        return None, 0, None
    tab = np.ascontiguousarray(params, dtype=np.uint32).reshape(-1)
    return tab.ctypes.data, tab.size // 3, tab


# ---- the C restatement ----------------------------------------------------
def domino_walk(t, steps, seed, cftp=False, params=None) -> np.ndarray:
    a, n = _tiling(t)
    p, np_, keep = _table(params)
    _check(oracle().orc_domino_walk(a.ctypes.data, n, steps, seed, p, np_, int(cftp)), "orc_domino_walk")
    return a


def domino_walk_epochs(t, steps, seeds, cftp=True, params=None) -> np.ndarray:
    a, n = _tiling(t)
    st = np.ascontiguousarray(steps, dtype=np.int64)
    se = np.ascontiguousarray(seeds, dtype=np.int64)
    p, np_, keep = _table(params)
    _check(oracle().orc_domino_walk_epochs(a.ctypes.data, n, st.ctypes.data, se.ctypes.data, st.size, p, np_,
                                           int(cftp)), "orc_domino_walk_epochs")
    return a


def domino_walk_weighted(t, steps, seeds, wh, wv, fast=False, single_walk=False, chain=0, params=None) -> np.ndarray:
    """The heat-bath domino walk with periodic weights (orc_domino_walk_weighted);
    steps / seeds are per epoch (one each for a single walk)."""
    a, n = _tiling(t)
    st = np.ascontiguousarray(np.atleast_1d(steps), dtype=np.int64)
    se = np.ascontiguousarray(np.atleast_1d(seeds), dtype=np.int64)
    h = np.ascontiguousarray(wh, dtype=np.float64)
    v = np.ascontiguousarray(wv, dtype=np.float64)
    p, np_, keep = _table(params)
    _check(oracle().orc_domino_walk_weighted(a.ctypes.data, n, st.ctypes.data, se.ctypes.data, st.size,
                                             int(single_walk), int(fast), chain, p, np_, h.shape[0], h.ctypes.data,
                                             v.ctypes.data), "orc_domino_walk_weighted")
    return a


def lozenge_walk_weighted(t, steps, seeds, w0, w1, w2, fast=False, chain=0, params=None) -> np.ndarray:
    """The uniform lozenge walk with periodic weights (orc_lozenge_walk_weighted);
    steps / seeds are per epoch."""
    a, n = _tiling(t)
    st = np.ascontiguousarray(np.atleast_1d(steps), dtype=np.int64)
    se = np.ascontiguousarray(np.atleast_1d(seeds), dtype=np.int64)
    w = [np.ascontiguousarray(x, dtype=np.float64) for x in (w0, w1, w2)]
    p, np_, keep = _table(params)
    _check(oracle().orc_lozenge_walk_weighted(a.ctypes.data, n, st.ctypes.data, se.ctypes.data, st.size, int(fast),
                                              chain, p, np_, w[0].shape[0], *(x.ctypes.data for x in w)),
           "orc_lozenge_walk_weighted")
    return a


def lozenge_walk(t, steps, seed, qweight=False, q=0.99, qcmp_double=False, params=None) -> np.ndarray:
    a, n = _tiling(t)
    p, np_, keep = _table(params)
    _check(oracle().orc_lozenge_walk(a.ctypes.data, n, steps, seed, p, np_, int(qweight), q, int(qcmp_double)),
           "orc_lozenge_walk")
    return a


def recttri_walk(t, steps, seed, weights=None, params=None) -> np.ndarray:
    a, n = _tiling(t)
    p, np_, keep = _table(params)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
    _check(oracle().orc_recttri_walk(a.ctypes.data, n, steps, seed, p, np_, None if w is None else w.ctypes.data),
           "orc_recttri_walk")
    return a


def tridimer_walk(t, steps, seed, params=None) -> np.ndarray:
    a, n = _tiling(t)
    p, np_, keep = _table(params)
    _check(oracle().orc_tridimer_walk(a.ctypes.data, n, steps, seed, p, np_), "orc_tridimer_walk")
    return a


def tridimer_arrays(t) -> np.ndarray:
    """The eight state arrays (H, L, R, U, D, BH, BL, BR) of a triangle-dimer
    tiling, shape (8, n/2, n/2) (rt_oracle.c: orc_tridimer_arrays)."""
    a, n = _tiling(t)
    out = np.zeros((8, n // 2, n // 2), dtype=np.int32)
    _check(oracle().orc_tridimer_arrays(a.ctypes.data, n, out.ctypes.data), "orc_tridimer_arrays")
    return out


def lozenge_walk_epochs(t, steps, seeds, qweight=False, q=0.99, qcmp_double=False, params=None) -> np.ndarray:
    a, n = _tiling(t)
    st = np.ascontiguousarray(steps, dtype=np.int64)
    se = np.ascontiguousarray(seeds, dtype=np.int64)
    p, np_, keep = _table(params)
    _check(oracle().orc_lozenge_walk_epochs(a.ctypes.data, n, st.ctypes.data, se.ctypes.data, st.size, p, np_,
                                            int(qweight), q, int(qcmp_double)), "orc_lozenge_walk_epochs")
    return a


# ---- fast mode (counter-based draws, cyclic colours) ----------------------
def philox4x32_10(ctr, key) -> list[int]:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    oracle().orc_philox4x32_10(c.ctypes.data, k.ctypes.data, out.ctypes.data)
    return [int(x) for x in out]


def _epochs(steps, keys):
    st = np.atleast_1d(np.ascontiguousarray(steps, dtype=np.int64))
    ke = np.atleast_1d(np.ascontiguousarray(np.asarray(keys, dtype=np.uint64).astype(np.int64), dtype=np.int64))
    assert st.size == ke.size
    return st, ke


def walk_fast(model: str, t, steps, keys, chain: int = 0, q: float = 0.99, qcmp_double: bool = False,
              weights=None) -> np.ndarray:
    """Fast-mode walk of `model` in {"domino", "domino_cftp", "lozenge",
    "qlozenge", "lozenge_q8", "recttri", "tridimer"}; steps / keys are one
    value or one per epoch (epochs: dominoes and lozenges).  "lozenge_q8" is
    the batched chains' volume-weighted int8 rule (add below 0.4 q, remove in
    [0.4, 0.8))."""
    a, n = _tiling(t)
    st, ke = _epochs(steps, keys)
    lib = oracle()
    if model in ("domino", "domino_cftp"):
        rc = lib.orc_domino_walk_fast(a.ctypes.data, n, st.ctypes.data, ke.ctypes.data, st.size, chain,
                                      int(model == "domino_cftp"))
    elif model in ("lozenge", "qlozenge", "lozenge_q8"):
        qmode = {"lozenge": 0, "qlozenge": 1, "lozenge_q8": 2}[model]
        rc = lib.orc_lozenge_walk_fast(a.ctypes.data, n, st.ctypes.data, ke.ctypes.data, st.size, chain,
                                       qmode, q, int(qcmp_double))
    elif model == "recttri":
        assert st.size == 1
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        rc = lib.orc_recttri_walk_fast(a.ctypes.data, n, int(st[0]), int(ke[0]), chain,
                                       None if w is None else w.ctypes.data)
    elif model == "tridimer":
        assert st.size == 1
        rc = lib.orc_tridimer_walk_fast(a.ctypes.data, n, int(st[0]), int(ke[0]), chain)
    else:
        raise ValueError(model)
    _check(rc, f"fast walk of {model}")
    return a


def walk_planes(model: str, t, steps, keys, chain: int = 0) -> np.ndarray:
    """Bit-plane mode walk of `model` in {"domino" (two-bit toggle),
    "domino_cftp" (heat bath), "lozenge" (heat bath)}; steps / keys are one
    value or one per epoch."""
    a, n = _tiling(t)
    st, ke = _epochs(steps, keys)
    lib = oracle()
    if model in ("domino", "domino_cftp"):
        rc = lib.orc_domino_walk_planes(a.ctypes.data, n, st.ctypes.data, ke.ctypes.data, st.size, chain,
                                        int(model == "domino_cftp"))
    elif model == "lozenge":
        rc = lib.orc_lozenge_walk_planes(a.ctypes.data, n, st.ctypes.data, ke.ctypes.data, st.size, chain)
    else:
        raise ValueError(model)
    _check(rc, f"bit-plane walk of {model}")
    return a


def cftp(tmax, tmin, first_steps: int, master_seed: int, schedule: str = "doubling", max_trials: int = 30,
         model: str = "domino_cftp", fast: bool = False, planes: bool = False, weights=None, **kw):
    """CFTP composed from the restated epoch walks, following
    Examples/AztecDiamondCftpEx.cpp:42-68 (seeds: successive mt19937 outputs,
    newest epoch first; in fast mode each seed is its epoch's Philox key).
    model: "domino_cftp", "lozenge" or "qlozenge" (kw: q, qcmp_double);
    weights: (wh, wv) periodic domino weights for "domino_cftp", (w0, w1, w2)
    periodic lozenge weights for "lozenge".
    Returns (tiling, trials, total_steps, coalesced)."""
    def run(t, steps, seeds):
        if weights is not None and model == "lozenge":
            return lozenge_walk_weighted(t, steps, seeds, *weights, fast=fast, **kw)
        if weights is not None:
            return domino_walk_weighted(t, steps, seeds, weights[0], weights[1], fast=fast, **kw)
        if planes:
            return walk_planes(model, t, steps, seeds, **kw)
        if fast:
            return walk_fast(model, t, steps, seeds, **kw)
        if model == "domino_cftp":
            return domino_walk_epochs(t, steps, seeds, cftp=True)
        return lozenge_walk_epochs(t, steps, seeds, qweight=model == "qlozenge", **kw)

    seeds_out = np.zeros(max_trials + 1, dtype=np.uint32)
    oracle().orc_mt19937_stream(master_seed, max_trials + 1, seeds_out.ctypes.data)
    steps, seeds = [first_steps], [int(seeds_out[0])]
    for trial in range(max_trials):
        top, bot = run(tmax, steps, seeds), run(tmin, steps, seeds)
        if np.array_equal(top, bot):
            return top, trial + 1, sum(steps), True
        steps.insert(0, 2 * steps[-1] if schedule == "reference" else sum(steps))
        seeds.insert(0, int(seeds_out[trial + 1]))
    return top, max_trials, sum(steps), False


def project_heights(model: str, domain, hmin, hmax, target) -> np.ndarray:
    """The oracle's height projection; model "domino" or "lozenge"."""
    d = np.ascontiguousarray(domain, dtype=np.int32).reshape(-1)
    lo = np.ascontiguousarray(hmin, dtype=np.int32).reshape(-1)
    hi = np.ascontiguousarray(hmax, dtype=np.int32).reshape(-1)
    t = np.ascontiguousarray(target, dtype=np.float32).reshape(-1)
    n = int(round(lo.size ** 0.5))
    out = np.zeros(n * n, dtype=np.int32)
    _check(oracle().orc_project_heights(0 if model == "domino" else 1, d.ctypes.data, d.size, lo.ctypes.data,
                                        hi.ctypes.data, t.ctypes.data, out.ctypes.data, n, None),
           "orc_project_heights")
    return out


def lozenge_q_divergence(t, seed: int, max_steps: int, q: float = 0.99) -> int:
    """First step count after which the q-weighted walk of t differs between
    the float32 and the double comparison of qlozengekernel.cl:25 (0: none
    within max_steps)."""
    a, n = _tiling(t)
    r = oracle().orc_lozenge_q_divergence(a.ctypes.data, n, seed, max_steps, q)
    if r < 0:
        raise RuntimeError("orc_lozenge_q_divergence failed")
    return int(r)


# ---- six-vertex model (sixv_oracle.c) ----------------------------------------
SIXV_UNIFORM = (1.0, 1.0, 1.0, 1.0, 1.0, 1.0)


def sixv_dwbc(n: int) -> tuple[np.ndarray, np.ndarray]:
    """(h_min, h_max) of the domain-wall boundary, (n+1)^2 int32 each."""
    lo = np.zeros((n + 1) ** 2, dtype=np.int32)
    hi = np.zeros((n + 1) ** 2, dtype=np.int32)
    oracle().orc_sixv_dwbc(n, lo.ctypes.data, hi.ctypes.data)
    return lo, hi


def sixv_thresholds(w=SIXV_UNIFORM) -> np.ndarray:
    ww = np.ascontiguousarray(w, dtype=np.float64)
    out = np.zeros(16, dtype=np.uint32)
    oracle().orc_sixv_thresholds(ww.ctypes.data, out.ctypes.data)
    return out


def sixv_walk(h, sweeps, keys, chain: int = 0, w=SIXV_UNIFORM) -> np.ndarray:
    """The six-vertex heat bath on heights h ((n+1)^2); sweeps / keys one value
    or one per epoch."""
    a = np.array(h, dtype=np.int32).reshape(-1).copy()
    n = int(round(a.size ** 0.5)) - 1
    st, ke = _epochs(sweeps, keys)
    ww = np.ascontiguousarray(w, dtype=np.float64)
    _check(oracle().orc_sixv_walk(a.ctypes.data, n, st.ctypes.data, ke.ctypes.data, st.size, chain, ww.ctypes.data),
           "orc_sixv_walk")
    return a


def sixv_step_rows(a: np.ndarray, s: int, key: int, lo: int, hi: int, chain: int = 0, w=SIXV_UNIFORM) -> None:
    """Colour step s (epoch key `key`) on the face rows [lo, hi) of the
    heights a ((n+1)^2 int32, contiguous), in place."""
    assert a.dtype == np.int32 and a.flags.c_contiguous
    n = int(round(a.size ** 0.5)) - 1
    ww = np.ascontiguousarray(w, dtype=np.float64)
    _check(oracle().orc_sixv_step_rows(a.ctypes.data, n, s, key & (2**64 - 1), chain, ww.ctypes.data, lo, hi),
           "orc_sixv_step_rows")


def sixv_cftp(n: int, first_sweeps: int, master_seed: int, max_trials: int = 30, w=SIXV_UNIFORM, chain: int = 0):
    """CFTP from the maximal and minimal heights as rt_sixv_cftp composes it:
    epoch keys are successive std::mt19937(master_seed) outputs, newest epoch
    first; the schedule doubles.  Returns (heights, trials, total sweeps,
    coalesced)."""
    lo, hi = sixv_dwbc(n)
    keys_out = np.zeros(max_trials + 1, dtype=np.uint32)
    oracle().orc_mt19937_stream(master_seed, max_trials + 1, keys_out.ctypes.data)
    sweeps, keys = [first_sweeps], [int(keys_out[0])]
    top = hi
    for trial in range(max_trials):
        top, bot = sixv_walk(hi, sweeps, keys, chain, w), sixv_walk(lo, sweeps, keys, chain, w)
        if np.array_equal(top, bot):
            return top, trial + 1, sum(sweeps), True
        sweeps.insert(0, sum(sweeps))
        keys.insert(0, int(keys_out[trial + 1]))
    return top, max_trials, sum(sweeps), False


def sixv_vertex_types(h) -> np.ndarray:
    """n x n vertex types (0..5: a1 a2 b1 b2 c1 c2) of heights h; -1 where invalid."""
    a = np.asarray(h, dtype=np.int64).reshape(-1)
    n1 = int(round(a.size ** 0.5))
    H = a.reshape(n1, n1)
    lib = oracle()
    return np.array([[lib.orc_sixv_vertex_type(int(H[i - 1, j - 1]), int(H[i - 1, j]), int(H[i, j - 1]), int(H[i, j]))
                      for j in range(1, n1)] for i in range(1, n1)], dtype=np.int32)


def sixv_enumerate(n: int) -> list[np.ndarray]:
    """Every domain-wall height function of the n x n grid (the alternating-sign
    matrices of order n), by depth-first filling of the interior faces in row
    order (small n only: 1, 2, 7, 42, 429, 7436 configurations)."""
    lo, hi = sixv_dwbc(n)
    N1 = n + 1
    h = lo.astype(np.int64).reshape(N1, N1).copy()
    lo2, hi2 = lo.reshape(N1, N1), hi.reshape(N1, N1)
    cells = [(i, j) for i in range(1, n) for j in range(1, n)]
    out = []

    def rec(k):
        if k == len(cells):
            out.append(h.reshape(-1).astype(np.int32).copy())
            return
        i, j = cells[k]
        for v in (h[i - 1, j] - 1, h[i - 1, j] + 1):
            if lo2[i, j] <= v <= hi2[i, j] and abs(v - h[i, j - 1]) == 1:
                h[i, j] = v
                rec(k + 1)
        h[i, j] = lo2[i, j]

    rec(0)
    return out


def sixv_weight(h, w=SIXV_UNIFORM) -> float:
    t = sixv_vertex_types(h)
    assert (t >= 0).all()
    return float(np.prod(np.asarray(w, dtype=np.float64)[t]))


# ---- the reference's own code (oracle/_ref) --------------------------------
# "qlozenge_f32": qlozengekernel.cl compiled with single-precision arithmetic (an fp32-only device)
REF_MODELS = {"domino": 0, "domino_cftp": 1, "lozenge": 2, "qlozenge": 3, "recttri": 4, "tridimer": 5,
              "qlozenge_f32": 6}


class RefTiler:
    """One reference Tiler object (its LoadTinyMT already done)."""

    def __init__(self, model: str, n_params: int, params=None, threads: int = 1):
        lib = ref()
        lib.ref_set_threads(threads)
        fd, path = tempfile.mkstemp(prefix="tinymt_", suffix=".txt")
        os.close(fd)
        try:
            if params is None:
                lib.ref_write_params(path.encode(), n_params, *TINYMT32J)
            else:
                tab = np.asarray(params, dtype=np.uint32).reshape(-1, 3)
                with open(path, "w") as f:
                    f.write("# table\n")
                    for i, (m1, m2, tm) in enumerate(tab[:n_params]):
                        f.write(f"tinymt32,{i},127,{m1:08x},{m2:08x},{tm:08x},0\n")
            self.h = lib.ref_tiler_create(REF_MODELS[model], path.encode(), n_params)
        finally:
            os.unlink(path)
        if not self.h:
            raise RuntimeError("ref_tiler_create failed")

    def walk(self, t, steps, seed) -> np.ndarray:
        a, n = _tiling(t)
        _check(ref().ref_tiler_walk(self.h, a.ctypes.data, a.size, steps, seed), "ref_tiler_walk")
        return a

    def walk_epochs(self, t, steps, seeds) -> np.ndarray:
        a, n = _tiling(t)
        st = np.ascontiguousarray(steps, dtype=np.int64)
        se = np.ascontiguousarray(seeds, dtype=np.int64)
        _check(ref().ref_tiler_walk_epochs(self.h, a.ctypes.data, a.size, st.ctypes.data, se.ctypes.data, st.size),
               "ref_tiler_walk_epochs")
        return a

    def close(self):
        if self.h:
            ref().ref_tiler_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


BUILD = {
    "domino_rectangle": 0, "domino_aztec": 1, "domino_aztec_rectangle": 2, "domino_max": 3, "domino_min": 4,
    "domino_vertices": 5, "domino_tiling_to_domain": 6, "domino_h2t": 7, "domino_t2h": 8,
    "lozenge_almost_hex": 10, "lozenge_max": 11, "lozenge_min": 12, "lozenge_vertices": 13,
    "lozenge_tiling_to_domain": 14, "lozenge_h2t": 15, "lozenge_t2h": 16,
    "recttri_max_hex": 20, "recttri_min_hex": 21, "recttri_slope_hex": 22, "recttri_from_lozenge": 23,
    "tridimer_ice_cream_cone": 30, "tridimer_test_butterfly": 31, "tridimer_triangle_flips": 32,
    "tridimer_butterfly_flips": 33, "tridimer_vertices": 34, "tridimer_domain": 35, "tridimer_dimer_indicator": 36,
}


def ref_build(what: str, a=None, b=None, p0: int = 0, p1: int = 0) -> np.ndarray:
    lib = ref()
    A = None if a is None else np.ascontiguousarray(a, dtype=np.int32).reshape(-1)
    B = None if b is None else np.ascontiguousarray(b, dtype=np.int32).reshape(-1)
    args = (BUILD[what], None if A is None else A.ctypes.data, 0 if A is None else A.size,
            None if B is None else B.ctypes.data, 0 if B is None else B.size, p0, p1)
    n = lib.ref_build(*args, None, 0)
    if n < 0:
        raise RuntimeError(f"ref_build({what}) failed")
    out = np.zeros(max(n, 1), dtype=np.int32)
    lib.ref_build(*args, out.ctypes.data, n)
    return out[:n]


REF_WRITE = {
    "domino_domain": 0, "domino_tiling": 1, "domino_maya": 2, "domino_dimer": 3, "domino_dimer_d": 4,
    "lozenge_domain": 10, "lozenge_tiling": 11, "lozenge_dimer": 12, "lozenge_dimer_d": 13, "lozenge_print_domain": 14,
    "recttri_tiling": 20, "tridimer_domain": 30, "tridimer_tiling": 31, "tridimer_dimer": 32, "tridimer_dimer_d": 33,
    "save_matrix": 40,
}


def ref_write(what: str, filename: str, a, b=None) -> None:
    """One of the reference's SVG / text writers, run through oracle/_ref."""
    A = np.ascontiguousarray(a, dtype=np.int32).reshape(-1)
    B = None if b is None else np.ascontiguousarray(b, dtype=np.int32).reshape(-1)
    rc = ref().ref_write(REF_WRITE[what], A.ctypes.data, A.size, None if B is None else B.ctypes.data,
                         0 if B is None else B.size, str(filename).encode())
    if rc != 0:
        raise RuntimeError(f"ref_write({what}) failed")
