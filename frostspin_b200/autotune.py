"""Autotuner of the sector-GEMM dispatch over the sector-size histogram.

One contraction gives one grouped GEMM launch of sector problems of very uneven
sizes (irrep degeneracies).  Each problem can run on the FP64 tensor-core path
(DMMA, 64 x 64 tiles, split-K for short launches) or on the mixed int8 path of
the current precision mode (256 x 256 CTA-pair tiles; Ozaki I digit slices or
Ozaki II moduli), and which one is faster depends on the shape: small M or N
waste most of a 256-wide tile, short K leaves the int8 pipeline and the CRT
epilogue unamortised.  The tuner measures, for every shape class present in a
recorded set of launches (classes = the bit lengths of M, N and K), a launch of
copies of the class's largest problem on each path with random operands, and
keeps the seconds per FLOP; grouped_gemm then sends each problem to the path
with the smaller predicted time.  Problems of classes that were never measured
take the choice of the nearest measured classes (bit lengths within 2), else the
analytic cost model.

Typical use: record the launches of one untimed iteration
(linalg.record_gemm_calls), then tune(records, mode) before timing.
"""

import time

import numpy as np
import torch

from . import device as dev

_TABLE = {}        # (mode, class) -> {"fp64": s/flop, "mixed": s/flop, "shape": (M, N, K)}
_ENABLED = {"on": False}

# a class is timed on a launch of copies of its representative problem, with N
# cut to at most this many columns, and enough copies for two waves of tiles
_MAX_N = 8192
_TARGET_TILES = 2 * 148
_MAX_BYTES = 4 << 30


def enabled():
    return _ENABLED["on"]


def set_enabled(flag):
    _ENABLED["on"] = bool(flag)


def clear():
    _TABLE.clear()


def shape_class(M, N, K):
    return (int(M).bit_length(), int(N).bit_length(), int(K).bit_length())


def table():
    """The measured table: {(mode, class): {"fp64": s/flop, "mixed": s/flop,
    "shape": representative (M, N, K)}}."""
    return dict(_TABLE)


def _time_launch(M, N, K, ta, tb, copies, modes, reps):
    """Best time of `reps` launches of the class on each path of `modes`, after
    one untimed launch each; the paths alternate launch by launch, so that a
    clock or power drift during the measurement affects them alike."""
    from . import linalg

    g = torch.Generator(device=dev.device())
    g.manual_seed(M * 131 + N * 7 + K)
    specs = []
    for _ in range(copies):
        dA = torch.randn(M * K, dtype=torch.float64, device=dev.device(), generator=g)
        dB = torch.randn(K * N, dtype=torch.float64, device=dev.device(), generator=g)
        dC = torch.empty(M * N, dtype=torch.float64, device=dev.device())
        specs.append({"A": dA, "a_off": 0, "a_trans": ta, "B": dB, "b_off": 0, "b_trans": tb,
                      "C": dC, "c_off": 0, "M": M, "N": N, "K": K})
    best = {m: float("inf") for m in modes}
    for r in range(reps + 1):
        for mode in modes:
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            with linalg.gemm_precision_mode(mode), linalg.ozaki_dispatch_mode("all"), \
                    _bypass():
                linalg.grouped_gemm(specs)
            e1.record()
            torch.cuda.synchronize()
            if r:
                best[mode] = min(best[mode], e0.elapsed_time(e1) * 1e-3)
    linalg.check_ozaki_flags()
    return best


class _bypass:
    """Disables the tuned dispatch while a class is being measured."""

    def __enter__(self):
        self.old = _ENABLED["on"]
        _ENABLED["on"] = False

    def __exit__(self, *exc):
        _ENABLED["on"] = self.old


def tune(records, mode, *, reps=3, min_flops=1e8):
    """Measure every shape class of the recorded launches (a list of
    GEMM_PROBLEM_DTYPE tables) not measured yet for `mode`; returns the number
    of classes measured and the seconds spent."""
    reps_by_class = {}
    for arr in records:
        M = arr["M"].astype(np.int64)
        N = arr["N"].astype(np.int64)
        K = arr["K"].astype(np.int64)
        for i in range(arr.size):
            f = 2.0 * M[i] * N[i] * K[i]
            if f < min_flops:
                continue
            key = shape_class(M[i], N[i], K[i])
            cur = reps_by_class.get(key)
            if cur is None or f > cur[0]:
                reps_by_class[key] = (f, int(M[i]), int(N[i]), int(K[i]),
                                      bool(arr["transA"][i]), bool(arr["transB"][i]))
    t0 = time.perf_counter()
    n = 0
    for key, (_, M, N, K, ta, tb) in sorted(reps_by_class.items()):
        if (mode, key) in _TABLE:
            continue
        Nc = min(N, _MAX_N)
        tiles = max(1, -(-M // 256) * -(-Nc // 256))
        per_copy = 8 * (M * K + K * Nc + M * Nc)
        copies = int(max(1, min(-(-_TARGET_TILES // tiles), _MAX_BYTES // max(per_copy, 1))))
        flops = 2.0 * M * Nc * K * copies
        t = _time_launch(M, Nc, K, ta, tb, copies, ("fp64", mode), reps)
        _TABLE[(mode, key)] = {"shape": (M, N, K), "copies": copies,
                               "fp64": t["fp64"] / flops, "mixed": t[mode] / flops}
        n += 1
    return n, time.perf_counter() - t0


def _choice(mode, key, max_dist):
    """True / False from the measured row of `key`, else from the measured
    classes nearest to it (L1 distance of the bit lengths, at most max_dist;
    FP64 when the nearest ones disagree), else None."""
    row = _TABLE.get((mode, key))
    if row is not None:
        return bool(row["mixed"] < row["fp64"])
    best, votes = None, set()
    for (m, k), r in _TABLE.items():
        if m != mode:
            continue
        d = sum(abs(a - b) for a, b in zip(k, key, strict=True))
        if d > max_dist or (best is not None and d > best):
            continue
        if best is None or d < best:
            best, votes = d, set()
        votes.add(bool(r["mixed"] < r["fp64"]))
    if best is None:
        return None
    return votes == {True}


def decide(arr, mode, *, max_dist=2):
    """Per problem of `arr`: True (mixed path), False (FP64) or None (no
    measured class within max_dist).  A class that was not measured (block
    sizes drift across a power of two between iterations) takes the decision of
    its nearest measured neighbours."""
    out = []
    memo = {}
    for i in range(arr.size):
        key = shape_class(arr["M"][i], arr["N"][i], arr["K"][i])
        if key not in memo:
            memo[key] = _choice(mode, key, max_dist)
        out.append(memo[key])
    return out


def predict(records, mode):
    """Seconds the recorded launches would take by the measured rates: every
    problem on FP64, every problem on the mixed path, and each on the path
    decide() picks (problems of classes with no measured neighbour count on
    FP64 in all three)."""
    out = {"fp64": 0.0, "mixed": 0.0, "chosen": 0.0}
    for arr in records:
        M = arr["M"].astype(np.float64)
        N = arr["N"].astype(np.float64)
        K = arr["K"].astype(np.float64)
        flops = 2.0 * M * N * K
        for i in range(arr.size):
            key = shape_class(arr["M"][i], arr["N"][i], arr["K"][i])
            row = _TABLE.get((mode, key))
            if row is None:
                near = [r for (m, k), r in _TABLE.items() if m == mode and
                        sum(abs(a - b) for a, b in zip(k, key, strict=True)) <= 2]
                row = min(near, key=lambda r: sum(abs(a - b) for a, b in zip(
                    shape_class(*r["shape"]), key, strict=True))) if near else None
            if row is None:
                continue
            f64, mx = row["fp64"] * flops[i], row["mixed"] * flops[i]
            out["fp64"] += f64
            out["mixed"] += mx
            out["chosen"] += min(f64, mx)
    return out

