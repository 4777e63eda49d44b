#!/usr/bin/env python
"""Benchmark driver: prints ONE JSON line (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ctmrg|u1_microbench|gemm|ising] [--precision fp64|ozakiS|ozaki2_N]

Workload "ctmrg" (default): double-layer CTMRG of the spin-1/2 Heisenberg
model on the square lattice.  The site tensors come from the finite-temperature
simple update (2-site checkerboard cell, tau = 0.01, second-order Trotter,
bond dimension target D) evolved to beta = 2 on the device; then
SequentialCTMRG on the AB/BA cell at corner dimension chi.  Default: SU(2)
symmetry, D = 24 (whole multiplets: Dmax = 28), chi = 256.  `--symmetry u1`
runs the same chain with U(1) sectors (defaults D = 12, chi = 64).  One step =
one CTMRG iteration (up, right, down, left moves).  The timed iterations start
from an environment warmed up for W iterations; the headline arithmetic
(`--precision`, default ozaki2_11: sector GEMMs on the tcgen05 int8 tensor
cores, one product per modulus for 11 moduli, CRT in FP64; the autotuner picks
the int8 or FP64 path per sector shape class) runs exactly K iterations after
one untimed iteration of its own, the plain FP64 run (DMMA tensor cores)
min(K, 3) iterations from a copy of the same environment, and the energies per
bond after the same number of iterations are compared.  11 moduli are the
fewest that keep every mixed parity test against the reference's runs within
its tolerance (10 moduli miss the simple-update logZ bound) and the energy
within 1e-12 of plain FP64 over 25 iterations.

Workload "u1_microbench": the U(1) kernel microbenchmark -- rank-4 float64
tensors whose legs carry charges -4..4 with degeneracies ~ exp(-q^2/8) rounded
(largest remainder) to 256 states per leg, only charge-conserving blocks filled
with seeded N(0,1) entries (17 blocks, 455 018 564 coefficients, 3.64 GB per
tensor).  One step = permute (0,2),(1,3) then the grouped matmul against a
second tensor of the same structure, the hot path of every CTMRG contraction.
Inputs are larger than the 126 MB L2, so no flush is needed between steps.

Workload "gemm": one square FP64 GEMM (--gemm-n) through the grouped path at
--precision, timed beside cuBLAS DGEMM (kernel-level measurement).

Multi-GPU: the path does not shard -- every rank runs an independent replica
(weak scaling), and the timed region is the max over ranks.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

# The chi = 256 working set is many sector buffers of very uneven sizes (tens of
# KB to ~11 GB) allocated and freed every move; with fixed segments the caching
# allocator fragments until a request of ~11 GB fails with ~100 GB reserved but
# unused.  Growable segments keep the reserved memory reusable.
os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "expandable_segments:True")

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "CTMRG iter/s, grouped mixed-prec vs plain FP64 on 1 B200 at 1e-9 energy err"
LEG_STATES = 256
QMAX = 4
SEED = 2024


def microbench_rep(total, qmax=QMAX):
    """Charges -qmax..qmax, degeneracy ~ exp(-q^2/8) with largest-remainder
    rounding to `total` states, sorted by charge."""
    q = np.arange(-qmax, qmax + 1)
    w = np.exp(-(q**2) / 8.0)
    raw = w / w.sum() * total
    deg = np.floor(raw).astype(int)
    rem = total - deg.sum()
    order = np.argsort(-(raw - deg), kind="stable")
    deg[order[:rem]] += 1
    return np.repeat(q, deg).astype(np.int8)


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


# ------------------------------------------------------------------- clocks


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.file = None

    def start(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL,
            )
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi missing"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except ValueError:
                continue
            try:
                power.append(float(r[3]))
            except ValueError:
                pass
            for name, val in zip(names, r[5:9], strict=True):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": float(max(smax)) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
            "power_w": float(np.median(power)) if power else None,
        }


# ---------------------------------------------------------------- workloads


class U1Microbench:
    name = "u1_microbench"

    def __init__(self, leg_states=LEG_STATES):
        from frostspin_b200 import U1SymmetricTensor

        self.cls = U1SymmetricTensor
        rep = microbench_rep(leg_states)
        self.rep = rep
        self.sig1 = np.array([False, False, True, True])
        self.sig2 = np.array([True, False, False, True])
        self.irr1, self.shapes1 = U1SymmetricTensor.get_block_sizes(
            (rep, rep), (rep, rep), self.sig1)
        self.irr2, self.shapes2 = U1SymmetricTensor.get_block_sizes(
            (rep, rep), (rep, rep), self.sig2)
        self.ncoeff = int((self.shapes1[:, 0] * self.shapes1[:, 1]).sum())

    def device_inputs(self):
        import torch

        g = torch.Generator(device="cuda")
        g.manual_seed(SEED)
        n2 = int((self.shapes2[:, 0] * self.shapes2[:, 1]).sum())
        f1 = torch.randn(self.ncoeff, dtype=torch.float64, device="cuda", generator=g)
        f2 = torch.randn(n2, dtype=torch.float64, device="cuda", generator=g)
        rep = self.rep
        t1 = self.cls.from_flat((rep, rep), (rep, rep), f1, self.irr1, self.sig1)
        t2 = self.cls.from_flat((rep, rep), (rep, rep), f2, self.irr2, self.sig2)
        return t1, t2

    def flops(self, p, t2):
        common, i1, i2 = np.intersect1d(p.block_irreps, t2.block_irreps,
                                        return_indices=True)
        m = p.block_shapes[i1, 0]
        k = p.block_shapes[i1, 1]
        n = t2.block_shapes[i2, 1]
        return float((2 * m * k * n).sum())

    @staticmethod
    def step(t1, t2, ev=None):
        if ev is not None:
            ev[0].record()
        p = t1.permute((0, 2), (1, 3))
        if ev is not None:
            ev[1].record()
        m = p @ t2
        if ev is not None:
            ev[2].record()
        return m


def measure_dgemm_peak():
    """cuBLAS DGEMM throughput (TFLOP/s) on 8192^3, best of 3: the measured FP64
    denominator for the FP64 GEMM roofline."""
    import torch

    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 0.0
    for _ in range(3):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * n**3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def tensor_ops_ozaki(p, t2, precision):
    """int8 tensor-core operations the mixed path issues on the padded tile
    grid: S(S+1)/2 digit-slice products of 2 M N K (ozakiS, 128 x 256 x 128
    tiles) or one product per modulus (ozaki2_N, 256 x 256 x 128 tiles)."""
    common, i1, i2 = np.intersect1d(p.block_irreps, t2.block_irreps, return_indices=True)
    m = p.block_shapes[i1, 0]
    k = p.block_shapes[i1, 1]
    n = t2.block_shapes[i2, 1]
    pad = lambda x, a: (x + a - 1) // a * a  # noqa: E731
    if precision.startswith("ozaki2_"):
        nmod = int(precision[7:])
        return float((2 * pad(m, 256) * pad(n, 256) * pad(k, 128)).sum() * nmod)
    S = int(precision[5:])
    return float((2 * pad(m, 128) * pad(n, 256) * pad(k, 128)).sum() * S * (S + 1) // 2)


def mixed_kernel_names(precision):
    if precision.startswith("ozaki2_"):
        return "k_oz_pair<CRT>"
    return "k_oz_pair / k_oz_gemm (+ k_oz_split, k_oz_exponents)"


# --------------------------------------------------------------- CPU baseline


def cpu_microbench_seconds(leg_states, nthreads):
    """Oracle (numpy restatement of the reference) permute + matmul on a reduced
    microbench; returns (t_permute, t_matmul, ncoeff, flops) of the sample."""
    os.environ.setdefault("OMP_NUM_THREADS", str(nthreads))
    from oracle import frostspin_oracle as fo

    rep = microbench_rep(leg_states)
    rng = np.random.default_rng(SEED)
    sig1 = np.array([False, False, True, True])
    irr, shapes = fo.get_block_sizes((rep, rep), (rep, rep), sig1)
    t1 = fo.OTensor((rep, rep), (rep, rep), [rng.standard_normal(tuple(s)) for s in shapes],
                    irr, sig1)
    sig2 = np.array([True, False, False, True])
    irr2, shapes2 = fo.get_block_sizes((rep, rep), (rep, rep), sig2)
    t2 = fo.OTensor((rep, rep), (rep, rep), [rng.standard_normal(tuple(s)) for s in shapes2],
                    irr2, sig2)
    t0 = time.perf_counter()
    p = fo.permute(t1, (0, 2), (1, 3))
    t1_ = time.perf_counter()
    fo.matmul(p, t2)
    t2_ = time.perf_counter()
    ncoeff = sum(b.size for b in t1.blocks)
    flops = 0.0
    for q, b in zip(p.block_irreps, p.blocks, strict=True):
        j = np.flatnonzero(t2.block_irreps == q)
        if j.size:
            flops += 2.0 * b.shape[0] * b.shape[1] * t2.blocks[j[0]].shape[1]
    return t1_ - t0, t2_ - t1_, ncoeff, flops


def cpu_baseline_full_step(full_ncoeff, full_flops, sample_states=128):
    nthreads = os.cpu_count() or 1
    tp, tm, nc, fl = cpu_microbench_seconds(sample_states, nthreads)
    t_full = tp * full_ncoeff / nc + tm * full_flops / fl
    return t_full, {
        "cores": nthreads,
        "kind": "port",
        "sample": (
            f"oracle numpy restatement of the reference permute+matmul on the same "
            f"microbench with {sample_states}-state legs ({nc} coeff, {fl:.3g} flop): "
            f"permute {tp:.3f} s, matmul {tm:.3f} s, scaled to the full step by "
            f"coefficients (permute) and flops (matmul)"
        ),
    }



# ------------------------------------------------------------ CTMRG workload

SDS_22 = np.array([[0.25, 0.0, 0.0, 0.0], [0.0, -0.25, 0.5, 0.0], [0.0, 0.5, -0.25, 0.0],
                   [0.0, 0.0, 0.0, 0.25]])


def heisenberg_u1():
    from frostspin_b200 import U1SymmetricTensor

    reps = (np.array([1, -1], dtype=np.int8),) * 2
    return U1SymmetricTensor.from_array(SDS_22.reshape(2, 2, 2, 2), reps, reps)


def heisenberg_su2():
    from frostspin_b200 import SU2SymmetricTensor

    r = np.array([[1], [2]])
    return SU2SymmetricTensor.from_array(SDS_22.reshape(2, 2, 2, 2), (r, r), (r, r))


def energy_per_bond(ctm):
    """Mean of tr(rho h) over the 4 inequivalent bonds of the AB/BA cell."""
    h = SDS_22.reshape(2, 2, 2, 2)
    es = []
    for x, y in ctm.site_coords:
        for r in (ctm.compute_rdm1x2(x, y), ctm.compute_rdm2x1(x, y)):
            es.append(float(np.einsum("ijkl,klij->", r.toarray(), h)))
    return float(np.mean(es))


def ctmrg_setup(args):
    import torch

    from frostspin_b200.ctmrg import SequentialCTMRG
    from frostspin_b200.simple_update import SimpleUpdate

    t0 = time.perf_counter()
    h = heisenberg_su2() if args.symmetry == "su2" else heisenberg_u1()
    su = SimpleUpdate.square_lattice_first_neighbor(h, args.D, 0.01,
                                                    rcutoff=1e-10, degen_ratio=0.9999)
    su.evolve(args.beta)
    tensors = su.get_tensors()
    torch.cuda.synchronize()
    t_su = time.perf_counter() - t0
    ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", tensors, args.chi, cutoff=1e-10,
                                                  degen_ratio=0.9999)
    return su, tensors, ctm, t_su


def timed_iterations(ctm, steps, precision, local):
    import torch

    from frostspin_b200 import _native, instrument, linalg

    linalg.set_gemm_precision(precision)
    clocks = ClockSampler(local)
    torch.cuda.synchronize()
    n0 = _native.kernel_launches()
    instrument.enable()
    clocks.start()
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    # NVTX range for profilers: "timed_fp64" or "timed_mixed"
    torch.cuda.nvtx.range_push("timed_fp64" if precision == "fp64" else "timed_mixed")
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    s.record()
    for i in range(steps):
        ctm.iterate()
        marks[i].record()
    e.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    clk = clocks.stop()
    instrument.disable()
    kernels = instrument.summary()
    kernels["per_iteration_s"] = [round(a.elapsed_time(b) * 1e-3, 4)
                                  for a, b in zip([s, *marks[:-1]], marks, strict=True)]
    launches = _native.kernel_launches() - n0
    linalg.check_ozaki_flags()
    return s.elapsed_time(e) * 1e-3, clk, kernels, launches


def _split_roofline(sp, hbm):
    """The Ozaki II operand split (k_oz2_exponents + k_oz2_split) against the
    copy bandwidth: per operand entry 8 bytes read twice (row maxima, then the
    split) and one residue byte written per modulus."""
    if not sp or not sp.get("ms"):
        return None
    gbs = sp["bytes"] / (sp["ms"] * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": "k_oz2_exponents + k_oz2_split", "achieved": gbs,
            "peak": hbm, "unit": "GB/s", "frac": gbs / hbm, "launches": sp["launches"],
            "ms": sp["ms"]}


def _fused_roofline(fz, hbm):
    """The fused SU(2) permute (k_su2_fused) against the copy bandwidth: 16
    bytes per coefficient (one read, one write)."""
    if not fz or not fz.get("ms"):
        return None
    gbs = fz["bytes"] / (fz["ms"] * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": "k_su2_fused", "achieved": gbs, "peak": hbm,
            "unit": "GB/s", "frac": gbs / hbm, "launches": fz["launches"], "ms": fz["ms"]}


def _kernel_table(kern):
    return {k: (v if k == "per_iteration_s" else {kk: round(vv, 4) for kk, vv in v.items()})
            for k, v in kern.items()}


def run_ctmrg(args, world, rank, local):
    import torch

    from frostspin_b200 import linalg

    mixed = args.precision if args.precision != "fp64" else "ozaki2_11"
    su, tensors, ctm, t_su = ctmrg_setup(args)
    linalg.set_gemm_precision("fp64")
    # the warm-up iterations record the sector GEMM launches; the tuner
    # measures their shape classes on both paths before timing
    records = []
    for w in range(args.warmup):
        if args.autotune == "on":
            with linalg.record_gemm_calls() as rec:
                ctm.iterate()
                if w == args.warmup - 1:
                    # the end-to-end loop evaluates the energy every step:
                    # its rdm contractions are tuned too
                    energy_per_bond(ctm)
            records += rec
        else:
            ctm.iterate()
    torch.cuda.synchronize()
    tune_info = None
    if args.autotune == "on" and args.precision != "fp64":
        from frostspin_b200 import autotune

        n_cls, t_tune = autotune.tune(records, mixed)
        autotune.set_enabled(True)
        pred = autotune.predict(records, mixed)
        tune_info = {"classes_measured": n_cls, "seconds": t_tune,
                     "predicted_gemm_s_per_warmup_iteration": {
                         k: v / max(args.warmup, 1) for k, v in pred.items()},
                     "classes_mixed": sum(1 for (m, _), r in autotune.table().items()
                                          if m == mixed and r["mixed"] < r["fp64"]),
                     "classes_total": sum(1 for (m, _) in autotune.table() if m == mixed)}
    start_env = ctm.copy()
    headline_mixed = args.precision != "fp64"
    if headline_mixed:
        # one untimed mixed iteration on a throwaway copy: the warm-up above
        # ran the FP64 path only, and the first int8 iteration pays one-time
        # costs (slice workspaces and residue scratch growing the allocator's
        # segments, plans of the new launch shapes)
        warm = start_env.copy()
        linalg.set_gemm_precision(mixed)
        warm.iterate()
        del warm
        linalg.set_gemm_precision("fp64")
        torch.cuda.synchronize()
    # the headline run times exactly `steps` iterations; the comparison run
    # (the other arithmetic, same start environment) is capped at 3 iterations
    # and both energies are taken after the same number of iterations
    n_cmp = min(args.steps, 3)
    n64 = args.steps if not headline_mixed else n_cmp
    nmx = args.steps if headline_mixed else n_cmp
    # energies after the same number of iterations from the same start; each
    # environment is dropped as soon as its energy is known (four chi = 256
    # environments plus the rdm intermediates do not fit at once)
    barrier(world)
    t64, clk64, k64, l64 = timed_iterations(ctm, n64, "fp64", local)
    chi_values = [int(c) for c in ctm.chi_values]
    e64 = energy_per_bond(ctm) if n64 == n_cmp else None
    # freed, not released: the mixed run reuses the mapped segments (releasing
    # them made its first iteration map tens of GB again)
    del ctm
    ctm_mixed = start_env.copy()
    barrier(world)
    tmx, clkmx, kmx, lmx = timed_iterations(ctm_mixed, nmx, mixed, local)
    emx = energy_per_bond(ctm_mixed) if nmx == n_cmp else None
    if args.symmetry != "u1":
        del ctm_mixed
    for prec in ("fp64", mixed):
        if (e64 if prec == "fp64" else emx) is not None:
            continue
        env = start_env.copy()
        linalg.set_gemm_precision(prec)
        for _ in range(n_cmp):
            env.iterate()
        if prec == "fp64":
            e64 = energy_per_bond(env)
        else:
            emx = energy_per_bond(env)
        del env
    t64 = max_over_ranks(t64, world)
    tmx = max_over_ranks(tmx, world)
    t_head = tmx if headline_mixed else t64
    kern = kmx if headline_mixed else k64

    # end to end through the public API: site tensors uploaded from pinned host
    # buffers each step, energy (reduced density matrices) read back
    hostA = [t.data.cpu().pin_memory() for t in tensors]
    e2e_env = start_env.copy()
    linalg.set_gemm_precision(mixed if headline_mixed else "fp64")
    e2e_steps = args.steps
    torch.cuda.synchronize()
    es = torch.cuda.Event(enable_timing=True)
    ee = torch.cuda.Event(enable_timing=True)
    es.record()
    for _ in range(e2e_steps):
        new = [type(t).from_flat(t.row_reps, t.col_reps, h, t.block_irreps, t.signature)
               for t, h in zip(tensors, hostA, strict=True)]
        e2e_env.set_tensors(new)
        e2e_env.iterate()
        energy_per_bond(e2e_env)
    ee.record()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(es.elapsed_time(ee) * 1e-3, world)
    del e2e_env, new
    h2d = int(sum(h.numel() * 8 for h in hostA))
    d2h = int(4 * 2 * 16 * 8)  # four 2x2x2x2 reduced density matrices per site pair

    # the same workload at the smaller chi the CPU arm measures, so that a
    # same-configuration GPU/CPU ratio exists next to the chi=256 extrapolation
    same_cfg = {}
    for chi_c in (int(c) for c in args.compare_chis.split(",") if c):
        from frostspin_b200.ctmrg import SequentialCTMRG

        c_env = SequentialCTMRG.from_elementary_tensors("AB\nBA", tensors, chi_c, cutoff=1e-10,
                                                        degen_ratio=0.9999)
        linalg.set_gemm_precision("fp64")
        c_env.iterate()
        row = {}
        for prec in ("fp64", mixed):
            env = c_env.copy()
            linalg.set_gemm_precision(prec)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            env.iterate()
            e1.record()
            torch.cuda.synchronize()
            row["gpu_s_per_iter_" + ("fp64" if prec == "fp64" else "mixed")] = \
                max_over_ranks(e0.elapsed_time(e1) * 1e-3, world)
        same_cfg[str(chi_c)] = row
    linalg.check_ozaki_flags()

    hbm, bf16, peak_kind = load_peaks()
    fp64_peak = measure_dgemm_peak()
    gem = kern.get("gemm_ozaki") if headline_mixed else kern.get("gemm_fp64")
    if gem is None:
        gem = kern.get("gemm_fp64", {"ms": 1.0, "flops": 0.0, "launches": 0})
    perm = kern.get("permute", {"ms": 1.0, "bytes": 0.0, "launches": 0})
    if headline_mixed and "gemm_ozaki" in kern:
        ach = gem["int8_ops"] / (gem["ms"] * 1e-3) / 1e12
        roof = {"bound": "tensor", "kernel": mixed_kernel_names(mixed),
                "achieved": ach, "peak": 2.0 * bf16, "unit": "TOP/s (int8)",
                "frac": ach / (2.0 * bf16),
                "peak_kind": f"2 x {peak_kind} bf16 dense (int8 dense rate is twice bf16)",
                "traffic": None, "launches": gem["launches"], "ms": gem["ms"],
                "effective_fp64_tflops": gem["flops"] / (gem["ms"] * 1e-3) / 1e12}
    else:
        ach = gem["flops"] / (gem["ms"] * 1e-3) / 1e12
        roof = {"bound": "tensor", "kernel": "k_grouped_dgemm", "achieved": ach,
                "peak": fp64_peak, "unit": "TFLOP/s", "frac": ach / fp64_peak,
                "peak_kind": "measured in-run cuBLAS DGEMM 8192^3", "traffic": None,
                "launches": gem["launches"], "ms": gem["ms"]}
    perm_gbs = perm["bytes"] / (perm["ms"] * 1e-3) / 1e9
    value = world * args.steps / t_head
    fp64_rate = world * n64 / t64
    mixed_rate = world * nmx / tmx
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "iter/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_head / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if not headline_mixed else f"f64 via int8 {mixed}",
        "data": "synthetic (site tensors from the device simple update, seeded)",
        "impl": "ours",
        "config": {
            "workload": f"ctmrg_heisenberg_{args.symmetry}",
            "model": ("spin-1/2 Heisenberg square lattice, AB/BA cell, "
                      + ("SU(2) multiplets" if args.symmetry == "su2" else "U(1) sectors")),
            "beta": args.beta, "D_target": args.D, "Dmax": su.Dmax, "chi": args.chi,
            "chi_values": chi_values,
            "precision": mixed if headline_mixed else "fp64",
            "ozaki_pair": args.ozaki_pair,
            "autotune": tune_info,
            "fp64_iter_per_s": fp64_rate, "fp64_steps": n64,
            "mixed_iter_per_s": mixed_rate, "mixed_steps": nmx,
            "mixed_over_fp64": mixed_rate / fp64_rate,
            "energy_iterations_compared": n_cmp,
            "energy_fp64": e64, "energy_mixed": emx,
            "energy_rel_err_mixed_vs_fp64": abs(emx - e64) / abs(e64),
            "kernels_fp64_run": _kernel_table(k64),
            "kernels_mixed_run": _kernel_table(kmx),
            "simple_update_setup_s": t_su,
            "l2": "working set > 126 MB L2 (no flush needed)",
            "parallelism": f"replicas x{world}",
        },
        "roofline": roof,
        "roofline_permute": {"bound": "hbm", "kernel": "k_perm_gather", "achieved": perm_gbs,
                             "peak": hbm, "unit": "GB/s", "frac": perm_gbs / hbm,
                             "launches": perm["launches"], "ms": perm["ms"]},
        "roofline_permute_fused": _fused_roofline(kern.get("permute_fused"), hbm),
        "roofline_ozaki_split": _split_roofline(kern.get("ozaki_split"), hbm),
        "e2e": {"value": world * e2e_steps / t_e2e, "unit": "iter/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "same_config_points": same_cfg,
        "gpu_launches": lmx if headline_mixed else l64,
        "clocks": clkmx if headline_mixed else clk64,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        if args.symmetry == "u1":
            t_cpu, info = cpu_ctmrg_seconds(tensors, ctm_mixed, args.chi)
            info["value"] = 1.0 / t_cpu
            info["unit"] = "iter/s"
        else:
            info = cpu_ctmrg_sample(args.symmetry, args.chi, chis=(16, 32))
        line["cpu_baseline"] = info
    return line


SU_FIXTURES = {"su2": "su2_d24_beta2", "u1": "heisenberg_d12_beta2"}


def fixture_site_tensors(symmetry):
    """The reference's own simple-update site tensors at beta = 2 (committed
    fixtures written by tests/golden/make_golden.py) as oracle tensors."""
    from oracle import frostspin_oracle as fo
    from oracle import su2_oracle as so

    m = so if symmetry == "su2" else fo
    d = np.load(os.path.join(ROOT, "tests", "golden", SU_FIXTURES[symmetry] + ".npz"))
    out = []
    for p in ("A0", "A1"):
        nrr = int(d[p + "_n_row_reps"])
        ncr = int(d[p + "_n_col_reps"])
        irr = d[p + "_block_irreps"]
        out.append(m.OTensor([d[f"{p}_row_rep_{i}"] for i in range(nrr)],
                             [d[f"{p}_col_rep_{i}"] for i in range(ncr)],
                             [d[f"{p}_block_{i}"] for i in range(irr.size)], irr,
                             d[p + "_signature"]))
    return out


def cpu_ctmrg_sample(symmetry, chi_target, *, chis=(32, 64), timed=1, one_thread=True):
    """Bounded CPU sample of the CTMRG workload: the numpy oracle (restating the
    reference) from the reference's own site tensors, with BLAS on every host
    core (pinned through threadpoolctl); at each chi of `chis` one untimed
    iteration grows the environment to that chi, then `timed` iterations are
    timed.  The value at chi_target is a power law t = t(chis[-1]) (chi /
    chis[-1])^p fitted on the last two measured points, labelled as an
    extrapolation when chi_target is not among them.  With one_thread, one more
    iteration of the first chi's environment is timed with BLAS on one thread
    (the 1-thread number of the baseline protocol)."""
    from threadpoolctl import threadpool_info, threadpool_limits

    from oracle import ctmrg_oracle as co

    cores = os.cpu_count() or 1
    A, B = fixture_site_tensors(symmetry)
    times = {}
    first_env = None
    with threadpool_limits(limits=cores):
        threads = sorted({int(d.get("num_threads", 0)) for d in threadpool_info()})
        for chi in chis:
            c = co.SequentialCTMRG(A, B, chi, cutoff=1e-10, degen_ratio=0.9999)
            c.iterate()
            t0 = time.perf_counter()
            for _ in range(timed):
                c.iterate()
            times[chi] = (time.perf_counter() - t0) / timed
            if first_env is None:
                first_env = c
    one = None
    if one_thread and first_env is not None:
        with threadpool_limits(limits=1):
            t0 = time.perf_counter()
            first_env.iterate()
            one = {"chi": int(chis[0]), "s_per_iter": time.perf_counter() - t0, "threads": 1}
    measured = chi_target in times
    if measured:
        t_target, p = times[chi_target], None
    else:
        c0, c1 = chis[-2], chis[-1]
        p = float(np.log(times[c1] / times[c0]) / np.log(c1 / c0))
        t_target = times[c1] * (chi_target / c1) ** max(p, 0.0)
    pts = ", ".join(f"{v:.1f} s at chi={k}" for k, v in times.items())
    return {
        "value": 1.0 / t_target, "unit": "iter/s", "cores": cores, "kind": "port",
        "blas_threads": threads,
        "sample": (f"numpy oracle SequentialCTMRG ({symmetry}) from the reference's own "
                   f"simple-update tensors (D=24 target, beta=2), BLAS on {cores} host cores; "
                   f"one warm-up then {timed} timed iteration(s) per chi: {pts}"
                   + ("" if measured else
                      f"; value = power-law fit (exponent {p:.2f}) on the last two points, "
                      f"extrapolated to chi={chi_target} ({t_target:.0f} s/iteration), "
                      f"labelled as an extrapolation")),
        "measured_s_per_iter": {str(k): v for k, v in times.items()},
        "one_thread": one,
        "fit_exponent": p, "extrapolated": not measured,
    }


def env_to_oracle(dev_ctm, chi):
    """Oracle CTMRG warm-started from a device environment (host copies)."""
    from oracle import ctmrg_oracle as co
    from oracle import frostspin_oracle as fo

    def ot(t):
        return co.OT(fo.OTensor(t.row_reps, t.col_reps, t.host_blocks(), t.block_irreps,
                                t.signature))

    env = dev_ctm.environment
    A, B = env.elementary_tensors
    oc = co.SequentialCTMRG(ot(A).o, ot(B).o, chi, cutoff=1e-10, degen_ratio=0.9999)
    for name in ("C1", "C2", "C3", "C4", "T1", "T2", "T3", "T4"):
        oc.t[name] = [ot(t) for t in env.tensors(name)]
    return oc


def cpu_ctmrg_seconds(tensors, dev_ctm, chi):
    """One iteration of the numpy oracle CTMRG (restating the reference), warm
    started from the device environment at the same chi and D."""
    oc = env_to_oracle(dev_ctm, chi)
    t0 = time.perf_counter()
    oc.iterate()
    t = time.perf_counter() - t0
    return t, {"cores": os.cpu_count() or 1, "kind": "port",
               "sample": (f"one iteration of the numpy oracle SequentialCTMRG (dense "
                          f"sector SVDs, BLAS with all host threads) at the same D and "
                          f"chi={chi}, warm-started from the device environment: {t:.2f} s")}

# ------------------------------------------------------------------- driver


def dist_init(gpus):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def run_ours(args, world, rank, local):
    import torch

    from frostspin_b200 import _native

    from frostspin_b200 import linalg

    linalg.set_gemm_precision(args.precision)
    wl = U1Microbench(args.leg_states)
    t1, t2 = wl.device_inputs()
    m = wl.step(t1, t2)
    flops = wl.flops(t1.permute((0, 2), (1, 3)), t2)
    del m
    for _ in range(args.warmup):
        wl.step(t1, t2)
    torch.cuda.synchronize()

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record()
    for k in range(args.steps):
        wl.step(t1, t2, evs[k])
    end.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    elapsed = max_over_ranks(start.elapsed_time(end) * 1e-3, world)
    perm_ms_in_step = float(np.mean([e[0].elapsed_time(e[1]) for e in evs]))
    gemm_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in evs]))

    # the permute kernel timed alone (inside the step it runs at the clocks the
    # power-capped GEMM leaves it)
    for _ in range(3):
        t1.permute((0, 2), (1, 3))
    pclk = ClockSampler(local)
    pclk.start()
    ps = torch.cuda.Event(enable_timing=True)
    pe = torch.cuda.Event(enable_timing=True)
    n_perm = 20
    ps.record()
    for _ in range(n_perm):
        t1.permute((0, 2), (1, 3))
    pe.record()
    torch.cuda.synchronize()
    perm_clk = pclk.stop()
    perm_ms = ps.elapsed_time(pe) / n_perm

    # end-to-end through the public API from pinned host buffers
    rep = wl.rep
    h1 = t1.data.cpu().pin_memory()
    h2 = t2.data.cpu().pin_memory()
    out_host = torch.empty(int(t1.data.numel()), dtype=torch.float64).pin_memory()
    e2e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    barrier(world)
    es = torch.cuda.Event(enable_timing=True)
    ee = torch.cuda.Event(enable_timing=True)
    es.record()
    for _ in range(e2e_steps):
        a = wl.cls.from_flat((rep, rep), (rep, rep), h1, wl.irr1, wl.sig1)
        b = wl.cls.from_flat((rep, rep), (rep, rep), h2, wl.irr2, wl.sig2)
        r = wl.step(a, b)
        out_host[: r.data.numel()].copy_(r.data, non_blocking=True)
        del a, b, r
    ee.record()
    torch.cuda.synchronize()
    e2e_elapsed = max_over_ranks(es.elapsed_time(ee) * 1e-3, world)

    hbm, bf16, peak_kind = load_peaks()
    fp64_peak = measure_dgemm_peak()
    linalg.check_ozaki_flags()
    perm_bytes = 16.0 * wl.ncoeff
    perm_gbs = perm_bytes / (perm_ms * 1e-3) / 1e9
    gemm_tf = flops / (gemm_ms * 1e-3) / 1e12
    value = world * args.steps / elapsed
    if args.precision.startswith("ozaki"):
        int8_ops = tensor_ops_ozaki(t1.permute((0, 2), (1, 3)), t2, args.precision)
        int8_peak = 2.0 * bf16
        gemm_roofline = {
            "bound": "tensor",
            "kernel": mixed_kernel_names(args.precision),
            "achieved": int8_ops / (gemm_ms * 1e-3) / 1e12,
            "peak": int8_peak,
            "unit": "TOP/s (int8)",
            "frac": int8_ops / (gemm_ms * 1e-3) / 1e12 / int8_peak,
            "peak_kind": f"2 x {peak_kind} bf16 dense (int8 dense rate is twice bf16)",
            "traffic": None,
            "int8_ops_per_step": int8_ops,
            "note": "ms includes the digit-split kernels",
        }
    else:
        gemm_roofline = {
            "bound": "tensor",
            "kernel": "k_grouped_dgemm",
            "achieved": gemm_tf,
            "peak": fp64_peak,
            "unit": "TFLOP/s",
            "frac": gemm_tf / fp64_peak,
            "peak_kind": "measured in-run cuBLAS DGEMM 8192^3 (no FP64 figure in the peaks file)",
            "traffic": None,
        }
    line = {
        "metric": "U(1) microbench permute+grouped-matmul steps/s",
        "value": value,
        "unit": "step/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": elapsed / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded N(0,1) blocks)",
        "impl": "ours",
        "config": {
            "workload": wl.name,
            "legs": "4 x 256 states, U(1) charges -4..4, degeneracies [7,17,32,46,52,46,32,17,7]",
            "ncoeff": wl.ncoeff,
            "gemm_flop_per_step": flops,
            "gemm_precision": args.precision,
            "l2": "inputs 3.64 GB per tensor > 126 MB L2; no flush needed",
            "parallelism": f"replicas x{world}",
        },
        "roofline": gemm_roofline,
        "gemm_vs_cublas_dgemm": gemm_tf / fp64_peak,
        "roofline_permute": {
            "bound": "hbm",
            "kernel": "k_perm_gather",
            "achieved": perm_gbs,
            "peak": hbm,
            "unit": "GB/s",
            "frac": perm_gbs / hbm,
            "peak_kind": f"{peak_kind} copy bandwidth (burst)",
            "ms": perm_ms,
            "timing": "20 back-to-back launches timed alone with CUDA events",
            "ms_inside_step": perm_ms_in_step,
            "clocks": perm_clk,
        },
        "e2e": {
            "value": world * e2e_steps / e2e_elapsed,
            "unit": "step/s",
            "h2d_bytes_per_step": int(h1.numel() * 8 + h2.numel() * 8),
            "d2h_bytes_per_step": int(t1.data.numel() * 8),
        },
        "gpu_launches": (2 if args.precision == "fp64" else 4) * args.steps,
        "clocks": clk,
    }
    if rank == 0 and not args.no_cpu_baseline:
        t_cpu, info = cpu_baseline_full_step(wl.ncoeff, flops)
        info["value"] = 1.0 / t_cpu
        info["unit"] = "step/s"
        line["cpu_baseline"] = info
    del _native
    return line


def run_gemm(args, world, rank, local):
    """One FP64 GEMM (n^3 with n = --gemm-n, or --gemm-shape M,N,K) through the grouped sector-GEMM path
    at --precision (fp64: DMMA; ozakiS: tcgen05 int8, every problem on the int8
    path), timed with CUDA events beside cuBLAS DGEMM on the same operands."""
    import torch

    from frostspin_b200 import linalg

    n = args.gemm_n
    M, N, K = (int(x) for x in args.gemm_shape.split(",")) if args.gemm_shape else (n, n, n)
    g = torch.Generator(device="cuda").manual_seed(SEED)
    A = torch.randn(M, K, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(K, N, dtype=torch.float64, device="cuda", generator=g)
    C = torch.empty(M, N, dtype=torch.float64, device="cuda")
    spec = [{"A": A.reshape(-1), "a_off": 0, "a_trans": False, "B": B.reshape(-1), "b_off": 0,
             "b_trans": False, "C": C.reshape(-1), "c_off": 0, "M": M, "N": N, "K": K}]

    def step():
        with linalg.gemm_precision_mode(args.precision), linalg.ozaki_dispatch_mode("all"):
            linalg.grouped_gemm(spec)

    def timed(f):
        for _ in range(args.warmup):
            f()
        torch.cuda.synchronize()
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(args.steps):
            f()
        e.record()
        torch.cuda.synchronize()
        return s.elapsed_time(e) * 1e-3 / args.steps

    clocks = ClockSampler(local)
    clocks.start()
    t = max_over_ranks(timed(step), world)
    clk = clocks.stop()
    linalg.check_ozaki_flags()
    err = float((C - A @ B).abs().max() / (A.abs().max() * B.abs().max() * K))
    t_cublas = timed(lambda: torch.matmul(A, B, out=C))
    flops = 2.0 * M * N * K
    return {
        "metric": "square GEMM, effective FP64 TFLOP/s", "value": world * flops / t / 1e12,
        "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else f"f64 via int8 {args.precision}",
        "data": "synthetic (seeded N(0,1))", "impl": "ours",
        "config": {"workload": "gemm", "shape": [M, N, K], "precision": args.precision,
                   "cublas_dgemm_tflops": flops / t_cublas / 1e12,
                   "max_err_rel_to_maxA_maxB_n": err},
        "clocks": clk,
        "roofline": _gemm_roofline(args.precision, M, N, K, t, clk),
    }


def _gemm_roofline(precision, M, N, K, t, clk):
    """Tensor roofline of one GEMM launch: int8 operations on the padded tile
    grid (Ozaki forms) or FP64 flops (DMMA) per second against the peak, and
    the same fraction per SM clock cycle (the kernel runs at the power cap, so
    the clock it gets is part of the result)."""
    pad = lambda x, a: (x + a - 1) // a * a  # noqa: E731
    hbm, bf16, kind = load_peaks()
    if precision.startswith("ozaki2_"):
        ops = 2.0 * pad(M, 256) * pad(N, 256) * pad(K, 128) * int(precision[7:])
        peak, unit, name = 2.0 * bf16, "TOP/s (int8)", "k_oz_pair<CRT>"
    elif precision.startswith("ozaki"):
        S = int(precision[5:])
        ops = 2.0 * pad(M, 128) * pad(N, 256) * pad(K, 128) * S * (S + 1) / 2
        peak, unit, name = 2.0 * bf16, "TOP/s (int8)", "k_oz_gemm_pair"
    else:
        return None
    ach = ops / t / 1e12
    out = {"bound": "tensor", "kernel": name, "achieved": ach, "peak": peak, "unit": unit,
           "frac": ach / peak, "peak_kind": f"2 x {kind} bf16 dense", "traffic": None}
    if clk.get("sm_mhz") and clk.get("sm_max_mhz"):
        out["frac_per_clock"] = ach / peak * clk["sm_max_mhz"] / clk["sm_mhz"]
    return out


def run_reference_ctmrg(args, world):
    """The reference arm of the CTMRG workload: the CPU oracle port (the
    reference is Python + numba and does not travel to the GPU box)."""
    chis = tuple(int(c) for c in args.cpu_chis.split(","))
    info = cpu_ctmrg_sample(args.symmetry, args.chi, chis=chis)
    value = info["value"]
    return {
        "metric": METRIC,
        "value": value, "unit": "iter/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (the reference's own simple-update site tensors, committed fixture)",
        "impl": "reference",
        "config": {"workload": f"ctmrg_heisenberg_{args.symmetry}", "beta": args.beta,
                   "D_target": args.D, "chi": args.chi,
                   "precision": "fp64 (numpy / OpenBLAS)",
                   "parallelism": "host threads"},
        "cpu_baseline": info,
        "e2e": {"value": value, "unit": "iter/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


ISING_BETA = 0.44
ISING_CHI = 32
ISING_ITERS = 100


def run_ising(args, world, rank, local):
    """Config 1: C4v classical Ising CTMRG (Z2 sectors), beta = 0.44, chi = 32,
    the reference example's seeded start; one step = one iteration
    (examples/ising_classical_ctmrg.py:115-204).  W untimed then K timed
    iterations, then untimed iterations up to 100 in total, after which the
    energy per bond and the correlation length are reported."""
    import torch

    from frostspin_b200 import _native
    from frostspin_b200.ctmrg import (correlation_length, energy_per_bond,
                                      ising_initial_environment, ising_site_tensors,
                                      iterate_c4v)

    a, a2, a0d, mopd = ising_site_tensors(ISING_BETA)
    s, T = ising_initial_environment(ISING_CHI, np.random.default_rng(42))
    for _ in range(args.warmup):
        s, T = iterate_c4v(s, T, a, a2, ISING_CHI)
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    n0 = _native.kernel_launches()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        s, T = iterate_c4v(s, T, a, a2, ISING_CHI)
    ev1.record()
    torch.cuda.synchronize()
    launches = _native.kernel_launches() - n0
    clk = clocks.stop()
    t = max_over_ranks(ev0.elapsed_time(ev1) * 1e-3, world)
    done = args.warmup + args.steps
    for _ in range(max(0, ISING_ITERS - done)):
        s, T = iterate_c4v(s, T, a, a2, ISING_CHI)
    e = energy_per_bond(s, T, a0d, mopd)
    xi = correlation_length(T)
    line = {
        "metric": "C4v Ising CTMRG iter/s (chi=32)", "value": world * args.steps / t,
        "unit": "iter/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (the reference example's seeded start)", "impl": "ours",
        "config": {"workload": "ising_c4v", "beta": ISING_BETA, "chi": ISING_CHI,
                   "iterations_total": max(done, ISING_ITERS),
                   "energy_per_bond": e, "correlation_length": xi,
                   "l2": "blocks of at most 16 x 32: launch-bound, L2-resident",
                   "parallelism": f"replicas x{world}"},
        "gpu_launches": launches, "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_ising_sample(max(args.steps, 20))
    return line


def cpu_simple_update_sample(symmetry, D, warmup, *, budget_s=15.0):
    """Bounded CPU sample of the simple-update workload: the numpy oracle
    (restating the reference) on the same model, from the same infinite-
    temperature start; the first cycle and `warmup` more untimed, then cycles
    (evolve(4 tau) each, as on the device) timed until `budget_s` has passed
    (at least three), with BLAS on every host core, then two cycles on one
    BLAS thread."""
    from threadpoolctl import threadpool_limits

    from oracle import frostspin_oracle as fo
    from oracle import simple_update_oracle as suo
    from oracle import su2_oracle as so

    cores = os.cpu_count() or 1
    if symmetry == "su2":
        r = np.array([[1], [2]])
        h = so.from_array(SDS_22.reshape(2, 2, 2, 2), (r, r), (r, r))
    else:
        rep = np.array([1, -1], dtype=np.int8)
        h = fo.from_array(SDS_22.reshape(2, 2, 2, 2), (rep, rep), (rep, rep))
    cycle = 4 * 0.01
    with threadpool_limits(limits=cores):
        su = suo.SimpleUpdate(h, D, 0.01, rcutoff=1e-10, degen_ratio=0.9999)
        for _ in range(1 + warmup):
            su.evolve(cycle)
        n, t0 = 0, time.perf_counter()
        while n < 3 or time.perf_counter() - t0 < budget_s:
            su.evolve(cycle)
            n += 1
        t = time.perf_counter() - t0
    with threadpool_limits(limits=1):
        t1 = time.perf_counter()
        for _ in range(2):
            su.evolve(cycle)
        one = (time.perf_counter() - t1) / 2
    return {"value": n / t, "unit": "cycle/s", "cores": cores, "kind": "port",
            "sample": (f"numpy oracle simple update ({symmetry}, D={D} target, tau=0.01) from "
                       f"beta=0: {1 + warmup} untimed cycles, then {n} timed cycles in "
                       f"{t:.1f} s with BLAS on {cores} host cores (beta "
                       f"{(1 + warmup) * cycle:.2f} to {(1 + warmup + n) * cycle:.2f})"),
            "one_thread": {"s_per_cycle": one, "threads": 1}}


def run_simple_update(args, world, rank, local):
    """Config 3: the SU(2) finite-temperature simple update of the spin-1/2
    Heisenberg model (2-site checkerboard cell, second-order Trotter, tau =
    0.01, bond dimension target D = 24: whole multiplets) on the device.  One
    step = one second-order Trotter cycle (beta += 4 tau).  The first cycle
    (structural precompute: CG trees and recoupling tables) is reported
    separately; W further untimed cycles, K timed, then untimed cycles up to
    beta = 4, where Dmax and logZ are reported."""
    import torch

    from frostspin_b200.simple_update import SimpleUpdate

    h = heisenberg_su2() if args.symmetry == "su2" else heisenberg_u1()
    su = SimpleUpdate.square_lattice_first_neighbor(h, args.D, 0.01, rcutoff=1e-10,
                                                    degen_ratio=0.9999)
    cycle = 4 * 0.01
    t0 = time.perf_counter()
    su.evolve(cycle)
    torch.cuda.synchronize()
    t_first = time.perf_counter() - t0
    for _ in range(args.warmup):
        su.evolve(cycle)
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    ev0.record()
    for _ in range(args.steps):
        su.evolve(cycle)
    ev1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    clk = clocks.stop()
    t = max_over_ranks(ev0.elapsed_time(ev1) * 1e-3, world)
    while su.beta < 4.0 - 1e-9:
        su.evolve(cycle)
    return {
        "metric": "SU(2) simple update Trotter cycles/s (D=24 target)",
        "value": world * args.steps / t, "unit": "cycle/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (infinite-temperature start)", "impl": "ours",
        "config": {"workload": "simple_update_" + args.symmetry, "D_target": args.D,
                   "tau": 0.01, "beta_final": su.beta, "Dmax": su.Dmax, "logZ": su.logZ,
                   "first_cycle_s": t_first, "wall_s_timed": wall,
                   "l2": "bond tensors of a few MB: L2-resident, launch-bound",
                   "parallelism": f"replicas x{world}"},
        "clocks": clk,
        **({"cpu_baseline": cpu_simple_update_sample(args.symmetry, args.D, args.warmup)}
           if rank == 0 and world == 1 and not args.no_cpu_baseline else {}),
    }


def run_deviation(args, world, rank, local):
    """Accuracy of the mixed path over a long run: from the same warmed-up
    chi = 256 environment, plain FP64 and the mixed precision iterate side by
    side; after each iteration count in --deviation the energies per bond are
    compared and the truncation decisions (chi after every move) checked for
    equality; at the end the horizontal correlation lengths are compared."""
    import torch

    from frostspin_b200 import autotune, linalg

    mixed = args.precision if args.precision != "fp64" else "ozaki2_11"
    points = sorted(int(x) for x in args.deviation.split(","))
    su, tensors, ctm, _ = ctmrg_setup(args)
    linalg.set_gemm_precision("fp64")
    records = []
    for _ in range(args.warmup):
        if args.autotune == "on":
            with linalg.record_gemm_calls() as rec:
                ctm.iterate()
            records += rec
        else:
            ctm.iterate()
    if args.autotune == "on":
        autotune.tune(records, mixed)
        autotune.set_enabled(True)
    mix = ctm.copy()
    rows = []
    same_chi = True
    t0 = time.perf_counter()
    for it in range(1, points[-1] + 1):
        linalg.set_gemm_precision("fp64")
        ctm.iterate()
        linalg.set_gemm_precision(mixed)
        mix.iterate()
        same_chi = same_chi and list(ctm.chi_values) == list(mix.chi_values)
        if it in points:
            linalg.set_gemm_precision("fp64")
            e64 = energy_per_bond(ctm)
            linalg.set_gemm_precision(mixed)
            emx = energy_per_bond(mix)
            rows.append({"iterations": it, "energy_fp64": e64, "energy_mixed": emx,
                         "rel_err": abs(emx - e64) / abs(e64),
                         "chi_decisions_identical": same_chi,
                         "elapsed_s": time.perf_counter() - t0})
            print(json.dumps(rows[-1]), file=sys.stderr, flush=True)
    linalg.check_ozaki_flags()
    xi = None
    if args.deviation_xi == "on":
        linalg.set_gemm_precision("fp64")
        x64 = ctm.compute_corr_length_h(0)
        linalg.set_gemm_precision(mixed)
        xmx = mix.compute_corr_length_h(0)
        xi = {"xi_fp64": x64, "xi_mixed": xmx, "rel_err": abs(xmx - x64) / abs(x64)}
    torch.cuda.synchronize()
    return {"metric": "relative energy deviation, mixed vs plain FP64 CTMRG",
            "value": rows[-1]["rel_err"], "unit": "relative", "n_gpus": world,
            "steps": points[-1], "warmup": args.warmup, "higher_is_better": False,
            "impl": "ours", "dtype": f"f64 via int8 {mixed}",
            "config": {"workload": f"ctmrg_heisenberg_{args.symmetry}", "chi": args.chi,
                       "D_target": args.D, "beta": args.beta, "precision": mixed,
                       "points": rows, "correlation_length_h0": xi,
                       "chi_values_fp64": [int(c) for c in ctm.chi_values],
                       "chi_values_mixed": [int(c) for c in mix.chi_values]}}


BATCH_RUNS = 64
BATCH_CHIS = (16, 32, 64, 96)


def batched_specs(seed=SEED):
    """The 64 Z2 Ising runs of the batched workload: beta uniform in
    [0.30, 0.60] and chi drawn from {16, 32, 64, 96} with a fixed seed."""
    rng = np.random.default_rng(seed)
    betas = rng.uniform(0.30, 0.60, BATCH_RUNS)
    chis = rng.choice(BATCH_CHIS, BATCH_RUNS)
    return [(float(b), int(c)) for b, c in zip(betas, chis, strict=True)]


def run_batched(args, world, rank, local):
    """Config 5 (its Z2 half): 64 independent C4v Ising CTMRG runs of uneven
    chi advanced in lock step by iterate_c4v_many, each step one grouped GEMM
    launch and one multi-buffer permute launch for all runs.  One step = one
    iteration of every run; value = run-iterations per second."""
    import torch

    from frostspin_b200 import _native
    from frostspin_b200.ctmrg import (energy_per_bond, ising_initial_environment,
                                      ising_site_tensors, iterate_c4v_many)

    specs = batched_specs()
    runs = []
    for i, (beta, chi) in enumerate(specs):
        a, a2, a0d, mopd = ising_site_tensors(beta)
        s, T = ising_initial_environment(chi, np.random.default_rng(42 + i))
        runs.append([s, T, a, a2, chi, a0d, mopd])

    def step():
        res = iterate_c4v_many([r[:5] for r in runs])
        for r, (s, T) in zip(runs, res, strict=True):
            r[0], r[1] = s, T

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    n0 = _native.kernel_launches()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        step()
    ev1.record()
    torch.cuda.synchronize()
    launches = _native.kernel_launches() - n0
    clk = clocks.stop()
    t = max_over_ranks(ev0.elapsed_time(ev1) * 1e-3, world)
    energies = [energy_per_bond(r[0], r[1], r[5], r[6]) for r in runs[:4]]
    line = {
        "metric": "batched C4v CTMRG run-iterations/s (64 Z2 Ising runs, uneven chi)",
        "value": world * BATCH_RUNS * args.steps / t, "unit": "run-iter/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded betas, chis and starting environments)", "impl": "ours",
        "config": {"workload": "batched_ising_c4v", "runs": BATCH_RUNS,
                   "beta_range": [0.30, 0.60], "chis": list(BATCH_CHIS),
                   "chi_counts": {str(c): sum(1 for _, x in specs if x == c) for c in BATCH_CHIS},
                   "energies_first_runs": energies,
                   "u1_runs": "not built: the reference gives no U(1) classical C4v model",
                   "parallelism": f"replicas x{world}"},
        "gpu_launches": launches, "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_batched_sample()
    return line


def cpu_batched_sample():
    """The oracle's C4v iteration of every run of the batched workload in a
    sequential loop, one BLAS thread: one untimed and one timed pass."""
    from threadpoolctl import threadpool_limits

    from oracle import frostspin_oracle as fo

    specs = batched_specs()
    runs = []
    for i, (beta, chi) in enumerate(specs):
        a, a2, _, _ = fo.ising_tensors(beta)
        sb, si, T = fo.ising_initial_env(chi, np.random.default_rng(42 + i))
        runs.append([sb, si, T, a, a2, chi])
    with threadpool_limits(limits=1):
        times = []
        for _ in range(2):
            t0 = time.perf_counter()
            for r in runs:
                r[0], r[1], r[2] = fo.ising_c4v_iteration(r[0], r[1], r[2], r[3], r[4], r[5])
            times.append(time.perf_counter() - t0)
    t = times[-1]
    return {"value": BATCH_RUNS / t, "unit": "run-iter/s", "cores": 1, "kind": "port",
            "sample": f"numpy oracle C4v iteration of all {BATCH_RUNS} runs in a loop, one "
                      f"pass after one warm-up pass: {t:.2f} s per pass"}


def cpu_ising_sample(n):
    """The oracle's C4v iteration (numpy restatement of the reference example)
    from the same seeded start, one BLAS thread: mean time of n iterations
    after 3."""
    from threadpoolctl import threadpool_limits

    from oracle import frostspin_oracle as fo

    a, a2, _, _ = fo.ising_tensors(ISING_BETA)
    sb, si, T = fo.ising_initial_env(ISING_CHI, np.random.default_rng(42))
    with threadpool_limits(limits=1):
        for _ in range(3):
            sb, si, T = fo.ising_c4v_iteration(sb, si, T, a, a2, ISING_CHI)
        t0 = time.perf_counter()
        for _ in range(n):
            sb, si, T = fo.ising_c4v_iteration(sb, si, T, a, a2, ISING_CHI)
        t = (time.perf_counter() - t0) / n
    return {"value": 1.0 / t, "unit": "iter/s", "cores": 1, "kind": "port",
            "sample": f"numpy oracle C4v iteration, chi={ISING_CHI}, mean of {n} after 3: "
                      f"{t * 1e3:.2f} ms/iteration"}


def run_reference(args, world, rank):
    if rank != 0:
        return None
    if args.workload == "ctmrg":
        return run_reference_ctmrg(args, world)
    if args.workload == "batched":
        info = cpu_batched_sample()
        v = info["value"]
        return {"metric": "batched C4v CTMRG run-iterations/s (64 Z2 Ising runs, uneven chi)",
                "value": v, "unit": "run-iter/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * BATCH_RUNS / v,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": "batched_ising_c4v", "runs": BATCH_RUNS},
                "cpu_baseline": info,
                "e2e": {"value": v, "unit": "run-iter/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
    if args.workload == "simple_update":
        info = cpu_simple_update_sample(args.symmetry, args.D, args.warmup)
        v = info["value"]
        return {"metric": "SU(2) simple update Trotter cycles/s (D=24 target)", "value": v,
                "unit": "cycle/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (infinite-temperature start)", "impl": "reference",
                "config": {"workload": "simple_update_" + args.symmetry, "D_target": args.D,
                           "tau": 0.01},
                "cpu_baseline": info,
                "e2e": {"value": v, "unit": "cycle/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
    if args.workload == "ising":
        info = cpu_ising_sample(max(args.steps, 20))
        v = info["value"]
        return {"metric": "C4v Ising CTMRG iter/s (chi=32)", "value": v, "unit": "iter/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "impl": "reference", "config": {"workload": "ising_c4v", "beta": ISING_BETA,
                                                "chi": ISING_CHI},
                "cpu_baseline": info,
                "e2e": {"value": v, "unit": "iter/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
    if args.workload == "gemm":
        rng = np.random.default_rng(SEED)
        n = args.gemm_n
        A = rng.standard_normal((n, n))
        B = rng.standard_normal((n, n))
        times = []
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            A @ B
            if i >= args.warmup:
                times.append(time.perf_counter() - t0)
        value = 2.0 * n**3 / float(np.mean(times)) / 1e12
        info = {"value": value, "unit": "TFLOP/s", "cores": os.cpu_count() or 1,
                "kind": "port", "sample": f"numpy (OpenBLAS) dgemm {n}^3, all host threads"}
        return {"metric": "square GEMM, effective FP64 TFLOP/s", "value": value,
                "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic (seeded N(0,1))", "impl": "reference",
                "config": {"workload": "gemm", "n": n}, "cpu_baseline": info,
                "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
    wl_states = LEG_STATES
    from frostspin_b200.symmetric_tensor.abelian_plan import GroupInfo  # noqa: F401

    rep = microbench_rep(wl_states)
    from oracle import frostspin_oracle as fo

    sig1 = np.array([False, False, True, True])
    irr, shapes = fo.get_block_sizes((rep, rep), (rep, rep), sig1)
    ncoeff = int((shapes[:, 0] * shapes[:, 1]).sum())
    # flops of the full step from block shapes (permuted blocks are square)
    sigp = np.array([False, True, False, True])
    irrp, shp = fo.get_block_sizes((rep, rep), (rep, rep), sigp)
    flops = float((2 * shp[:, 0] * shp[:, 1] * shp[:, 1]).sum())
    times = []
    info = None
    for i in range(args.warmup + args.steps):
        t, info = cpu_baseline_full_step(ncoeff, flops)
        if i >= args.warmup:
            times.append(t)
    value = 1.0 / float(np.mean(times))
    info["value"] = value
    info["unit"] = "step/s"
    return {
        "metric": "U(1) microbench permute+grouped-matmul steps/s",
        "value": value,
        "unit": "step/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 / value,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded N(0,1) blocks)",
        "impl": "reference",
        "config": {"workload": "u1_microbench", "ncoeff": ncoeff,
                   "gemm_flop_per_step": flops},
        "cpu_baseline": info,
        "e2e": {"value": value, "unit": "step/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["ctmrg", "u1_microbench", "gemm", "ising",
                                           "simple_update", "batched"],
                    default="ctmrg")
    ap.add_argument("--gemm-n", type=int, default=4096, help="matrix size of the gemm workload")
    ap.add_argument("--gemm-shape", default=None, help="M,N,K of the gemm workload (else n,n,n)")
    ap.add_argument("--symmetry", choices=["u1", "su2"], default="su2")
    ap.add_argument("--D", type=int, default=None,
                    help="simple-update bond dimension target (default 12 for U(1), 24 for SU(2))")
    ap.add_argument("--chi", type=int, default=None,
                    help="CTMRG corner dimension target (default 64 for U(1), 256 for SU(2))")
    ap.add_argument("--beta", type=float, default=2.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fused-permute", choices=["on", "off"], default="on",
                    help="thin SU(2) simple blocks in the one-pass fused permute kernel")
    ap.add_argument("--deviation", default="",
                    help="iteration counts (e.g. 10,25,50) at which a side-by-side FP64 and "
                         "mixed CTMRG run compares energies (accuracy study, not a bench line)")
    ap.add_argument("--deviation-xi", choices=["on", "off"], default="on")
    ap.add_argument("--autotune", choices=["on", "off"], default="on",
                    help="measure the sector-GEMM shape classes of a warm-up iteration on "
                         "both paths and dispatch by the measurement")
    ap.add_argument("--compare-chis", default="64,128",
                    help="smaller chi values also timed on the GPU (one iteration each)")
    ap.add_argument("--cpu-chis", default="32,64",
                    help="chi values the CPU reference arm of the ctmrg workload measures")
    ap.add_argument("--ozaki-pair", choices=["on", "off"], default="on",
                    help="large int8 sector GEMMs on CTA pairs (tcgen05 cta_group::2)")
    ap.add_argument("--precision", default="ozaki2_11",
                    help="sector GEMM arithmetic: fp64, ozakiS (S = 3..8 int8 digit slices) "
                         "or ozaki2_N (N = 8..14 int8 moduli, CRT)")
    ap.add_argument("--leg-states", type=int, default=LEG_STATES,
                    help="states per leg (256 = the benchmark; smaller for profiling)")
    args = ap.parse_args()
    if args.D is None:
        args.D = 24 if args.symmetry == "su2" else 12
    if args.chi is None:
        args.chi = 256 if args.symmetry == "su2" else 64
    args.warmup_requested = args.warmup
    if args.warmup < 3:
        # the timing rules need at least 3 untimed steps; the line reports both
        args.warmup = 3
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        line = run_reference(args, world, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    world, rank, local = dist_init(args.gpus)
    from frostspin_b200 import linalg

    linalg.set_ozaki_pair(args.ozaki_pair == "on")
    from frostspin_b200.symmetric_tensor import lie_group_symmetric_tensor

    lie_group_symmetric_tensor.set_fused_permute(args.fused_permute == "on")
    if args.workload == "ctmrg" and args.deviation:
        line = run_deviation(args, world, rank, local)
    elif args.workload == "ctmrg":
        line = run_ctmrg(args, world, rank, local)
    elif args.workload == "gemm":
        line = run_gemm(args, world, rank, local)
    elif args.workload == "ising":
        line = run_ising(args, world, rank, local)
    elif args.workload == "simple_update":
        line = run_simple_update(args, world, rank, local)
    elif args.workload == "batched":
        line = run_batched(args, world, rank, local)
    else:
        line = run_ours(args, world, rank, local)
    if rank == 0:
        if args.warmup_requested != args.warmup:
            line["warmup_requested"] = args.warmup_requested
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
