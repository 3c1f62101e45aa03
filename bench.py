"""Benchmark: Fock-build seconds per SCF iteration on one B200 (mixed tensor-core form vs FP64).

One step = one direct-form RCS Fock build (Coulomb + exchange r12 contractions, Fock assembly and
energy) for the workload's density on its radial x Lebedev grid.  `value` is device time per step
with every input resident in HBM; `e2e` is the same through the public C ABI from host buffers
(grid upload, device basis evaluation, Fock build, G/Fock/energy back to the host).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload kr|ne|he|batch|scf]
                  [--precision bf16x3|fp64|tf32]

Under torchrun (N > 1) every rank runs an independent replica (the Fock build does not shard in
this design); rank 0 prints the whole-job line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def load_peaks() -> tuple[dict, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def scf_guess_density(basis, Z: int, nocc: int):
    """Core-Hamiltonian guess (the reference's first iteration: zero density -> F = h), solved in the
    real-harmonic basis with canonical orthogonalisation (the even-tempered overlap is
    ill-conditioned), so the closed-shell density is real there; returned in the reference basis."""
    from tcscf_b200 import api
    from tcscf_b200.basis import real_harmonic_unitary

    S, h = api.overlap_core(basis, Z)
    U = real_harmonic_unitary(basis)
    SR = np.real(U.conj() @ S @ U.T)
    hR = np.real(U.conj() @ h @ U.T)
    s, V = np.linalg.eigh(SR)
    keep = s > 1e-10 * s.max()
    X = V[:, keep] / np.sqrt(s[keep])
    e, Cp = np.linalg.eigh(X.T @ hR @ X)
    CR = X @ Cp[:, :nocc]
    DR = CR @ CR.T
    D = U.T @ DR @ U.conj()
    return np.ascontiguousarray(D.astype(np.complex128)), h


def workload(name: str):
    from tcscf_b200 import basis as wl

    return {"kr": wl.kr, "ne": wl.ne, "he": wl.he}[name]()


def cpu_reference(w, grid, D, h, budget_s: float, threads: int | None = None) -> dict:
    """The reference algorithm (precomputeIntegrand + computeF once, then calculateIaa / calculateFai /
    assembly per iteration) timed on the host cores through the oracle port on a sample of r1 rows
    with the full r2 grid, extrapolated linearly to all rows (rows are independent and of equal cost)."""
    import oracle

    if threads:
        oracle.set_threads(threads)
    cores = oracle.threads()
    vals2 = oracle.basis_values(grid.points, w.basis)
    rng = np.random.default_rng(0)
    # calibrate with one row per thread, then size the sample to the budget
    rows = cores
    t_row = None
    sample_rows = rows
    for _ in range(2):
        idx = np.sort(rng.choice(grid.n, sample_rows, replace=False))
        p1 = np.ascontiguousarray(grid.points[:, idx])
        t0 = time.perf_counter()
        F = oracle.compute_F(p1, grid.points, grid.weights, vals2, w.nb)
        t_pre = time.perf_counter() - t0
        vals1 = np.ascontiguousarray(vals2[idx])
        t0 = time.perf_counter()
        oracle.fock_build(F, vals1, np.ascontiguousarray(grid.weights[idx]), D, h)
        t_it = time.perf_counter() - t0
        t_row = (t_pre + t_it) / sample_rows
        want = int(max(cores, min(grid.n, budget_s / max(t_row, 1e-9))))
        want = (want // cores) * cores or cores
        if want <= sample_rows * 1.2:
            break
        sample_rows = want
    scale = grid.n / sample_rows
    # per SCF iteration the reference rebuilds the Fock matrix from its precomputed F; computeF runs
    # once per SCF and is reported beside it
    return {"s_per_iter": t_it * scale, "precompute_s": t_pre * scale, "iteration_s": t_it * scale,
            "cores": cores, "rows": sample_rows, "sample": f"{sample_rows} of {grid.n} r1 rows x all {grid.n} r2 points: "
            "per-iteration Fock build (calculateIaa/calculateFai/assembly) from the precomputed F, extrapolated linearly "
            "to all rows; the one-off computeF precompute is reported as precompute_s"}


def run_reference(args, rank: int) -> None:
    from tcscf_b200 import grids

    if rank != 0:
        return
    w = workload(args.workload)
    if args.nrad:
        w.nrad = args.nrad
    g = grids.product_grid(w.nrad, w.order)
    D, h = scf_guess_density(w.basis, w.Z, w.n_up)
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_reference(w, g, D, h, budget_s=args.ref_seconds)
        if i >= args.warmup:
            vals.append(r["s_per_iter"])
    v = statistics.median(vals)
    dropped, near = grids.coincident_pairs(g, g)   # r1 = r2 grid: the diagonal pairs contribute 0
    line = {"metric": METRIC, "value": v, "unit": "s/iter", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": f"{w.name} RCS Fock build", "n_points": g.n, "n_basis": w.nb, "n_occ": w.n_up,
                       "dropped_pairs": dropped, "near_coincident_pairs": near},
            "cpu_baseline": {"value": v, "unit": "s/iter", "cores": r["cores"], "kind": "port", "sample": r["sample"],
                             "precompute_s": r["precompute_s"]},
            "e2e": {"value": v, "unit": "s/iter", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def roofline(prec: int, n: int, nb: int, nocc: int, c_ms: float, peaks: dict, peak_kind: str, fp64_peak: float, traffic) -> dict:
    """The line's roofline object for one Fock build of n points (r1 = r2 grid) whose contraction
    kernel took c_ms milliseconds."""
    from tcscf_b200 import ffi

    # algorithmic work per Fock build: F_alg = 2 N^2 (nb nocc + 1), the pair-density count of the direct
    # build (nb nocc exchange pair densities and the Coulomb density per (r1, r2) pair); this kernel
    # contracts the same sum in factored form, 2 N^2 (nocc + nb + 1) flops (rho GEMM, exchange GEMM,
    # Coulomb), reported beside it as kernel_algorithm_tflops
    flops = 2.0 * n * n * (nb * nocc + 1)
    kernel_flops = 2.0 * n * n * (nocc + nb + 1)
    achieved = flops / (c_ms / 1e3) / 1e12
    kernel_achieved = kernel_flops / (c_ms / 1e3) / 1e12
    numerator = {"achieved_numerator": "F_alg = 2 N^2 (nb nocc + 1) flops per build (pair-density count)",
                 "kernel_algorithm_tflops": kernel_achieved}
    if prec == ffi.PREC_FP64:
        roof = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                "traffic": None, "peak_source": "nominal B200 FP64 dense rate (--fp64-peak or TCSCF_FP64_PEAK_TFLOPS overrides)",
                **numerator}
    elif prec == ffi.PREC_TF32:
        # TF32 dense rate is half the BF16 rate (nominal 1.1 vs 2.25 PFLOP/s): half the measured BF16 burst
        peak = peaks["bf16_tflops"] / 2
        RP = 32                            # TF32 launches hold rank 32 (larger ranks run in chunks)
        NB = 64 if nb <= 64 else 128
        chunks = -(-nocc // RP)
        issued = n * n * chunks * (2.0 * RP + 2.0 * NB) / (c_ms / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": None, "peak_source": f"tf32 dense = half the bf16 dense burst, {peak_kind}",
                "issued_tensor_tflops": issued, "issued_frac": issued / peak, **numerator}
    else:
        peak = peaks["bf16_tflops"]
        # tensor work the kernel issues per (r1, r2) pair: GEMM1 6 slice products of K = RP; GEMM2 6 of
        # N = NB with 24-bit X (rank padding 32), 4 with 16-bit X (rank padding 64)
        RP = 32 if nocc <= 32 else 64   # real closed-shell guess density: factor rank = n_occ
        NB = 64 if nb <= 64 else 128
        issued = n * n * (2.0 * 6 * RP + 2.0 * (6 if RP == 32 else 4) * NB) / (c_ms / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": f"bf16 dense burst, {peak_kind}",
                "issued_tensor_tflops": issued, "issued_frac": issued / peak, **numerator}
    return roof


METRIC = "Fock-build s/iter, mixed vs FP64 GPU at |dE|<=1 uEh; % of roofline"


def profiled_traffic(name: str):
    """DRAM bytes per launch of the tensor contraction kernel for this workload, as recorded in the
    committed ncu summary (profiles/kflashtc_dram_traffic.md: 'traffic_bytes_per_launch <name> <bytes>')."""
    path = Path(__file__).resolve().parent / "profiles" / "kflashtc_dram_traffic.md"
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        parts = line.strip("` ").split()
        if len(parts) == 3 and parts[0] == "traffic_bytes_per_launch" and parts[1].lower() == name.lower():
            return float(parts[2])
    return None


def run_ours(args, rank: int, world: int) -> None:
    import torch

    from tcscf_b200 import api, ffi, grids, replicas

    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    prec = {"fp64": ffi.PREC_FP64, "bf16x3": ffi.PREC_BF16X3, "tf32": ffi.PREC_TF32}[args.precision]
    w = workload(args.workload)
    if args.nrad:
        w.nrad = args.nrad
    g = grids.product_grid(w.nrad, w.order)
    D, h = scf_guess_density(w.basis, w.Z, w.n_up)
    peaks, peak_kind = load_peaks()

    ctx = api.Context(local)
    if args.autotune:
        ctx.set_autotune(True)
    G = api.QMCGrid(ctx, g)
    G.setBasisFunctions(w.basis)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    dD = torch.from_numpy(D[None].view(np.float64).copy()).to(dev)
    dH = torch.from_numpy(h).to(dev)
    dE = torch.zeros(1, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def step(precision: int) -> None:
        ffi.check(ffi.lib().tcscf_fock_build_device(ctx.handle, G.id, G.id, 1, dD.data_ptr(), dH.data_ptr(), 1, precision,
                                                    None, None, dE.data_ptr()), ctx.handle)

    def timed(precision: int, steps: int, warmup: int):
        for _ in range(warmup):
            step(precision)
        torch.cuda.synchronize()
        ms, contraction, launches = [], [], 0
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            replicas.barrier(world)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step(precision)
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
            c, _, n = ctx.last_timing()
            contraction.append(c)
            launches += n
        return ms, contraction, launches, float(dE.item())

    with ClockSampler(local) as clk:
        ms, cms, launches, E = timed(prec, args.steps, args.warmup)
    total_ms = replicas.max_over_ranks(sum(ms), world, dev)
    s_per_iter = replicas.whole_job_seconds_per_build(total_ms, args.steps, world)

    # FP64 comparison (the plain FP64 GPU form) at the same density
    fp64 = None
    if prec != ffi.PREC_FP64 and not args.skip_fp64:
        fsteps = max(1, min(args.steps, args.fp64_steps))
        fms, fcms, _, E64 = timed(ffi.PREC_FP64, fsteps, 1)
        fp64 = {"s_per_iter": statistics.median(fms) / 1e3, "energy": E64, "dE_mixed_vs_fp64": E - E64,
                "contraction_ms": statistics.median(fcms)}

    # end-to-end through the public C ABI from pinned host buffers
    e2e = None
    if not args.skip_e2e:
        pts = torch.from_numpy(g.points).pin_memory().numpy()
        wts = torch.from_numpy(g.weights).pin_memory().numpy()
        Dh = torch.from_numpy(D[None].view(np.float64).copy()).pin_memory().numpy().view(np.complex128)
        e_times = []
        for i in range(max(1, args.e2e_steps) + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            Gg = api.QMCGrid(ctx, grids.QuadratureGrid(pts, wts))
            Gg.setBasisFunctions(w.basis)
            Gm, Fm, Em = api.fock_build(Gg, Gg, Dh, h, precision=prec)
            Gg.close()
            torch.cuda.synchronize()
            if i > 0:
                e_times.append(time.perf_counter() - t0)
        nb = w.nb
        # whole job, like `value`: the slowest rank's time per build over the builds of all ranks
        e2e = {"value": replicas.max_over_ranks(statistics.median(e_times), world, dev) / world, "unit": "s/iter",
               "h2d_bytes_per_step": int(pts.nbytes + wts.nbytes + Dh.nbytes + h.nbytes),
               "d2h_bytes_per_step": int(2 * 16 * nb * nb + 8)}

    if rank != 0:
        return
    n = g.n
    dropped, near = grids.coincident_pairs(g, g)   # r1 = r2 grid: the diagonal pairs contribute 0
    c_ms = statistics.median(cms)
    roof = roofline(prec, n, w.nb, w.n_up, c_ms, peaks, peak_kind, args.fp64_peak, profiled_traffic(w.name))
    cpu = None
    if not args.skip_cpu:
        r = cpu_reference(w, g, D, h, budget_s=args.cpu_seconds)
        cpu = {"value": r["s_per_iter"], "unit": "s/iter", "cores": r["cores"], "kind": "port", "sample": r["sample"],
               "precompute_s": r["precompute_s"], "iteration_s": r["iteration_s"]}
    line = {"metric": METRIC, "value": s_per_iter, "unit": "s/iter", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp64": "f64", "bf16x3": "bf16", "tf32": "tf32"}[args.precision],
            "data": "synthetic",
            "config": {"workload": f"{w.name} RCS Fock build (direct form)", "Z": w.Z, "n_points": n, "n_basis": w.nb,
                       "n_occ": w.n_up, "grid": f"{w.nrad} radial (Gauss-Chebyshev, r=(1+x)/(1-x)) x Lebedev order {w.order}",
                       "precision": {"fp64": "fp64",
                                     "bf16x3": "bf16 fixed-point slices (24-bit factors and kernel tile), exact fp32 "
                                               "accumulation of the leading slices per 64-point block, double-float across blocks",
                                     "tf32": "tf32 operands (10-bit mantissa, round to nearest), fp32 accumulation per 64-point "
                                             "block, double-float across blocks"}[args.precision],
                       "l2": "flushed (256 MB write) between timed steps",
                       "density": "core-Hamiltonian guess (canonical orthogonalisation)",
                       "dropped_pairs": dropped, "near_coincident_pairs": near,
                       "schedule": "autotuned r2 split (tuned in the warm-up: shapes, batches, measurements = %s)" % (ctx.autotune_stats(),)
                       if args.autotune else "fixed rule"},
            "energy": E, "contraction_ms": c_ms, "gpu_launches": launches, "roofline": roof, "fp64": fp64,
            "speedup_vs_fp64": (fp64["s_per_iter"] / (total_ms / args.steps / 1e3)) if fp64 else None,
            "e2e": e2e, "cpu_baseline": cpu, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_batch(args, rank: int) -> None:
    """The 64-instance batched configuration: closed-shell atoms/ions with Z ~ U{2..36}, 10-80 even-tempered
    STOs, 40-200 radial x Lebedev 110-1202 points (seeded).  Times the batched mixed-precision build (one
    persistent tensor-core launch per tile class), the same builds one at a time, and reports every
    instance's energy error against its FP64 build."""
    import torch

    from tcscf_b200 import api, ffi, grids
    from tcscf_b200 import basis as wl

    if rank != 0:
        return
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    ctx = api.Context(int(os.environ.get("LOCAL_RANK", 0)))
    if args.autotune:
        ctx.set_autotune(True)
    inst = wl.batch()
    Gs, Ds, hs, npts = [], [], [], []
    for w in inst:
        g = grids.product_grid(w.nrad, w.order)
        G = api.QMCGrid(ctx, g)
        G.setBasisFunctions(w.basis)
        D, h = scf_guess_density(w.basis, w.Z, w.n_up)
        Gs.append(G); Ds.append(D); hs.append(h); npts.append(g.n)
    prec = ffi.PREC_BF16X3

    def batched():
        return api.fock_build_batch(Gs, Gs, Ds, hs, precision=prec)

    def one_by_one():
        return np.array([api.fock_build(G, G, D, h, precision=prec)[2] for G, D, h in zip(Gs, Ds, hs)])

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts), out

    with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
        tb, Eb = timed(batched, args.steps, args.warmup)
    t1, E1 = timed(one_by_one, max(1, min(args.steps, 2)), 1)
    E64 = np.array([api.fock_build(G, G, D, h, precision=ffi.PREC_FP64)[2] for G, D, h in zip(Gs, Ds, hs)])
    err = np.abs(Eb - E64)
    line = {"metric": "batched RCS Fock builds (64 atoms/ions) per second", "value": len(inst) / tb, "unit": "instances/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": tb * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
            "config": {"workload": "64 closed-shell atoms/ions, Z ~ U{2..36}, 10-80 even-tempered STOs, 40-200 radial x "
                                   "Lebedev 110-1202 points (seed 20261203), core-Hamiltonian guess densities",
                       "points_total": int(sum(npts)), "points_max": int(max(npts)), "timing": "host wall clock around the "
                       "public batched call, inputs resident on the device except the densities"},
            "one_at_a_time_s": t1, "batch_speedup": t1 / tb, "batched_equals_one_at_a_time": bool(np.array_equal(Eb, E1)),
            "dE_vs_fp64_max": float(err.max()), "dE_vs_fp64_median": float(np.median(err)),
            "dE_rel_vs_fp64_max": float((err / np.abs(E64)).max()), "clocks": clk.summary(),
            "schedule": {"autotune": bool(args.autotune), "tuned_shapes_batches_measurements": ctx.autotune_stats()}}
    print(json.dumps(line), flush=True)


def run_scf(args, rank: int) -> None:
    """Full RCS SCF of the Kr configuration to |dE| < 1e-8 Eh: split-BF16 and FP64 Fock builds in the plain
    Roothaan iteration of the reference (at most --scf-max-iter iterations), split BF16 with Pulay DIIS
    (history --diis), and the FP64 SCF converged to 1e-10 Eh as the energy reference; all with the
    real-harmonic eigen-solve (real densities throughout, one contraction per build).  Each SCF starts
    from the zero density (core-Hamiltonian first step, as the reference); wall time around the public
    call."""
    import torch

    from tcscf_b200 import api, ffi, grids

    if rank != 0:
        return
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    w = workload("kr")
    if args.nrad:
        w.nrad = args.nrad
    g = grids.product_grid(w.nrad, w.order)
    ctx = api.Context(int(os.environ.get("LOCAL_RANK", 0)))
    G = api.QMCGrid(ctx, g)
    G.setBasisFunctions(w.basis)
    S, h = api.overlap_core(w.basis, w.Z)
    # the 1e-8 runs time the configuration; the mixed-precision energy is compared with the FP64 SCF
    # converged to 1e-10 (the split-BF16 energy settles to its own precision, ~1e-9 Eh per build, so it
    # is not itself run to 1e-10)
    runs = [("bf16x3_plain", ffi.PREC_BF16X3, 0, 1e-8), ("bf16x3_diis", ffi.PREC_BF16X3, args.diis, 1e-8),
            ("fp64_plain", ffi.PREC_FP64, 0, 1e-8), ("fp64_plain_1e-10", ffi.PREC_FP64, 0, 1e-10)]
    res = {}
    with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
        for name, prec, nd, tol in runs:
            hf = api.RCSHartreeFock(w.n_up, w.n_down, w.nb)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            try:
                E, ok = hf.compute(S, h, G, G, precision=prec, tol=tol, max_iter=args.scf_max_iter, diis=nd,
                                   real_eigensolve=True), True
            except ffi.TcscfError as e:
                if e.code != ffi.ERR_NOT_CONVERGED:
                    raise
                E, ok = None, False
            torch.cuda.synchronize()
            res[name] = {"converged": ok, "energy": E, "iterations": hf.numberOfConvergenceLoops(),
                         "seconds": time.perf_counter() - t0, "diis": nd, "tol": tol}
    m, f, ft = res["bf16x3_plain"], res["fp64_plain"], res["fp64_plain_1e-10"]
    line = {"metric": "Kr RCS SCF to |dE| < 1e-8 Eh, wall s (split-BF16 Fock builds)", "value": m["seconds"], "unit": "s",
            "n_gpus": 1, "steps": 1, "warmup": 0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16", "data": "synthetic",
            "config": {"workload": f"Kr RCS SCF (direct-form Fock builds), {w.nrad} radial x Lebedev order {w.order}",
                       "n_points": g.n, "n_basis": w.nb, "n_occ": w.n_up, "start": "zero density (core-Hamiltonian step)"},
            "runs": res,
            "dE_mixed_vs_fp64_converged": (m["energy"] - ft["energy"]) if m["converged"] and ft["converged"] else None,
            "speedup_vs_fp64": f["seconds"] / m["seconds"], "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="kr", choices=["kr", "ne", "he", "batch", "scf"],
                    help="scf: full Kr SCF to 1e-8 Eh (split BF16 and FP64, plain iteration and DIIS)")
    ap.add_argument("--diis", type=int, default=8, help="DIIS history of --workload scf")
    ap.add_argument("--scf-max-iter", type=int, default=50, help="iteration limit of --workload scf (the reference's RCS limit)")
    ap.add_argument("--precision", default="bf16x3", choices=["bf16x3", "fp64", "tf32"])
    ap.add_argument("--nrad", type=int, default=0, help="override the workload's radial points (smaller profiling cases)")
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--fp64-peak", type=float, default=float(os.environ.get("TCSCF_FP64_PEAK_TFLOPS", "37.0")))
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-seconds", type=float, default=10.0)
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--autotune", action="store_true",
                    help="measure the tensor launch's r2 split per build shape / batch on first use (inside the warm-up)")
    args = ap.parse_args()

    from tcscf_b200 import replicas

    rank, world, local = replicas.env_ranks()
    replicas.init(world, local)
    try:
        if args.impl == "reference":
            run_reference(args, rank)
        elif args.workload == "batch":
            run_batch(args, rank)
        elif args.workload == "scf":
            run_scf(args, rank)
        else:
            run_ours(args, rank, world)
    finally:
        replicas.finalize(world)


if __name__ == "__main__":
    main()
