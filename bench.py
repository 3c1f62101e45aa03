"""Benchmark: Fock-build seconds per SCF iteration on one B200 (mixed tensor-core form vs FP64).

One step = one direct-form RCS Fock build (Coulomb + exchange r12 contractions, Fock assembly and
energy) for the workload's density on its radial x Lebedev grid.  `value` is device time per step
with every input resident in HBM; `e2e` is the same through the public C ABI from host buffers
(grid upload, device basis evaluation, Fock build, G/Fock/energy back to the host).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload kr|ne|he|batch|scf|be_tc]
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


def guess_from(S, h, basis, nocc: int):
    """Core-Hamiltonian guess (the reference's first iteration: zero density -> F = h), solved in the
    real-harmonic basis with canonical orthogonalisation (the even-tempered overlap is
    ill-conditioned), so the closed-shell density is real there; returned in the reference basis.
    numpy only: both bench arms take their density from here."""
    from tcscf_b200.basis import real_harmonic_unitary

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
    return np.ascontiguousarray(D.astype(np.complex128))


def scf_guess_density(basis, Z: int, nocc: int):
    """The guess density of the GPU arm, from the library's analytic S and h."""
    from tcscf_b200 import api

    S, h = api.overlap_core(basis, Z)
    return guess_from(S, h, basis, nocc), h


def workload(name: str):
    from tcscf_b200 import basis as wl

    return {"kr": wl.kr, "ne": wl.ne, "he": wl.he}[name]()


def workload_config(w, n_points: int, dropped: int, near: int) -> dict:
    """The `config` object of a direct-form workload, identical in both arms."""
    return {"workload": f"{w.name} RCS Fock build", "Z": w.Z, "n_points": n_points, "n_basis": w.nb, "n_occ": w.n_up,
            "grid": f"{w.nrad} radial (Gauss-Chebyshev, r=(1+x)/(1-x)) x Lebedev order {w.order}",
            "density": "core-Hamiltonian guess (canonical orthogonalisation)",
            "l2": "GPU arm: flushed (256 MB write) between timed steps",
            "dropped_pairs": dropped, "near_coincident_pairs": near}


def host_cpu() -> dict:
    """lscpu's model name, sockets, cores per socket and threads per core of the host."""
    out = {}
    try:
        txt = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
    except Exception:
        return out
    keys = {"Model name": "model", "Socket(s)": "sockets", "Core(s) per socket": "cores_per_socket",
            "Thread(s) per core": "threads_per_core", "CPU(s)": "cpus"}
    for line in txt.splitlines():
        k, _, v = line.partition(":")
        if k.strip() in keys and keys[k.strip()] not in out:
            out[keys[k.strip()]] = v.strip()
    return out


def stratified_rows(n: int, k: int) -> np.ndarray:
    """k row indices spread evenly over the n points (the product grid orders them radial shell by
    radial shell, so the sample covers every radial range and angular position)."""
    k = max(1, min(n, k))
    return np.unique((np.arange(k) * (n / k) + n / (2 * k)).astype(np.int64).clip(0, n - 1))


# FP64 RCS SCF iterations of the Kr configuration from the zero density to |dE| < 1e-8 Eh
# (`bench.py --workload scf`, fp64_plain): the reference's precompute is amortised over these
SCF_ITERATIONS_KR = 9
PER_ITERATION_ROWS = 1024


def cpu_reference(w, grid, D, h, budget_s: float, threads: int | None = None, calib: dict | None = None) -> dict:
    """The reference algorithm timed on the host cores through the oracle port: precomputeIntegrand +
    computeF (HartreeFock.hpp:23-180) on a stratified sample of r1 rows against the full r2 grid, then
    the per-iteration calculateIaa / calculateFai / assembly (HartreeFock.cpp:144-213, 817-850) on
    1,024 stratified rows; both extrapolated linearly to all rows (rows are independent and of equal
    cost).  `calib` carries the sample size between steps."""
    import oracle

    if threads:
        oracle.set_threads(threads)
    cores = oracle.threads()
    if calib is None:
        calib = {}
    if "rows" not in calib:
        # one row per thread times the per-row precompute cost, then the sample is sized to the budget
        idx = stratified_rows(grid.n, cores)
        vals2 = oracle.basis_values(grid.points, w.basis)
        t0 = time.perf_counter()
        oracle.compute_F(np.ascontiguousarray(grid.points[:, idx]), grid.points, grid.weights, vals2, w.nb)
        per_row = (time.perf_counter() - t0) / len(idx)
        want = int(max(cores, min(grid.n, budget_s / max(per_row, 1e-9))))
        calib["rows"] = max(cores, (want // cores) * cores)
        calib["vals2"] = vals2
    vals2 = calib.get("vals2")
    if vals2 is None:
        vals2 = calib["vals2"] = oracle.basis_values(grid.points, w.basis)
    idx = stratified_rows(grid.n, calib["rows"])
    t0 = time.perf_counter()
    F = oracle.compute_F(np.ascontiguousarray(grid.points[:, idx]), grid.points, grid.weights, vals2, w.nb)
    t_pre = (time.perf_counter() - t0) / len(idx)
    # per-iteration build on 1,024 stratified rows: their basis values and weights, with the sampled
    # rows' F repeated (the per-row arithmetic of calculateIaa / calculateFai does not depend on F's values)
    it_idx = stratified_rows(grid.n, PER_ITERATION_ROWS)
    reps = -(-len(it_idx) // len(idx))
    F_it = np.ascontiguousarray(np.concatenate([F] * reps)[: len(it_idx)])
    vals1 = np.ascontiguousarray(vals2[it_idx])
    w1 = np.ascontiguousarray(grid.weights[it_idx])
    t0 = time.perf_counter()
    oracle.fock_build(F_it, vals1, w1, D, h)
    t_it = (time.perf_counter() - t0) / len(it_idx)
    T_pre, T_it = t_pre * grid.n, t_it * grid.n
    return {"s_per_iter": T_it, "precompute_s": T_pre, "iteration_s": T_it,
            "amortised_s_per_iter": T_pre / SCF_ITERATIONS_KR + T_it, "amortised_over_iterations": SCF_ITERATIONS_KR,
            "cores": cores, "rows": len(idx),
            "sample": f"precompute (precomputeIntegrand + computeF) on {len(idx)} stratified r1 rows x all {grid.n} r2 "
                      f"points; per-iteration Fock build (calculateIaa/calculateFai/assembly from the precomputed F) on "
                      f"{len(it_idx)} stratified r1 rows; both extrapolated linearly to all {grid.n} rows; value = the "
                      f"per-iteration cost, the one-off precompute reported as precompute_s and amortised over "
                      f"{SCF_ITERATIONS_KR} SCF iterations as amortised_s_per_iter"}


def reference_inputs(w):
    """Grid, guess density and h of the reference arm from the oracle, scipy's Lebedev rule and numpy:
    the product library is not loaded in that process."""
    import oracle
    from tcscf_b200 import ffi
    from tcscf_b200.grids import QuadratureGrid, lebedev_table

    r, wr = oracle.radial_grid(w.nrad, ffi.MAP_ONE_PLUS_X)
    pts, wts = oracle.product_grid(r, wr, lebedev_table(w.order))
    S, h = oracle.overlap_core(w.basis, w.Z)
    return QuadratureGrid(pts, wts), guess_from(S, h, w.basis, w.n_up), h


def product_library_loaded() -> bool:
    """Whether libtcscf_gpu.so is mapped into this process."""
    try:
        return "libtcscf_gpu.so" in Path("/proc/self/maps").read_text()
    except OSError:
        return False


def run_reference(args, rank: int) -> None:
    from tcscf_b200 import grids

    if rank != 0:
        return
    w = workload(args.workload)
    if args.nrad:
        w.nrad = args.nrad
    g, D, h = reference_inputs(w)
    vals, calib = [], {}
    for i in range(args.warmup + args.steps):
        r = cpu_reference(w, g, D, h, budget_s=args.ref_seconds, calib=calib)
        if i >= args.warmup:
            vals.append(r)
    v = statistics.median(x["s_per_iter"] for x in vals)
    pre = statistics.median(x["precompute_s"] for x in vals)
    amort = statistics.median(x["amortised_s_per_iter"] for x in vals)
    dropped, near = grids.coincident_pairs(g, g)   # r1 = r2 grid: the diagonal pairs contribute 0
    if product_library_loaded():
        raise RuntimeError("the reference arm must not load the product library")
    line = {"metric": METRIC, "value": v, "unit": "s/iter", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": workload_config(w, g.n, dropped, near),
            "cpu_baseline": {"value": v, "unit": "s/iter", "cores": r["cores"], "kind": "port", "sample": r["sample"],
                             "precompute_s": pre, "amortised_s_per_iter": amort,
                             "amortised_over_iterations": r["amortised_over_iterations"], "lscpu": host_cpu()},
            "e2e": {"value": v, "unit": "s/iter", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def measure_matmul_peaks(dev, n: int = 8192, reps: int = 10) -> dict:
    """Dense FP64 and TF32 matmul rates of this GPU, measured the way the BF16 peak of the peaks file
    is (torch.matmul of n x n operands, best of reps, CUDA events): the denominators of the FP64 and
    TF32 rooflines."""
    import torch

    out = {}
    saved = torch.backends.cuda.matmul.allow_tf32
    try:
        for name, dtype, tf32 in (("fp64_tflops", torch.float64, False), ("tf32_tflops", torch.float32, True)):
            torch.backends.cuda.matmul.allow_tf32 = tf32
            g = torch.Generator(device=dev).manual_seed(0)
            a = torch.randn(n, n, dtype=dtype, device=dev, generator=g)
            b = torch.randn(n, n, dtype=dtype, device=dev, generator=g)
            torch.matmul(a, b)
            torch.cuda.synchronize()
            best = float("inf")
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                torch.matmul(a, b)
                e1.record()
                torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1))
            out[name] = 2.0 * n ** 3 / (best / 1e3) / 1e12
            del a, b
    finally:
        torch.backends.cuda.matmul.allow_tf32 = saved
    torch.cuda.empty_cache()
    return out


def symmetric_pairs(n: int, fp64: bool = False) -> int:
    """(r1, r2) pairs the symmetric contraction computes on an n-point grid used as both r1 and r2:
    each 128-point r1 tile takes the r2 points from its own first row on (its diagonal tile in full, at
    half weight).  Split BF16 works in 64-point r2 blocks over the padded grid, sum_p 128 * 64 (nBlocks
    - 2 p); the FP64 kernel (128-row tiles, 8 x 8 register tiles) stops at the last point, sum_p 128
    (n - 128 p)."""
    tiles, blocks = -(-n // 128), -(-n // 64)
    if fp64:
        return sum(128 * (n - 128 * p) for p in range(tiles))
    return sum(128 * 64 * (blocks - 2 * p) for p in range(tiles))


def roofline(prec: int, n: int, nb: int, nocc: int, c_ms: float, peaks: dict, peak_kind: str, traffic, sym: bool = False,
             traffic_per_pair_sym=None) -> dict:
    """The line's roofline object for one Fock build of n points (r1 = r2 grid) whose contraction
    kernel took c_ms milliseconds.  peaks: the BF16 peak (bf16_tflops) and the FP64 / TF32 matmul rates
    (fp64_tflops, tf32_tflops) when measured.  sym: the split-BF16 kernel computed only the pairs on and
    above the diagonal tiles (X = g rho is symmetric when r1 = r2 and psi1 = psi2); its work counts those
    pairs, and traffic is traffic_per_pair_sym times them when that figure (measured on a symmetric
    launch) is given, else the full-launch figure scaled by them."""
    from tcscf_b200 import ffi

    # algorithmic work per Fock build: F_alg = 2 P (nb nocc + 1), the pair-density count of the direct
    # build (nb nocc exchange pair densities and the Coulomb density per (r1, r2) pair) over the P pairs
    # the build needs: N^2, or with the symmetric contraction each unordered pair once (the diagonal
    # tiles in full); the kernels contract the same sum in factored form, 2 P (nocc + nb + 1) flops
    # (rho GEMM, exchange GEMM, Coulomb), reported beside it as kernel_algorithm_tflops
    sym = sym and prec in (ffi.PREC_BF16X3, ffi.PREC_FP64)   # TF32 keeps the full contraction
    pairs = float(symmetric_pairs(n, fp64=prec == ffi.PREC_FP64)) if sym else float(n) * n
    flops = 2.0 * pairs * (nb * nocc + 1)
    kernel_flops = 2.0 * pairs * (nocc + nb + 1)
    achieved = flops / (c_ms / 1e3) / 1e12
    kernel_achieved = kernel_flops / (c_ms / 1e3) / 1e12
    numerator = {"achieved_numerator": "F_alg = 2 P (nb nocc + 1) flops per build (pair-density count over the P pairs computed)",
                 "pairs": pairs, "symmetric": bool(sym),
                 "full_pairs_tflops": 2.0 * n * n * (nb * nocc + 1) / (c_ms / 1e3) / 1e12,
                 "kernel_algorithm_tflops": kernel_achieved,
                 "frac_kind": "effective",
                 "frac_note": "frac counts F_alg, the pair-density work the factored form avoids; issued_frac (the "
                              "slice products the tensor pipe executes) and ncu's tensor-pipe activity measure the hardware"}
    if sym and prec != ffi.PREC_FP64 and traffic_per_pair_sym is not None:
        traffic = traffic_per_pair_sym * pairs
    elif traffic is not None and sym and prec != ffi.PREC_FP64:   # the full-launch figure, scaled by the units
        traffic = traffic * pairs / (float(-(-n // 128) * 128) * (-(-n // 64) * 64))
    if prec == ffi.PREC_FP64:
        # the FP64 kernel runs on the FP64 pipe: its roofline counts the flops it performs
        peak = peaks.get("fp64_tflops", 37.0)
        src = "fp64 dense matmul (torch, 8192^3), measured in this run" if "fp64_tflops" in peaks else "nominal B200 FP64 rate"
        roof = {"bound": "fp64", "achieved": kernel_achieved, "peak": peak, "unit": "TFLOP/s", "frac": kernel_achieved / peak,
                "traffic": None, "peak_source": src,
                "achieved_numerator": "2 P (nocc + nb + 1) flops per build (the factored contraction the kernel performs over "
                                      "the P pairs it computes)",
                "pairs": pairs, "symmetric": bool(sym), "effective_tflops": achieved}
    elif prec == ffi.PREC_TF32:
        if "tf32_tflops" in peaks:
            peak, src = peaks["tf32_tflops"], "tf32 dense matmul (torch, 8192^3), measured in this run"
        else:
            peak, src = peaks["bf16_tflops"] / 2, f"tf32 dense = half the bf16 dense burst, {peak_kind}"
        RP = 32                            # TF32 launches hold rank 32 (larger ranks run in chunks)
        NB = 64 if nb <= 64 else 128
        chunks = -(-nocc // RP)
        issued = pairs * chunks * (2.0 * RP + 2.0 * NB) / (c_ms / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": None, "peak_source": src,
                "issued_tensor_tflops": issued, "issued_frac": issued / peak, **numerator}
    else:
        peak = peaks["bf16_tflops"]
        # tensor work the kernel issues per (r1, r2) pair: GEMM1 6 slice products of K = RP; GEMM2 6 of
        # N = NB with 24-bit X (rank padding 32), 4 with 16-bit X (rank padding 64)
        RP = 32 if nocc <= 32 else 64   # real closed-shell guess density: factor rank = n_occ
        NB = 64 if nb <= 64 else 128
        issued = pairs * (2.0 * 6 * RP + 2.0 * (6 if RP == 32 else 4) * NB) / (c_ms / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": f"bf16 dense burst, {peak_kind}",
                "issued_tensor_tflops": issued, "issued_frac": issued / peak, **numerator}
    return roof


METRIC = "Fock-build s/iter, mixed vs FP64 GPU at |dE|<=1 uEh; % of roofline"


# DRAM bytes per launch of the split-BF16 contraction kernel (kFlashTc<128,32,3>) on the Kr workload:
# ncu's dram__bytes_read.sum + dram__bytes_write.sum of one launch on the 263,900-point Kr grid
# (130 radial x Lebedev 77) was 11.94 GB + 0.268 GB = 1.221e10 B; a launch re-streams the r2 operands
# once per (r1 tile, r2 block) unit where L2 misses, so the figure scales with the unit count,
# 3172 x 6344 at 406,000 points against 2062 x 4124 (x 2.366), to 2.889e10 B
TRAFFIC_BYTES_PER_LAUNCH = {"Kr": 2.889e10}
# The symmetric launch (r1 = r2 grid, psi1 = psi2) of the same kernel, its work items dealt by weight in
# snake order (so the CTAs running at a time hold tiles of similar index, whose r2 streams overlap in L2):
# one launch on the 263,900-point grid read 2.457 GB and wrote 0.237 GB for its 3.4848e10 computed pairs,
# 0.0773 B per pair (6.37e9 B for the 8.245e10 pairs at 406,000 points).  With the tiles in index order
# it was 13.81 GB, 0.3964 B per pair.
TRAFFIC_BYTES_PER_PAIR_SYM = {"Kr": (2.4566e9 + 0.2366e9) / 3.4848e10}


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
    # FP64 / TF32 matmul rates of this GPU (untimed region): the FP64 and TF32 roofline denominators
    mm_peaks = {} if args.skip_peaks else measure_matmul_peaks(dev)
    n = g.n
    dropped, near = grids.coincident_pairs(g, g)   # r1 = r2 grid: the diagonal pairs contribute 0
    c_ms = statistics.median(cms)
    allpeaks = dict(peaks, **mm_peaks)
    # one grid object serves as r1 and r2 and the guess density is real and positive semi-definite, so
    # the split-BF16 and FP64 builds take the symmetric contraction
    roof = roofline(prec, n, w.nb, w.n_up, c_ms, allpeaks, peak_kind,
                    TRAFFIC_BYTES_PER_LAUNCH.get(w.name) if prec == ffi.PREC_BF16X3 and args.nrad == 0 else None,
                    sym=True, traffic_per_pair_sym=TRAFFIC_BYTES_PER_PAIR_SYM.get(w.name) if prec == ffi.PREC_BF16X3 else None)
    if fp64 is not None:
        fp64["roofline"] = roofline(ffi.PREC_FP64, n, w.nb, w.n_up, fp64["contraction_ms"], allpeaks, peak_kind, None, sym=True)
    cpu = None
    if not args.skip_cpu:
        r = cpu_reference(w, g, D, h, budget_s=args.cpu_seconds)
        cpu = {"value": r["s_per_iter"], "unit": "s/iter", "cores": r["cores"], "kind": "port", "sample": r["sample"],
               "precompute_s": r["precompute_s"], "iteration_s": r["iteration_s"],
               "amortised_s_per_iter": r["amortised_s_per_iter"], "amortised_over_iterations": r["amortised_over_iterations"],
               "lscpu": host_cpu()}
    line = {"metric": METRIC, "value": s_per_iter, "unit": "s/iter", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp64": "f64", "bf16x3": "bf16", "tf32": "tf32"}[args.precision],
            "data": "synthetic",
            "config": workload_config(w, n, dropped, near),
            "form": "direct (no stored Fji)",
            "precision": {"fp64": "fp64",
                          "bf16x3": "bf16 fixed-point slices (24-bit factors and kernel tile), exact fp32 accumulation of "
                                    "the leading slices per 64-point block, double-float across blocks",
                          "tf32": "tf32 operands (10-bit mantissa, round to nearest), fp32 accumulation per 64-point block, "
                                  "double-float across blocks"}[args.precision],
            "schedule": "autotuned r2 split (tuned in the warm-up: shapes, batches, measurements = %s)" % (ctx.autotune_stats(),)
            if args.autotune else "fixed rule",
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
    # device times of the last batched call: the persistent tensor launches alone, and the whole call
    batch_contraction_ms, batch_total_ms, batch_launches = ctx.last_timing()
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
            "contraction_ms": batch_contraction_ms, "device_total_ms": batch_total_ms, "launches": batch_launches,
            "one_at_a_time_s": t1, "batch_speedup": t1 / tb, "batched_equals_one_at_a_time": bool(np.array_equal(Eb, E1)),
            "dE_vs_fp64_max": float(err.max()), "dE_vs_fp64_median": float(np.median(err)),
            "dE_rel_vs_fp64_max": float((err / np.abs(E64)).max()), "clocks": clk.summary(),
            "schedule": {"autotune": bool(args.autotune), "tuned_shapes_batches_measurements": ctx.autotune_stats()}}
    print(json.dumps(line), flush=True)


def run_scf(args, rank: int) -> None:
    """Full RCS SCF of the Kr configuration to |dE| < 1e-8 Eh: split-BF16 and FP64 Fock builds in the plain
    Roothaan iteration of the reference (at most --scf-max-iter iterations), each as the device loop in
    one CUDA graph (tcscf_scf_graph) and as the host-driven loop (tcscf_scf), optionally split BF16 with
    Pulay DIIS (--diis), and the FP64 device loop converged to 1e-10 Eh as the energy reference; all
    with the real-harmonic eigen-solve (real densities throughout, one contraction per build).  Each SCF
    starts from the zero density (core-Hamiltonian first step, as the reference); wall time around the
    public call."""
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
    # is not itself run to 1e-10).  "graph": the whole loop on the device as one CUDA graph launch
    # (tcscf_scf_graph); "host": the host-driven loop (tcscf_scf, real-harmonic eigen-solve)
    runs = [("bf16x3_graph", ffi.PREC_BF16X3, "graph", 0, 1e-8), ("fp64_graph", ffi.PREC_FP64, "graph", 0, 1e-8),
            ("bf16x3_host", ffi.PREC_BF16X3, "host", 0, 1e-8), ("fp64_host", ffi.PREC_FP64, "host", 0, 1e-8),
            ("fp64_graph_1e-10", ffi.PREC_FP64, "graph", 0, 1e-10)]
    if args.diis:
        runs.append(("bf16x3_host_diis", ffi.PREC_BF16X3, "host", args.diis, 1e-8))
    res = {}
    with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
        for name, prec, mode, nd, tol in runs:
            hf = api.RCSHartreeFock(w.n_up, w.n_down, w.nb)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            try:
                if mode == "graph":
                    E = hf.computeOnDevice(S, h, G, G, precision=prec, tol=tol, max_iter=args.scf_max_iter, capture=True)
                else:
                    E = hf.compute(S, h, G, G, precision=prec, tol=tol, max_iter=args.scf_max_iter, diis=nd, real_eigensolve=True)
                ok = True
            except ffi.TcscfError as e:
                if e.code != ffi.ERR_NOT_CONVERGED:
                    raise
                E, ok = None, False
            torch.cuda.synchronize()
            res[name] = {"converged": ok, "energy": E, "iterations": hf.numberOfConvergenceLoops(),
                         "seconds": time.perf_counter() - t0, "loop": mode, "diis": nd, "tol": tol}
    m, f, ft = res["bf16x3_graph"], res["fp64_graph"], res["fp64_graph_1e-10"]
    line = {"metric": "Kr RCS SCF to |dE| < 1e-8 Eh, wall s (split-BF16 Fock builds, device loop in one CUDA graph)",
            "value": m["seconds"], "unit": "s",
            "n_gpus": 1, "steps": 1, "warmup": 0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16", "data": "synthetic",
            "config": {"workload": f"Kr RCS SCF (direct-form Fock builds), {w.nrad} radial x Lebedev order {w.order}",
                       "n_points": g.n, "n_basis": w.nb, "n_occ": w.n_up, "start": "zero density (core-Hamiltonian step)"},
            "runs": res,
            "dE_mixed_vs_fp64_converged": (m["energy"] - ft["energy"]) if m["converged"] and ft["converged"] else None,
            "speedup_vs_fp64": f["seconds"] / m["seconds"],
            "speedup_vs_fp64_host_loop": res["fp64_host"]["seconds"] / m["seconds"], "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_be_tc(args, rank: int) -> None:
    """The Be transcorrelated configuration: 24 STOs, three 2^16-point scrambled-Sobol grids, Jastrow
    u = r12 / (2 (1 + b r12)), b = 1.  Per precision (split BF16 and FP64): the precompute
    (computeF of the same- and opposite-spin TC scalar kernels on r1 x r2, computeV of grad u on r1 x r3,
    HartreeFockTest.cpp:261-319), the TC SCF on those tensors to |dE| < 1e-8 Eh (TCHartreeFock,
    HartreeFock.cpp:1105-1362), and the per-iteration TC Fock build timed on its own.  value = the mixed
    precompute amortised over the SCF's iterations plus one per-iteration build (s/iter); the FP64
    figure beside it; device time on the context stream for the precompute, wall time around the
    synchronous per-iteration call."""
    import torch

    from tcscf_b200 import api, ffi, grids
    from tcscf_b200 import basis as wl

    if rank != 0:
        return
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    w = wl.be_tc()
    n = args.qmc_points or w.qmc_points
    jd = wl.be_tc_jastrow(w)
    u = ffi.ochi_struct(jd["a"], jd["a12"], jd["terms"])
    seed = w.extra["seed"]
    g = [grids.qmc_grid(3, n, seed + k) for k in range(3)]
    ctx = api.Context(local)
    G = [api.QMCGrid(ctx, gk) for gk in g]
    G[0].setBasisFunctions(w.basis, storeGradients=True)
    G[1].setBasisFunctions(w.basis)
    G[2].setBasisFunctions(w.basis)
    S, h = api.overlap_core(w.basis, w.Z)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))
    peaks, peak_kind = load_peaks()
    np_ = w.nb * (w.nb + 1) // 2

    def precompute(prec):
        ts, cms = [], []
        for kern, fn, grid in ((ffi.K_TC_SCALAR_SAME, api.computeF, G[1]), (ffi.K_TC_SCALAR_OPPO, api.computeF, G[1]),
                               (ffi.K_GRAD_U_SAME, api.computeV, G[2]), (ffi.K_GRAD_U_OPPO, api.computeV, G[2])):
            _, t = fn(G[0], grid, kern, u, keep=True, copy=False, precision=prec)
            ts.append(t)
            cms.append(ctx.last_timing()[0])
        return ts, cms

    res = {}
    with ClockSampler(local) as clk:
        for name, prec in (("bf16x3", ffi.PREC_BF16X3), ("fp64", ffi.PREC_FP64)):
            steps = args.steps if prec == ffi.PREC_BF16X3 else max(1, min(args.steps, args.fp64_steps))
            warm = args.warmup if prec == ffi.PREC_BF16X3 else 1
            pre_ms, kern_ms, launches = [], [], 0
            for i in range(warm + steps):
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                l0 = ctx.last_timing()[2]
                e0.record(stream)
                ts, cms = precompute(prec)
                e1.record(stream)
                torch.cuda.synchronize()
                if i >= warm:
                    pre_ms.append(e0.elapsed_time(e1))
                    kern_ms.append(cms)
                if i < warm + steps - 1:
                    for t in ts:
                        t.close()
            scf = api.TCHartreeFock(w.n_up, w.n_down)
            t0 = time.perf_counter()
            E = scf.compute(S, h, G[0], *ts, tol=1e-8, max_iter=200)
            scf_s = time.perf_counter() - t0
            occ = []
            for s_, nocc in ((0, w.n_up), (1, w.n_down)):
                # occupied orbitals of the converged density (its leading eigenvectors) for the timed build
                ev, V = np.linalg.eigh(scf.density[s_])
                occ.append((V[:, ::-1][:, :nocc] * np.sqrt(np.maximum(ev[::-1][:nocc], 0))).T.copy())
            it_s = []
            for i in range(3 + steps):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                api.tc_fock_build(G[0], *ts, w.n_up, w.n_down, scf.density, occ[0], occ[1], h)
                torch.cuda.synchronize()
                if i >= 3:
                    it_s.append(time.perf_counter() - t0)
            for t in ts:
                t.close()
            T_pre = statistics.median(pre_ms) / 1e3
            T_it = statistics.median(it_s)
            res[name] = {"precompute_s": T_pre, "iteration_s": T_it, "scf_iterations": scf.iterations, "scf_wall_s": scf_s,
                         "energy": E, "s_per_iter": T_pre / scf.iterations + T_it,
                         "contraction_ms": [statistics.median(k[j] for k in kern_ms) for j in range(4)]}
    m, f = res["bf16x3"], res["fp64"]
    # roofline of the dominant kernel (one computeV component launch of kPairTc): algorithmic flops
    # 2 N1 N2 np per launch (np = nb (nb+1)/2 real basis-pair columns); issued slice products
    # 6 x 2 x NBtot per pair (NBtot = np rounded up to whole 128-column chunks)
    NB = 64 if np_ <= 64 else 128
    nbtot = -(-np_ // NB) * NB
    c_ms = m["contraction_ms"][2] / 3   # computeV: three component launches
    alg = 2.0 * n * n * np_ / (c_ms / 1e3) / 1e12
    issued = 12.0 * nbtot * n * n / (c_ms / 1e3) / 1e12
    peak = peaks["bf16_tflops"]
    line = {"metric": "Be-TC Fock-build s/iter (precompute amortised over the TC-SCF iterations), mixed vs FP64 GPU",
            "value": m["s_per_iter"], "unit": "s/iter", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": m["s_per_iter"] * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16", "data": "synthetic",
            "config": {"workload": "Be transcorrelated HF (precompute form)", "Z": w.Z, "n_basis": w.nb,
                       "n_up": w.n_up, "n_down": w.n_down, "points_per_grid": n, "grids": "3 scrambled-Sobol sets "
                       f"(seeds {seed}..{seed + 2}), reference QMC map", "jastrow": "u = r12/(2(1+b r12)), b = 1, "
                       "c = -a12/2 (opposite), -a12/4 (same)", "scf_tol": 1e-8},
            "mixed": m, "fp64": f, "dE_mixed_vs_fp64": m["energy"] - f["energy"],
            "precompute_speedup_vs_fp64": f["precompute_s"] / m["precompute_s"],
            "speedup_vs_fp64": f["s_per_iter"] / m["s_per_iter"],
            "roofline": {"bound": "tensor", "achieved": alg, "peak": peak, "unit": "TFLOP/s", "frac": alg / peak, "traffic": None,
                         "kernel": "kPairTc (computeV component)", "peak_source": f"bf16 dense burst, {peak_kind}",
                         "issued_tensor_tflops": issued, "issued_frac": issued / peak,
                         "achieved_numerator": "2 N1 N2 nb(nb+1)/2 flops per launch"},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="kr", choices=["kr", "ne", "he", "batch", "scf", "be_tc"],
                    help="scf: full Kr SCF to 1e-8 Eh (split BF16 and FP64, plain iteration and DIIS); "
                         "be_tc: the Be transcorrelated configuration (precompute, TC SCF, per-iteration build)")
    ap.add_argument("--qmc-points", type=int, default=0, help="override the be_tc points per grid (smaller profiling cases)")
    ap.add_argument("--diis", type=int, default=0, help="add a split-BF16 host-loop run with this DIIS history to --workload scf")
    ap.add_argument("--scf-max-iter", type=int, default=50, help="iteration limit of --workload scf (the reference's RCS limit)")
    ap.add_argument("--precision", default="bf16x3", choices=["bf16x3", "fp64", "tf32"])
    ap.add_argument("--nrad", type=int, default=0, help="override the workload's radial points (smaller profiling cases)")
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--skip-peaks", action="store_true", help="do not measure the FP64 / TF32 matmul rates")
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
        elif args.workload == "be_tc":
            run_be_tc(args, rank)
        else:
            run_ours(args, rank, world)
    finally:
        replicas.finalize(world)


if __name__ == "__main__":
    main()
