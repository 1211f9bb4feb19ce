#!/usr/bin/env python
"""Benchmark: solves/s of the mixed-precision refined dense solve vs the FP64 LU.

Workload (one GPU): T-PMCHWT dielectric sphere, radius 0.5 m, eps_r = 4,
mu_r = 1, ka = pi (k0 = 2 pi, f = c0), class-I geodesic mesh with 2000 faces
and 3000 RWG edges (N = 6000 unknowns, J and M), Dunavant rule 17 assembly,
one x-polarised plane wave along +z. Synthetic: the mesh and excitation are
generated here, the system is assembled by the library.

A step is one solve of the assembled system: randomized-butterfly transform,
complex64 LU with split-TF32 tensor-core trailing updates, FP64 GMRES
refinement against the complex128 Z until the relative residual <= 1e-10.
Z (576 MB) is resident in HBM and larger than L2 (126 MB), so no separate L2
flush is needed between steps. The FP64 comparison is cusolverDnZgetrf +
Zgetrs on the same Z (the reference's own solver path).

Multi-GPU (torchrun): replicas, one independent solve stream per GPU (a
single dense system is not sharded); value = solves on all ranks / max time.

--impl reference times the reference's own CPU path for the same solve
(Eigen PartialPivLU in the reference's host build, oracle/_ref) on the host
cores, rank 0 only.
"""

from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "sie-gstc-2026_b200"))
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

C0 = 299792458.0
METRIC = "solves/s mixed-prec+IR vs FP64 LU at rel.res≤1e-10 (1 B200); adjoint grads/s"
WORKLOAD = ("T-PMCHWT dielectric sphere r=0.5 m, eps_r=4, mu_r=1, ka=pi; geodesic mesh 2000 faces / "
            "3000 RWG edges (N=6000); Dunavant rule 17; 1 plane-wave RHS")
# DRAM bytes (read + write) per trailing-update launch, mean over the 92
# launches of one factorization of this workload, from one ncu capture of
# the trailing GEMM (dram__bytes_read.sum + dram__bytes_write.sum).
GEMM_DRAM_BYTES_PER_LAUNCH = 158.4e6
# FP64 flops per Green evaluation (one point pair, one wavenumber) of the
# T-PMCHWT regular pass, counted from the kernel's source with an FMA as 2:
# the point-pair geometry shared by the two wavenumbers (distance, r_p.r_q,
# r_p x r_q, weights: 23 flops, half each), the kernel values (11) and the
# 8 TL + 10 TK complex moments (72); one sqrt, one reciprocal and one sincos
# per evaluation are not counted.
ASSEMBLY_FLOPS_PER_EVAL = 95
# Rotated-testing (nTL / nTK) pair kernel: per wavenumber 15 flops of kernel
# values and products with the weight, 30 for the 8 G-weighted and 44 for the
# 11 g-weighted complex moments; 51 flops of point-pair geometry shared by the
# two wavenumbers (FMA = 2; sqrt, reciprocal, sincos not counted).
N_ASSEMBLY_FLOPS_PER_EVAL = 115
# FP64 flops per field evaluation (one observation point, one face, one
# quadrature point) of the surface-field kernel, counted from its source with
# an FMA as 2: G and grad G (26), then for each of the three half-RWG
# functions rho (3), the L vector (36) and the K vector (36), plus the face's
# edge-length scaling and E/H accumulation spread over the rule's 61 points
# (~6); one sqrt, two divisions and one sincos are not counted.
FIELDS_FLOPS_PER_EVAL = 257


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def build_problem(rule: int = 17):
    import sieb200
    mesh = sieb200.geodesic_sphere(0.5, 10)
    opts = sieb200.DielectricOptions(frequency_hz=C0, quadrature_rule=rule,
                                     interior=sieb200.IsotropicMedium(4.0, 1.0))
    return mesh, opts


def bench_config(world: int) -> dict:
    """The workload key both arms print (the driver compares them)."""
    return {"workload": WORKLOAD, "N": 6000, "rule": 17, "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (Z complex128 576 MB resident)"}


class ClockSampler:
    """SM clocks, power and clock-event reasons sampled during the timed
    region: NVML polled every 10 ms from a thread (so that a short region
    still gets many samples), nvidia-smi at 200 ms when NVML is missing."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown"}
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int, period_s: float = 0.01):
        self.index = index
        self.period = period_s
        self.rows = []  # (sm_mhz, max_mhz, power_w, reasons)
        self.proc = None
        self.thread = None
        self.stop = threading.Event()
        self.source = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            for i in range(pynvml.nvmlDeviceGetCount()):
                h = pynvml.nvmlDeviceGetHandleByIndex(i)
                u = pynvml.nvmlDeviceGetUUID(h)
                u = u.decode() if isinstance(u, bytes) else u
                if u.replace("GPU-", "") == uuid.replace("GPU-", ""):
                    return pynvml, h
        except Exception:
            pass
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _poll_nvml(self, nv, h):
        reasons_fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1e3
                bits = reasons_fn(h)
                self.rows.append((float(sm), float(mx), pw, [n for b, n in self.REASONS.items() if bits & b]))
            except Exception:
                pass
            self.stop.wait(self.period)

    def _read_smi(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            if len(r) > 8 and r[1].replace(".", "").isdigit():
                reasons = [nm for nm, v in zip(names, r[5:9]) if v.lower() == "active"]
                pw = float(r[3]) if r[3].replace(".", "").isdigit() else None
                self.rows.append((float(r[1]), float(r[2]), pw, reasons))

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.source = "nvml 10 ms"
            self.thread = threading.Thread(target=self._poll_nvml, args=(nv, h), daemon=True)
            self.thread.start()
            return self
        except Exception:
            pass
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi 200 ms"
            self.thread = threading.Thread(target=self._read_smi, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [r[0] for r in self.rows]
        pw = [r[2] for r in self.rows if r[2] is not None]
        reasons = sorted({n for r in self.rows for n in r[3]})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(r[1] for r in self.rows),
                "sm_min_mhz": min(sm), "power_w_median": statistics.median(pw) if pw else None,
                "reasons": reasons, "samples": len(self.rows), "sampler": self.source}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def cpu_reference_solve(Zh: np.ndarray, bh: np.ndarray, threads: int):
    """The reference's CPU solve (Eigen PartialPivLU, oracle/_ref); seconds, x."""
    from oracle import oracle as O
    ref = O.reference()
    n = Zh.shape[0]
    Zf = np.asfortranarray(Zh)
    x = np.zeros(n, np.complex128)
    if ref is not None:
        secs = ref.ref_lu_solve(n, Zf.ctypes.data, bh.ctypes.data, x.ctypes.data, 1, threads)
        return secs, x, "reference", "Eigen PartialPivLU (reference host build, oracle/_ref)"
    t0 = time.perf_counter()
    x = np.linalg.solve(Zh, bh)
    return time.perf_counter() - t0, x, "port", "LAPACK zgesv via numpy (reference harness not built)"


def run_reference(args):
    """The reference's CPU solve of the benchmark system, on the host cores.

    Nothing of this library is loaded: the sphere comes from the oracle's own
    generator (vertex- and index-equal to the library's), the system and the
    right-hand side from the reference's host quadrature (oracle/_ref), the
    solve is the reference's Eigen PartialPivLU."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from oracle import oracle as O
    ref = O.reference()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference host build (oracle/_ref) missing"}))
        return
    mesh = O.geodesic_sphere(0.5, 10)
    threads = os.cpu_count() or 1
    # The reference's host assembly of this system at rule 17 (~3e10 Green
    # evaluations) is far beyond a bounded CPU sample. The LU does not depend
    # on the rule, so the solved system is assembled with Dunavant rule 1:
    # same size, same block structure, same operator.
    s = O.kernel_scalars(1, C0, eps_r=(4.0, 1.0))
    t0 = time.perf_counter()
    Z = O.assemble(ref, 1, mesh, 1, s, threads=threads, fn="ref_assemble")
    t_asm = time.perf_counter() - t0
    k = s["omega"] * math.sqrt(s["mu0"] * s["eps0"])
    eta = math.sqrt(s["mu0"] / s["eps0"])
    b = np.zeros(Z.shape[0], np.complex128)
    V = np.ascontiguousarray(mesh.vertices)
    E0 = np.array([1.0, 0, 0])
    kh = np.array([0, 0, 1.0])
    ref.ref_rhs_plane_wave(1, V.ctypes.data, mesh.faces.ctypes.data, mesh.faces_edges.ctypes.data,
                           mesh.num_faces, mesh.num_edges, 17, E0.ctypes.data, kh.ctypes.data, k, eta, 2,
                           s["mu0"], s["eps0"], b.ctypes.data, 0, 1.0, 1.0)
    steps = args.steps if args.steps is not None else 20
    times = []
    x = None
    for i in range(args.warmup + steps):
        secs, x, kind, desc = cpu_reference_solve(Z, b, threads)
        if i >= args.warmup:
            times.append(secs)
    tot = sum(times)
    value = len(times) / tot
    rres = float(np.linalg.norm(Z @ x - b) / np.linalg.norm(b))
    sample = (f"one full N={Z.shape[0]} complex128 factor+solve per step ({desc}), {threads} host threads")
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": bench_config(world), "impl": "reference",
        "solved_system": {"assembly": "reference host quadrature, Dunavant rule 1 (the LU cost does not depend "
                                      "on the rule; rule 17 on the host is ~3e10 Green evaluations)",
                          "assembly_seconds": t_asm, "N": int(Z.shape[0]), "faces": mesh.num_faces,
                          "edges": mesh.num_edges},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "relative_residual": rres,
    }), flush=True)


def run(args):
    import torch
    import torch.distributed as dist

    import sieb200

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ctx = sieb200.Context(local)
    try:
        out = measure(args, ctx, rank, world, local, barrier, max_over_ranks)
        if rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        # Orderly teardown: every tensor and solver of measure() is gone once
        # it returns; free torch's cached blocks (some were last used on the
        # library's stream) while that stream still exists, then the context.
        import gc
        gc.collect()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        ctx.close()
        if world > 1:
            dist.destroy_process_group()


def measure(args, ctx, rank: int, world: int, local: int, barrier, max_over_ranks) -> dict:
    """The timed work of one rank; returns rank 0's JSON line as a dict."""
    import torch

    import sieb200

    if args.steps is None:
        args.steps = 200
    stream = torch.cuda.ExternalStream(ctx.stream)
    mesh, opts = build_problem(args.rule)
    N = 2 * mesh.num_edges

    # Assembly (reported, not part of a solve): one warm-up, one timed.
    Z = torch.empty((N, N), dtype=torch.complex128, device="cuda")
    sieb200.assemble_matrix_device(mesh, opts, Z.data_ptr(), ctx=ctx)
    ctx.synchronize()
    t0 = time.perf_counter()
    sieb200.assemble_matrix_device(mesh, opts, Z.data_ptr(), ctx=ctx)
    ctx.synchronize()
    t_asm = time.perf_counter() - t0
    Q = 61 if args.rule == 17 else sieb200.lib().sieb200_quadrature_rule(args.rule, None, None)
    evals = 2.0 * mesh.num_faces ** 2 * Q * Q  # Green evaluations (two wavenumbers)
    fp64_peak = ctx.fp64_fma_peak()
    # The same system with rotated (n x RWG) testing, N-PMCHWT surface form:
    # nTL / nTK face-pair quadrature in place of TL / TK, same placement.
    opts_n = dataclasses.replace(opts, formulation="N_PMCHWT")
    sieb200.assemble_matrix_device(mesh, opts_n, Z.data_ptr(), ctx=ctx)
    ctx.synchronize()
    t0 = time.perf_counter()
    sieb200.assemble_matrix_device(mesh, opts_n, Z.data_ptr(), ctx=ctx)
    ctx.synchronize()
    t_asm_n = time.perf_counter() - t0
    variants = {
        "n_pmchwt": {
            "workload": "N-PMCHWT (n x RWG testing, surface nTL form) of the same sphere, rule 17",
            "assembly_seconds": t_asm_n, "t_pmchwt_assembly_seconds": t_asm,
            "green_evals_per_s": evals / t_asm_n,
            "roofline": {"bound": "fp64 pipe", "unit": "TFLOP/s", "flops_per_eval": N_ASSEMBLY_FLOPS_PER_EVAL,
                         "achieved": evals * N_ASSEMBLY_FLOPS_PER_EVAL / t_asm_n / 1e12, "peak": fp64_peak,
                         "frac": evals * N_ASSEMBLY_FLOPS_PER_EVAL / t_asm_n / 1e12 / fp64_peak},
        }
    }
    sieb200.assemble_matrix_device(mesh, opts, Z.data_ptr(), ctx=ctx)
    ctx.synchronize()
    b = torch.from_numpy(sieb200.assemble_rhs(mesh, opts, [sieb200.PlaneWaveExcitation()], ctx=ctx)[:, 0].copy()).cuda()
    x = torch.empty_like(b)

    solver = sieb200.DenseLuSolver(N, "mixed_ir", ctx=ctx)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def step():
        solver.factorize(Z.data_ptr())
        with torch.cuda.stream(stream):
            x.copy_(b)
        it = solver.solve(x.data_ptr(), tolerance=1e-10, max_iterations=60)
        return it

    # Warm-up: the second factorization of the same operand is captured as
    # a CUDA graph, later ones replay it.
    for _ in range(args.warmup):
        step()
    barrier()
    launches0 = sieb200.lib().sieb200_launch_count()
    iters = []
    with ClockSampler(local) as clocks:
        e0, e1 = ev(), ev()
        e0.record(stream)
        for _ in range(args.steps):
            iters.append(step())
        e1.record(stream)
        e1.synchronize()
    barrier()
    launches = sieb200.lib().sieb200_launch_count() - launches0
    t_mixed = max_over_ranks(e0.elapsed_time(e1) / 1e3)

    # The same K steps again with a CUDA-event pair around every hot launch
    # (per-kernel durations for the roofline): ~560 event records per
    # factorization would add ~1.3 ms to each step of the timed region above.
    ctx.profile(True)
    step()
    ctx.profile(True)
    p0, p1 = ev(), ev()
    p0.record(stream)
    for _ in range(args.steps):
        step()
    p1.record(stream)
    p1.synchronize()
    t_prof = p0.elapsed_time(p1) / 1e3
    gemm = ctx.profile_read(0)
    trsv = ctx.profile_read(1)
    gemv = ctx.profile_read(2)
    prof = {name: ctx.profile_read(i) for i, name in
            [(3, "diag_lu"), (4, "panels"), (6, "factorization"), (7, "refined_solve")]}
    # One more step with the per-launch timeline: the largest trailing update
    # (block step 0) on its own, against its roofline.
    ctx.profile(True, timeline=True)
    step()
    ctx.synchronize()
    first_gemm = next(((a, b2) for k, a, b2 in sorted(ctx.profile_timeline(), key=lambda v: v[1]) if k == 0), None)
    ctx.profile(False)

    # Accuracy of the mixed solution against the FP64 matrix.
    r = b.clone()
    torch.cuda.synchronize()
    sieb200.matvec(N, Z.data_ptr(), x.data_ptr(), r.data_ptr(), beta=-1.0, ctx=ctx)
    ctx.synchronize()
    rel_res = float(torch.linalg.vector_norm(r).item() / torch.linalg.vector_norm(b).item())
    x_mixed = x.clone()

    # The solved sphere against the Mie series (discretization error of the
    # far field; physical currents from the public solver call).
    try:
        mie_err = rcs_error_vs_mie(ctx, mesh, opts, 0.5, 4.0)
    except Exception as e:  # noqa: BLE001
        mie_err = {"error": repr(e)}
    try:
        ref_gpu = reference_gpu_section(ctx, mesh, opts, t_asm) if rank == 0 and not args.skip_sections else None
    except Exception as e:  # noqa: BLE001
        ref_gpu = {"error": repr(e)}

    # FP64 LU (cuSOLVER) on the same system, for the speed-up and the error.
    fp64 = sieb200.DenseLuSolver(N, "lu_cusolver", ctx=ctx)
    Zw = torch.empty_like(Z)
    fp64_times = []
    for i in range(1 + max(2, min(args.steps, 5))):
        with torch.cuda.stream(stream):
            Zw.copy_(Z)
            x.copy_(b)
        a, c = ev(), ev()
        a.record(stream)
        fp64.factorize(Zw.data_ptr())
        fp64.solve(x.data_ptr())
        c.record(stream)
        c.synchronize()
        if i > 0:
            fp64_times.append(a.elapsed_time(c) / 1e3)
    t_cusolver = max_over_ranks(statistics.mean(fp64_times))
    x_fp64 = x.clone()
    rel_diff = float(torch.linalg.vector_norm(x_mixed - x_fp64).item() / torch.linalg.vector_norm(x_fp64).item())
    del Zw
    fp64.close()
    # The library's own FP64 LU (complex128 butterfly LU, FP64 GEMM trailing
    # update, FP64 refinement) on the same system; Z stays intact.
    own = sieb200.DenseLuSolver(N, "lu_fp64", ctx=ctx)
    own_times = []
    for i in range(1 + max(2, min(args.steps, 5))):
        with torch.cuda.stream(stream):
            x.copy_(b)
        a, c = ev(), ev()
        a.record(stream)
        own.factorize(Z.data_ptr())
        own.solve(x.data_ptr(), tolerance=1e-10, max_iterations=5)
        c.record(stream)
        c.synchronize()
        if i > 0:
            own_times.append(a.elapsed_time(c) / 1e3)
    own.close()
    t_own = max_over_ranks(statistics.mean(own_times))
    own_rel_diff = float(torch.linalg.vector_norm(x - x_fp64).item() / torch.linalg.vector_norm(x_fp64).item())
    # the FP64 baseline is the faster of the two FP64 LUs
    t_fp64 = min(t_cusolver, t_own)

    # End to end through the public API with host buffers, every step: the
    # H2D copy of that step's Z and b from pinned memory, factor + refine,
    # the D2H copy of x. Two device buffers let the upload of step i+1 (on a
    # copy stream) overlap step i's factorization and refinement, as a
    # caller streaming systems through the solver would; the first upload is
    # not hidden.
    Zh = Z.cpu().pin_memory()
    bh = b.cpu().pin_memory()
    xh = [torch.empty_like(bh).pin_memory() for _ in range(2)]
    Zd = [torch.empty_like(Z) for _ in range(2)]
    xd = [torch.empty_like(b) for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    uploaded = [torch.cuda.Event() for _ in range(2)]
    released = [torch.cuda.Event() for _ in range(2)]
    for e in released:
        e.record(stream)
    e2e_steps = max(3, args.steps)

    def upload(i):
        j = i % 2
        with torch.cuda.stream(copy_stream):
            copy_stream.wait_event(released[j])  # the step that last used buffer j is done
            Zd[j].copy_(Zh, non_blocking=True)
            xd[j].copy_(bh, non_blocking=True)
            uploaded[j].record(copy_stream)

    def compute(i):
        j = i % 2
        stream.wait_event(uploaded[j])
        solver.factorize(Zd[j].data_ptr())
        solver.solve(xd[j].data_ptr(), tolerance=1e-10, max_iterations=60)
        with torch.cuda.stream(stream):
            xh[j].copy_(xd[j], non_blocking=True)
            released[j].record(stream)

    def e2e_run(k):
        upload(0)
        for i in range(k):
            if i + 1 < k:
                upload(i + 1)
            compute(i)

    e2e_run(4)  # both buffers: first sight, then capture of the factorization graphs
    torch.cuda.synchronize()
    barrier()
    a, c = ev(), ev()
    a.record(stream)
    e2e_run(e2e_steps)
    c.record(stream)
    c.synchronize()
    barrier()
    t_e2e = max_over_ranks(a.elapsed_time(c) / 1e3)
    solver.close()

    # CPU baseline (rank 0, one GPU only): the reference's CPU solve of this system.
    def section(fn, *a):
        # A side section that fails is reported in its key; the headline
        # solve above is never skipped by it.
        try:
            return fn(*a)
        except Exception as e:  # noqa: BLE001
            log(f"section {fn.__name__} failed: {e!r}")
            return {"error": repr(e)}

    fields = section(fields_section, ctx, mesh, fp64_peak, rank == 0 and world == 1 and not args.no_cpu)
    adjoint = section(adjoint_section, ctx, args.adjoint_steps, max_over_ranks) if args.adjoint_steps > 0 else None
    if adjoint is not None and "grads_per_s" in adjoint:
        adjoint["grads_per_s"] *= world
        adjoint["fp64_grads_per_s"] *= world
    with_cpu = rank == 0 and world == 1 and not args.no_cpu
    pec = section(pec_section, ctx, with_cpu) if not args.skip_sections else None
    # the FP64 complex GEMM runs on the FP64 tensor cores: its roof is their measured rate
    fp64_mma_peak = ctx.fp64_mma_peak()
    multi = section(multi_rhs_section, ctx, fp64_mma_peak, max_over_ranks) if not args.skip_sections else None
    sweep = section(sweep_section, ctx, max_over_ranks) if not args.skip_sections else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        secs, xc, kind, desc = cpu_reference_solve(Zh.numpy(), bh.numpy(), threads)
        cpu = {"value": 1.0 / secs, "unit": "solves/s", "cores": threads, "kind": kind,
               "sample": f"one N={N} complex128 factor+solve of the same assembled system ({desc})"}

    out = {}
    if rank == 0:
        peaks = measured_peaks()
        gemm_s = gemm["ms"] / 1e3
        total_dev_s = t_prof
        shares = {"tf32_gemm": gemm_s / total_dev_s, "trsv": trsv["ms"] / 1e3 / total_dev_s,
                  "fp64_matvec": gemv["ms"] / 1e3 / total_dev_s}
        tf32_peak = peaks["bf16_tflops"] / 2.0
        gemm_tflops = gemm["flops"] / gemm_s / 1e12 if gemm_s > 0 else 0.0
        gemm_gbs = gemm["bytes"] / gemm_s / 1e9 if gemm_s > 0 else 0.0
        # Which roof binds: the kernel's algorithmic intensity (flops per
        # byte of C read and written plus the packed operands) against the
        # ridge of the two measured peaks.
        intensity = gemm["flops"] / gemm["bytes"] if gemm["bytes"] else 0.0
        ridge = tf32_peak * 1e12 / (peaks["hbm_gbs"] * 1e9)
        hbm_bound = intensity < ridge
        roofline = {
            "kernel": "gemm_tf32_sub_persistent_kernel (split-TF32 trailing update, tcgen05)",
            "bound": "hbm" if hbm_bound else "tensor",
            "achieved": gemm_gbs if hbm_bound else gemm_tflops,
            "peak": peaks["hbm_gbs"] if hbm_bound else tf32_peak,
            "unit": "GB/s" if hbm_bound else "TFLOP/s",
            "frac": gemm_gbs / peaks["hbm_gbs"] if hbm_bound else gemm_tflops / tf32_peak,
            "intensity_flop_per_byte": intensity, "ridge_flop_per_byte": ridge,
            "tensor_tflops_achieved": gemm_tflops, "tensor_peak_tflops": tf32_peak,
            "tensor_frac": gemm_tflops / tf32_peak,
            "traffic": GEMM_DRAM_BYTES_PER_LAUNCH,
            "traffic_note": "mean dram read+write bytes per trailing-update launch, ncu over the 92 "
                            "launches of one N=6000 factorization",
            "algorithmic_bytes_per_launch": gemm["bytes"] / gemm["launches"] if gemm["launches"] else None,
            "peak_note": f"TF32 dense = {peaks['source']} bf16 {peaks['bf16_tflops']} TFLOP/s / 2",
            "launches": gemm["launches"], "hbm_gbs_achieved": gemm_gbs,
            "hbm_frac": gemm_gbs / peaks["hbm_gbs"], "time_share": shares,
            "trsv_gbs": trsv["bytes"] / (trsv["ms"] / 1e3) / 1e9 if trsv["ms"] > 0 else None,
            "fp64_matvec_gbs": gemv["bytes"] / (gemv["ms"] / 1e3) / 1e9 if gemv["ms"] > 0 else None,
            # mean device time per launch (ms) of the chain kernels and of the
            # two phases of a step (spans on the launching streams)
            "mean_ms": {k: (v["ms"] / v["launches"] if v["launches"] else None)
                        for k, v in [("tf32_gemm", gemm), ("trsv", trsv), *prof.items()]},
            "largest_launch": largest_launch_roofline(first_gemm, peaks, tf32_peak),
        }
        value = world * args.steps / t_mixed
        out = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_mixed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64+tf32x3/c128", "data": "synthetic",
            "config": bench_config(world),
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": world * e2e_steps / t_e2e, "unit": "solves/s",
                    "h2d_bytes_per_step": int(16 * N * N + 16 * N), "d2h_bytes_per_step": int(16 * N),
                    "steps": e2e_steps,
                    "pipelining": "step i+1's H2D copy overlaps step i (copy stream, two device buffers)"},
            "gpu_launches": int(launches), "clocks": clocks.summary(),
            "fp64_lu_solves_per_s": world / t_fp64, "speedup_vs_fp64_lu": (value / world) * t_fp64,
            "fp64_baseline": "own FP64 LU" if t_own <= t_cusolver else "cuSOLVER Zgetrf/Zgetrs",
            "fp64_cusolver_solves_per_s": world / t_cusolver, "fp64_own_lu_solves_per_s": world / t_own,
            "own_fp64_vs_cusolver_rel_diff": own_rel_diff,
            "relative_residual": rel_res, "rel_diff_vs_fp64_lu": rel_diff,
            "rcs_rel_rms_error_vs_mie": mie_err,
            "reference_gpu": ref_gpu,
            "refinement_iterations": max(iters), "assembly_seconds": t_asm,
            "assembly_green_evals_per_s": evals / t_asm,
            "assembly_roofline": {
                "bound": "fp64 pipe", "unit": "TFLOP/s",
                "flops_per_eval": ASSEMBLY_FLOPS_PER_EVAL,
                "achieved": evals * ASSEMBLY_FLOPS_PER_EVAL / t_asm / 1e12,
                "peak": fp64_peak, "peak_note": "measured FP64 FMA rate (sieb200_fp64_fma_peak)",
                "frac": evals * ASSEMBLY_FLOPS_PER_EVAL / t_asm / 1e12 / fp64_peak,
                "z_write_gbs": 16.0 * N * N / t_asm / 1e9,
            },
            "fields": fields,
            "pec_efie": pec,
            "multi_rhs": multi,
            "sweep": sweep,
            "adjoint": adjoint,
            "variants": variants,
        }
    torch.cuda.synchronize()
    return out if rank == 0 else {}


ADJOINT_WORKLOAD = ("SIE-GSTC adjoint synthesis: circular-arc spindle (arc radius 1.5 m, half-angle 60 deg), "
                    "revolved mesh 9800 faces / 14700 RWG edges (N=58800), f=300 MHz, Dunavant rule 5; "
                    "omega parameters (B, X, chi) per face (29400 reals, seeded, |chi^2-BX|>=0.25); "
                    "objective = far-field power in a 10 deg cone about +z; x-polarised plane wave along +z")


def fields_section(ctx, mesh, fp64_peak: float, with_cpu: bool) -> dict:
    """Surface-integral field values on a cut around the sphere: 361
    directions (phi = 0 and 90 degrees, theta in 1-degree steps) at 0.55 m
    (faces within 0.1 lambda of a point take the analytic part) and 3 m,
    seeded synthetic currents, vacuum, Dunavant rule 17. Timed through the
    public call (host points and currents in, host fields out)."""
    import sieb200
    th = np.radians(np.arange(181.0))
    dirs = np.concatenate([np.column_stack([np.sin(th), np.zeros_like(th), np.cos(th)]),
                           np.column_stack([np.zeros_like(th[1:-1]), np.sin(th[1:-1]), np.cos(th[1:-1])])])
    pts = np.concatenate([0.55 * dirs, 3.0 * dirs])
    rng = np.random.default_rng(5)
    ne = mesh.num_edges
    J = rng.standard_normal(ne) + 1j * rng.standard_normal(ne)
    M = 377.0 * (rng.standard_normal(ne) + 1j * rng.standard_normal(ne))
    call = lambda p: sieb200.evaluate_surface_integral_fields(mesh, J, M, p, C0, None, 17, ctx=ctx)  # noqa: E731
    call(pts)
    reps = 5
    t0 = time.perf_counter()
    for _ in range(reps):
        call(pts)
    t = (time.perf_counter() - t0) / reps
    Q = 61
    evals = float(pts.shape[0]) * mesh.num_faces * Q
    out = {"points": int(pts.shape[0]), "faces": mesh.num_faces, "rule": 17, "seconds": t,
           "points_per_s": pts.shape[0] / t, "evals_per_s": evals / t,
           "roofline": {"bound": "fp64 pipe", "flops_per_eval": FIELDS_FLOPS_PER_EVAL,
                        "achieved": evals * FIELDS_FLOPS_PER_EVAL / t / 1e12, "peak": fp64_peak,
                        "unit": "TFLOP/s", "frac": evals * FIELDS_FLOPS_PER_EVAL / t / 1e12 / fp64_peak}}
    if with_cpu:
        from oracle import oracle as O
        ref = O.reference()
        if ref is not None:
            sample = pts[::45]
            t0 = time.perf_counter()
            O.surface_fields(ref, mesh, J, M, sample, C0, rule=17)
            tc = time.perf_counter() - t0
            out["cpu_reference"] = {"points_per_s": sample.shape[0] / tc, "cores": 1, "kind": "reference",
                                    "sample": f"{sample.shape[0]} of the cut's points, the reference's own "
                                              "per-face helpers on one host thread (oracle/_ref)"}
    return out


def rcs_error_vs_mie(ctx, mesh, opts, radius: float, eps_r) -> dict:
    """Relative RMS difference of the bistatic RCS (181 theta in the phi = 0
    and 90 degree cuts) of the mixed solve from the Mie series (oracle/mie.py,
    pinned to the reference's spherical-wave solver); eps_r None: PEC."""
    import dataclasses as dc
    import sieb200
    from oracle import mie
    o = dc.replace(opts, solver="mixed_ir")
    if eps_r is None:
        r = sieb200.solve_pec_dense(mesh, o, sieb200.PlaneWaveExcitation(), ctx=ctx)
        J, M = r.currents, None
    else:
        r = sieb200.solve_dielectric_dense(mesh, o, sieb200.PlaneWaveExcitation(), ctx=ctx)
        J, M = r.currents[:mesh.num_edges], r.currents[mesh.num_edges:]
    mu0, eps0 = 1.25663706212e-6, 8.8541878128e-12
    k = 2 * math.pi * C0 * math.sqrt(mu0 * eps0)
    eta = math.sqrt(mu0 / eps0)
    th = np.linspace(0.0, np.pi, 181)
    num = den = 0.0
    for phi in (0.0, np.pi / 2):
        ph = np.full_like(th, phi)
        r_hat, t_hat, p_hat = sieb200.spherical_frames(th, ph)
        ft, fp, _ = sieb200.far_field(mesh, J, M, k, eta, r_hat, t_hat, p_hat, ctx=ctx)
        rcs = 4 * np.pi * (np.abs(ft) ** 2 + np.abs(fp) ** 2)
        ref = mie.bistatic_rcs(k, radius, eps_r, th, ph)
        num += float(np.sum((rcs - ref) ** 2))
        den += float(np.sum(ref ** 2))
    return math.sqrt(num / den)


def reference_gpu_section(ctx, mesh, opts, t_asm_lib: float):
    """The reference's own GPU path on this box (solve_dielectric_dense built
    for sm_100a from its sources: its assembly kernels, cusolverDnZgetrf /
    Zgetrs, its residual) on the benchmark system, against the library's
    currents (mixed solve) and assembly time."""
    import dataclasses as dc
    import sieb200
    from oracle import oracle as O
    lib = O.reference_gpu()
    if lib is None:
        return {"unavailable": "oracle/_ref/libsieref_gpu.so not built (make -C oracle ref_gpu REF=...)"}
    cur, t = O.reference_gpu_dielectric(lib, mesh, C0, 4.0, opts.quadrature_rule)
    r = sieb200.solve_dielectric_dense(mesh, dc.replace(opts, solver="mixed_ir"), sieb200.PlaneWaveExcitation(),
                                       ctx=ctx)
    t["currents_rel_diff_vs_library_mixed"] = float(np.linalg.norm(r.currents - cur) / np.linalg.norm(cur))
    t["library_assembly_seconds"] = t_asm_lib
    t["assembly_speedup"] = t["assembly_seconds"] / t_asm_lib
    t["what"] = ("the reference's solve_dielectric_dense compiled for sm_100a from its sources (oracle/Makefile "
                 "ref_gpu): assembly kernels, cuSOLVER Zgetrf/Zgetrs, residual (second assembly + Zgemv); "
                 "timings are the reference's own metrics")
    return t


PEC_WORKLOAD = ("PEC sphere r=1 m, T-EFIE, SphericalSurface(1, 3): 1280 faces / 1920 RWG edges (N=1920), "
                "k=2 pi (f=c0), Dunavant rule 5 (7 points), threshold 0.1 lambda0, x-polarised plane wave along +z, "
                "bistatic RCS at 181 theta in the phi=0 and phi=90 deg cuts")


def pec_section(ctx, with_cpu: bool) -> dict:
    """The PEC workload end to end through the public solver call (host mesh
    in, host currents out: assembly, factorization, solve, residual), its
    device-resident parts timed with CUDA events, the bistatic RCS cuts, and
    the reference's host path on the same inputs (its quadrature and Eigen
    LU from oracle/_ref; the far-field projection of its Python script as
    the oracle's C restatement)."""
    import torch
    import sieb200
    m = sieb200.icosphere(1.0, 3)
    N = m.num_edges
    th = np.linspace(0.0, np.pi, 181)
    frames = [sieb200.spherical_frames(th, np.full_like(th, ph)) for ph in (0.0, np.pi / 2)]
    r_hat = np.concatenate([f[0] for f in frames])
    t_hat = np.concatenate([f[1] for f in frames])
    p_hat = np.concatenate([f[2] for f in frames])
    out = {"workload": PEC_WORKLOAD, "N": N}
    for solver in ("lu_cusolver", "mixed_ir"):
        o = sieb200.PecOptions(frequency_hz=C0, quadrature_rule=5, singularity_threshold_lambda0=0.1, solver=solver)
        r = sieb200.solve_pec_dense(m, o, sieb200.PlaneWaveExcitation(), ctx=ctx)  # warm-up
        reps = 5
        t0 = time.perf_counter()
        for _ in range(reps):
            r = sieb200.solve_pec_dense(m, o, sieb200.PlaneWaveExcitation(), ctx=ctx)
        t = (time.perf_counter() - t0) / reps
        out[solver] = {"end_to_end_seconds": t, "solves_per_s": 1.0 / t,
                       "assembly_seconds": r.metrics["assembly_seconds"],
                       "factorization_seconds": r.metrics["factorization_seconds"],
                       "solve_seconds": r.metrics["solve_seconds"],
                       "relative_residual": r.metrics["relative_residual"]}
        if solver == "lu_cusolver":
            x64 = r.currents
        else:
            out["mixed_vs_fp64_rel_diff"] = float(np.linalg.norm(r.currents - x64) / np.linalg.norm(x64))
    s = {"mu0": 1.25663706212e-6, "eps0": 8.8541878128e-12}
    k = 2 * math.pi * C0 * math.sqrt(s["mu0"] * s["eps0"])
    eta = math.sqrt(s["mu0"] / s["eps0"])
    sieb200.far_field(m, x64, None, k, eta, r_hat, t_hat, p_hat, ctx=ctx)
    reps = 20
    t0 = time.perf_counter()
    for _ in range(reps):
        ft, fp, _ = sieb200.far_field(m, x64, None, k, eta, r_hat, t_hat, p_hat, ctx=ctx)
    t_ff = (time.perf_counter() - t0) / reps
    rcs = 4 * np.pi * (np.abs(ft) ** 2 + np.abs(fp) ** 2)
    out["rcs"] = {"directions": int(r_hat.shape[0]), "seconds": t_ff,
                  "monostatic_m2": float(rcs[180]), "forward_m2": float(rcs[0]),
                  "rel_rms_error_vs_mie": rcs_error_vs_mie(
                      ctx, m, sieb200.PecOptions(frequency_hz=C0, quadrature_rule=5,
                                                 singularity_threshold_lambda0=0.1), 1.0, None)}
    if with_cpu:
        from oracle import oracle as O
        ref = O.reference()
        lib = O.oracle()
        if ref is not None:
            threads = os.cpu_count() or 1
            sc = O.kernel_scalars(0, C0)
            om = O.icosphere(1.0, 3)
            t0 = time.perf_counter()
            Z = O.assemble(ref, 0, om, 5, sc, threads=threads, fn="ref_assemble")
            t_asm = time.perf_counter() - t0
            b = np.zeros(N, np.complex128)
            V = np.ascontiguousarray(om.vertices)
            E0, kh = np.array([1.0, 0, 0]), np.array([0, 0, 1.0])
            ref.ref_rhs_plane_wave(0, V.ctypes.data, om.faces.ctypes.data, om.faces_edges.ctypes.data,
                                   om.num_faces, om.num_edges, 5, E0.ctypes.data, kh.ctypes.data, k, eta, 2,
                                   sc["mu0"], sc["eps0"], b.ctypes.data, 0, 1.0, 1.0)
            t_lu, xc, kind, desc = cpu_reference_solve(Z, b, threads)
            t0 = time.perf_counter()
            O.far_field(lib, om, xc, None, k, eta, r_hat, t_hat, p_hat)
            t_ffc = time.perf_counter() - t0
            tot = t_asm + t_lu + t_ffc
            out["cpu_reference"] = {
                "seconds": tot, "solves_per_s": 1.0 / tot, "assembly_seconds": t_asm, "lu_seconds": t_lu,
                "far_field_seconds": t_ffc, "cores": threads, "kind": "reference",
                "sample": "the whole workload once: the reference's host quadrature and Eigen PartialPivLU "
                          "(oracle/_ref, all host threads), far field by the oracle's C restatement of "
                          "plot_far_field.py (one thread)",
                "currents_rel_diff_vs_gpu_fp64": float(np.linalg.norm(xc - x64) / np.linalg.norm(xc))}
            out["gpu_vs_cpu_end_to_end"] = tot / out["mixed_ir"]["end_to_end_seconds"]
    return out


MULTI_WORKLOAD = ("SIE-GSTC omega-bianisotropic sphere r=1 m, geodesic mesh 2880 faces / 4320 RWG edges "
                  "(N=17280: [J1, M1, J2, M2] per edge), f=c0 (ka=2 pi), Dunavant rule 17; per-face lossless "
                  "omega records (B, X, chi uniform in [-2, 2], seeded, |chi^2-BX|>=0.25); 64 plane waves, "
                  "theta uniform in [0, pi] (k in the xz-plane, E perpendicular in it), solved as one batch")


def multi_rhs_section(ctx, fp64_peak: float, max_over_ranks) -> dict:
    """Batch solves/s for 64 right-hand sides: the mixed factorization and
    the tensor-core multi-right-hand-side refinement against cuSOLVER
    Zgetrf + Zgetrs(nrhs = 64) on the same system, inputs resident."""
    import torch
    import sieb200
    m = sieb200.geodesic_sphere(1.0, 12)
    nf = m.num_faces
    rng = np.random.default_rng(2026)
    B_, X_, chi = (rng.uniform(-2, 2, nf) for _ in range(3))
    bad = np.abs(chi ** 2 - B_ * X_) < 0.25
    while bad.any():
        B_[bad], X_[bad], chi[bad] = (rng.uniform(-2, 2, int(bad.sum())) for _ in range(3))
        bad = np.abs(chi ** 2 - B_ * X_) < 0.25
    t = sieb200.omega_records(B_, X_, chi).numpy().reshape(nf, 32)
    o = sieb200.GstcSieOptions(frequency_hz=C0, quadrature_rule=17)
    N = 4 * m.num_edges
    nrhs = 64
    th = np.linspace(0.0, np.pi, nrhs)
    srcs = [sieb200.PlaneWaveExcitation(electric_amplitude=(np.cos(a), 0.0, -np.sin(a)),
                                        propagation_direction=(np.sin(a), 0.0, np.cos(a))) for a in th]
    stream = torch.cuda.ExternalStream(ctx.stream)
    Z = torch.empty((N, N), dtype=torch.complex128, device="cuda")
    t0 = time.perf_counter()
    sieb200.assemble_matrix_device(m, o, Z.data_ptr(), tensors=t, ctx=ctx)
    ctx.synchronize()
    t_asm = time.perf_counter() - t0
    Bh = sieb200.assemble_rhs(m, o, srcs, ctx=ctx)  # (N, nrhs) column-major
    B = torch.from_numpy(np.ascontiguousarray(Bh.T)).cuda()  # row c = column c: column-major N x nrhs
    X = torch.empty_like(B)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def timed(fn, reps):
        ts = []
        for _ in range(reps):
            a, c = ev(), ev()
            a.record(stream)
            fn()
            c.record(stream)
            c.synchronize()
            ts.append(a.elapsed_time(c) / 1e3)
        return ts

    mixed = sieb200.DenseLuSolver(N, "mixed_ir", ctx=ctx)
    iters = []

    def mixed_step():
        mixed.factorize(Z.data_ptr())
        with torch.cuda.stream(stream):
            X.copy_(B)
        iters.append(mixed.solve(X.data_ptr(), nrhs=nrhs, tolerance=1e-10, max_iterations=60))

    timed(mixed_step, 2)
    ctx.profile(True)
    mixed_step()
    prof = {name: ctx.profile_read(i) for i, name in [(0, "tf32_gemm"), (2, "fp64_gemm"), (5, "block_trsm"),
                                                      (6, "factorization"), (7, "refined_solve")]}
    ctx.profile(False)
    t_mixed = max_over_ranks(statistics.mean(timed(mixed_step, 3)))
    # accuracy: every column's FP64 residual
    R = B.clone()
    torch.cuda.synchronize()
    sieb200.zgemm(N, nrhs, N, Z.data_ptr(), X.data_ptr(), R.data_ptr(), alpha=-1.0, beta=1.0, ctx=ctx)
    res = (torch.linalg.vector_norm(R, dim=1) / torch.linalg.vector_norm(B, dim=1)).max().item()
    X_mixed = X.clone()
    mixed.close()
    fp64 = sieb200.DenseLuSolver(N, "lu_cusolver", ctx=ctx)
    Zw = torch.empty_like(Z)

    def fp64_step():
        with torch.cuda.stream(stream):
            Zw.copy_(Z)
            X.copy_(B)
        fp64.factorize(Zw.data_ptr())
        fp64.solve(X.data_ptr(), nrhs=nrhs)

    timed(fp64_step, 1)
    t_fp64 = max_over_ranks(statistics.mean(timed(fp64_step, 2)))
    rel = (torch.linalg.vector_norm(X_mixed - X) / torch.linalg.vector_norm(X)).item()
    fp64.close()
    del Zw
    np_ = ((N + 3) // 4) * 4
    trsm = prof["block_trsm"]
    gemm64 = prof["fp64_gemm"]
    tri_tflops = trsm["flops"] / (trsm["ms"] / 1e3) / 1e12 if trsm["ms"] > 0 else None
    return {
        "workload": MULTI_WORKLOAD, "N": N, "nrhs": nrhs, "assembly_seconds": t_asm,
        "batch_solves_per_s": 1.0 / t_mixed, "ms_per_batch": 1e3 * t_mixed,
        "rhs_per_s": nrhs / t_mixed, "fp64_batch_solves_per_s": 1.0 / t_fp64,
        "fp64_ms_per_batch": 1e3 * t_fp64, "speedup_vs_fp64_lu": t_fp64 / t_mixed,
        "max_relative_residual": res, "rel_diff_vs_fp64_lu": rel, "refinement_iterations": max(iters),
        "fp64": "cusolverDnZgetrf + Zgetrs with nrhs=64 on a copy of Z (the reference's batch solve path)",
        "profile_ms": {k: v["ms"] for k, v in prof.items()},
        "block_trsm": {"launches_of_applications": trsm["launches"],
                       "tf32_tflops": tri_tflops,
                       "packed_factor_gbs": trsm["bytes"] / (trsm["ms"] / 1e3) / 1e9 if trsm["ms"] > 0 else None,
                       "work_note": f"24 np^2 nrhs TF32 flops and 32 np^2 bytes of split [hi | lo] packed "
                                    f"factors per application, np={np_}"},
        "fp64_gemm": {"launches": gemm64["launches"],
                      "tflops": gemm64["flops"] / (gemm64["ms"] / 1e3) / 1e12 if gemm64["ms"] > 0 else None,
                      "peak_tflops": fp64_peak,
                      "peak_note": "measured FP64 tensor-core rate (sieb200_fp64_mma_peak)",
                      "frac": gemm64["flops"] / (gemm64["ms"] / 1e3) / 1e12 / fp64_peak if gemm64["ms"] > 0 else None},
    }


SWEEP_WORKLOAD = ("Batched sweep: 32 SIE-GSTC spheres r=1 m of uneven size (geodesic frequency n uniform in "
                  "6..14: 1080-5880 RWG edges, N=4320-23520), ka uniform in [pi, 4 pi], per-face reciprocal 4x4 "
                  "maps [[Y, K], [-K^T, Z]] with uniform complex entries (Y, Z symmetric, +2 I), seeded; Dunavant "
                  "rule 5; one x-polarised plane wave each; mixed solve to rel. residual 1e-10")


def sweep_instances(count: int = 32, seed: int = 4):
    import sieb200
    rng = np.random.default_rng(seed)
    insts = []
    for _ in range(count):
        n = int(rng.integers(6, 15))
        ka = float(rng.uniform(np.pi, 4 * np.pi))
        m = sieb200.geodesic_sphere(1.0, n)
        nf = m.num_faces
        c = lambda *sh: rng.uniform(-1, 1, sh) + 1j * rng.uniform(-1, 1, sh)  # noqa: E731
        Y = c(nf, 2, 2)
        Y = (Y + Y.transpose(0, 2, 1)) / 2 + 2 * np.eye(2)
        Zm = c(nf, 2, 2)
        Zm = (Zm + Zm.transpose(0, 2, 1)) / 2 + 2 * np.eye(2)
        K = 0.5 * c(nf, 2, 2)
        L = np.concatenate([np.concatenate([Y, K], 2), np.concatenate([-K.transpose(0, 2, 1), Zm], 2)], 1)
        t = np.concatenate([L.reshape(nf, 16), np.linalg.inv(L).reshape(nf, 16)], 1)
        o = sieb200.GstcSieOptions(frequency_hz=ka * C0 / (2 * np.pi), quadrature_rule=5, solver="mixed_ir")
        insts.append(sieb200.SweepInstance(m, t, o, exterior=sieb200.PlaneWaveExcitation()))
    return insts


def sweep_section(ctx, max_over_ranks) -> dict:
    """Config-4 sweep through sieb200_solve_gstc_sweep: the instances one
    after another (one lane) against the autotuned lane count (each
    candidate timed once here and cached by sieb200.autotune)."""
    import sieb200
    from sieb200 import autotune
    insts = sweep_instances()
    sizes = [4 * i.mesh.num_edges for i in insts]
    res, _ = sieb200.solve_gstc_sweep_batched(insts, concurrency=4, ctx=ctx)  # warm-up
    best, timings = autotune.tune_sweep(insts, ctx=ctx)
    t_seq = max_over_ranks(timings[1])
    t_best = max_over_ranks(timings[best])
    res, _ = sieb200.solve_gstc_sweep_batched(insts, concurrency=best, ctx=ctx)
    flops = sum(8.0 * float(n) ** 3 for n in sizes)  # split-TF32 LU: 3 x (8/3) N^3
    return {"workload": SWEEP_WORKLOAD, "instances": len(insts), "N_min": min(sizes), "N_max": max(sizes),
            "sequential_seconds": t_seq, "sequential_solves_per_s": len(insts) / t_seq,
            "batched_seconds": t_best, "batched_solves_per_s": len(insts) / t_best,
            "speedup_vs_sequential": t_seq / t_best, "autotuned_concurrency": best,
            "seconds_by_concurrency": {str(k): v for k, v in timings.items()},
            "max_relative_residual": max(r.metrics["relative_residual"] for r in res),
            "max_refinement_iterations": max(r.metrics["refinement_iterations"] for r in res),
            "tf32_tflops_effective": flops / t_best / 1e12,
            "timing": "wall clock around the library call (host tensors in, host currents out)"}


def adjoint_section(ctx, steps: int, max_over_ranks):
    """Gradients/s of a far-field objective with respect to the per-face omega
    parameters: assembly, factorization and refined solve forward, one
    conjugate-transpose solve plus the tensor contraction backward."""
    import torch
    import sieb200
    m = sieb200.revolved_spindle()
    o = sieb200.GstcSieOptions(frequency_hz=3e8, quadrature_rule=5)
    rng = np.random.default_rng(20260)
    nf = m.num_faces
    B, X, chi = (rng.uniform(-2, 2, nf) for _ in range(3))
    bad = np.abs(chi ** 2 - B * X) < 0.25
    while bad.any():
        B[bad], X[bad], chi[bad] = (rng.uniform(-2, 2, int(bad.sum())) for _ in range(3))
        bad = np.abs(chi ** 2 - B * X) < 0.25
    params = [torch.tensor(v, dtype=torch.float64, requires_grad=True) for v in (B, X, chi)]
    b = torch.from_numpy(sieb200.assemble_rhs(m, o, [sieb200.PlaneWaveExcitation()], ctx=ctx)[:, 0].copy()).cuda()
    obj = sieb200.FarFieldConeObjective(m, o, half_angle_deg=10.0, ctx=ctx)

    def grad(method):
        for p in params:
            p.grad = None
        x = sieb200.gstc_solve(sieb200.omega_records(*params), b, m, o, method=method, tolerance=1e-10, ctx=ctx)
        L = obj(x)
        L.backward()
        return float(L.detach()), torch.cat([p.grad for p in params]).clone()

    def timed(method, n):
        out = None
        t = []
        for _ in range(n):
            torch.cuda.synchronize()
            a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            out = grad(method)
            c.record()
            c.synchronize()
            t.append(a.elapsed_time(c) / 1e3)
        return out, t

    grad("mixed_ir")  # warm-up (workspaces, module loading)
    (L_mx, g_mx), t_mx = timed("mixed_ir", steps)
    (L_64, g_64), t_64 = timed("lu_cusolver", 1)
    t_mx_s = max_over_ranks(statistics.mean(t_mx))
    t_64_s = max_over_ranks(statistics.mean(t_64))
    return {
        "workload": ADJOINT_WORKLOAD, "N": 4 * m.num_edges, "method": "mixed_ir (split-TF32 LU + FP64 FGMRES, "
        "adjoint: conjugate-transpose FGMRES on the same factors)",
        "grads_per_s": 1.0 / t_mx_s, "ms_per_grad": 1e3 * t_mx_s, "steps": steps,
        "fp64_grads_per_s": 1.0 / t_64_s, "speedup_vs_fp64": t_64_s / t_mx_s,
        "objective": L_mx, "objective_rel_diff_vs_fp64": abs(L_mx - L_64) / abs(L_64),
        "grad_rel_diff_vs_fp64": float((g_mx - g_64).norm() / g_64.norm()),
        "timing": "CUDA events around device-synchronized gradient evaluations",
    }


def largest_launch_roofline(span, peaks, tf32_peak):
    """The first trailing update of the N = 6016 factorization (block step
    0: C = 2m x (m - 64) real with m = 5952, split packs 256 wide) from its
    in-situ timeline span: time against max(bytes / HBM, flops / TF32)."""
    if not span:
        return None
    np_, nb = 6016, 64
    m = np_ - nb
    rows, cols, k = 2 * m, m - nb, 256
    alg_bytes = 4.0 * (2.0 * rows * cols + (rows + cols) * k)
    flops = 2.0 * rows * cols * 384
    t = (span[1] - span[0]) / 1e3
    roof = max(alg_bytes / (peaks["hbm_gbs"] * 1e9), flops / (tf32_peak * 1e12))
    return {"us": t * 1e6, "algorithmic_bytes": alg_bytes, "tf32_flops": flops, "roofline_us": roof * 1e6,
            "frac_of_roofline": roof / t, "hbm_frac": alg_bytes / t / (peaks["hbm_gbs"] * 1e9),
            "tensor_frac": flops / t / (tf32_peak * 1e12)}


def timeline_summary(spans):
    """Critical path of one factorization and solve from the library's
    timeline [(kind, start_ms, end_ms)]: kinds 0 trailing GEMM, 1 triangular
    solve, 2 FP64 matvec, 3 diagonal block, 4 panels, 6 factorization,
    7 refined solve. A block step runs panels(k), then the GEMM of step k
    beside the next diagonal block. Split panels (a head launch on the
    lookahead stream beside the rest) overlap in time and count as one
    panels span of their step."""
    span = {k: [(a, b) for kk, a, b in spans if kk == k] for k in range(8)}
    total = {name: sum(b - a for a, b in span[k]) for k, name in
             [(0, "gemm_ms"), (1, "trsv_ms"), (2, "matvec_ms"), (3, "diag_ms"), (4, "panels_ms")]}
    pan = []
    for a, b in sorted(span[4]):
        if pan and a <= pan[-1][1] + 0.005:
            pan[-1] = (pan[-1][0], max(pan[-1][1], b))
        else:
            pan.append((a, b))
    gem, dia = span[0], span[3]
    steps = []
    for k in range(len(pan) - 1):
        g = [b - a for a, b in gem if pan[k][1] - 1e-6 <= a < pan[k + 1][0]]
        d = [b - a for a, b in dia if pan[k][0] - 1e-6 <= a < pan[k + 1][0]]
        steps.append((pan[k + 1][0] - pan[k][1], g[0] if g else 0.0, d[0] if d else 0.0))
    fact = span[6][0][1] - span[6][0][0] if span[6] else None
    solve = span[7][0][1] - span[7][0][0] if span[7] else None
    return {"factorization_ms": fact, "refined_solve_ms": solve, **total,
            "steps_bound_by_gemm": sum(1 for _, g, d in steps if g > d),
            "steps_bound_by_diag": sum(1 for _, g, d in steps if g <= d),
            "sum_max_gemm_diag_ms": sum(max(g, d) for _, g, d in steps),
            "gaps_ms": sum(t - max(g, d) for t, g, d in steps),
            "trsv_us": [round(1e3 * (b - a), 1) for a, b in span[1]],
            "matvec_us": [round(1e3 * (b - a), 1) for a, b in span[2]]}


def run_case(args):
    """One small workload for a profiler capture (ncu -k <kernel> -c <n>):
    no timing, one short JSON summary. Cases:
      assembly       T-PMCHWT assembly of the 2000-face sphere, Dunavant rule 17 (twice)
      assembly_small T-PMCHWT assembly of a 320-face icosphere (r = 0.5), rule 17 (twice)
      factorization  mixed factorization of that system (N = 6000), twice
      multi_rhs      mixed solve of 64 plane-wave right-hand sides of it
      fp64_lu        own FP64 LU factorization and solve of it
      residual       four FP64 residual matvecs b - Z x of that system (576 MB each)
      timeline       one mixed factorization and refined solve of it with the
                     library's per-launch timeline (after three warm-up solves);
                     prints the critical-path summary
    """
    import torch
    import sieb200
    ctx = sieb200.Context(0)
    mesh, opts = build_problem(17)
    if args.case == "assembly_small":
        mesh = sieb200.icosphere(0.5, 2)
    N = 2 * mesh.num_edges
    Z = torch.empty((N, N), dtype=torch.complex128, device="cuda")
    for _ in range(2 if args.case.startswith("assembly") else 1):
        sieb200.assemble_matrix_device(mesh, opts, Z.data_ptr(), ctx=ctx)
    ctx.synchronize()
    out = {"case": args.case, "N": N}
    if args.case == "factorization":
        s = sieb200.DenseLuSolver(N, "mixed_ir", ctx=ctx)
        for _ in range(2):
            s.factorize(Z.data_ptr())
        ctx.synchronize()
        s.close()
    elif args.case in ("multi_rhs", "fp64_lu"):
        th = np.linspace(0.0, np.pi, 64 if args.case == "multi_rhs" else 1)
        srcs = [sieb200.PlaneWaveExcitation(electric_amplitude=(np.cos(a), 0.0, -np.sin(a)),
                                            propagation_direction=(np.sin(a), 0.0, np.cos(a))) for a in th]
        B = torch.from_numpy(np.ascontiguousarray(sieb200.assemble_rhs(mesh, opts, srcs, ctx=ctx).T)).cuda()
        s = sieb200.DenseLuSolver(N, "mixed_ir" if args.case == "multi_rhs" else "lu_fp64", ctx=ctx)
        s.factorize(Z.data_ptr())
        torch.cuda.synchronize()
        out["iterations"] = s.solve(B.data_ptr(), nrhs=len(srcs), tolerance=1e-10, max_iterations=60)
        ctx.synchronize()
        s.close()
    elif args.case == "residual":
        g = torch.Generator(device="cuda").manual_seed(5)
        x = torch.randn(N, dtype=torch.complex128, device="cuda", generator=g)
        y = torch.randn(N, dtype=torch.complex128, device="cuda", generator=g)
        torch.cuda.synchronize()
        for _ in range(4):
            sieb200.matvec(N, Z.data_ptr(), x.data_ptr(), y.data_ptr(), beta=-1.0, ctx=ctx)
        ctx.synchronize()
        out["y_norm"] = float(y.norm())
    elif args.case == "timeline":
        b = torch.from_numpy(sieb200.assemble_rhs(mesh, opts, [sieb200.PlaneWaveExcitation()], ctx=ctx)[:, 0]
                             .copy()).cuda()
        s = sieb200.DenseLuSolver(N, "mixed_ir", ctx=ctx)
        for i in range(4):
            if i == 3:
                ctx.profile(True, timeline=True)
            s.factorize(Z.data_ptr())
            x = b.clone()
            torch.cuda.synchronize()
            s.solve(x.data_ptr(), tolerance=1e-10, max_iterations=60)
            ctx.synchronize()
        spans = sorted(ctx.profile_timeline(), key=lambda v: v[1])
        ctx.profile(False)
        s.close()
        out.update(timeline_summary(spans))
    elif not args.case.startswith("assembly"):
        raise SystemExit(f"unknown case {args.case}")
    del Z
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    ctx.close()
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 200; the reference arm, one CPU solve per step, 20)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sieb200", choices=["sieb200", "reference"])
    ap.add_argument("--rule", type=int, default=17)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline solve")
    ap.add_argument("--skip-sections", action="store_true",
                    help="time only the headline solve (no PEC or 64-right-hand-side sections)")
    ap.add_argument("--adjoint-steps", type=int, default=2,
                    help="timed adjoint gradients on the spindle workload (0 skips them)")
    ap.add_argument("--case", default=None, help="run one small profiling workload (see run_case) and exit")
    args = ap.parse_args()
    if args.case:
        run_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run(args)


if __name__ == "__main__":
    main()
