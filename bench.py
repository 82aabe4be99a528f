"""Benchmark: acc solve ms per k-point, mixed vs FP64 at |d eps| <= 1e-8 eV,
plus the force-adjoint cost, on the 12-atom HfO2-like cell (Gamma, 48^3 box,
~3400 plane waves, 64 bands, PBE, MIMIC_US D_ij) -- synthetic seeded inputs
with the reference's CHGCAR/POTCAR formats.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = one complete acc solve of every k point this rank owns, from
operator preparation to converged eigenpairs, through the C ABI.  `value`
is the whole-job ms per k-point (max over ranks / k points of all ranks).
k points are independent units: ranks take them cyclically (the reference's
MPI ownership rule); a workload with fewer k points than ranks runs replicas.
There is no data-path collective.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "deepaw-half_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "acc solve ms per k-point, mixed vs FP64 at |d eps|<=1e-8 eV; force-adjoint ms"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="hfo2")
    p.add_argument("--tol", type=float, default=2e-5,
                   help="ACC residual tolerance (eV); 2e-5 keeps |d eps| below 1e-8 eV on this workload in both modes")
    p.add_argument("--max-iter", type=int, default=2000)
    p.add_argument("--block", type=int, default=16)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp64", action="store_true", help="skip the FP64-mode comparison run")
    p.add_argument("--cpu-sample-s", type=float, default=15.0)
    p.add_argument("--no-check", action="store_true",
                   help="skip the dense FP64 reference eigenvalues (profiling runs; |d eps| reported as null)")
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def owned(kpts, rank, world):
    from halfb200.shard import owned_indices
    idx = owned_indices(len(kpts), rank, world)
    return kpts[idx] if len(idx) else kpts[:1]


class Clocks:
    """nvidia-smi sampler running during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], 0.0, set()
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 7:
                    continue
                try:
                    sm.append(float(f[0]))
                    mx = max(mx, float(f[1]))
                except ValueError:
                    continue
                for n, v in zip(names, f[3:7]):
                    if v.lower() == "active":
                        reasons.add(n)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def committed_traffic():
    """Per-launch DRAM traffic of the local-operator kernels from the committed
    ncu summary (profiles/local_operator_hfo2.md), if present."""
    path = os.path.join(ROOT, "profiles", "local_operator_hfo2.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_band:"):
                return float(line.split(":")[1])
    except (OSError, ValueError):
        pass
    return None


class CpuBaseline:
    """The oracle's FP64 acc restatement timed on this host for a bounded number
    of iterations, scaled to the iteration count the FP64 solve of the same
    workload needs (same algorithm, same tolerance)."""

    def __init__(self, w, ch, po):
        from oracle import hamiltonian as H
        try:
            from threadpoolctl import threadpool_info
            self.cores = max((i.get("num_threads", 1) for i in threadpool_info()), default=1)
        except Exception:
            self.cores = os.cpu_count() or 1
        self.w = w
        self.sysm = H.load_system(ch, po, w.encut, use_pbe=(w.xc == "pbe"), use_uspp=True)
        from oracle.basis import build_basis
        self.npw = build_basis(self.sysm.crystal, w.grid, w.encut, w.kpoints[0]).npw

    def measure(self, fp64_iterations, sample_s):
        from oracle import hamiltonian as H, acc
        w = self.w
        t0 = time.perf_counter()
        op = H.prepare(self.sysm, w.kpoints[0])
        t_prep = time.perf_counter() - t0
        iters = 1
        while True:   # grow the sample until it uses the budget
            t0 = time.perf_counter()
            acc.solve_acc(op, w.nbands, tol=1e-300, max_iterations=iters)
            dt = time.perf_counter() - t0
            t_it = dt / iters
            if dt * 2.5 > sample_s or iters >= 64:
                break
            iters *= 2
        ms = (t_prep + t_it * max(fp64_iterations, 1)) * 1e3
        return {"value": ms, "unit": "ms/k-point", "cores": int(self.cores), "kind": "port",
                "sample": f"oracle FP64 acc restatement (numpy/scipy), {w.name} Gamma: operator preparation + "
                          f"{iters} iterations timed ({t_it * 1e3:.1f} ms/iteration), scaled to the "
                          f"{fp64_iterations} iterations the FP64 solve needs at this tolerance"}


def workload_config(w, npw, args, nk, world, l2):
    """The `config` object both arms print for the same workload."""
    return {"workload": f"{w.name}: {w.nions} atoms, Gamma, {w.grid[0]}^3 box, {npw} plane waves, "
                        f"{w.nbands} bands, PBE, MIMIC_US D_ij", "tol_eV": args.tol,
            "block": args.block, "kpoints_per_rank": nk, "l2": l2,
            "parallelism": f"k-point ownership x{world}" if world > 1 else "single GPU"}


def cpu_baseline(w, ch, po, fp64_iterations, sample_s):
    return CpuBaseline(w, ch, po).measure(fp64_iterations, sample_s)


def write_inputs(w, rank):
    from halfb200 import synth
    d = os.path.join(tempfile.gettempdir(), f"half_bench_{w.name}_{os.getpid()}_{rank}")
    return synth.write_inputs(w, d)


def run_reference(args, rank, world):
    if rank != 0:
        return
    from halfb200 import synth
    w = synth.workload(args.workload)
    ch, po = write_inputs(w, rank)
    iters = reference_iterations(args) or args.max_iter
    base = CpuBaseline(w, ch, po)
    samples = []
    budget = max(2.0, 4 * args.cpu_sample_s / max(1, args.warmup + args.steps))
    for i in range(max(args.warmup, 0) + max(args.steps, 1)):
        cb = base.measure(iters, budget)
        if i >= args.warmup:
            samples.append(cb["value"])
    v = statistics.mean(samples)
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "ms/k-point", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": workload_config(w, base.npw, args, len(owned(w.kpoints, 0, 1)), 1, "n/a (host)"),
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "ms/k-point", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# Iterations the reference acc algorithm (the oracle's FP64 restatement, LAPACK
# small solves) needs to reach a residual tolerance on a workload, from
# complete oracle runs to convergence on one host: hfo2 at 3e-5 eV, 234
# iterations (228 s, max |d eps| = 5.8e-9 eV against the dense solve); at
# 2e-5 eV, 267 iterations (267 s, 5.7e-9 eV).  A complete run is minutes of
# CPU time, so the reference arm times a bounded sample of iterations and
# scales it by this count.
REFERENCE_ITERATIONS = {("hfo2", 3e-5): 234, ("hfo2", 2e-5): 267}


def reference_iterations(args):
    for (name, tol), its in REFERENCE_ITERATIONS.items():
        if name == args.workload and abs(args.tol - tol) < 1e-12:
            return its
    return None


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import halfb200
    from halfb200 import synth
    halfb200.load_library()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    w = synth.workload(args.workload)
    ch, po = write_inputs(w, rank)
    kpts = owned(w.kpoints, rank, world)
    nk = len(kpts)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > L2

    # ---- FP64 dense reference eigenvalues (untimed)
    if args.no_check:
        dense = None
    else:
        with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="evd") as dctx:
            dense = [dctx.solve(k, w.nbands)[0] for k in kpts]

    def run_mode(ctx, precision, steps, warmup):
        ctx.set_acc(tol=args.tol, max_iterations=args.max_iter, block_size=args.block, precision=precision)
        dev_ms, wall_ms, infos, errs = [], [], [], []
        for i in range(warmup + steps):
            flush.fill_(float(i))
            torch.cuda.synchronize()
            barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eig = ctx.solve_kpoints(kpts, w.nbands)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            barrier()
            inf = ctx.info()
            if i >= warmup:
                dev_ms.append(max_over_ranks(inf["device_ms"]))
                wall_ms.append(max_over_ranks((t1 - t0) * 1e3))
                infos.append(inf)
                if dense is not None:
                    errs.append(max(float(np.abs(e - d).max()) for e, d in zip(eig, dense)))
        return dev_ms, wall_ms, infos, errs

    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="acc") as ctx:
        fp64 = fp64g = None
        if not args.no_fp64:
            fp64 = run_mode(ctx, "fp64", max(1, min(args.steps, 2)), 1)
            fp64g = run_mode(ctx, "fp64_guarded", max(1, min(args.steps, 2)), 1)
        with Clocks(local) as clk:
            dev_ms, wall_ms, infos, errs = run_mode(ctx, "mixed", args.steps, args.warmup)
        clocks = clk.summary()
        # ---- end-to-end through the C ABI with host buffers: half_solve_kpoint with an eigenvector buffer
        ctx.set_acc(tol=args.tol, max_iterations=args.max_iter, block_size=args.block, precision="mixed")
        e2e_ms = []
        npw = [ctx.npw(k) for k in kpts]
        for i in range(max(1, args.steps)):
            flush.fill_(float(i))
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            for k in kpts:
                ctx.solve(k, w.nbands, vectors=True)
            t1 = time.perf_counter()
            barrier()
            e2e_ms.append(max_over_ranks((t1 - t0) * 1e3))
        # ---- force adjoint vs one forward sweep (FP64), on the dense eigenpairs of the first k point
        k0 = kpts[0]
        with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="evd") as fctx:
            e0, v0, _, _ = fctx.solve(k0, w.nbands, vectors=True)
            occ = np.where(np.arange(w.nbands) < int(w.nelect // 2), 2.0, 0.0)
            adj, sweep = [], []
            for i in range(3 + max(1, args.steps)):
                fctx.nonlocal_forces(k0, v0, e0, occ, 1.0)
                a = fctx.info()["adjoint_ms"]
                fctx.apply_hs(k0, v0)
                s = fctx.info()["sweep_ms"]
                if i >= 3:
                    adj.append(a)
                    sweep.append(s)
    nk_total = nk * world
    ms_step = statistics.mean(dev_ms)
    value = ms_step / nk_total
    peaks, peak_kind = measured_peaks()
    loc_ms = sum(i["local_ms"] for i in infos)
    loc_bytes = sum(i["local_bytes"] for i in infos)
    loc_cols = sum(i["local_columns"] for i in infos)
    sweeps = max(1, sum(i["sweep_columns"] for i in infos) // max(1, w.nbands))
    achieved = loc_bytes / (loc_ms * 1e-3) / 1e9 if loc_ms > 0 else None
    traffic_per_band = committed_traffic()
    fp64_iters = int(statistics.mean(i["iterations"] for i in fp64[2])) if fp64 else None
    line = {
        "metric": METRIC, "value": value, "unit": "ms/k-point", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64/c128 (mixed: FP32 operator and GEMMs, FP64 small solves and refinement)",
        "data": "synthetic (seeded CHGCAR/POTCAR in the reference formats)",
        "config": workload_config(w, npw[0], args, nk, world, "flushed between steps (256 MB write)"),
        "max_abs_d_eps_eV": max(errs) if errs else None,
        "per_step": [{"ms": round(t, 3), "iterations": i["iterations"], "fp64_iterations": i["fp64_iterations"]}
                     for t, i in zip(dev_ms, infos)],
        "iterations": int(statistics.mean(i["iterations"] for i in infos)),
        "fp64_refinement_iterations": int(statistics.mean(i["fp64_iterations"] for i in infos)),
        "wall_ms_per_step": statistics.mean(wall_ms),
        "fp64_mode": ({"ms_per_k": statistics.mean(fp64[0]) / nk_total, "iterations": fp64_iters,
                       "max_abs_d_eps_eV": max(fp64[3]) if fp64[3] else None} if fp64 else None),
        "mixed_speedup_vs_fp64": (statistics.mean(fp64[0]) / ms_step) if fp64 else None,
        "fp64_guarded_mode": ({"ms_per_k": statistics.mean(fp64g[0]) / nk_total,
                               "iterations": int(statistics.mean(i["iterations"] for i in fp64g[2])),
                               "max_abs_d_eps_eV": max(fp64g[3]) if fp64g[3] else None} if fp64g else None),
        "mixed_speedup_vs_fp64_guarded": (statistics.mean(fp64g[0]) / ms_step) if fp64g else None,
        "force_adjoint_ms": statistics.mean(adj), "forward_sweep_ms": statistics.mean(sweep),
        "force_over_sweep": statistics.mean(adj) / statistics.mean(sweep),
        "roofline": {"kernel": "local operator (K1 sphere->planes, K2 x-lines*Veff, K3 planes->sphere), FP32",
                     "bound": "hbm", "achieved": achieved, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                     "frac": (achieved / peaks["hbm_gbs"]) if achieved else None,
                     "peak_source": peak_kind,
                     "traffic": (traffic_per_band * loc_cols / max(1, sweeps)) if traffic_per_band else None,
                     "algorithmic_bytes_per_launch": loc_bytes / max(1, sweeps)},
        "clocks": clocks,
        "gpu_launches": int(sum(i["kernel_launches"] for i in infos)),
        "e2e": {"value": statistics.mean(e2e_ms) / nk_total, "unit": "ms/k-point",
                "h2d_bytes_per_step": 24 * nk,
                "d2h_bytes_per_step": sum(8 * w.nbands + 16 * n * w.nbands for n in npw)},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref_iters = reference_iterations(args)
        line["cpu_baseline"] = cpu_baseline(w, ch, po, ref_iters or fp64_iters or line["iterations"],
                                            args.cpu_sample_s)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
