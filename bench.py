"""Benchmark of the B200 pour engine: simulated seconds per wall second of the 4 mm gentle pour.

One step is one substep of the pour (binning, particle-to-grid, pressure solve, extrapolation,
density correction, advection). The timed region runs K substeps after W warm-up substeps, from a
mid-pour state (by default 3 s into the pour: the pot tilted, liquid in the spout), each substep one
launch of the production substep graph bracketed by CUDA events on the engine's stream, with a
256 MiB buffer written before each substep (outside the bracket) so every substep starts with a cold
L2. The reported value is the simulated time those K substeps covered divided by their summed
device time. The per-stage split comes from a second replica from the same start whose graph holds
stage events.

`e2e` repeats the measurement through the public C ABI call a host program makes per substep
(pl_step: host->device control block, the substep, device->host stats block), timed by the host
clock around each call. `whole_pour` runs the reference's own benchmark loop (benchmarks/run3d.ts:
the whole pour until 1.5 s after the controller is done, pl_advance in 0.5 s chunks) with the
Chebyshev and the multigrid preconditioner, and compares the poured volume and layer shares with the
reference CPU solver's result. The reference arm (--impl reference) times the CPU FP64 restatement of
the reference solver on the same workload (the reference itself is TypeScript and no JavaScript
runtime exists on the box).

Supplementary measurements in the same line: `poisson_batch` solves the isolated pressure-Poisson
batch (64 snapshots of 128^3 per GPU) with multigrid- and MIC(0)-preconditioned CG, each timed with
CUDA events around the public pl_poisson_solve call on inputs resident in HBM (671 MB, larger than
L2), beside the CPU FP64 oracle on a bounded sample; `full_domain` and `ensemble` time the 2.5 mm
full-domain APIC pour and the 256-pour ensemble.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU: torchrun --nproc-per-node N bench.py --gpus N: every rank runs its own replica of the
pour (the single pour does not shard); value is the sum over ranks, timed as the max over ranks. The
Poisson batch and the ensemble are partitioned over the ranks by estimated cost.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "gentle 400 mL pour, 4 mm cells, half pot (81x81x22 grid, 88,856 parcels), seed 1"
# kernels per substep: controller, bin count/scan/place/permute, p2g cells + faces, density, solve set-up,
# 2x extrapolation, advect, and the solves: MIC(0) one kernel per system; Chebyshev one cluster launch for both
# systems plus the two gated MIC(0) fallbacks (at the default 16 x 512 shape four cells per thread add no
# capacity, so no second cluster launch); multigrid its set-up, one cluster launch and one fallback per system
KERNELS_PER_SUBSTEP = {"mic0": 14, "cheb": 15, "mg": 17}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cell-mm", type=float, default=4.0)
    ap.add_argument("--precond", default="cheb", choices=["mic0", "mg", "cheb"])
    ap.add_argument("--solve-shape", default="16x512",
                    help="cluster CTAs x threads of the cluster solves, or 'auto' (pl_autotune_solver, untimed)")
    ap.add_argument("--precision", default="mixed", choices=["f64", "mixed"],
                    help="solver vectors: mixed = FP32 stencils/Chebyshev with FP64 inner products and FP64 "
                         "true-residual refinement; f64 = all FP64")
    ap.add_argument("--start", type=float, default=3.0,
                    help="simulated seconds to advance before warm-up (3 s: the pot tilted, liquid in the spout)")
    ap.add_argument("--whole-pour", type=int, default=1,
                    help="1: also time the whole pour (run3d.ts rule) with Chebyshev and multigrid PCG")
    ap.add_argument("--cpu-sample", type=int, default=60, help="substeps of the CPU baseline sample")
    ap.add_argument("--poisson-n", type=int, default=128, help="grid of the isolated Poisson batch (0: skip it)")
    ap.add_argument("--poisson-count", type=int, default=64, help="snapshots of the isolated Poisson batch per GPU")
    ap.add_argument("--poisson-cpu-sample", type=int, default=4, help="snapshots the CPU oracle solves as its sample")
    ap.add_argument("--full-mm", type=float, default=2.5,
                    help="cell size of the full-domain APIC pour on the grid-scale solves (0: skip it)")
    ap.add_argument("--full-start", type=float, default=1.5, help="simulated seconds before its timed substeps")
    ap.add_argument("--full-steps", type=int, default=100, help="its timed substeps (grid-scale multigrid PCG)")
    ap.add_argument("--learned-train-s", type=float, default=45.0,
                    help="seconds of network training for its learned-PCG leg (0: skip the leg)")
    ap.add_argument("--learned-steps", type=int, default=10, help="timed substeps of the learned-PCG leg")
    ap.add_argument("--ensemble-count", type=int, default=256, help="pours of the seeded ensemble (0: skip it)")
    ap.add_argument("--ensemble-mm", type=float, default=5.0, help="cell size of the ensemble's pours")
    ap.add_argument("--ensemble-steps", type=int, default=40, help="timed substeps per pour of the ensemble")
    return ap.parse_args()


def make_cfg(args):
    from teapotfluidsimulation_b200 import abi

    cfg = abi.gentle_pour(args.cell_mm, 20.0)
    cfg.preconditioner = {"mic0": abi.PRECOND_MIC0, "mg": abi.PRECOND_MG, "cheb": abi.PRECOND_CHEB}[args.precond]
    cfg.solve_precision = abi.SOLVE_MIXED if args.precision == "mixed" else abi.SOLVE_F64
    if args.solve_shape != "auto":
        cfg.solve_cluster, cfg.solve_threads = (int(v) for v in args.solve_shape.split("x"))
    else:
        if not hasattr(make_cfg, "tuned"):
            from teapotfluidsimulation_b200 import engine as E

            make_cfg.tuned = E.autotune_solver(cfg, 8)[:2]
        cfg.solve_cluster, cfg.solve_threads = make_cfg.tuned
    return cfg


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def allmax(x: float, world: int, device: str = "cuda") -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allsum(x: float, world: int, device: str = "cuda") -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


class Clocks:
    """nvidia-smi samples of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        import tempfile

        self.path = os.path.join(tempfile.gettempdir(), f"pourlab_clocks_{os.getpid()}.csv")

    def start(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    mx = float(p[2])
                except ValueError:
                    continue
                for name, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(name)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the pressure PCG kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "k_chebpcg_4mm_full.md")
    try:
        with open(path) as f:
            for line in f:
                m = re.match(r"\s*traffic_bytes_per_launch:\s*([0-9.eE+]+)", line)
                if m:
                    return float(m.group(1))
    except OSError:
        pass
    return None


def pcg_bytes_per_iteration(m: int, precond: str, precision: str) -> float:
    """Algorithmic bytes of one PCG iteration over m liquid cells, each array counted once per pass.

    MIC(0) in FP64: apply A (s, 6 neighbour indices, diagonal, write As: 8+24+8+8), s.As (16),
    q/r update (read q, s, r, As, write q, r: 48), the two MIC(0) sweeps (r or qv, pc, 3 neighbour
    indices, 3 neighbour values, write: 2 x 48), z.r (16), direction update (24): 248 B per cell.
    Chebyshev (degree 12) with vectors of w bytes: s and A s formed from z and the old s
    (z, s, 6 u16 indices, diagonal, write s and As: 4w+12+4), q/r update (q 16, s, r r/w, As: 4w+16),
    and per Chebyshev step the direction (read + write), residual (read + write), z (read + write),
    inverse diagonal, diagonal and indices (7w+16), plus z.r and max|r| (2w).
    """
    if precond == "mic0":
        return 248.0 * m
    w = 4.0 if precision == "mixed" else 8.0
    deg = 12
    return m * ((4 * w + 16) + (4 * w + 16) + deg * (7 * w + 16) + 2 * w)


def poisson_bytes_per_iteration(m: int) -> float:
    """Algorithmic bytes of one MG-preconditioned PCG iteration over m unknowns (FP32 vectors, each array
    once per pass): the PCG part (apply A 9, axpys 24, direction 12 = 45 B) plus one V-cycle, (4 smoothing
    sweeps x 13 + residual 13 + transfer 8) x 8/7 (the coarse levels add 1/7) = 83.4 B."""
    return m * (45.0 + (4 * 13 + 13 + 8) * 8.0 / 7.0)


def mic0_bytes_per_iteration(m: int) -> float:
    """The same for MIC(0): the PCG part plus the two triangular sweeps (26 B)."""
    return m * (45.0 + 26.0)


def run_poisson(args, world: int, rank: int) -> dict | None:
    """The isolated pressure-Poisson batch: `count` snapshots of n^3 (rank r solves its own snapshots), MG- and
    MIC(0)-preconditioned CG in FP32 vectors with FP64 inner products and refinement at the max-norm 1e-6
    rule, each against an FP64 MG-PCG solve to 1e-12 of the same snapshots."""
    if args.poisson_n <= 0:
        return None
    import torch

    from teapotfluidsimulation_b200 import abi
    from teapotfluidsimulation_b200 import engine as E

    from teapotfluidsimulation_b200 import sharding

    n = args.poisson_n
    t0 = time.perf_counter()
    mine = shard_snapshots(n, args.poisson_count * world, rank, world)
    count = len(mine)
    cell = np.zeros((count, n ** 3), np.uint8)
    b = np.zeros((count, n ** 3), np.float32)
    at = 0
    for first, k in sharding.contiguous_runs(mine):
        cell[at:at + k], b[at:at + k] = E.poisson_generate(n, first, k)
        at += k
    gen_s = time.perf_counter() - t0
    m_each = ((cell & 3) == abi.FLUID).sum(axis=1)  # unknowns per snapshot (border cells are SOLID)
    dc = torch.from_numpy(cell).cuda()
    db = torch.from_numpy(b).cuda()
    del cell

    def solve(method, precision, tol, reps):
        x = torch.zeros((count, n ** 3), dtype=torch.float64, device="cuda")
        pb = E.PoissonBatch(n, count, method, precision)
        best = None
        for _ in range(reps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            it, res, conv = pb.solve(dc.data_ptr(), db.data_ptr(), x.data_ptr(), tol, 4000)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = (ms, it, conv) if best is None or ms < best[0] else best
        dev_bytes = pb.device_bytes
        pb.destroy()
        return x, best, dev_bytes

    ref, (ref_ms, ref_it, ref_conv), _ = solve(E.POISSON_MG, abi.SOLVE_F64, 1e-12, 1)
    refn = ref.abs().amax(dim=1).clamp_min(1e-300)
    peaks, peak_kind = measured_peaks()
    out = {"workload": f"{args.poisson_count} snapshots of {n}^3 per GPU (cylinder wall, slab, 1-8 mulberry32 "
                       f"spheres; rhs = -div of a Gaussian random face field), seeds 1000.."
                       f"{1000 + args.poisson_count * world - 1}, partitioned over ranks by unknowns",
           "snapshots_this_rank": count,
           "unknowns": int(m_each.sum()), "generate_s": gen_s, "tolerance": "max|r| <= 1e-6 max|b|",
           "reference": {"method": "MG-PCG FP64 to 1e-12 (GPU; pinned to the CPU FP64 oracle in the tests)",
                         "ms": ref_ms, "iterations_mean": float(ref_it.mean()), "converged": bool(ref_conv.all())}}
    for name, method, reps, per_it in [("mg", E.POISSON_MG, 3, poisson_bytes_per_iteration),
                                       ("mic0", E.POISSON_MIC0, 1, mic0_bytes_per_iteration)]:
        x, (ms, it, conv), dev_bytes = solve(method, abi.SOLVE_MIXED, 1e-6, reps)
        err = ((x - ref).abs().amax(dim=1) / refn).max().item()
        del x
        ms_max = allmax(ms, world)
        work = float(sum(per_it(int(m)) * int(k) for m, k in zip(m_each, it)))
        achieved = work / (ms / 1e3) / 1e9
        out[name] = {"ms_per_batch": ms_max, "ms_per_snapshot": ms_max / count,
                     "snapshots_per_s": args.poisson_count * world / (ms_max / 1e3),
                     "iterations_mean": float(it.mean()), "iterations_max": int(it.max()),
                     "converged": bool(conv.all()), "max_rel_err_vs_fp64_1e-12": err, "device_gb": dev_bytes / 1e9,
                     "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                                  "frac": achieved / peaks.get("hbm_gbs", 1.0), "peak_kind": peak_kind}}
    out["mg_speedup_vs_mic0"] = out["mic0"]["ms_per_batch"] / out["mg"]["ms_per_batch"]
    if rank == 0 and args.poisson_cpu_sample > 0:  # the CPU FP64 oracle (MIC(0)-PCG) on a bounded sample
        from oracle import oracle as O

        cs, bs = E.poisson_generate(n, 0, args.poisson_cpu_sample)
        t0 = time.perf_counter()
        for q in range(args.poisson_cpu_sample):
            O.poisson_solve(cs[q], bs[q].astype(np.float64), n, tol=1e-6, max_iter=4000)
        wall = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": args.poisson_cpu_sample / wall, "unit": "snapshots/s", "cores": 1,
                               "kind": "port", "sample": f"{args.poisson_cpu_sample} snapshots of {n}^3, FP64 "
                               f"MIC(0)-PCG (the C++ restatement of Pcg3D.solve) at the same 1e-6 rule"}
    return out


UNET_FLOP_PER_CELL = 2 * 27 * (  # the 11 convolutions as computed (channels padded to 16), per fine cell
    (16 * 16 + 16 * 16 + 48 * 16 + 16 * 16 + 16 * 16)  # full resolution
    + (16 * 32 + 32 * 32 + 96 * 32 + 32 * 32) / 8  # half
    + (32 * 64 + 64 * 64) / 64)  # quarter


def unet_throughput(net, box, pairs) -> dict:
    """The network's forward pass (the preconditioner application: BF16 tensor-core convolutions) on two
    boxes, CUDA-event timed, as FLOP/s against the measured dense BF16 peak."""
    import torch

    X, Y, Z = box
    dc = torch.from_numpy(np.ascontiguousarray(pairs[0])).cuda()
    dr = torch.from_numpy(np.ascontiguousarray(pairs[1])).cuda()
    dz = torch.zeros_like(dr)
    count = dc.shape[0]
    for _ in range(2):
        net.apply(dc.data_ptr(), dr.data_ptr(), dz.data_ptr(), X, Y, Z, count)
    reps = 5
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        net.apply(dc.data_ptr(), dr.data_ptr(), dz.data_ptr(), X, Y, Z, count)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    flop = UNET_FLOP_PER_CELL * X * Y * Z * count
    peaks, kind = measured_peaks()
    tf = flop / (ms / 1e3) / 1e12
    return {"boxes": count, "box": [X, Y, Z], "ms_per_apply": ms, "gflop_per_apply": flop / 1e9,
            "roofline": {"bound": "tensor", "achieved": tf, "peak": peaks.get("bf16_tflops"), "unit": "TFLOP/s",
                         "frac": tf / peaks.get("bf16_tflops", 1.0), "peak_kind": kind},
            "kernels": "k_conv: implicit-GEMM 3x3x3 convolutions, BF16 mma.sync m16n8k16, FP32 accumulation"}


def run_full_domain(args, world: int, rank: int) -> dict | None:
    """The full-domain APIC pour (both halves of the pot; at 2.5 mm 126 x 126 x 64 cells and 752,630
    parcels) on the grid-scale pressure solves: multigrid PCG, then learned flexible CG (network trained
    here on residual/correction pairs of the same pour, multigrid fall-back) from the same state. Both end
    every solve on the reference's max-norm 1e-6 rule; device time from the substep graph's stage events
    (the correction solve runs beside the pressure solve, so both are in the "pressure" stage)."""
    if args.full_mm <= 0:
        return None
    import torch

    import teapotfluidsimulation_b200 as pkg
    from teapotfluidsimulation_b200 import abi
    from teapotfluidsimulation_b200 import engine as E
    from teapotfluidsimulation_b200 import learned as Lr

    def make(pre):
        cfg = abi.gentle_pour(args.full_mm, 20, domain=abi.DOMAIN_FULL, transfer=abi.TRANSFER_APIC)
        cfg.preconditioner = pre
        cfg.solve_precision = abi.SOLVE_MIXED
        cfg.device = torch.cuda.current_device()
        return pkg.Simulation3D(cfg)

    def timed(sim, k):
        sim.enable_stage_timing(True)
        acc, its, cits = {}, [], []
        d0 = sim.diagnostics()
        for _ in range(k):
            sim.enqueue(1)
            sim.sync()
            for name, v in sim.stage_times().items():
                acc[name] = acc.get(name, 0.0) + v
            d = sim.diagnostics()
            its.append(d["pressureIterations"])
            cits.append(d["correctionIterations"])
        d1 = sim.diagnostics()
        ms = allmax(sum(v for name, v in acc.items() if name != "density"), world)  # density overlaps P2G
        return {"substeps": k, "ms_per_substep": ms / k,
                "sim_s_per_wall_s": allsum(d1["time"] - d0["time"], world) / (ms / 1e3),
                "pressure_ms_per_substep": acc["pressure"] / k, "correction_ms_per_substep": acc["correction"] / k,
                "pressure_iterations_mean": float(np.mean(its)), "correction_iterations_mean": float(np.mean(cits)),
                "pressure_failures": d1["pressureFailures"] - d0["pressureFailures"],
                "stages_ms_per_substep": {name: v / k for name, v in acc.items()}}

    mg = make(abi.PRECOND_BOX_MG)
    mg.advance(args.full_start)
    out = {"workload": f"gentle pour at {args.full_mm} mm, full domain (no symmetry plane), APIC, "
                       f"timed from t = {args.full_start} s; the liquid system embedded in a power-of-two box",
           "parcels": mg.n, "grid": [mg.nx, mg.ny, mg.nz], "liquid_cells": mg.diagnostics()["liquidCells"]}
    out["mg"] = timed(mg, args.full_steps)
    if args.learned_train_s > 0:
        t0 = time.perf_counter()
        box, cells, r, e = Lr.harvest_pour_systems(cell_mm=args.full_mm, count=12, every=25, seconds=20.0,
                                                   preconditioner=abi.PRECOND_BOX_MG, domain=abi.DOMAIN_FULL,
                                                   transfer=abi.TRANSFER_APIC)
        tc, tr, te = Lr.residual_pairs(box, cells, r, e, iters=(1, 2, 4))
        harvest_s = time.perf_counter() - t0
        npairs = int(tc.shape[0])
        cells_for_timing = (tc[:2].copy(), tr[:2].copy())
        del cells, r, e
        net = E.UNet(seed=2)
        net.set_loss(E.UNET_LOSS_ENERGY)
        t0 = time.perf_counter()
        hist = Lr.train(net, box, tc, tr, te, steps=1_000_000, batch=2, lr=1e-3, time_limit=args.learned_train_s)
        train_s = time.perf_counter() - t0
        del tc, tr, te
        out["unet_conv"] = unet_throughput(net, box, cells_for_timing)
        del cells_for_timing
        ln = make(abi.PRECOND_LEARNED)
        ln.set_unet(net)
        ln.set_state(mg.get_state(), mg.particles())
        ln.set_affine(mg.affine())
        mg_again = timed(mg, args.learned_steps)  # the same stretch of the pour with multigrid
        ln_res = timed(ln, args.learned_steps)
        ln_res["training"] = {"pairs": npairs, "box": list(box), "steps": len(hist), "seconds": train_s,
                              "harvest_and_pairs_s": harvest_s, "loss_first": hist[0],
                              "loss_last20": float(np.mean(hist[-20:])), "loss": "energy norm",
                              "pairs_from": "12 pressure systems of the same pour and MG-PCG iterates 1, 2, 4"}
        out["learned"] = ln_res
        out["mg_same_stretch"] = mg_again
        out["learned_over_mg_pressure_time"] = ln_res["pressure_ms_per_substep"] / mg_again["pressure_ms_per_substep"]
        ln.destroy()
        net.destroy()
    mg.destroy()
    return out


def shard_pours(cfgs: list, rank: int, world: int) -> list[int]:
    """Indices of the ensemble's pours this rank runs: a partition by estimated cost (cells + parcels times
    estimated substeps), the same on every rank without communication; no collective on the data path."""
    from teapotfluidsimulation_b200 import sharding

    if world == 1:
        return list(range(len(cfgs)))
    return sharding.partition_by_cost(sharding.pour_costs(cfgs), world)[rank]


def shard_snapshots(n: int, total: int, rank: int, world: int) -> list[int]:
    """Snapshot indices of the Poisson batch this rank solves: a partition of all ranks' snapshots by their
    unknowns (masks generated on every rank, cheap: no rhs)."""
    from teapotfluidsimulation_b200 import sharding

    if world == 1:
        return list(range(total))
    return sharding.partition_by_cost(sharding.snapshot_costs(n, 0, total), world)[rank]


def run_ensemble(args, world: int, rank: int) -> dict | None:
    """A seeded ensemble of pours (fill U[0.6, 1.0] L, peak tilt U[60, 110] deg, tilt-in ramp U[4, 12] s;
    uneven grids), sharded round-robin over the ranks, each pour on its own stream with the substeps of all
    pours interleaved; timed by the host clock around the whole set (every pour's stream synchronised),
    against the same pours run one after another."""
    if args.ensemble_count <= 0:
        return None
    import torch

    from teapotfluidsimulation_b200 import abi
    from teapotfluidsimulation_b200 import engine as E

    from teapotfluidsimulation_b200 import sharding

    cfgs = E.ensemble_configs(2026, args.ensemble_count, args.ensemble_mm, 20.0)
    mine_idx = shard_pours(cfgs, rank, world)
    mine = [cfgs[i] for i in mine_idx]
    for c in mine:
        c.preconditioner = abi.PRECOND_CHEB
        c.solve_precision = abi.SOLVE_MIXED
        # 4-CTA clusters: a 5 mm pour solves as fast as on 16, and 4x as many pours' solves fit at once
        c.solve_cluster, c.solve_threads = 4, 512
        c.device = torch.cuda.current_device()
    t0 = time.perf_counter()
    ens = E.Ensemble(mine)
    create_s = time.perf_counter() - t0
    grids = [m.nx * m.ny * m.nz for m in ens.members]
    parcels = sum(m.n for m in ens.members)
    ens.advance(0.6)  # past the start delay, into the tilt
    ens.enqueue(3)
    t_before = [m.diagnostics()["time"] for m in ens.members]
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ens.enqueue(args.ensemble_steps)
    torch.cuda.synchronize()
    wall = allmax(time.perf_counter() - t0, world)
    sim_s = sum(m.diagnostics()["time"] - t for m, t in zip(ens.members, t_before))
    fails = sum(m.diagnostics()["pressureFailures"] for m in ens.members)
    # per-pour stats (about a hundred bytes each), gathered from every rank
    local = {}
    for i, m in zip(mine_idx, ens.members):
        d = m.diagnostics()
        local[i] = {"time": d["time"], "steps": d["steps"], "discharged_ml": d["dischargedMl"],
                    "pressure_failures": d["pressureFailures"], "cells": m.nx * m.ny * m.nz}
    stats = sharding.gather_stats(local, world)
    # the same kind of work one pour at a time (the first few pours), for the concurrency gain
    seq_wall, seq_sim = 0.0, 0.0
    for m in ens.members[: min(8, len(ens.members))]:
        t = m.diagnostics()["time"]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m.enqueue(args.ensemble_steps)
        m.sync()
        seq_wall += time.perf_counter() - t0
        seq_sim += m.diagnostics()["time"] - t
    ens.destroy()
    total_sim = allsum(sim_s, world)
    return {"workload": f"{args.ensemble_count} seeded gentle pours at {args.ensemble_mm} mm (half pot), "
                        f"{args.ensemble_steps} substeps each from t = 0.6 s, Chebyshev solves on 4-CTA clusters",
            "pours": args.ensemble_count, "pours_per_gpu": len(mine), "parcels_per_gpu": parcels,
            "cells_min": min(grids), "cells_max": max(grids), "create_s": create_s,
            "sim_s_per_wall_s": total_sim / wall, "pour_substeps_per_s": allsum(len(mine), world) * args.ensemble_steps / wall,
            "wall_s": wall, "pressure_failures": fails,
            "pours_gathered": len(stats), "cells_total": sum(v["cells"] for v in stats.values()),
            "sharding": "pours partitioned by estimated cost (cells + parcels) x substeps; stats gathered "
                        "from every rank",
            "one_at_a_time_sim_s_per_wall_s": seq_sim / seq_wall if seq_wall > 0 else None,
            "concurrency_gain": (sim_s / wall) / (seq_sim / seq_wall) if seq_wall > 0 and seq_sim > 0 else None,
            "timing": "host clock around the interleaved launches and every pour's synchronisation"}


def run_cpu_baseline(args, substeps: int, state=None) -> dict:
    """The CPU FP64 restatement of the reference solver on a bounded sample of the same workload, from
    the engine's state at the start of the timed window when one is given."""
    from oracle import oracle as O

    sim = O.OracleSim(make_cfg(args))
    if state is not None:
        sim.set_state(*state)
    elif args.start > 0:
        sim.advance(args.start)
    t_sim0 = sim.diagnostics()["time"]
    t0 = time.perf_counter()
    for _ in range(substeps):
        sim.step(-1.0)
    wall = time.perf_counter() - t0
    t_sim = sim.diagnostics()["time"] - t_sim0
    sim.close()
    return {"value": t_sim / wall, "unit": "sim-s/wall-s", "cores": 1, "kind": "port",
            "sample": f"{substeps} substeps of the same pour from t={t_sim0:.3f} s, C++ FP64 restatement "
                      f"of src/sim3d (one thread; the reference is single-threaded TypeScript)",
            "wall_s": wall, "sim_s": t_sim, "ms_per_substep": 1000 * wall / substeps}


def reference_pour_result(cell_mm: float) -> dict | None:
    """The reference CPU solver's whole-pour result at this cell size (benchmarks/run3d.json, committed
    as a test fixture)."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "reference_goldens.json")) as f:
            rows = json.load(f)["run3d"]
    except (OSError, KeyError):
        return None
    for r in rows:
        if abs(r["cellMm"] - cell_mm) < 1e-9:
            return {"discharged_ml": r["dischargedMl"], "shares": r["dischargedFractions"],
                    "simulated_s": r.get("simulatedSeconds"), "wall_s_reference_laptop": r.get("wallSeconds")}
    return None


def run_whole_pour(args, precond: str) -> dict:
    """The reference's own benchmark loop (benchmarks/run3d.ts:14-23): advance in 0.5 s chunks until 1.5 s
    after the controller is done, through the public pl_advance call, timed by the host clock (end to end)
    and by CUDA events on the engine's stream; then the same pour again with stage events, one substep per
    launch, for the per-stage device time. No L2 flush: this is the continuous run the reference times."""
    import torch

    import teapotfluidsimulation_b200 as pkg

    a = argparse.Namespace(**vars(args))
    a.precond = precond

    def make():
        cfg = make_cfg(a)
        cfg.device = torch.cuda.current_device()
        return pkg.Simulation3D(cfg)

    sim = make()
    stream = torch.cuda.ExternalStream(sim.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record(stream)
    done_at = -1.0
    while not sim.finished:
        d = sim.advance(0.5)
        if d["phase"] == "done" and done_at < 0:
            done_at = d["time"]
        if done_at >= 0 and d["time"] > done_at + 1.5:
            break
    e1.record(stream)
    e1.synchronize()
    wall = time.perf_counter() - t0
    dev_s = e0.elapsed_time(e1) / 1e3
    d = sim.diagnostics()
    sh = sim.discharged_fractions()
    sim_s, substeps = d["time"], d["steps"]
    sim.destroy()
    out = {"simulated_s": sim_s, "substeps": substeps, "wall_s": wall, "sim_s_per_wall_s": sim_s / wall,
           "device_s": dev_s, "sim_s_per_device_s": sim_s / dev_s,
           "discharged_ml": d["dischargedMl"], "shares": None if sh is None else [float(v) for v in sh],
           "spilled_ml": d["spilledMl"], "lost_ml": d["lostMl"], "pressure_failures": d["pressureFailures"]}
    ref = reference_pour_result(args.cell_mm)
    if ref is not None:
        out["reference"] = ref
        out["volume_rel_err"] = d["dischargedMl"] / ref["discharged_ml"] - 1
        if sh is not None:
            out["shares_max_abs_err"] = float(np.abs(np.array(sh) - np.array(ref["shares"])).max())
    # the stage split of the same pour (one substep per launch, stage events in the graph)
    sim = make()
    sim.enable_stage_timing(True)
    acc, its, cits, n = {}, [], [], 0
    done_at = -1.0
    while not sim.finished:
        sim.enqueue(1)
        sim.sync()
        for k, v in sim.stage_times().items():
            acc[k] = acc.get(k, 0.0) + v
        dd = sim.diagnostics()
        its.append(dd["pressureIterations"])
        cits.append(dd["correctionIterations"])
        n += 1
        if dd["phase"] == "done" and done_at < 0:
            done_at = dd["time"]
        if done_at >= 0 and dd["time"] > done_at + 1.5:
            break
    sim.destroy()
    out["stages_ms_per_substep"] = {k: v / max(n, 1) for k, v in acc.items()}
    out["pressure_ms_per_substep"] = acc.get("pressure", 0.0) / max(n, 1)
    out["correction_ms_per_substep"] = acc.get("correction", 0.0) / max(n, 1)
    out["pressure_iterations_mean"] = float(np.mean(its)) if its else 0.0
    out["correction_iterations_mean"] = float(np.mean(cits)) if cits else 0.0
    out["pressure_iterations_max"] = int(max(its)) if its else 0
    return out


def run_reference(args):
    world, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    from oracle import oracle as O

    sim = O.OracleSim(make_cfg(args))
    if args.start > 0:
        sim.advance(args.start)
    for _ in range(args.warmup):
        sim.step(-1.0)
    t_sim0 = sim.diagnostics()["time"]
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.step(-1.0)
    wall = time.perf_counter() - t0
    t_sim = sim.diagnostics()["time"] - t_sim0
    value = t_sim / wall
    line = {
        "impl": "reference", "metric": "sim-s/wall-s", "value": value, "unit": "sim-s/wall-s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cell_mm": args.cell_mm, "substeps_timed": args.steps,
                   "note": "C++ FP64 restatement of the reference CPU solver (TypeScript reference not runnable: "
                           "no JavaScript runtime)"},
        "cpu_baseline": {"value": value, "unit": "sim-s/wall-s", "cores": 1, "kind": "port",
                         "sample": f"{args.steps} substeps after {args.warmup} warm-up substeps"},
        "e2e": {"value": value, "unit": "sim-s/wall-s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_ours(args):
    import torch

    world, rank, local = dist_init()
    import teapotfluidsimulation_b200 as pkg

    torch.cuda.set_device(local)
    cfg = make_cfg(args)
    cfg.device = local
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > 126 MB L2

    def started():
        sim = pkg.Simulation3D(cfg)
        if args.start > 0:
            sim.advance(args.start)
        return sim, torch.cuda.ExternalStream(sim.stream, device=torch.device("cuda", local))

    # value: the production substep graph (no stage events), one graph launch per substep bracketed by CUDA
    # events on the engine's stream, the L2 flushed before each substep outside the bracket
    sim, stream = started()
    start_state = (sim.get_state(), sim.particles())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def substep() -> float:
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0.record(stream)
        sim.enqueue(1)
        e1.record(stream)
        sim.sync()
        return e0.elapsed_time(e1)

    for _ in range(args.warmup):
        substep()
    d0 = sim.diagnostics()
    clocks = Clocks(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    dev_ms = 0.0
    steps_done = 0
    torch.cuda.cudart().cudaProfilerStart()  # the timed window alone, for `ncu --profile-from-start off`
    for _ in range(args.steps):
        if sim.finished:
            break
        dev_ms += substep()
        steps_done += 1
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStop()
    barrier(world)
    d1 = sim.diagnostics()
    sim_s = d1["time"] - d0["time"]
    max_ms = allmax(dev_ms, world)
    value = allsum(sim_s, world) / (max_ms / 1000.0)
    sim.destroy()

    # stage split of the same window: a second replica from the same start with stage events in its graph
    ssim, sstream = started()
    ssim.enable_stage_timing(True)
    for _ in range(args.warmup):
        with torch.cuda.stream(sstream):
            flush.fill_(1.0)
        ssim.enqueue(1)
        ssim.sync()
    stage_acc: dict = {}
    pcg_work, iters, corr_iters = 0.0, [], []
    for _ in range(steps_done):
        with torch.cuda.stream(sstream):
            flush.fill_(1.0)
        ssim.enqueue(1)
        ssim.sync()
        for k, v in ssim.stage_times().items():
            stage_acc[k] = stage_acc.get(k, 0.0) + v
        d = ssim.diagnostics()
        iters.append(d["pressureIterations"])
        corr_iters.append(d["correctionIterations"])
        # the Chebyshev launch solves both systems (on two clusters at once): count both
        solved = d["pressureIterations"] + (d["correctionIterations"] if args.precond == "cheb" else 0)
        pcg_work += pcg_bytes_per_iteration(d["liquidCells"], args.precond, args.precision) * solved
    ssim.destroy()

    # end to end through the C ABI: pl_step per substep (control block in, stats block out) from the same start
    e2e_sim, _ = started()
    for _ in range(args.warmup):
        e2e_sim.step(-1.0)
    e2e_t0 = e2e_sim.diagnostics()["time"]
    wall = 0.0
    for _ in range(steps_done):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_sim.step(-1.0)
        wall += time.perf_counter() - t0
    e2e_s = e2e_sim.diagnostics()["time"] - e2e_t0
    e2e_value = allsum(e2e_s, world) / allmax(wall, world)
    scalars = int(e2e_sim.sizes.step_copy_bytes)  # the device scalar block, copied each way per pl_step
    e2e_sim.destroy()

    whole = None
    if args.whole_pour:
        whole = {"workload": f"the whole gentle pour at {args.cell_mm:g} mm from t = 0 until 1.5 s after the "
                             f"controller is done (benchmarks/run3d.ts), pl_advance in 0.5 s chunks, no L2 flush"}
        for pre in ("cheb", "mg"):
            whole[pre] = run_whole_pour(args, pre)
    clk = clocks.stop()

    peaks, peak_kind = measured_peaks()
    n = max(steps_done, 1)
    pres_ms = stage_acc.get("pressure", 0.0) / n
    achieved = (pcg_work / n) / (pres_ms / 1000.0) / 1e9 if pres_ms > 0 else 0.0
    traffic = profile_traffic()
    line = {
        "metric": "sim-s/wall-s", "value": value, "unit": "sim-s/wall-s", "n_gpus": world, "steps": steps_done,
        "warmup": args.warmup, "ms_per_step": max_ms / n, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": ("f32 solve vectors, f64 inner products/refinement" if args.precision == "mixed" else "f64 solve")
                 + " / f32 parcels and faces, f64 transfer weights", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cell_mm": args.cell_mm, "preconditioner": args.precond,
                   "solve_shape": f"{cfg.solve_cluster}x{cfg.solve_threads}",
                   "solve_precision": args.precision,
                   "start_s": args.start, "simulated_s": sim_s, "l2": "256 MiB buffer written between substeps",
                   "timing": "CUDA events around each substep graph launch (no stage events in the graph)",
                   "parallelism": f"replicas x{world}"},
        "pressure_ms_per_substep": pres_ms,
        "pressure_iterations_mean": (sum(iters) / len(iters)) if iters else 0,
        "correction_iterations_mean": (sum(corr_iters) / len(corr_iters)) if corr_iters else 0,
        "stages_ms_per_substep": {k: v / n for k, v in stage_acc.items()},
        "stages_note": "a separate replica from the same start with stage events in its graph; density runs "
                       "beside P2G on a second stream (its time overlaps P2G's)",
        "gpu_launches": KERNELS_PER_SUBSTEP[args.precond] * steps_done,
        "e2e": {"value": e2e_value, "unit": "sim-s/wall-s", "h2d_bytes_per_step": scalars,
                "d2h_bytes_per_step": scalars},
        "roofline": {"kernel": "pressure solve stage (k_solve_setup + %s%s)" % (
                         "k_pcg" if args.precond == "mic0" else "k_chebpcg" if args.precond == "cheb" else "k_mgpcg",
                         "; pressure and correction systems on two clusters" if args.precond == "cheb" else ""),
                     "bound": "hbm", "achieved": achieved,
                     "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                     "frac": achieved / peaks.get("hbm_gbs", 1.0), "peak_kind": peak_kind,
                     "traffic": traffic},
    }
    if whole is not None:
        line["whole_pour"] = whole
    if clk:
        line["clocks"] = clk
    if rank == 0 and world == 1 and args.cpu_sample > 0:
        line["cpu_baseline"] = run_cpu_baseline(args, args.cpu_sample, start_state)
    pois = run_poisson(args, world, rank)
    if pois is not None:
        line["poisson_batch"] = pois
    full = run_full_domain(args, world, rank)
    if full is not None:
        line["full_domain"] = full
    ens = run_ensemble(args, world, rank)
    if ens is not None:
        line["ensemble"] = ens
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
