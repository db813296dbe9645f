"""A profiler window over a running pour: the substeps of a whole pour as `pl_advance` runs them
(warm caches, no L2 flush), for `ncu --profile-from-start off`.

The pour (gentle 400 mL, `--mm` cells, Chebyshev cluster solves with FP32 vectors and FP64
refinement unless `--precond` says otherwise) advances to `--start` seconds outside the window; then
`cudaProfilerStart`, `--substeps` substeps queued on the engine's stream, `cudaProfilerStop`.

    python -m teapotfluidsimulation_b200.profile_window --mm 4 --start 3.0 --substeps 10
"""
from __future__ import annotations

import argparse

from . import abi

PRECONDS = {"cheb": (abi.PRECOND_CHEB, abi.SOLVE_MIXED), "mg": (abi.PRECOND_MG, abi.SOLVE_MIXED),
            "box_mg": (abi.PRECOND_BOX_MG, abi.SOLVE_MIXED), "mic0": (abi.PRECOND_MIC0, abi.SOLVE_F64)}


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--mm", type=float, default=4.0, help="cell size in millimetres")
    ap.add_argument("--start", type=float, default=3.0, help="simulated seconds before the window")
    ap.add_argument("--substeps", type=int, default=10, help="substeps inside the window")
    ap.add_argument("--precond", default="cheb", choices=sorted(PRECONDS))
    args = ap.parse_args(argv)

    import torch

    from .engine import Simulation3D

    cfg = abi.gentle_pour(args.mm, 20)
    cfg.preconditioner, cfg.solve_precision = PRECONDS[args.precond]
    cfg.device = torch.cuda.current_device()
    sim = Simulation3D(cfg)
    sim.advance(args.start)
    sim.enqueue(3)  # the window's first substeps are not the first after a host synchronisation
    sim.sync()
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStart()
    sim.enqueue(args.substeps)
    sim.sync()
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStop()
    d = sim.diagnostics()
    print(f"window of {args.substeps} substeps at {args.mm} mm from t = {args.start} s: now t = {d['time']:.4f} s, "
          f"{d['steps']} substeps, pressure iterations {d['pressureIterations']}, "
          f"correction iterations {d['correctionIterations']}")
    sim.destroy()


if __name__ == "__main__":
    main()
