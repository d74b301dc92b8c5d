"""Runs one of the synthetic workloads through the library and prints its
device-timed throughput: ``python -m aerocfd_b200.run --case sa_plate``.

Cases (all generated, seeded where random): ``bump`` (Euler bump channel
97 x 49 x 5, M 0.5, CFL 5), ``naca`` (laminar NACA0012 O-grid 4 x 129 x 65 x 3,
M 0.5, Re 5000, AoA 2, CFL 2), ``sa_plate`` (SA flat plate 193 x 129 x 33 in 8
blocks along x, M 0.2, Re 5e6, CFL 5) and ``batch`` (64 bump channels of
uneven size, seed 0, as one batch).  Used for profiling single workloads."""
from __future__ import annotations

import argparse
import ctypes
import json

from . import _lib, grids, solver
from .case import Config, IFLAG_EULERSOLVER, IFLAG_NSSOLVER


def make(name: str, inviscid: int):
    if name == "bump":
        return grids.bump_channel(cfg=Config(solver=IFLAG_EULERSOLVER, ma=0.5, re=1.0e6, cfl=5.0, inviscid=inviscid)), None
    if name == "naca":
        return grids.naca_ogrid(cfg=Config(solver=IFLAG_NSSOLVER, ma=0.5, re=5000.0, aoa_deg=2.0, cfl=2.0,
                                           inviscid=inviscid)), None
    if name == "sa_plate":
        cfg = Config(solver=IFLAG_NSSOLVER, turbulence=2, ma=0.2, re=5.0e6, cfl=5.0, nutinf=3.0, inviscid=inviscid)
        return grids.flat_plate(nbi=8, nbj=1, nbk=1, cfg=cfg), None
    if name == "batch":
        return grids.batch_case(grids.bump_batch(64, seed=0))
    raise ValueError(f"unknown case {name}")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--case", default="naca", choices=["bump", "naca", "sa_plate", "batch"])
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--inviscid", type=int, default=4, help="4 Roe + WENO3, 5 SW + WENO5, 8 WCNS5")
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--sweep-cluster", type=int, default=0, help="CTAs per block of the LU-SGS sweep (0: autotune)")
    ap.add_argument("--sweep-exchange", choices=["l2", "shared", "slab", "shared2"], default=None,
                    help="plane exchange of a cluster sweep (default: the autotuner's or L2)")
    ap.add_argument("--sa-sweep-cluster", type=int, default=0, help="CTAs per block of the SA sweep (0: autotune)")
    ap.add_argument("--sweep-prefetch", type=int, choices=[2, 3, 4], default=0,
                    help="L2 prefetch distance of the bulk-exchange sweep (default: the autotuner's)")
    ap.add_argument("--register-bound", type=int, choices=[0, 1], default=None,
                    help="register-bounded viscous part a (default: the autotuner's)")
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="default launch shapes")
    ap.add_argument("--tuning", type=int, nargs=5, metavar=("INV_TILE", "EW", "VISC", "MATS", "NST"),
                    help="launch shapes as aero_set_tuning takes them (instead of the autotuner)")
    args = ap.parse_args(argv)
    case, params = make(args.case, args.inviscid)
    gc = solver.GpuCase(case, block_params=params) if params else solver.GpuCase(case)
    try:
        gc.compute_geometry()
        gc.init_flowfield()
        gc.start()
        gc.set_precision(args.mixed)
        if args.tuning:
            gc.set_tuning(*args.tuning)
            tuning = ""
        else:
            tuning = "" if args.no_autotune else gc.autotune(3)
        if args.sweep_cluster:
            gc.set_sweep_cluster(args.sweep_cluster)
        if args.sweep_exchange:
            gc.set_sweep_exchange(args.sweep_exchange)
        if args.sa_sweep_cluster:
            gc.set_sa_sweep_cluster(args.sa_sweep_cluster)
        if args.register_bound is not None:
            gc.set_register_bound(args.register_bound == 1)
        if args.sweep_prefetch:
            gc.set_sweep_prefetch(args.sweep_prefetch)
        gc.use_graphs(not args.no_graphs)
        gc.step(args.warmup, history=False)
        ms = ctypes.c_double(0.0)
        _lib.check(gc.L.aero_step_timed(ctypes.c_int(args.steps), ctypes.c_int(1), ctypes.byref(ms)), "timed")
        gc.L.aero_tuning.restype = ctypes.c_char_p
        print(json.dumps({"case": args.case, "nodes": case.nodes, "steps": args.steps,
                          "value": case.nodes * args.steps / (ms.value / 1e3) / 1e6, "unit": "Mcell-iter/s",
                          "ms_per_step": ms.value / args.steps, "tuning": gc.L.aero_tuning().decode(),
                          "autotuned": tuning, "device_status": gc.status()}))
    finally:
        gc.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
