"""Run one of the measured forging cases for a few increments and print what every increment did.

    python -m impressionfea_b200.run_case --case closed_die --tets 60000 --increments 3 --fp32
    python -m impressionfea_b200.run_case --case upsetting --increments 5
    python -m impressionfea_b200.run_case --case 2d --increments 20

Meant for looking at one configuration at a time (a profiler run, a timing of one form) without the whole bench.
The closed-die case takes the library's host remeshing; --fp32 selects the single-precision factorisation with
double-precision refinement and the Newton tolerance 2e-4.
"""
import argparse
import dataclasses
import json
import time


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", choices=["closed_die", "upsetting", "2d"], default="closed_die")
    ap.add_argument("--tets", type=int, default=200000, help="closed-die billet size (isosurface-stuffed tets)")
    ap.add_argument("--increments", type=int, default=3)
    ap.add_argument("--fp32", action="store_true")
    ap.add_argument("--no-remesh", action="store_true")
    args = ap.parse_args(argv)

    from . import workloads

    if args.case == "2d":
        from .forging2d import ForgingSolver2D

        s = ForgingSolver2D(workloads.upsetting_2d())
        keys = ("n_factor",)
    else:
        from .forging3d import Forging3DSolver

        if args.case == "closed_die":
            cfg, mesh, dies = workloads.closed_die_gear_blank(target_tets=args.tets)
        else:
            cfg, mesh, dies = workloads.upsetting_drop_in()
        if args.fp32:
            cfg = dataclasses.replace(cfg, tol=2e-4)
        s = Forging3DSolver(cfg, mesh, dies)
        if args.fp32:
            s.set_scalar("factor_fp32", 1)
        if args.case == "closed_die" and not args.no_remesh:
            s.set_scalar("remesh", 1)
        keys = ("n_fact", "remesh_count", "t_factor", "t_pcg", "t_remesh", "ne")
    for k in range(args.increments):
        t0 = time.perf_counter()
        info = s.step()
        out = {"increment": k + 1, "seconds": round(time.perf_counter() - t0, 4), "iterations": info["iterations"],
               "load": info["load"]}
        out.update({q: s.scalar(q) for q in keys})
        print(json.dumps(out), flush=True)
    s.close()


if __name__ == "__main__":
    main()
