"""Benchmark: stroke increments per second of the 3D upsetting drop-in on B200, FP32-factor form vs plain FP64.

Workload (one "step" = one forging increment, Forging3DSolver.Step): quarter model of a cylindrical billet
d = 30 mm, h = 45 mm, ~30k linear tets (seeded Delaunay fill, node jitter +-10 % of h), flat dies as two-triangle
height fields, C = 150 MPa, eps0 = 0.01, n = 0.1, m = 0.12, friction m_f = 0.4, 40 % height reduction in 80
increments (ds = 0.225 mm), reference defaults otherwise (ram 50 mm/s, tolerance 1e-3). Synthetic data.

Arms:
  default            the CUDA path (libifea_gpu.so) — one JSON line, device-timed with CUDA events. `value` is the
                     warm-started single-precision-factor form (the reference's extrapolated start v_n + (v_n -
                     v_n-1); FP32 multifrontal Cholesky, every solve refined by FP64 PCG to 1e-7); `plain_fp64` is
                     the reference's default (previous-step start, FP64 factor, direct solve) on the same
                     increments, and `error_vs_plain_fp64` compares the two increment by increment;
  --impl reference   the reference algorithm on the host cores (the C# reference cannot run here; its CPU
                     restatement under oracle/ is timed instead, OpenMP element phase on all host threads).

Multi-GPU: a forging case does not shard (one mesh, one sparse factorisation); N GPUs run N independent replicas
of the case ("scaling": "weak"), one process per GPU, timing = max over ranks.
"""
import argparse
import dataclasses
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "stroke steps/s on 1 B200, warm-start+FP32 vs plain FP64, at <=0.5% load error"
UNIT = "stroke steps/s"
R, H, SHUT_RED, STEPS_TOTAL = 15.0, 45.0, 0.40, 80
TARGET_TETS = 30000


def workload():
    from impressionfea_b200.workloads import upsetting_drop_in
    return upsetting_drop_in()


def config_dict(cfg, mesh, extra=None):
    d = {"workload": "3D upsetting drop-in (quarter cylinder d30 x h45, flat dies, 40% in 80 steps)",
         "tets": int(mesh.ne), "nodes": int(mesh.nn), "dof": int(3 * mesh.nn), "h_mm": cfg.h, "ds_mm": cfg.ds,
         "friction": cfg.friction, "tolerance": cfg.tol, "global_batch": 1, "parallelism": "replicas"}
    if extra:
        d.update(extra)
    return d


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index=0):
        self.samples = []
        self.index = index
        self._stop = threading.Event()
        self._proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                           "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            t0 = time.time()  # sampling is live before the timed region starts
            while not self.samples and time.time() - t0 < 5.0:
                time.sleep(0.01)
            self._n0 = len(self.samples)
        except Exception:
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            self.samples.append([s.strip() for s in line.split(",")])

    def __exit__(self, *a):
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()

    def summary(self):
        # the samples taken while the timed region ran (the ones before it only proved that sampling was live)
        if len(self.samples) > getattr(self, "_n0", 0):
            self.samples = self.samples[self._n0:]
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if len(s) > 7 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 7 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples if len(s) > 7 for i in range(4) if s[4 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def assembly_algorithmic_bytes(ne, nn, nnz):
    """Algorithmic bytes of one matrix assembly (conn, gradients, volume, strain, element fields out; velocities,
    frames; K_vol read, K write, row index; residual and fixed flags)."""
    ndof = 3 * nn
    return ne * (16 + 96 + 8 + 8 + 64) + nn * (24 + 72) + nnz * (8 + 8 + 4) + ndof * (8 + 1)


def cpu_baseline_sample(budget_s=25.0, threads=None):
    """Time the CPU restatement on the same workload for a bounded number of increments."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from build_oracle import build_oracle
    build_oracle()
    threads = threads or os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import Oracle3D
    cfg, mesh, dies = workload()
    o = Oracle3D(cfg, mesh, dies)
    o.step()  # first increment includes the symbolic analysis; not timed
    t0 = time.perf_counter()
    n = 0
    while n < 50 and time.perf_counter() - t0 < budget_s:
        o.step()
        n += 1
    el = time.perf_counter() - t0
    return {"value": n / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} increments (steps 2..{n + 1}) of the same workload after one untimed increment; "
                      f"C restatement, OpenMP element phase, serial scatter and up-looking sparse Cholesky"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    s = cpu_baseline_sample(budget_s=max(20.0, 8.0 * args.steps))
    cfg, mesh, _ = workload()
    line = {"impl": "reference", "metric": METRIC, "value": s["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / s["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_dict(cfg, mesh),
            "cpu_baseline": s, "e2e": {"value": s["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def _timed_steps(s, stream, flush, k, snap=None):
    """k increments of solver s, each bracketed by CUDA events on the solver's stream, L2 flushed in between."""
    import torch

    durs, infos, snaps = [], [], []
    for _ in range(k):
        if s.IsFinished:
            break
        flush.zero_()  # L2 flush between timed increments (outside the timed pair)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        infos.append(s.step())
        b.record(stream)
        b.synchronize()
        durs.append(a.elapsed_time(b))
        if snap:
            snaps.append({nm: s.array(nm).copy() for nm in snap})
    return durs, infos, snaps


FAST_TOL = 2e-4  # Newton tolerance of the timed form: five times tighter than the reference default


def closed_die_workload():
    from impressionfea_b200.workloads import closed_die_gear_blank
    return closed_die_gear_blank()


def run_closed_die(stream, flush, warmup=2, steps=8):
    """The closed-die case over its first increments (the mesh distorts past about 3 mm of stroke without the
    host-side remeshing, which is out of scope): plain FP64 against the FP32 factor with FP64 refinement at the
    same tolerance and start."""
    from impressionfea_b200.forging3d import Forging3DSolver

    cfg, mesh, dies = closed_die_workload()
    out = {"workload": "closed-die gear blank (d40 x h50 billet, ~205k tets), increments %d..%d of 200" % (warmup + 1, warmup + steps),
           "tets": int(mesh.ne), "nodes": int(mesh.nn), "dof": int(3 * mesh.nn)}
    res = {}
    for label, fp32 in (("plain_fp64", False), ("fp32_factor", True)):
        s = Forging3DSolver(cfg, mesh, dies)
        s.set_stream(stream.cuda_stream)
        if fp32:
            s.set_scalar("factor_fp32", 1)
        for _ in range(warmup):
            s.step()
        durs, infos, _ = _timed_steps(s, stream, flush, steps)
        res[label] = {"ms_per_step": float(sum(durs)) / len(durs), "newton_iterations": int(sum(i["iterations"] for i in infos)),
                      "factorisations": int(infos[-1]["n_factor"] - infos[0]["n_factor"]) + 1,
                      "loads": [i["load"] for i in infos]}
        out["factor"] = {q: s.scalar(q) for q in ("supernodes", "levels", "max_front", "factor_nnz")}
        s.close()
    out["plain_fp64_ms_per_step"] = res["plain_fp64"]["ms_per_step"]
    out["fp32_ms_per_step"] = res["fp32_factor"]["ms_per_step"]
    out["speedup"] = out["plain_fp64_ms_per_step"] / out["fp32_ms_per_step"]
    out["newton_iterations"] = {k: v["newton_iterations"] for k, v in res.items()}
    out["factorisations"] = {k: v["factorisations"] for k, v in res.items()}
    out["load_rel_max_vs_plain"] = max(abs(a / b - 1) for a, b in zip(res["fp32_factor"]["loads"], res["plain_fp64"]["loads"]))
    return out


def fast_form(cfg):
    """The timed form's configuration: the reference's extrapolated start (ExtrapolateStart) as the warm start and
    a Newton tolerance five times tighter than the plain form's; the single-precision factorisation is switched on
    per context (`factor_fp32`)."""
    return dataclasses.replace(cfg, extrapolate_start=True, tol=FAST_TOL)


def _count_launches(cfg, mesh, dies, stream, warmup, k, fp32):
    """Kernels of this library launched during k increments (after the same warm-up), counted by the CUDA
    profiler interface on a re-run of the timed increments."""
    import torch

    from impressionfea_b200.forging3d import Forging3DSolver

    try:
        s = Forging3DSolver(fast_form(cfg) if fp32 else cfg, mesh, dies)
        s.set_stream(stream.cuda_stream)
        if fp32:
            s.set_scalar("factor_fp32", 1)
        for _ in range(warmup):
            s.step()
        torch.cuda.synchronize()
        acts = [torch.profiler.ProfilerActivity.CUDA]
        with torch.profiler.profile(activities=acts) as prof:
            for _ in range(k):
                s.step()
            torch.cuda.synchronize()
        s.close()
        n = 0
        for e in prof.events():
            if e.device_type == torch.autograd.DeviceType.CUDA and "k_" in e.name and "at::" not in e.name:
                n += 1
        return n
    except Exception:
        return None


def whole_job_value(total_ms, k, world, device="cuda"):
    """Increments per second of the whole job: every rank ran k increments and the job took as long as its
    slowest rank (max over ranks of each rank's device time). Returns (value, that time in ms)."""
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([total_ms], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    return world * k / (total_ms / 1000.0), total_ms


def run_gpu(args, rank, world):
    import torch

    from impressionfea_b200.forging3d import Forging3DSolver

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    cfg, mesh, dies = workload()
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    snap = ("vg", "eps")

    # plain FP64 form (the reference's arithmetic: FP64 factorisation, direct solve after each factorisation)
    s64, durs64, infos64, snaps64 = None, [], [], []
    if args.form == "both":
        s64 = Forging3DSolver(cfg, mesh, dies)
        s64.set_stream(stream.cuda_stream)
        for _ in range(args.warmup):
            s64.step()
        torch.cuda.synchronize()
        durs64, infos64, snaps64 = _timed_steps(s64, stream, flush, args.steps, snap)

    # FP32 factorisation refined by FP64 PCG: the timed form
    s = Forging3DSolver(fast_form(cfg), mesh, dies)
    s.set_stream(stream.cuda_stream)
    s.set_scalar("factor_fp32", 1)
    for _ in range(args.warmup):
        s.step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        durs, infos, snaps = _timed_steps(s, stream, flush, args.steps, snap)
    torch.cuda.synchronize()
    k = len(durs)
    value, total_ms = whole_job_value(float(sum(durs)), k, world)
    ms64 = float(sum(durs64)) / len(durs64) if durs64 else None

    # a tightly converged FP64 reference (Newton tolerance 1e-6) over the same increments, untimed: the plain
    # form's own tolerance (1e-3) leaves errors of that order, so both forms are also compared with it
    tight = []
    if args.form == "both":
        st = Forging3DSolver(dataclasses.replace(cfg, tol=1e-6), mesh, dies)
        st.set_stream(stream.cuda_stream)
        for _ in range(args.warmup):
            st.step()
        for _ in range(len(infos)):
            inf = st.step()
            tight.append({"load": inf["load"], "vg": st.array("vg").copy(), "eps": st.array("eps").copy()})
        st.close()

    def errors(run_infos, run_snaps, ref):
        k2 = min(len(run_infos), len(ref))
        if k2 == 0:
            return None
        rl2 = lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
        return {"load_rel_max": max(abs(run_infos[i]["load"] / ref[i]["load"] - 1) for i in range(k2)),
                "velocity_rel_l2_max": max(rl2(run_snaps[i]["vg"], ref[i]["vg"]) for i in range(k2)),
                "strain_rel_l2_max": max(rl2(run_snaps[i]["eps"], ref[i]["eps"]) for i in range(k2)),
                "increments": k2}

    # error of the timed form against the plain FP64 form, increment by increment
    kk = min(len(infos), len(infos64))
    load_err = max((abs(infos[i]["load"] / infos64[i]["load"] - 1) for i in range(kk)), default=None)
    vel_err = max((float(np.linalg.norm(snaps[i]["vg"] - snaps64[i]["vg"]) / np.linalg.norm(snaps64[i]["vg"]))
                   for i in range(kk)), default=None)
    eps_err = max((float(np.linalg.norm(snaps[i]["eps"] - snaps64[i]["eps"]) / max(np.linalg.norm(snaps64[i]["eps"]), 1e-300))
                   for i in range(kk)), default=None)

    # roofline: the factor's triangular-solve sweep (forward + backward over every front, one captured graph per
    # solve), HBM-bound; algorithmic bytes = the factor read once per sweep direction (a wide front's pivot-block
    # inverse has as many entries as the triangle it replaces) plus the permuted vectors in and out
    s.set_scalar("profile_solves", 1)  # events around every solve (a host wait each): after the timed region
    solves0, solve_ms0 = s.scalar("solves"), s.scalar("solve_gpu_ms")
    for _ in range(2):
        s.step()
    n_solves = s.scalar("solves") - solves0
    solve_ms = (s.scalar("solve_gpu_ms") - solve_ms0) / max(n_solves, 1)
    s.set_scalar("profile_solves", 0)
    vb = 4
    lnnz = s.scalar("factor_nnz")
    ndof = 3 * mesh.nn
    sbytes = 2 * lnnz * vb + ndof * (8 + 8 + 4 * vb)
    peak, peak_kind = measured_peak()
    achieved = sbytes / (solve_ms / 1000.0) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "solve_traffic.json")
    if os.path.exists(tp):
        try:
            with open(tp) as f:
                traffic = json.load(f).get("bytes_per_solve")
        except Exception:
            traffic = None

    # assembly (element + column kernels), the per-iteration HBM pass the element path is measured by
    nnz = int(s.scalar("nnz"))
    s.prepare_step()
    for _ in range(3):
        s.assemble(1, 1)
    asm = []
    for _ in range(10):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s.assemble(1, 1)
        b.record(stream)
        b.synchronize()
        asm.append(a.elapsed_time(b))
    asm_ms = float(np.median(asm))
    abytes = assembly_algorithmic_bytes(mesh.ne, mesh.nn, nnz)
    a_achieved = abytes / (asm_ms / 1000.0) / 1e9

    # end to end through the public API with host buffers: mesh/die upload, K increments, snapshot read-back
    e2e_steps = args.steps
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s2 = Forging3DSolver(fast_form(cfg), mesh, dies)
    s2.set_scalar("factor_fp32", 1)
    t_setup = time.perf_counter() - t0
    d2h = 0
    for _ in range(e2e_steps):
        s2.step()
        for nm in ("x", "vg", "contact", "eps", "dmg", "el_sig", "el_rate", "el_mean"):
            d2h += s2.array(nm).nbytes
    e2e_s = time.perf_counter() - t0
    e2e_parts = {"construct_ms": 1000.0 * t_setup}
    for q in ("t_order", "t_symbolic", "t_symbolic_wait", "t_symbolic_dev", "t_graph_factor", "t_graph_solve",
              "t_factor", "t_pcg"):
        try:
            e2e_parts[q[2:] + "_ms"] = 1000.0 * s2.scalar(q)
        except Exception:
            pass
    s2.close()
    h2d = mesh.x.nbytes + mesh.tets.nbytes + mesh.on_x0.nbytes + mesh.on_y0.nbytes + sum(d.h.nbytes for d in dies)

    gpu_launches = _count_launches(cfg, mesh, dies, stream, args.warmup, k, True) if rank == 0 else None
    closed_die = None
    if rank == 0 and args.form == "both" and not args.no_closed_die:
        try:
            closed_die = run_closed_die(stream, flush)
        except Exception as e:  # reported, not fatal: the headline line stands on its own
            closed_die = {"error": str(e)}
    if rank == 0:
        clocks = clk.summary()
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": k, "warmup": args.warmup,
                "ms_per_step": total_ms / k, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64 (factorisation f32, refined in f64)", "data": "synthetic",
                "config": config_dict(cfg, mesh, {
                    "form": "extrapolated warm start (the reference's ExtrapolateStart) + FP32 multifrontal factor "
                            "with FP64 PCG refinement, Newton tolerance 2e-4 (plain FP64 form: 1e-3)",
                    "l2": "flushed (256 MiB write) between timed increments",
                    "newton_iterations": int(sum(i["iterations"] for i in infos)),
                    "factorisations": int(infos[-1]["n_factor"] - infos[0]["n_factor"]) + 1 if infos else 0,
                    "factor": {q: s.scalar(q) for q in ("supernodes", "levels", "front_pool_mb", "max_front",
                                                        "factor_nnz")}}),
                "plain_fp64": {"value": 1000.0 / ms64, "unit": UNIT, "ms_per_step": ms64, "steps": len(durs64),
                               "speedup_of_value": value / world / (1000.0 / ms64)} if ms64 else None,
                "error_vs_plain_fp64": {"load_rel_max": load_err, "velocity_rel_l2_max": vel_err,
                                        "strain_rel_l2_max": eps_err, "increments": kk},
                "error_vs_tight_fp64": {"reference": "FP64 form, Newton tolerance 1e-6, same increments",
                                        "timed_form": errors(infos, snaps, tight),
                                        "plain_fp64": errors(infos64, snaps64, tight)} if tight else None,
                "roofline": {"kernel": "multifrontal triangular-solve sweep (forward + backward, one graph per solve)",
                             "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                             "algorithmic_bytes": sbytes, "ms_per_launch": solve_ms, "launches": int(n_solves)},
                "roofline_assembly": {"kernel": "assembly (k_element<MATRIX> + k_columns<MATRIX,BC>)", "bound": "hbm",
                                      "achieved": a_achieved, "peak": peak, "unit": "GB/s", "frac": a_achieved / peak,
                                      "peak_kind": peak_kind, "algorithmic_bytes": abytes, "ms_per_launch": asm_ms},
                "e2e": {"value": e2e_steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d / e2e_steps,
                        "d2h_bytes_per_step": d2h / e2e_steps, "increments": e2e_steps,
                        "host_ms": {k: round(v, 2) for k, v in e2e_parts.items()}},
                "gpu_launches": gpu_launches, "clocks": clocks, "closed_die": closed_die}
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_sample(budget_s=args.cpu_budget)
        print(json.dumps(line))
    s.close()
    if s64:
        s64.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=25.0)
    ap.add_argument("--no-closed-die", action="store_true", help="skip the closed-die gear-blank measurement")
    ap.add_argument("--form", default="both", choices=["both", "fp32"],
                    help="both: time the FP32-factor form and the plain FP64 form; fp32: the timed form only")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_gpu(args, rank, world)


if __name__ == "__main__":
    main()
