"""Benchmark of the B200 step path on the turbulent boundary-layer workload
(814 x 257 x 193 = 40,375,214 cells, RK3 at CFL 0.5, synthetic initial field).

Metric: ns per cell per RK3 step (lower is better) of the mixed FP32/FP64
form, with the FP64 plain form timed on the same field beside it and the
relative L2 difference of the two stated.  One process per GPU; every rank
advances its own replica box (weak scaling, no collective on the data path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl reference times the CPU restatement of the reference step (oracle/)
on the host cores, one RK3 substep per timed step, on the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "boundary-layer-gpu_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "ns/cell/RK3 step, mixed vs FP64 plain on one B200 at stated L2 error; HBM GB/s"
UNIT = "ns/cell/step"
CELLS_NOTE = "cells = nx*ny*nz"
# algorithmic HBM bytes per cell per RK3 step: 73 compulsory element passes
# (RHS+RK 33, projection 3 x 13, pressure save 1)
PASSES_PER_STEP = 73


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nx", type=int, default=814)
    ap.add_argument("--ny", type=int, default=257)
    ap.add_argument("--nz", type=int, default=193)
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--err-steps", type=int, default=100)
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-les", action="store_true")
    ap.add_argument("--no-cufft", action="store_true")
    ap.add_argument("--no-transition", action="store_true")
    ap.add_argument("--no-closure", action="store_true")
    ap.add_argument("--les-steps", type=int, default=200)
    ap.add_argument("--ts-steps", type=int, default=2000)
    ap.add_argument("--ens-boxes", type=int, default=64)
    ap.add_argument("--ens-steps", type=int, default=20)
    ap.add_argument("--profile", default=None, choices=["mixed", "fp64", "ensemble"],
                    help="profiling driver: set up, warm up, then run --steps steps between "
                         "cudaProfilerStart/Stop (for ncu --profile-from-start off); prints one line")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        d = os.environ.get("BLGPU_CLOCKS_DIR")  # where to keep the raw samples (default: a temporary file)
        self.out = os.path.join(d, "clocks_rank%d.csv" % index) if d and os.path.isdir(d) else \
            "/tmp/blgpu_clocks_%d_%d.csv" % (os.getpid(), index)

    def start(self):
        try:
            self.fh = open(self.out, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,timestamp",
                 "--format=csv,noheader,nounits", "-lms", "20"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self, t0=None, t1=None):
        """Median SM clock, its maximum and the throttle reasons seen, over
        the samples taken between the host times t0 and t1 (the timed region;
        all samples when none fall inside)."""
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        import datetime
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []
        for line in open(self.out):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[9], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(f[1]), float(f[2]), {n for n, v in zip(names, f[5:9]) if v.lower() == "active"}))
            except ValueError:
                continue
        inside = [r for r in rows if t0 is not None and t0 <= r[0] <= t1]
        use = inside if inside else rows
        if not use:
            return None
        reasons = set().union(*(r[3] for r in use))
        return {"sm_mhz": float(np.median([r[1] for r in use])), "sm_max_mhz": float(max(r[2] for r in use)),
                "reasons": sorted(reasons), "samples": len(use), "in_timed_region": bool(inside)}


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local) if args.impl == "b200" else None
        backend = "nccl" if args.impl == "b200" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, world, local, pg


def barrier(pg, local):
    if pg is None:
        return
    import torch
    if torch.cuda.is_available():
        pg.barrier(device_ids=[local])
    else:
        pg.barrier()


def allmax(pg, v, local):
    if pg is None:
        return v
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device="cuda:%d" % local if torch.cuda.is_available() else "cpu")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


# DRAM bytes per cell of one launch of the mixed-form kernels, measured by
# ncu (dram__bytes_read.sum + dram__bytes_write.sum) on the 814x129x97 box
# (state 128 MB per field triple, every kernel's inputs above the 126 MB L2)
# and scaled by cells; the RHS figure is (substep 1 + 2 x substep 2) / 3.
# Writes still in L2 when a launch ends are not counted, so these run a few
# per cent under the compulsory bytes.
MEASURED_TRAFFIC_PER_CELL = {"rhs_rk": (318.22e6 + 2 * 473.18e6) / 3 / 10185342,
                             "project": 267.69e6 / 10185342}


def algorithmic_bytes(phase, cells, esz, spectral_cells):
    """compulsory bytes of one launch of a phase (element passes x size)"""
    return {
        "rhs_rk": 11.0 * cells * esz,       # average of 9 (s1) and 12 (s2, s3) passes
        "div_dct": 4.0 * cells * esz,       # read U,V,W; write the DCT lines
        "dft_z": 2.0 * spectral_cells * esz,
        "thomas": 2.0 * spectral_cells * esz,
        "idft_z": 2.0 * spectral_cells * esz,
        "idct": 2.0 * spectral_cells * esz,
        "project": 7.0 * cells * esz,       # read p, U, V, W; write U, V, W
    }.get(phase)


def run_reference(args, rank, world, pg):
    """CPU restatement of the reference step on the host cores.

    Each bench step is one RK3 substep of the full box (the stages cycle
    1 -> 2 -> 3, compute_dt before stage 1), so `steps` timed bench steps are
    steps/3 RK3 steps; `ms_per_step` is the time of one bench step and
    `value` is three substeps' time per cell (one RK3 step)."""
    if rank != 0:
        return
    import oracle
    from blgpu import cases
    threads = len(os.sched_getaffinity(0))
    case = cases.turbulent_case(nx=args.nx, ny=args.ny, nz=args.nz)
    o = oracle.oracle_for(case, threads=threads)
    o.compute_dt()
    stage = 1
    times = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        o.rk3_stage(stage)
        el = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(el)
        stage = stage % 3 + 1
        if stage == 1:
            o.compute_dt()
    per_sub = float(np.mean(times))
    v = 3.0 * per_sub / case.cells * 1e9
    sample = ("each timed step is one RK3 substep of the full %dx%dx%d box (stages cycling 1-2-3, %d timed = "
              "%.2f RK3 steps); value = 3 x mean substep time / cells" % (args.nx, args.ny, args.nz, args.steps,
                                                                          args.steps / 3.0))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_sub * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "turbulent BL DNS %dx%dx%d, RK3 CFL 0.5, Lund inflow, FP64 CPU restatement"
                                   % (args.nx, args.ny, args.nz), "cells": case.cells,
                       "bench_step": "one RK3 substep"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline(args):
    """The CPU restatement on the host cores: one warm-up substep, then one
    timed substep of each RK3 stage of the full box; value = the three
    substeps' time per cell (one RK3 step)."""
    import oracle
    from blgpu import cases
    threads = len(os.sched_getaffinity(0))
    case = cases.turbulent_case(nx=args.nx, ny=args.ny, nz=args.nz)
    o = oracle.oracle_for(case, threads=threads)
    o.compute_dt()
    o.rk3_stage(1)  # warm-up (page faults, thread pool)
    o.rk3_stage(2)
    o.rk3_stage(3)
    o.compute_dt()
    el = 0.0
    for stage in (1, 2, 3):
        t0 = time.perf_counter()
        o.rk3_stage(stage)
        el += time.perf_counter() - t0
    v = el / case.cells * 1e9
    return {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "one RK3 step (stages 1, 2, 3 timed after a warm-up step) of the full %dx%dx%d box"
                      % (args.nx, args.ny, args.nz)}


def ensemble_boxes(args, dev, seed_offset=0):
    """The batched ensemble: uneven turbulent boxes with Lund inflow, mixed form."""
    import blgpu
    from blgpu import cases
    cs = cases.ensemble_cases(nbox=args.ens_boxes, seed=2024 + seed_offset)
    return cs, [cases.solver_for(c, precision=blgpu.MIXED, device=dev) for c in cs]


def run_ensemble(args, dev, pg, local, world):
    """Aggregate cells*steps/s of the ensemble in one graph launch per step,
    against the same boxes advanced one after another."""
    import blgpu
    cs, box = ensemble_boxes(args, dev, seed_offset=int(os.environ.get("RANK", "0")))
    ens = blgpu.Ensemble(box)
    cells = ens.cells
    t0 = time.perf_counter()
    ens.advance(args.warmup)
    ens.sync()
    ms_default = ens.time(args.ens_steps) / args.ens_steps
    ms_seq_default = ens.time(args.ens_steps, sequential=True) / args.ens_steps
    ntuned = ens.autotune(steps=3)
    tune_s = time.perf_counter() - t0
    ens.advance(1)
    ens.sync()
    barrier(pg, local)
    ms = allmax(pg, ens.time(args.ens_steps), local) / args.ens_steps
    ms_seq = allmax(pg, ens.time(args.ens_steps, sequential=True), local) / args.ens_steps
    shapes = sorted({(s.nx, s.ny, s.nz) for s in box})
    tiles = {"%dx%dx%d" % sh: next(s.tiles() for s in box if (s.nx, s.ny, s.nz) == sh) for sh in shapes}
    out = {"boxes": len(box), "cells": cells, "steps_timed": args.ens_steps, "precision": "mixed",
           "recipe": "nx in {128,192,256}, ny 65, nz in {64,96}, Re_theta in [800,1500], Lund inflow, RK3 CFL 0.5",
           "ms_per_step": ms, "cells_steps_per_s": cells * world / (ms * 1e-3),
           "ns_per_cell_step": ms * 1e6 / (cells * world),
           "sequential_ms_per_step": ms_seq, "speedup_vs_sequential": ms_seq / ms,
           "before_autotune": {"ms_per_step": ms_default, "sequential_ms_per_step": ms_seq_default},
           "autotuned_shapes": ntuned, "tiles": tiles, "setup_and_tune_s": round(tune_s, 2),
           "graph_launches_per_step": 1, "kernels_per_step": None}
    l0 = ens.launches()
    ens.advance(1)
    out["kernels_per_step"] = ens.launches() - l0
    ens.close()
    for s in box:
        s.close()
    return out


def run_les(args, dev):
    """LES legs on the headline box in the mixed form: the device Smagorinsky
    (LES = 1) and dynamic Smagorinsky (LES = 2 z-averaged, 3 pointwise) eddy
    viscosity evaluated before every substep.  Fixed dt = 2e-4 so that the
    synthetic field stays finite under the eddy viscosity; the step is timed
    with CUDA events (advance_timed), one eddy-viscosity evaluation by wall
    clock around the synchronising blgpu_eddy_viscosity call."""
    import blgpu
    from blgpu import cases
    case = cases.turbulent_case(nx=args.nx, ny=args.ny, nz=args.nz)
    case.cfl = -2e-4
    out = {}
    for model in (1, 2, 3):
        s = cases.solver_for(case, precision=blgpu.MIXED, les_model=model, device=dev)
        s.advance(2)
        step = s.advance_timed(3) / 3
        s._ck(s.lib.blgpu_eddy_viscosity(s.ctx))
        t0 = time.perf_counter()
        for _ in range(3):
            s._ck(s.lib.blgpu_eddy_viscosity(s.ctx))
        ev = (time.perf_counter() - t0) / 3 * 1e3
        out["les%d" % model] = {"step_ms": step, "eddy_viscosity_ms": ev,
                                "nu_t_finite": bool(np.isfinite(s.nu_t()).all())}
        s.close()
    return out


def run_cufft(args, case, dev):
    """The cuFFT comparison path (poisson = BLGPU_POISSON_CUFFT) against the
    hand-written transforms on the same box: graph-replayed step time and the
    per-phase device times (CUDA events) of the Poisson solve, FP64 and mixed."""
    import blgpu
    from blgpu import cases
    out = {}
    for name, prec in (("fp64", blgpu.FP64), ("mixed", blgpu.MIXED)):
        s = cases.solver_for(case, precision=prec, device=dev, poisson=blgpu.POISSON_CUFFT)
        s.advance(2)
        n = 5
        ms = s.advance_timed(n) / n
        ph = s.phase_times(1)
        keep = ("div_dct", "dft_z", "thomas", "idft_z", "idct", "project")
        out[name] = {"ms_per_step": round(ms, 4),
                     "poisson_ms_per_step": round(sum(ph[k][0] for k in keep), 4),
                     "phases": {k: round(ph[k][0], 4) for k in keep}}
        s.close()
    return out


def run_transition(args, dev):
    """Tollmien-Schlichting transition on the 1024 x 129 x 128 box (400 x 20 x 40
    delta*, Re_delta* = 1000 at the inflow): a 2-D TS wave at omega = 0.1
    (amplitude 1e-3) and an oblique pair (1e-4, seeded phases) from the
    Orr-Sommerfeld solve, forced through the reference-format mode file, 2000
    steps at a fixed dt of 1/400 forcing period (CFL 0.4 on the x spacing);
    the spatial growth rate of the wave envelope, mixed against FP64."""
    import tempfile
    import blgpu
    from blgpu import files, transition
    lz = 40.0
    beta = 2.0 * np.pi / lz  # the box's spanwise wavenumber closest to 0.2
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "ts_modes.dat")
        info = transition.ts_mode_file(path, beta=beta)
        c = transition.transition_case(nx=1024, ny=129, nz=128, lx=400.0, ly=20.0, lz=lz)
        modes = files.read_temporal_modes(path, c.y)
    out = {"grid": [1024, 129, 128], "steps": args.ts_steps, "beta": beta, "os": info}
    t0 = time.perf_counter()
    g64, _, _ = transition.run_growth(c, modes, blgpu.FP64, steps=args.ts_steps, device=dev, x_fit=(20.0, 90.0))
    g32, _, _ = transition.run_growth(c, modes, blgpu.MIXED, steps=args.ts_steps, device=dev, x_fit=(20.0, 90.0))
    out.update({"growth_fp64": g64, "growth_mixed": g32, "rel_diff": abs(g32 - g64) / abs(g64),
                "wall_s": round(time.perf_counter() - t0, 1)})
    return out


def run_closure(args, dev):
    """The learned wall-stress closure: trained on the turbulent DNS recipe's
    own wall samples (814 x 257 x 193, 12 snapshots of the row at h = 0.1
    delta99 after 300 steps, 2 more held out), assessed on the held-out states
    against the resolved wall stress beside the equilibrium law of the wall,
    then both as the wall condition of the 512 x 96 x 256 wall-modelled LES."""
    from blgpu import wallmodel, WallNet
    t0 = time.perf_counter()
    net, hold = WallNet(seed=11), WallNet(seed=12)
    info = wallmodel.config2_training(net, hold, device=dev)
    l0 = net.eval()
    wallmodel.train(net)
    l1 = net.eval()
    e = wallmodel.holdout_errors(net, hold, info["tau_eq"])
    c = wallmodel.config4_case()
    jh = wallmodel.row_at(c, 0.1)
    cf_eq = wallmodel.run_cf(c, 1, jh=jh, steps=args.les_steps, device=dev)
    cf_net = wallmodel.run_cf(c, 2, net, jh=jh, steps=args.les_steps, device=dev)
    r = lambda v: float("%.5g" % v)
    return {"samples": info["samples"], "held_out": info["held_samples"], "dns_steps": info["steps"],
            "h": r(info["h"]), "loss": [r(l0), r(l1)],
            "held_out_cf": {"dns": r(e["cf_dns"]), "network": r(e["cf_net"]), "equilibrium": r(e["cf_eq"])},
            "held_out_rms_tau": {"network": r(e["rms_net"]), "equilibrium": r(e["rms_eq"])},
            "les_512x96x256_cf": {"equilibrium": r(cf_eq), "network": r(cf_net), "steps": args.les_steps},
            "wall_s": round(time.perf_counter() - t0, 1)}


def run_profile(args):
    """Small driver for ncu: set-up and warm-up outside the profiled range."""
    import torch
    import blgpu
    from blgpu import cases
    torch.cuda.set_device(0)
    if args.profile == "ensemble":
        _, box = ensemble_boxes(args, 0)
        ens = blgpu.Ensemble(box)
        ens.advance(args.warmup)
        ens.sync()
        torch.cuda.profiler.start()
        ens.advance(args.steps)
        ens.sync()
        torch.cuda.profiler.stop()
        print(json.dumps({"profile": "ensemble", "boxes": len(box), "steps": args.steps}))
        return
    case = cases.turbulent_case(nx=args.nx, ny=args.ny, nz=args.nz)
    prec = blgpu.MIXED if args.profile == "mixed" else blgpu.FP64
    s = cases.solver_for(case, precision=prec)
    s.advance(args.warmup)
    s.sync()
    torch.cuda.profiler.start()
    s.advance(args.steps)
    s.sync()
    torch.cuda.profiler.stop()
    print(json.dumps({"profile": args.profile, "grid": [args.nx, args.ny, args.nz], "steps": args.steps,
                      "max_div": s.check_divergence()}))


def main():
    args = parse()
    if args.profile:
        run_profile(args)
        return
    rank, world, local, pg = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, rank, world, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    import torch
    import blgpu
    from blgpu import cases
    dev = local
    torch.cuda.set_device(dev)
    case = cases.turbulent_case(nx=args.nx, ny=args.ny, nz=args.nz, seed=1234 + rank)
    cases.project_initial(case, device=dev)
    cells = case.cells
    N, M, NM = case.nx - 2, case.nz - 2, case.ny - 1
    spectral_cells = N * M * NM

    span = {}

    def timed_run(precision):
        s = cases.solver_for(case, precision=precision, device=dev)
        s.advance(args.warmup)
        s.sync()
        barrier(pg, local)
        l0 = s.kernel_launches()
        t0 = time.time()
        ms = s.advance_timed(args.steps)
        span[precision] = (t0, time.time())
        launches = s.kernel_launches() - l0
        barrier(pg, local)
        return s, ms, launches

    hbm, peak_kind = peaks()
    clocks = Clocks(dev)
    # ---- mixed form (headline) ----
    clocks.start()
    smix, ms_mix, launches = timed_run(blgpu.MIXED)
    clk = clocks.stop(*span[blgpu.MIXED])
    ms_mix = allmax(pg, ms_mix, local)
    ms_step_mix = ms_mix / args.steps
    value = ms_step_mix * 1e6 / (cells * world)
    # ---- FP64 plain form ----
    fp64 = None
    err = None
    if not args.no_fp64:
        s64, ms64, _ = timed_run(blgpu.FP64)
        ms64 = allmax(pg, ms64, local)
        ms_step64 = ms64 / args.steps
        fp64 = {"ns_per_cell_step": ms_step64 * 1e6 / (cells * world), "ms_per_step": ms_step64,
                "hbm_gbs_step": PASSES_PER_STEP * 8.0 * cells / (ms_step64 * 1e-3) / 1e9}
        Um, Vm, Wm, _, tm = smix.download_state()
        U6, V6, W6, _, t6 = s64.download_state()
        err = {"u": float(np.linalg.norm(Um - U6) / np.linalg.norm(U6)),
               "v": float(np.linalg.norm(Vm - V6) / np.linalg.norm(V6)),
               "w": float(np.linalg.norm(Wm - W6) / np.linalg.norm(W6)),
               "steps": args.warmup + args.steps, "t": t6,
               "max_div_mixed": smix.check_divergence(), "max_div_fp64": s64.check_divergence()}
        ph64 = s64.phase_times(1)
        s64.close()
        # error of the mixed form after ERR_STEPS RK3 steps from the same field
        a = cases.solver_for(case, precision=blgpu.FP64, device=dev)
        b = cases.solver_for(case, precision=blgpu.MIXED, device=dev)
        a.advance(args.err_steps)
        b.advance(args.err_steps)
        A, B = a.download_state()[:3], b.download_state()[:3]
        err["after_%d_steps" % args.err_steps] = {
            n: float(np.linalg.norm(x - y) / np.linalg.norm(y)) for n, x, y in zip("uvw", B, A)}
        a.close()
        b.close()
    # ---- per-phase device times (CUDA events on the solver stream) ----
    ph = smix.phase_times(2)
    step_ms = sum(v[0] for v in ph.values()) / 2.0
    dom = max((k for k in ph if algorithmic_bytes(k, cells, 4, spectral_cells)), key=lambda k: ph[k][0])
    dom_ms, dom_n = ph[dom]
    launch_ms = dom_ms / max(dom_n, 1)
    alg = algorithmic_bytes(dom, cells, 4, spectral_cells)
    achieved = alg / (launch_ms * 1e-3) / 1e9
    traffic = MEASURED_TRAFFIC_PER_CELL.get(dom)
    roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_kind": peak_kind,
            "traffic": traffic * cells if traffic is not None else None,
            "traffic_source": "ncu DRAM bytes at 814x129x97 scaled by cells" if traffic is not None else None,
            "algorithmic_bytes_per_launch": alg, "launch_ms": launch_ms}
    # ---- end to end through the C ABI with pinned host buffers ----
    # a stream of states through the solver: per step the FP64 Fortran-layout
    # state goes up, one RK3 step runs and the new state comes down; the
    # streamed calls let the upload of the next state, the step and the
    # download of the previous state overlap
    pin = lambda shape: torch.empty(int(np.prod(shape)), dtype=torch.float64, pin_memory=True).numpy().reshape(
        shape, order="F")
    Uh = pin(case.U.shape); Vh = pin(case.V.shape); Wh = pin(case.W.shape)
    Uh[...] = case.U; Vh[...] = case.V; Wh[...] = case.W
    Uo_ = pin(case.U.shape); Vo_ = pin(case.V.shape); Wo_ = pin(case.W.shape)
    e2e_n = max(1, args.e2e_steps)
    import ctypes
    lib = smix.lib
    dp = blgpu._lib.c_double_p
    ptr = lambda a: a.ctypes.data_as(dp)

    def e2e_step():
        blgpu._lib.check(lib.blgpu_upload_state_async(smix.ctx, ptr(Uh), ptr(Vh), ptr(Wh), 0.0), smix.ctx)
        blgpu._lib.check(lib.blgpu_advance(smix.ctx, 1), smix.ctx)
        blgpu._lib.check(lib.blgpu_download_state_async(smix.ctx, ptr(Uo_), ptr(Vo_), ptr(Wo_)), smix.ctx)

    e2e_step()  # staging buffers and transfer streams, outside the timed region
    smix.sync()
    barrier(pg, local)
    t0 = time.perf_counter()
    for _ in range(e2e_n):
        e2e_step()
    smix.sync()
    el = time.perf_counter() - t0
    el = allmax(pg, el, local)
    bytes_state = 8 * (Uh.size + Vh.size + Wh.size)
    e2e = {"value": el / e2e_n * 1e9 / (cells * world), "unit": UNIT, "h2d_bytes_per_step": bytes_state,
           "d2h_bytes_per_step": bytes_state, "steps": e2e_n,
           "what": "upload_state_async + advance(1) + download_state_async per step (FP64 Fortran-layout pinned "
                   "host arrays, copies overlapping the steps), wall clock to the final blgpu_sync"}
    smix.close()
    cufft = None
    if world == 1 and not args.no_cufft:
        cufft = run_cufft(args, case, dev)
        keep = ("div_dct", "dft_z", "thomas", "idft_z", "idct", "project")
        cufft["native_poisson_ms_per_step"] = {"mixed": round(sum(ph[k][0] for k in keep) / 2.0, 4),
                                               "fp64": round(sum(ph64[k][0] for k in keep), 4) if fp64 else None}
    ens = None
    if not args.no_ensemble:
        ens = run_ensemble(args, dev, pg, local, world)
    ts = None
    if world == 1 and not args.no_transition:
        ts = run_transition(args, dev)
    closure = None
    if world == 1 and not args.no_closure:
        closure = run_closure(args, dev)
    les = None
    if world == 1 and not args.no_les:
        les = run_les(args, dev)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args)
    if rank == 0:
        if ens is not None:  # per-shape launch shapes: detail for the log, kept off the result line
            print(json.dumps({"ensemble_tiles": ens.pop("tiles")}), file=sys.stderr, flush=True)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step_mix, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 fields / f64 y-solve", "data": "synthetic",
                "config": {"workload": "turbulent BL DNS %dx%dx%d, RK3 CFL 0.5, Lund inflow i=%d, mixed FP32/FP64"
                                       % (case.nx, case.ny, case.nz, case.lund[1]),
                           "cells": cells, "l2": "inputs larger than L2 (3 x %.0f MB per state)"
                                                  % (smix_bytes(case, 4) / 1e6),
                           "replicas_per_gpu": 1},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clk, "ensemble": ens, "les_mixed": les, "cufft_path": cufft, "transition": ts, "closure": closure,
                "phases_ms_per_step_mixed": {k: round(v[0] / 2.0, 4) for k, v in ph.items()},
                "phases_ms_per_step_fp64": ({k: round(v[0], 4) for k, v in ph64.items()} if fp64 else None),
                "eager_step_ms_mixed": step_ms,
                "hbm_gbs_step": PASSES_PER_STEP * 4.0 * cells / (ms_step_mix * 1e-3) / 1e9,
                # the headline's own evidence last, so that it stays in the tail of the line
                "fp64": fp64, "mixed_rel_l2_vs_fp64": err,
                "speedup_mixed_vs_fp64": (fp64["ms_per_step"] / ms_step_mix) if fp64 else None}
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


def smix_bytes(case, esz):
    return (case.nx + 1 + 31) // 32 * 32 * (case.ny + 1) * (case.nz + 1) * esz


if __name__ == "__main__":
    main()
