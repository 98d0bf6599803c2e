#!/usr/bin/env python
"""Benchmark of the explicit RHS + SSP-RK3 time step on B200.

Metric: cell-updates/s per RK3 stage = nx*ny*nz*3*steps / seconds.
Workload (one "step" = one TimeScheme::step, i.e. three RK stages):
  temporal double shear layer, 256^3 periodic cells on [0,2pi]^3, rho=1,
  p=1/(gamma M^2) with M=0.5, seeded SplitMix64 noise 1e-3 on v and w,
  FP64 characteristic-wise WENO-5 (Shu weights, Lax-Friedrichs splitting) +
  second-order centered viscous terms (mu = 6.283e-4, Pr = 0.72), CFL 0.5,
  reference semantics.  Synthetic input; the device state (2.9 GB) is larger
  than L2, so no flush is needed between timed steps.

Arms:
  default            our CUDA path (libns_b200.so through its C ABI)
  --impl reference   the reference's own CPU TimeScheme::step (compiled from its
                     sources into oracle/_ref, OpenMP on all host cores)
Multi-GPU (torchrun): every rank advances an independent replica (the path is
single-GPU by design: no collective on the data path); value sums the ranks,
time is the max over ranks.
"""
import argparse
import csv
import importlib
import io
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s per RK3 stage on 1 B200 (FP32+learned vs plain FP64) at stated L2 err"
UNIT = "cell-updates/s"

FORMS = {
    # name: (convection, precision, sensor, dtype label)
    "fp64_char": (2, 0, 0, "f64"),
    "fp64_comp": (1, 0, 0, "f64"),
    "fp32_char": (2, 1, 0, "f32 (f64 RK3 accumulation and reductions)"),
    "fp32_comp": (1, 1, 0, "f32 (f64 RK3 accumulation and reductions)"),
    "fp32_sensor": (2, 1, 1, "f32 + bf16 sensor (f64 RK3 accumulation and reductions)"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256, help="cells per axis of the shear-layer box")
    ap.add_argument("--form", default="fp64_char", choices=sorted(FORMS))
    ap.add_argument("--also", default="fp64_comp,fp32_char,fp32_comp,fp32_sensor",
                    help="extra forms timed after the headline (comma list, '' for none)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def workload_params(pkg, n, form):
    conv, prec, sensor, _ = FORMS[form]
    L = 2 * math.pi
    # mu = rho0 * dU * delta / Re with dU = 2, delta = 0.05*2pi, Re = 1000
    return pkg.make_params(n, n, n, L=(L, L, L), mu=2.0 * 0.05 * 2 * math.pi / 1000.0, Pr=0.72,
                           gamma=1.4, cfl=0.5, convection=conv, diffusion_order=2, precision=prec,
                           sensor=sensor)


def workload_name(n, form):
    return (f"shear_layer {n}^3 periodic [0,2pi]^3 M=0.5 Re=1000, {form} WENO-5 (Shu, LF alpha=3) "
            f"+ CD-2 viscous, SSP-RK3 CFL 0.5, reference semantics")


# ---------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv",
                                          "-lms", "200"], stdout=self.tmp, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.tmp.flush()
        self.tmp.seek(0)
        rows = list(csv.reader(io.StringIO(self.tmp.read())))
        os.unlink(self.tmp.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows[1:]:
            if len(r) < 9 or r[0].strip() != str(self.gpu):
                continue
            try:
                sm.append(float(r[1].split()[0]))
                smax = float(r[2].split()[0])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if "Active" in v and "Not" not in v:
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own TimeScheme::step (oracle/_ref) on host cores

def cpu_baseline(steps=2, warmup=1, n=256):
    from oracle import oracle as O
    pkg = importlib.import_module("3dnssolver_b200")
    threads = os.cpu_count() or 1
    p = workload_params(pkg, n, "fp64_char")
    if O.ref_available(strict=False):
        r = O.ref_bench(p, steps=steps, warmup=warmup, threads=threads, timed=True)
        return {"value": r["cell_updates_per_s"], "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": f"{steps} timed TimeScheme::step calls (after {warmup} warm-up) of the "
                          f"same workload at {n}^3, reference sources built with -O3 -ffast-math, "
                          f"OpenMP {threads} threads, 1 rank", "seconds": r["seconds"]}
    # the oracle port (strict IEEE C restatement) when the reference build is absent
    wl = importlib.import_module("3dnssolver_b200.workloads")
    n = 64
    p = workload_params(pkg, n, "fp64_char")
    W = wl.shear_layer(p, seed=1)
    O.run(p, W, 1)
    t0 = time.perf_counter()
    O.run(p, W, steps)
    sec = time.perf_counter() - t0
    return {"value": n ** 3 * 3 * steps / sec, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} steps at {n}^3 of the oracle port", "seconds": sec}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    # sample grid: keep the whole --warmup/--steps run within a few minutes
    n = 256 if args.warmup + args.steps <= 16 else 128
    try:
        from oracle import oracle as O
        if not O.ref_available(strict=False):
            print(json.dumps({"impl": "reference", "unavailable":
                              "oracle/_ref/ref_harness_timed not built (needs the reference tree)"}))
            return 0
        pkg = importlib.import_module("3dnssolver_b200")
        p = workload_params(pkg, n, "fp64_char")
        threads = os.cpu_count() or 1
        r = O.ref_bench(p, steps=args.steps, warmup=args.warmup, threads=threads, timed=True)
    except Exception as e:  # report, do not crash the driver
        print(json.dumps({"impl": "reference", "unavailable": f"reference run failed: {e}"}))
        return 0
    v = r["cell_updates_per_s"]
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * r["seconds"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(args.n, "fp64_char"), "sample_grid": [n, n, n],
                   "parallelism": "1 rank, OpenMP"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"each step one TimeScheme::step at {n}^3 (reference sources, "
                                   f"-O3 -ffast-math, OpenMP {threads} threads)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


# ---------------------------------------------------------------------------
# replicas: one rank per GPU, each advancing its own copy of the workload

def max_over_ranks(x, dist=None, device="cuda"):
    """Maximum of a per-rank float over all ranks (the job's time is its slowest rank)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, cells, steps, ms_max):
    """Whole-job cell-updates/s per RK3 stage: every rank advanced `cells` cells `steps` steps."""
    return world * cells * 3 * steps / (ms_max / 1000.0)


# ---------------------------------------------------------------------------
# rooflines of the dominant kernel

# Floating-point work per unit of each kernel class, counted by ncu on the 128^3
# shear layer (sm__sass_thread_inst_executed_op_{d,f}{fma,mul,add}[2]_pred_on.sum
# divided by the faces or cells of the launch; the counts do not depend on the data):
# (flop per unit with an FMA as 2, FP lane operations per unit with a packed f32x2
# operation as 2, pipe, unit).  The fused stage rows are the first two stages; the
# third adds the next step's start (about 70 FP64 instructions per cell).
COMPUTE_PER_UNIT = {
    ("fp64_char", "face_x"): (1325, 953, "fp64", "face"),
    ("fp64_char", "face_y"): (1325, 953, "fp64", "face"),
    ("fp64_char", "face_z"): (1318, 946, "fp64", "face"),
    ("fp64_comp", "face_x"): (965, 729, "fp64", "face"),
    ("fp64_comp", "face_y"): (965, 729, "fp64", "face"),
    ("fp64_comp", "face_z"): (941, 705, "fp64", "face"),
    ("fp64_char", "update"): (316, 205, "fp64", "cell"),
    ("fp64_comp", "update"): (316, 205, "fp64", "cell"),
    # x-faces marched with the update (second stage; measured per cell)
    ("fp64_char", "xface_update"): (1505, 1083, "fp64", "cell"),
    ("fp64_comp", "xface_update"): (1155, 856, "fp64", "cell"),
    # viscous terms, CD-2 reference semantics (measured per cell)
    ("fp64_char", "viscous"): (222, 135, "fp64", "cell"),
    ("fp64_comp", "viscous"): (222, 135, "fp64", "cell"),
    ("fp32_char", "stage_fused"): (4137, 2831, "fp32", "cell"),
    ("fp32_comp", "stage_fused"): (3177, 2218, "fp32", "cell"),
}
# DRAM bytes (read + write) per unit from the same capture; these kernels stream
# their inputs once at 128^3 and above, so the traffic scales with the units.
TRAFFIC_PER_UNIT = {
    ("fp64_char", "face_x"): 120.4, ("fp64_char", "face_y"): 118.6, ("fp64_char", "face_z"): 113.6,
    ("fp64_comp", "face_x"): 119.7, ("fp64_comp", "face_y"): 118.7, ("fp64_comp", "face_z"): 113.3,
    ("fp64_char", "update"): 283.7, ("fp64_comp", "update"): 283.7,
    ("fp64_char", "xface_update"): 332.7, ("fp64_comp", "xface_update"): 330.3,
    ("fp64_char", "viscous"): 51.2, ("fp64_comp", "viscous"): 51.2,
}


def profile(s, reps=3):
    """Mean per-class device ms of one step (events between the kernels)."""
    profs = [s.profile_step() for _ in range(reps)]
    return {k: statistics.mean(pr[k] for pr in profs) for k in profs[0]}


def rooflines(form, prof, n, peaks, fma):
    """HBM and compute rooflines of the form's dominant kernel class."""
    cells = n ** 3
    dom = max(prof, key=prof.get)
    launches = 1 if dom == "step_begin" else 3
    per_launch_ms = prof[dom] / launches
    # algorithmic bytes: a face-flux launch reads W and U (2 x 5 doubles per cell) and
    # writes 5 values per face; an update launch reads U, U0 and 3 face arrays and
    # writes U; a fused stage reads U_in and U0 and writes U_out: 120 B per cell (the
    # third stage also writes the next step's U0; the common 120 B/cell-stage unit is kept)
    elem = 4 if FORMS[form][1] == 1 else 8
    faces = (n + 1) * n * n
    face_bytes = cells * 80 + faces * 5 * elem
    alg = {"face_x": face_bytes, "face_y": face_bytes, "face_z": face_bytes,
           "update": cells * (3 * 40) + 3 * faces * 5 * elem + cells * 40,
           "fill_prim": (n + 6) ** 3 * 80, "step_begin": (n + 6) ** 3 * 120,
           "stage_fused": cells * 120,
           # per-step sensor flags: U0 read once per axis, one byte per face written
           "sensor": 3 * (cells * 40 + faces),
           # x-faces + update: W and U (x stencils), the y- and z-face fluxes and U0
           # read, U_out and the next stage's W written (+ the 4 viscous terms read)
           "xface_update": cells * 312,
           # viscous terms: W (rho, p, u, v) read, 4 doubles written per cell
           "viscous": cells * 64}
    kname = {"stage_fused": f"k_stage_march ({form})", "update": f"k_update ({form})",
             "sensor": f"k_sensor_mask ({form})", "xface_update": f"k_xface_update ({form})",
             "viscous": f"k_viscous ({form})"}.get(
        dom, f"k_face_flux ({dom}, {form})" if dom.startswith("face") else dom)
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    achieved = alg[dom] / (per_launch_ms / 1000.0) / 1e9
    units = faces if dom.startswith("face") else cells
    tpu = TRAFFIC_PER_UNIT.get((form, dom))
    hbm = {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
           "frac": round(achieved / hbm_peak, 4),
           "traffic": round(tpu * units) if tpu else None,
           "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per unit at 128^3, "
                             "scaled by the units of this launch" if tpu else None,
           "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peaks else "fallback 6650 GB/s",
           "algorithmic_bytes_per_launch": alg[dom], "launch_ms": round(per_launch_ms, 4)}
    comp = None
    row = COMPUTE_PER_UNIT.get((form, dom))
    if row:
        flop_u, inst_u, pipe, unit = row
        peak = fma[pipe]
        tflops = flop_u * units / (per_launch_ms / 1000.0) / 1e12
        # FP lane operations against the FMA rate (peak / 2 flops): a multiply or add
        # takes the same pipe slot as an FMA, so this is the pipe's busy fraction
        ops_rate = inst_u * units / (per_launch_ms / 1000.0) / 1e12
        comp = {"bound": pipe, "kernel": kname, "achieved": round(tflops, 2), "peak": round(peak, 2),
                "unit": "TFLOP/s", "frac": round(tflops / peak, 4),
                "pipe_frac": round(ops_rate / (peak / 2.0), 4),
                "peak_source": f"measured now: ns_fma_peak ({pipe} FMA chains on every SM)",
                "flop_per_" + unit: flop_u, "fp_ops_per_" + unit: inst_u}
        hbm["note"] = f"{pipe}-pipe bound: see compute_roofline"
    return hbm, comp


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)

    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    def rank_max(x):
        return max_over_ranks(x, dist)

    pkg = importlib.import_module("3dnssolver_b200")
    wl = importlib.import_module("3dnssolver_b200.workloads")
    n = args.n
    cells = n ** 3
    p = workload_params(pkg, n, args.form)
    W0 = wl.shear_layer(p, seed=1 + rank)
    # a dedicated stream: the context adopts it, so CUDA events recorded on it bracket
    # exactly the library's kernels (torch's default stream is the legacy NULL stream)
    stream = torch.cuda.Stream()

    sensor_w, sensor_info = None, None

    def time_form(form, steps, warmup, sample_clocks=False):
        nonlocal sensor_w, sensor_info
        pf = workload_params(pkg, n, form)
        if FORMS[form][2] and sensor_w is None:
            sensor_mod = importlib.import_module("3dnssolver_b200.sensor")
            X, y = sensor_mod.default_training_set()
            sensor_w, sensor_info = sensor_mod.train(X, y, seed=0)
            del X, y
        s = pkg.Solver(pf)
        s.set_stream(stream.cuda_stream)
        if FORMS[form][2]:
            s.set_sensor_weights(sensor_w)
        s.upload_primitive(W0)
        s.advance(warmup)
        torch.cuda.synchronize()
        clk = ClockSampler(local) if sample_clocks else None
        if clk:
            clk.start()
            # untimed steps for about a second, so that the sampler (200 ms period)
            # sees the GPU under this load right up to and through the timed region
            t0 = time.time()
            while time.time() - t0 < 1.0:
                s.advance(2)
                torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        l0 = s.launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.advance(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1)
        launches = s.launches - l0
        clocks = clk.stop() if clk else None
        diag = s.diagnostics()
        return s, ms, launches, clocks, diag

    s, ms, launches, clocks, diag = time_form(args.form, args.steps, args.warmup, sample_clocks=True)
    ms_max = rank_max(ms)
    value = job_rate(world, cells, args.steps, ms_max)

    # per-kernel device times of one step (events between kernels on the same stream)
    prof = profile(s)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    fma = {"fp64": pkg.fma_peak(True), "fp32": pkg.fma_peak(False)}
    roofline, compute_roofline = rooflines(args.form, prof, n, peaks, fma)

    # end to end through the C ABI with host buffers: ns_time_step uploads W from pinned
    # host memory, runs the step and downloads W every step
    Wh_t = torch.empty(W0.shape, dtype=torch.float64, pin_memory=True)
    Wh = Wh_t.numpy()
    Wh[...] = W0
    s.time_step(Wh)  # warm-up
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        s.time_step(Wh)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = rank_max(e0.elapsed_time(e1))
    e2e = {"value": job_rate(world, cells, args.e2e_steps, e2e_ms), "unit": UNIT,
           "h2d_bytes_per_step": int(Wh.nbytes), "d2h_bytes_per_step": int(Wh.nbytes),
           "steps": args.e2e_steps, "api": "ns_time_step (TimeScheme::step drop-in), pinned host W"}
    s.close()

    # extra forms on the same workload (same timing rules); every form advances the
    # same initial state by warmup + steps steps, so their states compare with the
    # headline form's: relative L2 error per conserved field against it
    g3 = slice(3, -3)
    forms = {args.form: {"value": value, "ms_per_step": ms_max / args.steps}}
    if FORMS[args.form][2]:
        forms[args.form]["sensor_fraction"] = diag["sensor_fraction"]
        forms[args.form]["sensor_training"] = sensor_info
    U_ref = None
    if args.also:
        s0 = pkg.Solver(p)
        if FORMS[args.form][2]:
            s0.set_sensor_weights(sensor_w)
        s0.upload_primitive(W0)
        s0.advance(args.warmup + args.steps)
        U_ref = s0.download_conservative()[g3, g3, g3]
        s0.close()
    names = ["rho", "rhoE", "rhou", "rhov", "rhow"]
    for f in [x for x in args.also.split(",") if x and x != args.form]:
        try:
            s2, ms2, l2, _, d2 = time_form(f, args.steps, args.warmup)
            U2 = s2.download_conservative()[g3, g3, g3]
            hbm2, comp2 = rooflines(f, profile(s2), n, peaks, fma)
            s2.close()
            ms2 = rank_max(ms2)
            num = np.sqrt(((U2 - U_ref) ** 2).reshape(-1, 5).sum(0))
            den = np.sqrt((U_ref ** 2).reshape(-1, 5).sum(0))
            forms[f] = {"value": job_rate(world, cells, args.steps, ms2),
                        "ms_per_step": ms2 / args.steps, "gpu_launches": l2,
                        "rel_l2_vs_" + args.form: {k: float(v) for k, v in zip(names, num / den)},
                        "roofline": hbm2, "compute_roofline": comp2}
            if FORMS[f][2]:
                forms[f]["sensor_fraction"] = d2["sensor_fraction"]
                forms[f]["sensor_training"] = sensor_info
        except Exception as e:
            forms[f] = {"error": str(e)}
    del U_ref

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(n=n)
        except Exception as e:
            cpu = {"error": str(e)}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": FORMS[args.form][3], "data": "synthetic",
            "config": {"workload": workload_name(n, args.form), "grid": [n, n, n], "form": args.form,
                       "l2": "no flush: device state 2.9 GB > 126 MB L2",
                       "parallelism": f"{world} independent replica(s), no data-path collective"},
            "roofline": roofline, "compute_roofline": compute_roofline,
            "kernel_ms_per_step": {k: round(v, 4) for k, v in prof.items()},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
            "forms": forms,
            "diagnostics": {"nonfinite": diag["nonfinite"], "dt": diag["dt"],
                            "mass": diag["mass"], "kinetic": diag["kinetic"]},
        }
        print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
