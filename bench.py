#!/usr/bin/env python
"""Benchmark of the explicit RHS + SSP-RK3 time step on B200.

Metric: cell-updates/s per RK3 stage = nx*ny*nz*3*steps / seconds.
Headline workload (one "step" = one TimeScheme::step, i.e. three RK stages):
  compressible Taylor-Green vortex, 512^3 periodic cells on [0,2pi]^3, rho = 1,
  M = 0.1, Re = 1600 (mu = 1/1600), Pr = 0.72, seeded SplitMix64 velocity
  noise 1e-4, WENO-5 + second-order centered viscous terms, SSP-RK3 at CFL 0.5,
  physical semantics (the reference's own semantics go non-finite on this case:
  its Lax-Friedrichs speed is the constant 3 while c = 10).  `value` is the
  plain FP64 characteristic-wise form; the FP32 forms and the FP32 + learned
  sensor form are timed beside it and compared with it field by field.
  Synthetic input: no dataset is involved.  The device state (22 GB at 512^3)
  is larger than L2, so no flush is needed between timed steps.
Also in the line: the Sod shock tube 512x128x128 run to t = 0.2 by every form
(per-field L2/Linf against FP64 characteristic-wise), the sensor's training
recipe with held-out precision/recall, the HBM roofline in algorithmic bytes
(120 B per cell-stage: read U_stage and U0, write U_next), the compute
roofline, the end-to-end rate through ns_time_step with host buffers, and the
reference's own CPU TimeScheme::step timed on the host cores.

Arms:
  default            our CUDA path (libns_b200.so through its C ABI)
  --impl reference   the reference's own CPU TimeScheme::step (compiled from its
                     sources into oracle/_ref, OpenMP on all host cores), on the
                     same workload's initial condition at 256^3 (a bounded sample)
Multi-GPU (torchrun, N > 1): the domain is split along x into one slab per rank
(weak scaling: every rank holds the workload's n^3 cells, the global grid is
(N n) x n x n with the x extent N times the single-GPU box); before every RK
stage each rank exchanges its 3 outer planes x 5 fields per side with its x
neighbours (NCCL send/recv over NVLink) and the CFL minimum is all-reduced once
per step (3dnssolver_b200/slab.py).  value = all ranks' cell-updates / the
slowest rank's device time.
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
BYTES_PER_CELL_STAGE = 120  # read U_stage and U0, write U_next: 3 x 5 doubles

# workloads: initial condition, grid, semantics and physical parameters
WORKLOADS = {
    "tgv": dict(ic="taylor_green", n=512, semantics=1, mu=1.0 / 1600.0, Pr=0.72, cfl=0.5,
                label="taylor_green {n}^3 periodic [0,2pi]^3 M=0.1 Re=1600, {form} WENO-5 + CD-{order} "
                      "viscous, SSP-RK3 CFL 0.5, physical semantics"),
    "shear": dict(ic="shear_layer", n=256, semantics=0, mu=2.0 * 0.05 * 2 * math.pi / 1000.0, Pr=0.72,
                  cfl=0.5, label="shear_layer {n}^3 periodic [0,2pi]^3 M=0.5 Re=1000, {form} WENO-5 (LF alpha=3) "
                                 "+ CD-{order} viscous, SSP-RK3 CFL 0.5, reference semantics"),
}

# forms: scheme, precision, sensor; `ref` is the form its state is compared with
FORMS = {
    "fp64_char": dict(conv=2, prec=0, dtype="f64"),
    "fp64_comp": dict(conv=1, prec=0, dtype="f64"),
    "fp32_char": dict(conv=2, prec=1, dtype="f32 (f64 RK3 accumulation and reductions)"),
    "fp32_comp": dict(conv=1, prec=1, dtype="f32 (f64 RK3 accumulation and reductions)"),
    "fp32_sensor": dict(conv=2, prec=1, sensor=1,
                        dtype="f32 + bf16 sensor (f64 RK3 accumulation and reductions)"),
    # the network evaluated every 4th step, its flags gating the steps in between
    "fp32_sensor_p4": dict(conv=2, prec=1, sensor=1, period=4,
                           dtype="f32 + bf16 sensor (f64 RK3 accumulation and reductions)"),
    # the rest of the operator surface at full size: CD-6 viscous terms and Borges weights
    "fp64_char_cd6_borges": dict(conv=2, prec=0, order=6, weights=1, ref=None, dtype="f64"),
    "fp32_char_cd6_borges": dict(conv=2, prec=1, order=6, weights=1, ref="fp64_char_cd6_borges",
                                 dtype="f32 (f64 RK3 accumulation and reductions)"),
}
FIELDS = ["rho", "rhoE", "rhou", "rhov", "rhow"]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tgv", choices=sorted(WORKLOADS))
    ap.add_argument("--n", type=int, default=0, help="cells per axis (0: the workload's own)")
    ap.add_argument("--form", default="fp64_char", choices=sorted(FORMS))
    ap.add_argument("--also", default="fp64_comp,fp32_char,fp32_comp,fp32_sensor,fp32_sensor_p4,"
                                      "fp64_char_cd6_borges,fp32_char_cd6_borges",
                    help="extra forms timed after the headline (comma list, '' for none)")
    ap.add_argument("--accuracy-steps", type=int, default=0,
                    help="steps of the per-form accuracy runs (0: warmup + steps)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sod", action="store_true", help="skip the 512x128x128 Sod comparison")
    ap.add_argument("--cpu-sample-n", type=int, default=256,
                    help="grid of the reference CPU sample (the same workload's IC)")
    return ap.parse_args()


def workload_params(pkg, wk, n, form):
    W, F = WORKLOADS[wk], FORMS[form]
    L = 2 * math.pi
    return pkg.make_params(n, n, n, L=(L, L, L), mu=W["mu"], Pr=W["Pr"], gamma=1.4, cfl=W["cfl"],
                           convection=F["conv"], weights=F.get("weights", 0),
                           diffusion_order=F.get("order", 2), precision=F["prec"],
                           semantics=W["semantics"], sensor=F.get("sensor", 0),
                           sensor_period=F.get("period", 1))


def workload_name(wk, n, form):
    return WORKLOADS[wk]["label"].format(n=n, form=form, order=FORMS[form].get("order", 2))


def initial_state(wl, wk, p, seed):
    return getattr(wl, WORKLOADS[wk]["ic"])(p, seed=seed)


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
# the reference's own TimeScheme::step (oracle/_ref) on host cores

def _ref_cpu_params(pkg, wk, n):
    # the reference has one semantics; the same initial condition and schemes otherwise
    p = workload_params(pkg, wk, n, "fp64_char")
    p.semantics = 0
    return p


def _ref_sample_text(wk, n, n_full, threads, steps):
    extra = ""
    if WORKLOADS[wk]["semantics"] == 1:
        extra = (" with the reference's own semantics (it has no physical form; its characteristic-wise "
                 "Taylor-Green run turns non-finite after a few tens of steps, which does not change the "
                 "work or the time of a step)")
    return (f"{steps} timed TimeScheme::step calls on the {WORKLOADS[wk]['ic']} initial condition at {n}^3 "
            f"({(n / n_full) ** 3:.3g} of the workload's {n_full}^3 cells){extra}; "
            f"reference sources built with -O3 -ffast-math -march=x86-64-v3 (its CMake uses -march=native; "
            f"x86-64-v3 so that the binary built here runs on the GPU host), OpenMP {threads} threads, 1 rank")


def cpu_baseline(pkg, wk, n, n_full, steps=2, warmup=1):
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    if not O.ref_available(strict=False):
        return {"error": "oracle/_ref/ref_harness_timed is not built (needs the reference tree)"}
    p = _ref_cpu_params(pkg, wk, n)
    r = O.ref_bench(p, steps=steps, warmup=warmup, threads=threads, timed=True,
                    ic="tgv" if WORKLOADS[wk]["ic"] == "taylor_green" else "shear")
    return {"value": r["cell_updates_per_s"], "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": _ref_sample_text(wk, n, n_full, threads, steps), "seconds": r["seconds"]}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wk = args.workload
    n_full = args.n or WORKLOADS[wk]["n"]
    n = min(args.cpu_sample_n, n_full)
    try:
        from oracle import oracle as O
        if not O.ref_available(strict=False):
            print(json.dumps({"impl": "reference", "unavailable":
                              "oracle/_ref/ref_harness_timed not built (needs the reference tree)"}))
            return 0
        pkg = importlib.import_module("3dnssolver_b200")
        threads = os.cpu_count() or 1
        p = _ref_cpu_params(pkg, wk, n)
        r = O.ref_bench(p, steps=args.steps, warmup=args.warmup, threads=threads, timed=True,
                        ic="tgv" if WORKLOADS[wk]["ic"] == "taylor_green" else "shear")
    except Exception as e:  # report, do not crash the driver
        print(json.dumps({"impl": "reference", "unavailable": f"reference run failed: {e}"}))
        return 0
    v = r["cell_updates_per_s"]
    sample = _ref_sample_text(wk, n, n_full, threads, args.steps)
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * r["seconds"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(wk, n_full, "fp64_char"), "grid": [n_full] * 3,
                   "sample_grid": [n, n, n], "sample": sample, "parallelism": "1 rank, OpenMP"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
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
# rooflines

# Floating-point work per unit of each kernel class, counted by ncu at 128^3
# (sm__sass_thread_inst_executed_op_{d,f}{fma,mul,add}[2]_pred_on.sum divided by
# the faces or cells of the launch; the counts do not depend on the data):
# (flop per unit with an FMA as 2, FP lane operations per unit with a packed
# f32x2 operation as 2, pipe, unit), keyed by (semantics, form, kernel class).
# Reference semantics: the shear layer; physical semantics: the Taylor-Green
# vortex.  The x-update and fused stage rows average the three stages (the
# third also forms the next step's start).
COMPUTE_PER_UNIT = {
    ("reference", "fp64_char", "face_y"): (1408, 996, "fp64", "face"),
    ("reference", "fp64_char", "face_z"): (1406, 994, "fp64", "face"),
    ("reference", "fp64_comp", "face_y"): (995, 748, "fp64", "face"),
    ("reference", "fp64_comp", "face_z"): (995, 748, "fp64", "face"),
    ("reference", "fp64_char", "xface_update"): (1533, 1079, "fp64", "cell"),
    ("reference", "fp64_comp", "xface_update"): (1134, 841, "fp64", "cell"),
    ("reference", "fp64_char", "viscous"): (221, 135, "fp64", "cell"),
    ("reference", "fp64_comp", "viscous"): (221, 135, "fp64", "cell"),
    ("reference", "fp32_char", "stage_fused"): (4216, 2885, "fp32", "cell"),
    ("reference", "fp32_comp", "stage_fused"): (3211, 2244, "fp32", "cell"),
    ("physical", "fp64_char", "face_y"): (1438, 1022, "fp64", "face"),
    ("physical", "fp64_char", "face_z"): (1438, 1022, "fp64", "face"),
    ("physical", "fp64_comp", "face_y"): (1091, 815, "fp64", "face"),
    ("physical", "fp64_comp", "face_z"): (1091, 815, "fp64", "face"),
    ("physical", "fp64_char", "xface_update"): (1590, 1123, "fp64", "cell"),
    ("physical", "fp64_comp", "xface_update"): (1233, 909, "fp64", "cell"),
    ("physical", "fp64_char", "viscous"): (378, 218, "fp64", "cell"),
    ("physical", "fp64_comp", "viscous"): (378, 218, "fp64", "cell"),
    ("physical", "fp32_char", "stage_fused"): (4440, 3037, "fp32", "cell"),
    ("physical", "fp32_comp", "stage_fused"): (3521, 2448, "fp32", "cell"),
}
# DRAM bytes (read + write) per unit from the same captures at 128^3 (inputs
# larger than L2; the kernels stream their inputs once at 128^3 and above, so
# traffic scales with the units), averaged over the three stages of a step
# like the counts above; "fill" is the steady-state k_fill_halo.
TRAFFIC_PER_UNIT = {
    ("reference", "fp64_char", "face_y"): 69.6, ("reference", "fp64_char", "face_z"): 63.5,
    ("reference", "fp64_comp", "face_y"): 66.3, ("reference", "fp64_comp", "face_z"): 63.4,
    ("reference", "fp64_char", "xface_update"): 319.9, ("reference", "fp64_comp", "xface_update"): 317.7,
    ("reference", "fp64_char", "viscous"): 61.6, ("reference", "fp64_comp", "viscous"): 61.7,
    ("reference", "fp64_char", "fill_prim"): 21.8, ("reference", "fp64_comp", "fill_prim"): 21.7,
    ("reference", "fp32_char", "stage_fused"): 119.2, ("reference", "fp32_comp", "stage_fused"): 119.4,
    ("physical", "fp64_char", "face_y"): 66.3, ("physical", "fp64_char", "face_z"): 62.9,
    ("physical", "fp64_comp", "face_y"): 65.9, ("physical", "fp64_comp", "face_z"): 62.7,
    ("physical", "fp64_char", "xface_update"): 319.6, ("physical", "fp64_comp", "xface_update"): 317.9,
    ("physical", "fp64_char", "viscous"): 61.9, ("physical", "fp64_comp", "viscous"): 61.9,
    ("physical", "fp64_char", "fill_prim"): 21.6, ("physical", "fp64_comp", "fill_prim"): 21.9,
    ("physical", "fp32_char", "stage_fused"): 118.9, ("physical", "fp32_comp", "stage_fused"): 119.0,
}
KERNEL_NAMES = {"stage_fused": "k_stage_march", "update": "k_update",
                "sensor": "k_sensor_prims + k_sensor_mask_tc + k_gate_delta/k_gate_apply",
                "xface_update": "k_xface_update_tma", "viscous": "k_viscous", "fill_prim": "k_fill_prim/k_fill_halo",
                "step_begin": "k_step_begin", "face_x": "k_face_flux<x>", "face_y": "k_face_flux<y>",
                "face_z": "k_face_flux<z>"}


def profile(s, reps=3):
    """Mean per-class device ms of one step (events between the kernels)."""
    profs = [s.profile_step() for _ in range(reps)]
    return {k: statistics.mean(pr[k] for pr in profs) for k in profs[0]}


def rooflines(form, prof, n, ms_per_step, peaks, fma, semantics):
    """HBM roofline (algorithmic bytes: 120 B per cell-stage) of the form's dominant
    kernel class and of the whole step, and the compute roofline of that kernel
    (per-unit counts of the workload's semantics)."""
    sem = "physical" if semantics else "reference"
    cells = n ** 3
    faces = (n + 1) * n * n
    dom = max(prof, key=prof.get)
    launches = 1 if dom == "step_begin" else 3
    per_launch_ms = prof[dom] / launches
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    alg = BYTES_PER_CELL_STAGE * cells  # one stage of every cell per launch
    achieved = alg / (per_launch_ms / 1e3) / 1e9
    units = faces if dom.startswith("face") else cells
    # CD-6/Borges forms have no counts of their own in the tables: no rows, not the CD-2 ones
    fkey = form if "_cd6" in form else ("fp64_char" if form.startswith("fp64_char") else form)
    key = (sem, fkey, dom)
    tpu = TRAFFIC_PER_UNIT.get(key)
    traffic = round(tpu * units) if tpu else None
    step_alg = 3 * alg
    step_achieved = step_alg / (ms_per_step / 1e3) / 1e9
    # measured traffic of all kernel classes of one step where the capture has them
    step_traffic = 0.0
    covered = True
    for cls, ms in prof.items():
        if ms <= 0:
            continue
        t = TRAFFIC_PER_UNIT.get((sem, fkey, cls))
        if t is None:
            covered = False
            continue
        step_traffic += t * (faces if cls.startswith("face") else cells) * (1 if cls == "step_begin" else 3)
    kname = KERNEL_NAMES.get(dom, dom)
    if sem == "physical" and dom in ("face_y", "face_z"):
        kname = kname.replace("k_face_flux", "k_face_flux_tma")
    if dom == "viscous":
        kname = "k_viscous_tma<%d>" % (FORMS[form].get("order", 2) // 2)
    kname += f" ({form})"
    hbm = {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
           "frac": round(achieved / hbm_peak, 4), "traffic": traffic,
           "traffic_over_algorithmic": round(traffic / alg, 3) if traffic else None,
           "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum per unit at 128^3, "
                              "scaled by the units of this launch") if tpu else None,
           "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peaks else "fallback 6650 GB/s",
           "algorithmic_bytes_per_launch": alg,
           "algorithmic_unit": "120 B per cell-stage (U_stage and U0 read, U_next written) x cells",
           "launch_ms": round(per_launch_ms, 4),
           "step": {"achieved": round(step_achieved, 1), "frac": round(step_achieved / hbm_peak, 4),
                    "algorithmic_bytes": step_alg,
                    "measured_traffic": round(step_traffic) if covered and step_traffic else None,
                    "traffic_over_algorithmic": round(step_traffic / step_alg, 3)
                    if covered and step_traffic else None}}
    comp = None
    row = COMPUTE_PER_UNIT.get(key)
    if row:
        flop_u, inst_u, pipe, unit = row
        peak = fma[pipe]
        tflops = flop_u * units / (per_launch_ms / 1e3) / 1e12
        # FP lane operations against the FMA rate (peak / 2 flops): a multiply or add
        # takes the same pipe slot as an FMA, so this is the pipe's busy fraction
        ops_rate = inst_u * units / (per_launch_ms / 1e3) / 1e12
        comp = {"bound": pipe, "kernel": kname, "achieved": round(tflops, 2), "peak": round(peak, 2),
                "unit": "TFLOP/s", "frac": round(tflops / peak, 4),
                "pipe_frac": round(ops_rate / (peak / 2.0), 4),
                "peak_source": f"measured now: ns_fma_peak ({pipe} FMA chains on every SM)",
                "counts_source": f"ncu per-opcode counts of the {sem}-semantics kernel at 128^3",
                "flop_per_" + unit: flop_u, "fp_ops_per_" + unit: inst_u}
        hbm["note"] = f"{pipe}-pipe bound: see compute_roofline"
    return hbm, comp


# ---------------------------------------------------------------------------
# accuracy: per-field errors against the comparison form, on the GPU

def interior_tensor(U):
    import torch
    return torch.from_numpy(U[3:-3, 3:-3, 3:-3]).cuda()


def field_errors(U, R):
    """Relative L2 and Linf of U against R per conserved field; the momentum
    components also against the momentum magnitude (a field like rhow can be
    noise-amplitude, where its own norm is no scale)."""
    import torch
    out = {"rel_l2": {}, "rel_linf": {}, "mom_l2": {}, "mom_linf": {}}
    mom_l2 = math.sqrt(float((R[..., 2:5] ** 2).sum().item()))
    mom_inf = float(torch.sqrt((R[..., 2:5] ** 2).sum(-1)).max().item())
    for q, f in enumerate(FIELDS):
        d = U[..., q] - R[..., q]
        l2 = math.sqrt(float((d * d).sum().item()))
        li = float(d.abs().max().item())
        out["rel_l2"][f] = l2 / max(math.sqrt(float((R[..., q] ** 2).sum().item())), 1e-300)
        out["rel_linf"][f] = li / max(float(R[..., q].abs().max().item()), 1e-300)
        if q >= 2:
            out["mom_l2"][f] = l2 / max(mom_l2, 1e-300)
            out["mom_linf"][f] = li / max(mom_inf, 1e-300)
    return out


def accuracy_run(pkg, params, W0, steps, sensor_w=None, every=1):
    """Advances a fresh context `steps` steps from W0, recording time, kinetic energy and
    enstrophy every `every` steps; returns (interior U on the GPU, history)."""
    hist = {"step": [], "time": [], "kinetic": [], "enstrophy": []}
    with pkg.Solver(params) as s:
        if sensor_w is not None:
            s.set_sensor_weights(sensor_w)
        s.upload_primitive(W0)
        d = s.diagnostics()
        for k in range(steps + 1):
            if k % every == 0 or k == steps:
                d = s.diagnostics()
                hist["step"].append(k)
                hist["time"].append(d["time"])
                hist["kinetic"].append(d["kinetic"])
                hist["enstrophy"].append(d["enstrophy"])
            if k < steps:
                s.advance(1)
        frac = d["sensor_fraction"]
        U = interior_tensor(s.download_conservative())
    return U, hist, frac


def sod_comparison(pkg, wl, sensor_w_ref, t_end=0.2):
    """The 512x128x128 Sod shock tube (Ly = Lz = 1, characteristic-wise, reference
    semantics at CFL 0.2) to t = 0.2 in every form; errors against FP64 characteristic-wise."""
    import torch
    sensor_mod = importlib.import_module("3dnssolver_b200.sensor")
    cfl = sensor_mod.sod_cfl(0)
    base = sensor_mod.sod_params(512, 128, 128, cfl=cfl)
    W0 = wl.sod(base, seed=3)
    out = {"workload": f"sod 512x128x128, x in [0,1] (Neumann), y,z in [0,1] periodic (dy = dz = 4 dx), "
                       f"interface x = 0.5 + 0.01 sin(2 pi y) sin(2 pi z), mu = 1e-4, CD-2, CFL {cfl}, "
                       f"reference semantics (its characteristic-wise run turns non-finite within 40 steps "
                       f"at CFL 0.4; finite to t = 0.2 at CFL 0.2)",
           "t_end": t_end, "forms": {}}
    # the FP64 characteristic-wise run sets the step count that reaches t_end
    with pkg.Solver(base) as s:
        s.upload_primitive(W0)
        steps, t = 0, 0.0
        while t < t_end and steps < 5000:
            s.advance(10)
            steps += 10
            t = s.get_dt()[1]
        d64 = s.diagnostics()
        Uref = interior_tensor(s.download_conservative())
    out["steps"], out["t_fp64_char"] = steps, t
    out["fp64_char_nonfinite"] = d64["nonfinite"]
    for form, kw in [("fp64_comp", dict(convection=1)), ("fp32_char", dict(precision=1)),
                     ("fp32_comp", dict(precision=1, convection=1)),
                     ("fp32_sensor", dict(precision=1, sensor=1)),
                     ("fp32_sensor_p4", dict(precision=1, sensor=1, sensor_period=4))]:
        p = sensor_mod.sod_params(512, 128, 128, cfl=cfl, **kw)
        with pkg.Solver(p) as s:
            if kw.get("sensor"):
                s.set_sensor_weights(sensor_w_ref)
            s.upload_primitive(W0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.advance(steps)
            s.synchronize()
            sec = time.perf_counter() - t0
            d = s.diagnostics()
            U = interior_tensor(s.download_conservative())
        e = field_errors(U, Uref)
        e["time"] = d["time"]
        e["sensor_fraction"] = d["sensor_fraction"] if kw.get("sensor") else None
        e["cell_updates_per_s"] = 512 * 128 * 128 * 3 * steps / sec
        out["forms"][form] = e
        del U
    del Uref
    torch.cuda.empty_cache()
    return out


def slab_bench(args, dist, rank, world, local):
    """N > 1: the headline form on a slab decomposition along x (weak scaling)."""
    import torch
    pkg = importlib.import_module("3dnssolver_b200")
    wl = importlib.import_module("3dnssolver_b200.workloads")
    slab = importlib.import_module("3dnssolver_b200.slab")
    wk = args.workload
    n = args.n or WORKLOADS[wk]["n"]
    p1 = workload_params(pkg, wk, n, args.form)
    # the global problem: N single-GPU boxes side by side along x (the same dx)
    pg = workload_params(pkg, wk, n, args.form)
    pg.nx, pg.Lx = n * world, p1.Lx * world
    W_local = initial_state(wl, wk, p1, seed=(5 if wk == "tgv" else 1) + rank)  # this rank's box
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        ex = slab.HaloExchange(rank, world, periodic=True, host_staged=False)
        s = slab.SlabSolver(pg, rank, world, ex, stream=stream)
        s.upload_primitive(W_local)
        s.advance(args.warmup)
        torch.cuda.synchronize()
        clk = ClockSampler(local)
        clk.start()
        t0 = time.time()
        while time.time() - t0 < 1.0:  # the sampler sees the GPU under load through the timed region
            s.advance(1)
            torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        l0 = s.solver.launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.advance(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        ms = max_over_ranks(e0.elapsed_time(e1), dist)
        launches = s.solver.launches - l0
        clocks = clk.stop()
        prof = profile(s.solver)
        # end to end: ns_time_step with the rank's host W (pinned), exchanges included
        Wh_t = torch.empty(W_local.shape, dtype=torch.float64, pin_memory=True)
        Wh = Wh_t.numpy()
        Wh[...] = W_local
        s.solver.time_step(Wh)
        dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.e2e_steps):
            s.solver.time_step(Wh)
        e1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist)
        diag = s.diagnostics()
        s.close()
    cells = n ** 3
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    fma = {"fp64": pkg.fma_peak(True), "fp32": pkg.fma_peak(False)}
    roofline, compute_roofline = rooflines(args.form, prof, n, ms / args.steps, peaks, fma,
                                           WORKLOADS[wk]["semantics"])
    halo_bytes = 2 * 15 * n * n * 8 * 3  # both sides, 3 planes x 5 fields, 3 stages per step
    if rank == 0:
        out = {
            "metric": METRIC, "value": job_rate(world, cells, args.steps, ms), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": FORMS[args.form]["dtype"], "data": "synthetic",
            "config": {"workload": workload_name(wk, n, args.form) + f", {world} slabs along x",
                       "grid": [n * world, n, n], "grid_per_gpu": [n, n, n], "form": args.form,
                       "l2": "no flush: device state per GPU larger than L2",
                       "parallelism": f"slab decomposition along x over {world} GPUs: NCCL send/recv of "
                                      f"3 planes x 5 fields per side before every RK stage, "
                                      f"all-reduce(min) of the CFL minimum per step",
                       "halo_bytes_per_step_per_gpu": halo_bytes},
            "roofline": roofline, "compute_roofline": compute_roofline,
            "kernel_ms_per_step": {k: round(v, 4) for k, v in prof.items() if v > 0},
            "cpu_baseline": None, "gpu_launches": launches, "clocks": clocks,
            "e2e": {"value": job_rate(world, cells, args.e2e_steps, e2e_ms), "unit": UNIT,
                    "h2d_bytes_per_step": int(Wh.nbytes), "d2h_bytes_per_step": int(Wh.nbytes),
                    "steps": args.e2e_steps, "api": "ns_time_step on every rank's slab, pinned host W"},
            "diagnostics": {"nonfinite": diag["nonfinite"], "dt": diag["dt"]},
        }
        print(json.dumps(out))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)

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
        try:
            return slab_bench(args, dist, rank, world, local)
        finally:
            dist.destroy_process_group()

    def barrier():
        if dist is not None:
            dist.barrier()

    def rank_max(x):
        return max_over_ranks(x, dist)

    pkg = importlib.import_module("3dnssolver_b200")
    wl = importlib.import_module("3dnssolver_b200.workloads")
    sensor_mod = importlib.import_module("3dnssolver_b200.sensor")
    wk = args.workload
    n = args.n or WORKLOADS[wk]["n"]
    cells = n ** 3
    p = workload_params(pkg, wk, n, args.form)
    W0 = initial_state(wl, wk, p, seed=(5 if wk == "tgv" else 1) + rank)
    # a dedicated stream: the context adopts it, so CUDA events recorded on it bracket
    # exactly the library's kernels (torch's default stream is the legacy NULL stream)
    stream = torch.cuda.Stream()
    forms_wanted = [args.form] + [f for f in args.also.split(",") if f and f != args.form]

    # the learned sensor, trained by its recipe in the semantics of each workload that uses it
    sensor_w, sensor_info = {}, {}

    def sensor_weights(sem):
        if sem not in sensor_w:
            sensor_w[sem], sensor_info[sem] = sensor_mod.train_recipe(semantics=sem, seed=0)
        return sensor_w[sem]

    def time_form(form, steps, warmup, sample_clocks=False):
        pf = workload_params(pkg, wk, n, form)
        s = pkg.Solver(pf)
        s.set_stream(stream.cuda_stream)
        if FORMS[form].get("sensor"):
            s.set_sensor_weights(sensor_weights(WORKLOADS[wk]["semantics"]))
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
                s.advance(1)
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
        return s, ms, launches, clocks

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    fma = {"fp64": pkg.fma_peak(True), "fp32": pkg.fma_peak(False)}

    # ---- headline form: timed, profiled, then the end-to-end rate
    if FORMS[args.form].get("sensor"):
        sensor_weights(WORKLOADS[wk]["semantics"])
    s, ms, launches, clocks = time_form(args.form, args.steps, args.warmup, sample_clocks=True)
    ms_max = rank_max(ms)
    value = job_rate(world, cells, args.steps, ms_max)
    prof = profile(s)
    roofline, compute_roofline = rooflines(args.form, prof, n, ms_max / args.steps, peaks, fma,
                                           WORKLOADS[wk]["semantics"])

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
           "steps": args.e2e_steps,
           "api": "ns_time_step (TimeScheme::step drop-in), pinned host W; the library overlaps the chunked "
                  "upload with the first stage and the chunked download with the third"}
    s.close()
    del Wh, Wh_t

    forms = {args.form: {"value": value, "ms_per_step": ms_max / args.steps, "gpu_launches": launches,
                         "kernel_ms_per_step": {k: round(v, 4) for k, v in prof.items() if v > 0}}}
    for f in forms_wanted[1:]:
        try:
            s2, ms2, l2, _ = time_form(f, args.steps, args.warmup)
            ms2 = rank_max(ms2)
            pr2 = profile(s2)
            hbm2, comp2 = rooflines(f, pr2, n, ms2 / args.steps, peaks, fma, WORKLOADS[wk]["semantics"])
            s2.close()
            forms[f] = {"value": job_rate(world, cells, args.steps, ms2), "ms_per_step": ms2 / args.steps,
                        "gpu_launches": l2, "vs_" + args.form: ms_max / ms2,
                        "kernel_ms_per_step": {k: round(v, 4) for k, v in pr2.items() if v > 0},
                        "roofline": hbm2, "compute_roofline": comp2}
        except Exception as e:
            forms[f] = {"error": str(e)}

    # ---- accuracy: every form advances the same initial state; errors against its comparison form
    acc_steps = args.accuracy_steps or (args.warmup + args.steps)
    every = max(1, acc_steps // 50)
    refs = {}
    for f in forms_wanted:
        if "error" in forms[f]:
            continue
        pf = workload_params(pkg, wk, n, f)
        sw = sensor_weights(WORKLOADS[wk]["semantics"]) if FORMS[f].get("sensor") else None
        U, hist, frac = accuracy_run(pkg, pf, W0, acc_steps, sensor_w=sw, every=every)
        forms[f]["history"] = hist
        if FORMS[f].get("sensor"):
            forms[f]["sensor_fraction"] = frac
        ref = FORMS[f].get("ref", args.form)
        if ref is not None and ref != f and ref in refs:
            forms[f]["errors_vs_" + ref] = dict(field_errors(U, refs[ref]), steps=acc_steps)
        if f == args.form or any(FORMS[g].get("ref", args.form) == f for g in forms_wanted if g != f):
            refs[f] = U  # a later form is compared with this one
        del U
    refs.clear()
    torch.cuda.empty_cache()

    sod = None
    if rank == 0 and not args.no_sod:
        try:
            sod = sod_comparison(pkg, wl, sensor_weights(0))
        except Exception as e:
            sod = {"error": str(e)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(pkg, wk, min(args.cpu_sample_n, n), n)
        except Exception as e:
            cpu = {"error": str(e)}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": FORMS[args.form]["dtype"], "data": "synthetic",
            "config": {"workload": workload_name(wk, n, args.form), "grid": [n, n, n], "form": args.form,
                       "l2": f"no flush: device state {5 * 8 * (n + 6) ** 3 * 4 / 1e9:.1f} GB > 126 MB L2",
                       "parallelism": f"{world} independent replica(s), no data-path collective"},
            "roofline": roofline, "compute_roofline": compute_roofline,
            "kernel_ms_per_step": {k: round(v, 4) for k, v in prof.items() if v > 0},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
            "forms": forms,
            "sensor_training": {("physical" if k else "reference"): v for k, v in sensor_info.items()},
            "sod_512x128x128": sod,
        }
        print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
