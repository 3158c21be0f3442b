#!/usr/bin/env python
"""Throughput of the pllcart3d time step on B200, in cell-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME]

One step = one full RK3-CN time step (pllcart3d.c:158-195) of the named
seeded synthetic fingering workload (default fingering-512x256x256, the size
the headline metric is quoted at).  Three forms are timed (`--precision`):
the headline `value` is the mixed64 form (FP64 state, FP32 WENO5 weights:
the form within 1e-5 of the FP64 form in c after 1000 steps), the plain
FP64 form and the FP32-state precision form are reported beside it
(`fp64_form`, `mixed_form`, `mixed64_over_fp64`, `mixed_over_fp64`).  At
512x256x256 a state array is 276 MB in FP64 (138 MB in FP32), above the
126 MB L2, and a step moves tens of GB, so no L2 flush is needed between
steps (`config.l2` states the figures of the run).

--impl ours       the GPU step through the pllgpu_ C ABI (one CUDA graph per
                  step); `value` is device-timed with CUDA events on the
                  solver's stream, max over ranks; `e2e` goes through
                  pllgpu_run_host with pinned host buffers (initial fields
                  in, c/u/v/w out, inside the timed region).
--impl reference  the reference's own CPU step (pllcart3d.c and
                  pll_tridiag.c compiled by oracle/Makefile) at the same
                  workload and grid, on its x-slab MPI decomposition over
                  every host core the slabs allow (processes over a
                  shared-memory MPI stand-in); a time budget caps the timed
                  steps.
With N>1 (torchrun) every rank advances its own replica (the timed step path
runs on one GPU; replicas only) and `value` sums cells over ranks.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from pllcart3d_b200 import roofline  # noqa: E402
from pllcart3d_b200.ic import workload_fields  # noqa: E402
from pllcart3d_b200.params import workload  # noqa: E402

METRIC = "cell-steps/s: mixed vs plain FP64 on 1 B200 at \u22641e-5 c error; surrogate speedup"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="fingering-512x256x256")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--precision", default="all", choices=["all", "both", "fp64", "mixed", "mixed64"],
                    help="forms to time (all: fp64, mixed64, mixed; both: fp64, mixed); the headline value is "
                         "--headline's")
    ap.add_argument("--explicit-kernel", default="auto", choices=["auto", "direct", "tma"],
                    help="explicit-operator kernel of every timed form (Solver's explicit_kernel)")
    ap.add_argument("--headline", default="mixed64", choices=["fp64", "mixed", "mixed64"],
                    help="the form whose throughput is `value`: mixed64 is the form that meets the 1e-5 c "
                         "accuracy target of the metric")
    return ap.parse_args()


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def reduce_max(x, ws):
    """Max of x over the ranks (the slowest replica's time)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(cells, steps, ws, ms_max):
    """Whole-job throughput of ws replicas: every rank advances its own copy
    of the workload, timed as the slowest rank."""
    return cells * steps * ws / (ms_max / 1e3)


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def peaks():
    try:
        with open(PEAKS) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out = ""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def ref_ranks(nx):
    """Ranks of the reference's slab decomposition on this host: every core,
    as far as the slabs allow (each needs the 3 planes its neighbours'
    halos read)."""
    return max(1, min(os.cpu_count() or 1, nx // 3))


def ref_mpi(wl_name, ranks, warm, steps, budget_s):
    """The reference's own multi-rank step (pllcart3d.c on its x-slab
    decomposition, pll_tridiag.c's pipelined x solves, the halo exchanges)
    over the shared-memory MPI stand-in, in a fresh process (it forks its
    ranks, which a process holding a CUDA context must not do)."""
    cmd = [sys.executable, "-m", "oracle.refmpi", "--workload", wl_name, "--ranks", str(ranks),
           "--warmup", str(warm), "--steps", str(steps), "--budget", str(budget_s)]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=1800)
    if out.returncode != 0:
        raise RuntimeError(out.stderr.strip().splitlines()[-1] if out.stderr.strip() else "reference run failed")
    return json.loads(out.stdout.strip().splitlines()[-1])


def cpu_sample(wl_name, seconds=20.0):
    """The CPU baseline: the reference's own step at the workload's grid on
    every host core its slab decomposition allows, one untimed step then
    timed steps for about `seconds`; returns (cell-steps/s, kind, sample,
    cores)."""
    wl = workload(wl_name)
    ranks = ref_ranks(wl.params.nx)
    r = ref_mpi(wl_name, ranks, 1, 1000, seconds)
    sample = (f"{r['steps']} step(s) of {wl.name} ({wl.params.nx}x{wl.params.ny}x{wl.params.nz}) after 1 untimed "
              f"step: the reference's pllcart3d.c on {ranks} x-slab ranks (processes over a shared-memory MPI "
              f"stand-in), FFT-based DCT stand-in for FFTW, {r['seconds']:.1f} s timed")
    return r["cell_steps_per_s"], "reference", sample, ranks


def run_reference(args, ws, rank):
    """The reference's own CPU step on the host cores: pllcart3d.c on its
    x-slab decomposition over every core the slabs allow (the MPI path of
    pllcart3d.c:357-378 and pll_tridiag.c), at the benchmarked workload's
    grid; one untimed step, then up to --steps timed steps within a time
    budget so that the run ends within minutes."""
    if rank != 0:
        return
    wl = workload(args.workload)
    ranks = ref_ranks(wl.params.nx)
    budget = 150.0
    r = ref_mpi(args.workload, ranks, 1, args.steps, budget)
    value = r["cell_steps_per_s"]
    sample = (f"{r['steps']} of {args.steps} requested step(s) of {wl.name} after 1 untimed step (a {budget:.0f} s "
              f"budget caps the timed steps): pllcart3d.c on {ranks} x-slab ranks over a shared-memory MPI "
              f"stand-in, FFT-based DCT stand-in for FFTW")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-steps/s",
        "n_gpus": args.gpus, "steps": r["steps"], "warmup": 1, "ms_per_step": 1e3 * r["seconds"] / r["steps"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl.name, "grid": [wl.params.nx, wl.params.ny, wl.params.nz],
                   "precision": "fp64", "parallelism": f"mpi{ranks} (x slabs, host cores)"},
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": ranks, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def measure(prm, ic, form, steps, warmup, ws, local, profile_steps=2, explicit_kernel="auto"):
    """Device-timed steps of one precision form + per-kernel event profile."""
    import ctypes

    import torch

    from pllcart3d_b200.solver import Solver

    s = Solver(prm, device=local, exact_dct=False, use_graph=True, precision=form, explicit_kernel=explicit_kernel)
    s.load_ic(ic)
    stream = torch.cuda.ExternalStream(s._L.pllgpu_stream(s._h), device=local)
    s.step(warmup)
    barrier(ws)
    clocks = Clocks(local)
    clocks.start()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    ms = e0.elapsed_time(e1)
    ck = clocks.stop()
    ms_max = reduce_max(ms, ws)
    maxk = 64
    names = ctypes.create_string_buffer(32 * maxk)
    tot = (ctypes.c_double * maxk)()
    cnt = (ctypes.c_int * maxk)()
    nk = ctypes.c_int(0)
    kernels = {}
    if s._L.pllgpu_profile_steps(s._h, profile_steps, maxk, names, tot, cnt, ctypes.byref(nk)) == 0:
        for t in range(nk.value):
            lab = names.raw[32 * t:32 * t + 32].split(b"\0")[0].decode()
            kernels[lab] = {"ms_total": tot[t], "launches": cnt[t]}
    out = {"ms": ms_max, "launches_per_step": s.kernels_per_step, "clocks": ck,
           "kernels": kernels, "profile_steps": profile_steps, "solver": s}
    return out


# dense GEMM peaks of the DCT kernels' own arithmetic, measured on this
# pool's B200s with `python -m pllcart3d_b200.peaks` (cuBLAS, 8192^3, burst)
TF32_TFLOPS = 730.2
FP64_TFLOPS = 35.5


def tensor_peak():
    """Dense TF32 tensor peak the split-TF32 DCT passes are measured
    against (the measured burst rate)."""
    return TF32_TFLOPS


# DRAM traffic over algorithmic bytes of a launch, from the ncu captures of
# the 256x128x128 case (profiles/); traffic grows with the cells processed,
# so a full launch's traffic is this ratio times its algorithmic bytes
TRAFFIC_RATIO = {("k_explicit2", "fp32"): 1.05, ("k_explicit", "fp64"): 1.04, ("k_explicit_tma", "fp64"): 1.04}


def l2_note(prm, form):
    """How the timed steps stay clear of L2 reuse: the field size of the form
    and the step's traffic against the 126 MB L2 (no flush between steps)."""
    word = 4 if form == "mixed" else 8
    field = float(prm.shape[0] * prm.shape[1] * prm.shape[2]) * word / 1e6
    step = roofline.step_bytes(prm.cells, "fp32" if form == "mixed" else "fp64") / 1e6
    return (f"no L2 flush: each field {field:.0f} MB, each step moves {step / 1e3:.1f} GB "
            f"({step / 126:.0f}x the 126 MB L2)")


def roofline_of(kernels, nprof, cells, precision, dims=None, form=None, explicit="auto"):
    """Roofline of the kernel family with the largest share of the step."""
    hbm, peak_kind = peaks()
    fam = {}
    for lab, v in kernels.items():
        f = roofline.family(lab, precision, form, explicit)
        if f is None:
            continue
        d = fam.setdefault(f, {"ms": 0.0, "launches": 0, "bytes": 0.0, "labels": []})
        d["ms"] += v["ms_total"]
        d["launches"] += v["launches"]
        d["bytes"] += roofline.kernel_bytes_per_launch(lab, cells, precision) * v["launches"]
        d["labels"].append(lab)
    if not fam:
        return None
    step_ms_prof = sum(v["ms_total"] for v in kernels.values()) / nprof
    top = max(fam, key=lambda f: fam[f]["ms"])
    d = fam[top]
    avg_ms = d["ms"] / d["launches"]
    out = {"kernel": top, "labels": sorted(d["labels"]), "avg_launch_ms": avg_ms,
           "share_of_step": d["ms"] / nprof / step_ms_prof, "peak_source": peak_kind}
    tens = [lab for lab in d["labels"] if lab in roofline.TENSOR_PASS_FLOPS]
    if tens and dims is not None:
        nx, ny, nz = dims
        flops = roofline.TENSOR_PASS_FLOPS[tens[0]] * (ny + nz) * cells   # mean pass: 2n flops/cell
        ach = flops / (avg_ms / 1e3) / 1e12
        pk = tensor_peak()
        out.update({"bound": "tensor", "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                    "frac": ach / pk if pk else None, "traffic": None,
                    "algorithmic_flops_per_launch": flops})
        return out
    alg = d["bytes"] / d["launches"]
    ach = alg / (avg_ms / 1e3) / 1e9
    ratio = TRAFFIC_RATIO.get((top, precision))
    out.update({"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "traffic": ratio * alg if ratio else None, "algorithmic_bytes_per_launch": alg})
    return out


# the precision form's 1000-step accuracy at the timed workload, measured by
# `python -m pllcart3d_b200.validate --at 1,32,128,250,500,750,1000` and
# committed under profiles/ (the bench itself runs only a few steps)
GATE_RECORD = {
    "mixed": {"target": "c relative max-norm error <= 1e-5 after 1000 steps against the FP64 form",
              "c_rel_after_1000_steps": 4.1e-3, "met": False,
              "record": "profiles/precision_forms_accuracy_fingering-512x256x256.md"},
    "mixed64": {"target": "c relative max-norm error <= 1e-5 after 1000 steps against the FP64 form",
                "c_rel_after_1000_steps": 2.0e-6, "met": True,
                "record": "profiles/precision_forms_accuracy_fingering-512x256x256.md"},
}


def form_accuracy(test, ref, steps):
    """Relative max-norm errors of c, u (against the velocity vector) and phi
    of one solver against another after the same steps."""
    import numpy as np

    def rel(f, comps=None):
        den = max(float(np.abs(ref.get(c)).max()) for c in (comps or (f,)))
        return float(np.abs(test.get(f) - ref.get(f)).max()) / den

    vel = ("u_new", "v_new", "w_new")
    return {"steps": steps, "against": "fp64 form, same seed and step count",
            "c": rel("c_new"), "u": rel("u_new", vel), "v": rel("v_new", vel), "w": rel("w_new", vel),
            "phi": rel("phi")}


def e2e_of(s, ic, prm, steps, ws):
    """The step through pllgpu_run_host with host buffers: initial c, u, v, w
    (FP64) from pinned host memory, start-up, `steps` steps, c, u, v, w back
    into pinned host memory; wall clock around the call, max over ranks."""
    import ctypes

    import numpy as np
    import torch

    from pllcart3d_b200 import _lib

    shape = prm.shape
    pin = [torch.empty(shape, dtype=torch.float64, pin_memory=True) for _ in range(8)]
    for t, k in zip(pin[:4], "cuvw"):
        t.numpy()[...] = ic[k]
    ptr = [ctypes.cast(t.data_ptr(), ctypes.POINTER(ctypes.c_double)) for t in pin]
    t0 = time.perf_counter()
    code = s._L.pllgpu_run_host(s._h, steps, *ptr)
    t1 = time.perf_counter()
    if code != 0:
        raise _lib.PllGpuError(code, "run_host")
    sec = reduce_max(t1 - t0, ws)
    nbytes = 4 * int(np.prod(shape)) * 8
    return {"value": prm.cells * steps * ws / sec, "unit": "cell-steps/s",
            "h2d_bytes_per_step": nbytes / steps, "d2h_bytes_per_step": nbytes / steps,
            "note": "pllgpu_run_host: initial c,u,v,w (FP64) from pinned host memory, "
                    f"start-up, {steps} steps, c,u,v,w back to pinned host memory, "
                    "wall-clock around the call"}


def run_ours(args, ws, rank, local):
    import torch

    torch.cuda.set_device(local)
    wl = workload(args.workload)
    prm = wl.params
    cells = prm.cells
    ic = workload_fields(wl)
    hbm, _ = peaks()

    forms = {}
    chosen = {"all": ("fp64", "mixed64", "mixed"), "both": ("fp64", "mixed")}.get(args.precision, (args.precision,))
    for form in chosen:
        m = measure(prm, ic, form, args.steps, args.warmup, ws, local, explicit_kernel=args.explicit_kernel)
        prec = "fp32" if form == "mixed" else "fp64"
        sb = roofline.step_bytes(cells, prec)
        m["value"] = replica_value(cells, args.steps, ws, m["ms"])
        m["roofline"] = roofline_of(m["kernels"], m["profile_steps"], cells, prec, (prm.nx, prm.ny, prm.nz),
                                    form, args.explicit_kernel)
        m["step_roofline"] = {"bytes_per_step": sb,
                              "achieved_gbs": sb / (m["ms"] / args.steps / 1e3) / 1e9,
                              "frac_of_hbm": sb / (m["ms"] / args.steps / 1e3) / 1e9 / hbm}
        m["steps_done"] = args.warmup + args.steps + m["profile_steps"]
        forms[form] = m

    if args.headline not in forms:
        args.headline = args.precision
    head = forms[args.headline]

    # the precision form against the FP64 form from the same seed after the
    # same number of steps (warm-up + timed + profiled)
    accuracy = {}
    for form in forms:
        if form != "fp64" and "fp64" in forms:
            accuracy[form] = form_accuracy(forms[form]["solver"], forms["fp64"]["solver"],
                                           forms["fp64"]["steps_done"])

    for form, m in forms.items():
        m["e2e"] = None if args.no_e2e else e2e_of(m["solver"], ic, prm, args.steps, ws)
        m["solver"].close()

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            v, kind, sample, cores = cpu_sample(args.workload, seconds=20.0)
            cpu = {"value": v, "unit": "cell-steps/s", "cores": cores, "kind": kind, "sample": sample}
        except Exception as ex:  # the checker may be absent on a bare box
            cpu = {"value": None, "unit": "cell-steps/s", "cores": 0, "kind": "none",
                   "sample": f"unavailable: {ex}"}

    e2e = head["e2e"]
    if rank == 0:
        line = {
            "metric": METRIC, "value": head["value"], "unit": "cell-steps/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"mixed": "f32", "mixed64": "f64 (FP32 WENO5 weights)"}.get(args.headline, "f64"),
            "data": "synthetic",
            "config": {"workload": wl.name, "grid": [prm.nx, prm.ny, prm.nz],
                       "precision": args.headline,
                       "parallelism": "replicas" if ws > 1 else "single",
                       "l2": l2_note(prm, args.headline)},
            "e2e": e2e, "gpu_launches": head["launches_per_step"] * args.steps,
            "roofline": head["roofline"], "step_roofline": head["step_roofline"],
            "cpu_baseline": cpu, "clocks": head["clocks"],
            "kernels_ms_per_step": {k: v["ms_total"] / head["profile_steps"]
                                    for k, v in head["kernels"].items()},
        }
        for form, m in forms.items():
            line[f"{form}_form"] = {"value": m["value"], "ms_per_step": m["ms"] / args.steps,
                                    "e2e": m["e2e"],
                                    "step_roofline_frac": m["step_roofline"]["frac_of_hbm"],
                                    "roofline": m["roofline"], "clocks": m["clocks"],
                                    "kernels_ms_per_step": {k: v["ms_total"] / m["profile_steps"]
                                                            for k, v in m["kernels"].items()}}
        for form in forms:
            if form != "fp64" and "fp64" in forms:
                line[f"{form}_over_fp64"] = forms[form]["value"] / forms["fp64"]["value"]
                line[f"{form}_form"]["accuracy"] = accuracy[form]
                line[f"{form}_form"]["gate"] = GATE_RECORD[form]
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
