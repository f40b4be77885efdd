"""Benchmark of the fused D3Q19 stream-collide step (GLUPS and % of HBM roofline).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--size L] [--precision fp64|fp32|fp16] [--scheme two_lattice|aa]

Default workload: decaying HIT, 256^3 periodic box, FP64 two-lattice, tau = 0.505
(svisc = 0.005/3), seeded random-phase solenoidal velocity with
E(k) ~ k^4 exp(-2 (k/k0)^2), k0 = 4, u_rms = 0.03, equilibrium init. A step is
one fused stream-collide update of the whole box (the reference's
boundaries + col_MC). Prints one JSON line.

- value: GLUPS with the populations resident in HBM, K steps timed with CUDA
  events on the library's stream (inputs are 5 GB, larger than L2).
- forms (default run, one GPU): the same box in FP32-deviation and
  FP16-scaled-deviation storage (default two-lattice kernels), each timed
  the same way over max(K, 200) steps with its own clock record, its GLUPS
  ratio to the FP64 value and its roofline.
- large (default run, one GPU): FP64 two-lattice at 512^3 (k0 = 6,
  tau = 0.503) and the AA pattern at 1024^3 in FP16 and FP32 storage (k0 = 8,
  tau = 0.502), initial field made on the GPU; max(K, 50) steps each, own
  clock record.
- e2e: the same K steps through the public C-ABI as a user drives them: the
  initial velocity field uploaded from pinned host memory, then
  boundaries + col_MC + diagnostic every step (diagnostics computed every
  icheck = 100 steps, the reference's default, SRC/input.F90:221, and read
  back to the host), all inside the timed region, after an untimed warm-up
  pass of the same calls (upload, init and W steps); split into the one-time
  part (upload + init, fixed_ms) and the per-step part (per_step_ms).
- roofline: algorithmic bytes of the stream-collide kernel (19 loads + 19
  stores per cell) per launch / average launch time, against the measured HBM
  copy bandwidth.
- cpu_baseline: the CPU oracle (C restatement of the reference's
  boundaries + col_MC, FP64, OpenMP over all host cores) on a bounded sample.
- --impl reference: times that CPU implementation on this workload (rank 0),
  with the same config and warm-up as the GPU arm.
Under torchrun (N > 1) the default is one box split along z (--decomp slabs,
bgk3d_hit_b200.slabs): each rank holds one size^3 slab of a
size x size x (N size) box (weak scaling), the face populations go straight
into the neighbours' ghost planes over NVLink (CUDA IPC) and a one-element
NCCL all-reduce on the slab's stream separates the steps; value is all
ranks' cell updates over the slowest rank's time. --decomp replicas runs N
independent boxes instead. On one GPU, --decomp slabs --local-slabs P
splits the size^3 box into P slabs in one process (the exchange and its
barrier measured without a second GPU).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_CELL = {"fp64": 304, "fp32": 152, "fp16": 76}
DTYPE = {"fp64": "f64", "fp32": "f32", "fp16": "f16"}
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32", "fp16"])
    ap.add_argument("--scheme", default="two_lattice", choices=["two_lattice", "aa"])
    ap.add_argument("--tau", type=float, default=0.505)
    ap.add_argument("--k0", type=float, default=4.0)
    ap.add_argument("--icheck", type=int, default=100)
    ap.add_argument("--kernel", type=int, default=0, choices=[0, 1, 2, 4, 8],
                    help="stream-collide kernel (0 automatic; 2/4 cells per thread apply to FP16; 8 TMA row pipeline)")
    ap.add_argument("--les-cs", type=float, default=0.0,
                    help="Smagorinsky constant: > 0 times the LES collision instead of BGK")
    ap.add_argument("--decomp", default=None, choices=["replicas", "slabs"],
                    help="one box split into z-slabs (default under torchrun) or independent replica boxes "
                         "(default on one GPU)")
    ap.add_argument("--local-slabs", type=int, default=2, help="--decomp slabs on one GPU: slabs per box")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-forms", action="store_true", help="skip the FP32 / FP16 lines of the default run")
    ap.add_argument("--no-large", action="store_true", help="skip the 512^3 / 1024^3 lines of the default run")
    a = ap.parse_args()
    if a.decomp is None:
        a.decomp = "slabs" if int(os.environ.get("WORLD_SIZE", "1")) > 1 else "replicas"
    return a


def workload_name(a):
    coll = f"Smagorinsky LES cteS={a.les_cs:g}" if a.les_cs > 0 else "BGK"
    return (f"decaying HIT {a.size}^3 D3Q19 {coll}, {a.precision} {a.scheme}, tau={a.tau}, k0={a.k0:g}, "
            f"u_rms=0.03, seed 1234")


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), ws


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.proc, self.path = device, None, None

    def start(self):
        try:
            import tempfile

            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.device)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        pw = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(pw) if pw else None}


# ------------------------------------------------------------ shared parts
N_ARRAYS = {"two_lattice": 37, "aa": 19}
ELEM = {"fp64": 8, "fp32": 4, "fp16": 2}
# the larger boxes of the default run: (size, precision, scheme, k0, tau)
LARGE = ((512, "fp64", "two_lattice", 6.0, 0.503), (1024, "fp16", "aa", 8.0, 0.502),
         (1024, "fp32", "aa", 8.0, 0.502))


def config_of(a, ws):
    """The run's config dict; both arms print the same one."""
    L = a.size
    pop_gb = N_ARRAYS[a.scheme] * ELEM[a.precision] * float(L) ** 3 / 1e9
    cfg = {"workload": workload_name(a), "box": L, "precision": a.precision, "scheme": a.scheme, "tau": a.tau,
           "k0": a.k0, "u_rms": 0.03, "seed": 1234, "cells_per_gpu": L ** 3, "kernel": a.kernel,
           "les_cs": a.les_cs,
           "l2": f"inputs larger than L2 ({pop_gb:.1f} GB of populations per GPU, L2 126 MB)"
           if pop_gb > 0.126 else "inputs may fit in L2"}
    if a.decomp == "slabs":
        nslab = ws if ws > 1 else a.local_slabs
        cfg["workload"] += f", split into {nslab} z-slabs"
        cfg["box"] = [L, L, L * ws if ws > 1 else L]
        cfg["slabs"] = nslab
        cfg["parallelism"] = (f"z-slabs, {'one per GPU' if ws > 1 else 'all on one GPU'}, ghost planes filled "
                              "by the step kernel (peer stores), barrier between steps")
    else:
        cfg["parallelism"] = f"{ws} independent replica box(es), one per GPU"
    return cfg


def kernel_key(precision, scheme, L, kernel=0, les=False):
    """Name of the stream-collide kernel a launch runs (the key of
    profiles/ncu_traffic.json)."""
    kern = f"{'k_two' if scheme == 'two_lattice' else 'k_aa'}_{precision}" + ("_les" if les else "")
    if precision == "fp32" and scheme == "aa" and kernel == 0:
        tpr = L // 4  # the odd step on four cells per thread, the even one on two
        if L % 4 == 0 and tpr & (tpr - 1) == 0 and (L * tpr) % 32 == 0:
            return "k_aa_f32w" + ("_les" if les else "")
    if precision == "fp32" and kernel in (0, 2):  # two cells per thread, both schemes, BGK and LES
        tpr = L // 2
        if L % 2 == 0 and tpr & (tpr - 1) == 0 and (L * tpr) % 32 == 0:
            return ("k_two_f32v" if scheme == "two_lattice" else "k_aa_f32v") + ("_les" if les else "")
    allowed = (0, 4) if (les or scheme == "aa") else (0, 2, 4)  # the LES collision runs on four cells only
    if precision == "fp16" and scheme == "aa" and not les and kernel == 0:
        tpr = L // 8  # the odd step on eight cells per thread, the even one on four
        if L % 8 == 0 and tpr & (tpr - 1) == 0 and (L * tpr) % 32 == 0:
            return "k_aa_f16w"
    if precision == "fp16" and kernel in allowed:
        v = 2 if kernel == 2 else 4
        tpr = L // v
        if L % v == 0 and tpr & (tpr - 1) == 0 and (L * tpr) % 32 == 0:  # cells per thread: 2 or 4
            kern = ("k_two_f16v2" if kernel == 2 else "k_two_f16v") if scheme == "two_lattice" else "k_aa_f16v"
            kern += "_les" if les else ""
    return kern


# -------------------------------------------------------------- CPU oracle
def cpu_baseline(a, seconds: float):
    """The oracle's FP64 boundaries + col_MC (reference algorithm) on the host
    cores, on the same box; steps sized to about `seconds` of CPU work."""
    from oracle import oracle as O

    O.set_num_threads(os.cpu_count() or 1)
    L = a.size
    orc = O.OracleLattice(L, L, L, form="f64")
    from bgk3d_hit_b200.hit import hit_velocity

    u, v, w = hit_velocity(L, a.k0, 0.03, 1234)
    orc.init_velocity(u, v, w, 1.0)
    orc.set_les(a.les_cs)
    svisc = (a.tau - 0.5) / 3.0
    t1 = orc.time_steps(svisc, 1)
    steps = max(1, min(200, int(seconds / max(t1, 1e-6))))
    t = orc.time_steps(svisc, steps)
    orc.close()
    return {"value": L ** 3 * steps / t / 1e9, "unit": "GLUPS", "cores": O.num_threads(), "kind": "port",
            "sample": f"{steps} steps of {L}^3 FP64 (step3 halo fill + col_MC, C restatement, OpenMP)"}


def run_reference(a):
    rank, _, ws = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O

    O.set_num_threads(os.cpu_count() or 1)
    L = a.size
    from bgk3d_hit_b200.hit import hit_velocity

    orc = O.OracleLattice(L, L, L, form="f64")
    u, v, w = hit_velocity(L, a.k0, 0.03, 1234)
    orc.init_velocity(u, v, w, 1.0)
    orc.set_les(a.les_cs)
    svisc = (a.tau - 0.5) / 3.0
    t1 = orc.time_steps(svisc, 1)
    # each timed step is a bounded sample: cap the whole run at a few minutes
    k = max(1, min(a.steps, int(120.0 / max(t1, 1e-6))))
    w_ = max(0, min(a.warmup, int(60.0 / max(t1, 1e-6))))
    orc.time_steps(svisc, w_)
    t = orc.time_steps(svisc, k)
    val = L ** 3 * k / t / 1e9
    cores = O.num_threads()
    line = {
        "impl": "reference", "metric": "GLUPS (fused D3Q19 stream-collide)", "value": val, "unit": "GLUPS",
        "n_gpus": ws, "steps": k, "warmup": w_, "ms_per_step": 1e3 * t / k, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": DTYPE["fp64"], "data": "synthetic",
        "config": config_of(a, ws),
        "cpu_baseline": {"value": val, "unit": "GLUPS", "cores": cores, "kind": "port",
                         "sample": f"{k} steps of {L}^3 FP64, C restatement of boundaries + col_MC "
                                   "(the Fortran/MPI reference cannot be built in this image)"},
        "e2e": {"value": val, "unit": "GLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------- GPU
def measured_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel_key: str):
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        return json.load(open(p)).get(kernel_key)
    except Exception:
        return None


def time_steps(box, steps, device):
    """K steps of a resident box between CUDA events on its stream, with a
    clock record of the region: (ms, launches, clocks)."""
    import torch

    stream = torch.cuda.ExternalStream(box.stream, device=device)
    clocks = ClockSampler(device)
    clocks.start()
    l0 = box.launch_count
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    box.synchronize()
    e0.record(stream)
    box.run(steps)
    e1.record(stream)
    box.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return ms, box.launch_count - l0, clocks.stop()


def roofline_of(precision, scheme, L, ms_per_step, kernel=0, les=False):
    bpc = BYTES_PER_CELL[precision]
    peak, peak_kind = measured_hbm()
    achieved = bpc * float(L) ** 3 / (ms_per_step * 1e-3) / 1e9
    kern = kernel_key(precision, scheme, L, kernel, les)
    tr = ncu_traffic(kern)
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": tr * float(L) ** 3 if tr else None, "peak_kind": peak_kind, "bytes_per_cell": bpc,
            "kernel": kern}


def form_line(a, precision, pin, device, fp64_value):
    """The default box in another storage form (default two-lattice kernel)."""
    import bgk3d_hit_b200 as B

    L = a.size
    steps = max(a.steps, 200)
    box = B.BGK3D(L, svisc=(a.tau - 0.5) / 3.0, u0=0.03, precision=precision, scheme="two_lattice",
                  icheck=a.icheck, device=device)
    try:
        box.init_velocity(*(p.numpy() for p in pin))
        box.run(a.warmup)
        ms, launches, clk = time_steps(box, steps, device)
    finally:
        box.close()
    value = float(L) ** 3 * steps / (ms * 1e-3) / 1e9
    rl = roofline_of(precision, "two_lattice", L, ms / steps)
    if rl["traffic"] is not None:
        rl["traffic_note"] = "ncu DRAM bytes per cell of the 256^3 capture x cells"
    return {"value": value, "unit": "GLUPS", "ratio_vs_fp64": value / fp64_value, "steps": steps,
            "warmup": a.warmup, "ms_per_step": ms / steps, "dtype": DTYPE[precision], "scheme": "two_lattice",
            "roofline": rl, "gpu_launches": launches, "clocks": clk}


def large_line(a, L, precision, scheme, k0, tau, device):
    """A larger box of the same path, initial field made on the GPU."""
    import torch

    import bgk3d_hit_b200 as B
    from bgk3d_hit_b200.hit import NUMPY_NOISE_MAX_CELLS, hit_velocity_device

    steps = max(a.steps, 50)
    t0 = time.time()
    box = B.BGK3D(L, svisc=(tau - 0.5) / 3.0, u0=0.03, precision=precision, scheme=scheme, icheck=a.icheck,
                  device=device)
    try:
        u = hit_velocity_device(L, k0, 0.03, 1234, device=device)
        box.init_velocity_device(*u)
        del u
        torch.cuda.empty_cache()
        init_s = time.time() - t0
        box.run(a.warmup)
        ms, launches, clk = time_steps(box, steps, device)
        dev_gb = box.device_bytes / 1e9
    finally:
        box.close()
    value = float(L) ** 3 * steps / (ms * 1e-3) / 1e9
    rl = roofline_of(precision, scheme, L, ms / steps)
    if rl["traffic"] is not None:
        rl["traffic_note"] = "ncu DRAM bytes per cell of the 256^3 capture x cells"
    noise = "numpy default_rng" if L ** 3 <= NUMPY_NOISE_MAX_CELLS else "torch CUDA generator"
    return {"workload": f"decaying HIT {L}^3 D3Q19 BGK, {precision} {scheme}, tau={tau}, k0={k0:g}, u_rms=0.03, "
                        f"seed 1234 ({noise} noise)", "box": L, "precision": precision, "scheme": scheme,
            "value": value, "unit": "GLUPS", "steps": steps, "warmup": a.warmup, "ms_per_step": ms / steps,
            "device_gb": dev_gb, "init_s": init_s, "roofline": rl, "gpu_launches": launches, "clocks": clk}


def run_ours(a):
    import torch

    import bgk3d_hit_b200 as B
    from bgk3d_hit_b200.hit import hit_velocity

    rank, local, ws = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    L = a.size
    svisc = (a.tau - 0.5) / 3.0
    u, v, w = hit_velocity(L, a.k0, 0.03, 1234)
    pin = [torch.from_numpy(x).pin_memory() for x in (u, v, w)]
    del u, v, w
    box = B.BGK3D(L, svisc=svisc, u0=0.03, precision=a.precision, scheme=a.scheme, icheck=a.icheck, device=local,
                  kernel=a.kernel, les_cs=a.les_cs)
    box.init_velocity(*(p.numpy() for p in pin))
    stream = torch.cuda.ExternalStream(box.stream, device=local)

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        box.synchronize()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    # warm-up
    box.run(a.warmup)
    barrier()
    # -------- timed: K fused steps, populations resident
    clocks = ClockSampler(local)
    clocks.start()
    l0 = box.launch_count
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    box.run(a.steps)
    e1.record(stream)
    barrier()
    ms = e0.elapsed_time(e1)
    launches = box.launch_count - l0
    clk = clocks.stop()
    ms_max = max_over_ranks(ms)
    lu = float(L) ** 3 * a.steps
    value = ws * lu / (ms_max * 1e-3) / 1e9
    roofline = roofline_of(a.precision, a.scheme, L, ms / a.steps, a.kernel, a.les_cs > 0)
    box.close()

    # -------- e2e through the C-ABI with host buffers
    e2e = None
    if not a.no_e2e:
        ev0, evi, ev1 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        box2 = B.BGK3D(L, svisc=svisc, u0=0.03, precision=a.precision, scheme=a.scheme, icheck=a.icheck,
                       device=local, kernel=a.kernel, les_cs=a.les_cs)
        stream2 = torch.cuda.ExternalStream(box2.stream, device=local)
        # warm-up pass of the same calls (upload, init, W steps), untimed: the
        # context's upload staging and the first-use costs of the pinned pages
        # stay out of the timed pass, which uploads and initialises again
        box2.init_velocity(*(p.numpy() for p in pin))
        for it in range(1, a.warmup + 1):
            box2.boundaries(it)
            box2.col_MC(it)
        box2.synchronize()
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        ev0.record(stream2)
        box2.init_velocity(*(p.numpy() for p in pin))
        evi.record(stream2)
        ndiag = 0
        for it in range(1, a.steps + 1):
            box2.boundaries(it)
            box2.col_MC(it)
            if box2.diagnostic(it) is not None or it == a.steps:
                ndiag += 1
        if a.steps % a.icheck:
            box2.diagno(a.steps)
        ev1.record(stream2)
        box2.synchronize()
        ms2 = max_over_ranks(ev0.elapsed_time(ev1))
        fixed = max_over_ranks(ev0.elapsed_time(evi))
        per_step = (ms2 - fixed) / a.steps
        diag_bytes = 11 * 8
        e2e = {"value": ws * lu / (ms2 * 1e-3) / 1e9, "unit": "GLUPS",
               "h2d_bytes_per_step": 3 * 8 * L ** 3 / a.steps,
               "d2h_bytes_per_step": diag_bytes * ndiag / a.steps,
               "fixed_ms": fixed, "per_step_ms": per_step,
               "value_at_2000_steps": ws * float(L) ** 3 * 2000 / ((fixed + 2000 * per_step) * 1e-3) / 1e9,
               "includes": f"velocity upload from pinned host memory and init (fixed_ms), {a.steps} x "
                           f"(boundaries + col_MC + diagnostic gated by icheck={a.icheck}), diagnostics read back "
                           "(per_step_ms); value_at_2000_steps = the same split at the 2000 steps of the HIT "
                           "256^3 run"}
        box2.close()

    default_run = (ws == 1 and a.precision == "fp64" and a.scheme == "two_lattice" and a.les_cs == 0
                   and a.kernel == 0)
    forms = None
    if default_run and not a.no_forms:
        forms = {"fp64": {"value": value, "unit": "GLUPS", "ratio_vs_fp64": 1.0, "note": "the headline line"}}
        for prec in ("fp32", "fp16"):
            forms[prec] = form_line(a, prec, pin, local, value)
    large = None
    if default_run and not a.no_large:
        large = []
        for (Lb, prec, sch, k0, tau) in LARGE:
            try:
                large.append(large_line(a, Lb, prec, sch, k0, tau, local))
            except Exception as ex:  # a box that does not fit is reported, not fatal
                large.append({"box": Lb, "precision": prec, "scheme": sch, "error": str(ex)[:200]})
            torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu:
        try:
            cpu = cpu_baseline(a, a.cpu_seconds)
        except Exception as ex:  # the CPU baseline is optional for the GPU number
            cpu = {"value": None, "unit": "GLUPS", "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": "GLUPS (fused D3Q19 stream-collide)", "value": value, "unit": "GLUPS", "n_gpus": ws,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE[a.precision], "data": "synthetic",
            "config": config_of(a, ws), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": clk,
        }
        if forms is not None:
            line["forms"] = forms
        if large is not None:
            line["large"] = large
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def run_slabs(a):
    """The z-slab decomposition: value = all slabs' cell updates / the slowest
    slab's device time for K steps (each step: the slab kernels, then the
    barrier)."""
    import torch

    from bgk3d_hit_b200.hit import hit_velocity
    from bgk3d_hit_b200.slabs import DistSlabs, LocalSlabs, fp16_scale_for_velocity

    rank, local, ws = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    if a.scheme != "two_lattice":
        raise SystemExit("--decomp slabs runs the two-lattice scheme")
    L = a.size
    svisc = (a.tau - 0.5) / 3.0
    u, v, w = hit_velocity(L, a.k0, 0.03, 1234)
    kw = dict(svisc=svisc, u0=0.03, precision=a.precision, icheck=a.icheck, les_cs=a.les_cs)
    if a.precision == "fp16":
        kw["fp16_scale"] = fp16_scale_for_velocity(u, v, w)
    if ws > 1:
        drv = DistSlabs(L, L, L * ws, device=local, **kw)
        boxes, nslab, cells = [drv.box], ws, float(L) ** 3 * ws
    else:
        drv = LocalSlabs(L, L, L, a.local_slabs, devices=(local,), **kw)
        boxes, nslab, cells = drv.slabs, a.local_slabs, float(L) ** 3
    drv.init_velocity(u, v, w)
    streams = [torch.cuda.ExternalStream(b.stream, device=local) for b in boxes]
    drv.run(a.warmup)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = sum(b.launch_count for b in boxes)
    e0 = [torch.cuda.Event(enable_timing=True) for _ in boxes]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in boxes]
    drv.barrier()
    for e, s in zip(e0, streams):
        e.record(s)
    drv.run(a.steps)
    for e, s in zip(e1, streams):
        e.record(s)
    torch.cuda.synchronize()
    ms = max(e0[0].elapsed_time(e) for e in e1)
    if ws > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    launches = sum(b.launch_count for b in boxes) - l0
    clk = clocks.stop()
    # the edge-plane kernel of the last step (device events), slowest slab
    edge_us = max(b.slab_edge_time_us() for b in boxes)
    if ws > 1:
        t = torch.tensor([edge_us], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        edge_us = float(t.item())
    value = cells * a.steps / (ms * 1e-3) / 1e9
    bpc = BYTES_PER_CELL[a.precision]
    peak, peak_kind = measured_hbm()
    achieved = bpc * (cells / ws) / (ms * 1e-3 / a.steps) / 1e9
    # per step, every slab stores 5 populations of each of its two boundary
    # planes into its neighbours' ghost planes
    exch = len(boxes) * 2 * 5 * L * L * ELEM[a.precision]
    if rank == 0:
        line = {
            "metric": "GLUPS (fused D3Q19 stream-collide)", "value": value, "unit": "GLUPS", "n_gpus": ws,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE[a.precision], "data": "synthetic",
            "config": config_of(a, ws),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind, "bytes_per_cell": bpc,
                         "kernel": f"k_slab_{a.precision}", "per": "whole step of this GPU's slabs"},
            "exchange": {"bytes_per_step_per_gpu": exch, "peer": ws > 1,
                         "what": "2 faces x 5 populations x lx*ly x element size per slab, stored by the edge "
                                 "kernel into the neighbours' ghost planes",
                         "edge_kernel_us": edge_us, "edge_share_of_step": edge_us * 1e-3 / (ms / a.steps),
                         "edge_kernel_note": "device time of the last step's edge-plane kernel (boundary planes "
                                             "and their peer stores), running beside the interior kernel; "
                                             "slowest slab"},
            "cpu_baseline": None, "e2e": None, "gpu_launches": launches, "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    drv.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.decomp == "slabs":
        run_slabs(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
