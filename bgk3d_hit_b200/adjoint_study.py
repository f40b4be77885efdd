"""Checks and costs of the discrete adjoint on decaying HIT.

    python -m bgk3d_hit_b200.adjoint_study [--size 128] [--steps 1000] [--ckpt 32]
        [--tau 0.51] [--k0 4] [--dirs 64] [--h 1e-6] [--precision fp64] [--cache-gb 0]
        [--mode recompute|rebuild]

Initial velocity: seeded HIT field (seed 1234, E(k) ~ k^4 exp(-2 (k/k0)^2),
u_rms = 0.03); target u_tgt: the same generator with a second seed (4321).
Loss = 0.5 mean |u(T) - u_tgt|^2. Reports, as one JSON object:
- fd: the relative error of <grad, d> against central differences
  (L(u0 + h d) - L(u0 - h d)) / 2h over `dirs` seeded random unit directions d
  (max and median), and the same for tau;
- fd_sweep: the same with a step chosen per direction by the usual h-sweep:
  central differences at h = 1e-3 ... 1e-7 (`sweep` values), and the step
  whose estimate agrees best with the next smaller step's (the plateau
  between truncation error at large h and rounding noise at small h);
- tangent: the relative difference between <grad, d> + grad_tau dtau and the
  tangent-linear derivative along (d, dtau) for a few directions;
- cost: wall time of the adjoint call (forward with checkpoints, recomputation,
  backward) over the wall time of a forward-only call of the same length
  (medians of 5 calls each);
  with --cache-gb G, bgk_adjoint keeps up to G GB of forward states between
  checkpoints instead of recomputing them (bgk_adjoint_cache); with
  --mode rebuild the backward pass rebuilds the states between checkpoints
  from the one after them (bgk_adjoint_mode BGK_ADJ_REBUILD), and
  vs_recompute gives the relative L2 difference of its gradient from the
  recomputing mode's;
- vs_fp64 (FP32 storage only): the relative L2 difference between the FP32
  gradient and the FP64 adjoint gradient of the same problem (central
  differences of an FP32 loss over 1000 steps are dominated by its rounding,
  so the FP32 gradient is compared with FP64 instead).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import _abi
from .hit import hit_velocity
from .solver import BGK3D

DP = C.POINTER(C.c_double)


def _p(a):
    return a.ctypes.data_as(DP)


def _adj(box, u0, ut, T, K, grads):
    n = box.ncell
    loss, gt = C.c_double(), C.c_double()
    g = np.zeros(3 * n) if grads else None
    rc = box._lib.bgk_adjoint(box._h, _p(u0[0]), _p(u0[1]), _p(u0[2]), _p(ut[0]), _p(ut[1]), _p(ut[2]), T, K,
                              C.byref(loss), _p(g) if grads else None, C.byref(gt) if grads else None)
    if rc:
        raise RuntimeError(box._lib.bgk_last_error().decode())
    return loss.value, g, gt.value


def run(size=128, steps=1000, ckpt=32, tau=0.51, k0=4.0, u_rms=0.03, dirs=64, h=1e-6, precision="fp64", ntan=4,
        cache_gb=0.0, reps=5, sweep=(1e-3, 1e-4, 1e-5, 1e-6, 1e-7), mode="recompute"):
    svisc = (tau - 0.5) / 3.0
    u0 = [np.ascontiguousarray(a) for a in hit_velocity(size, k0, u_rms, 1234)]
    ut = [np.ascontiguousarray(a) for a in hit_velocity(size, k0, u_rms, 4321)]
    box = BGK3D(size, svisc=svisc, u0=u_rms, precision=precision)
    if cache_gb > 0:
        box._lib.bgk_adjoint_cache(box._h, int(cache_gb * 1e9))
    if mode == "rebuild":
        if not box._lib.bgk_adjoint_rebuilds(_abi.PRECISIONS[precision], box.omega, ckpt):
            raise ValueError("rebuild mode does not apply to tau %g with a checkpoint every %d steps" % (tau, ckpt))
        box._lib.bgk_adjoint_mode(box._h, _abi.BGK_ADJ_REBUILD)
    tau_used = 1.0 / box.omega
    # cost: forward-only and full adjoint, each the median of `reps` calls
    # after one warm-up call
    _adj(box, u0, ut, steps, ckpt, False)
    tf = []
    for _ in range(reps):
        t0 = time.perf_counter()
        loss, _, _ = _adj(box, u0, ut, steps, ckpt, False)
        tf.append(time.perf_counter() - t0)
    t_fwd = float(np.median(tf))
    _adj(box, u0, ut, steps, ckpt, True)
    ta = []
    for _ in range(reps):
        t0 = time.perf_counter()
        loss2, g, gtau = _adj(box, u0, ut, steps, ckpt, True)
        ta.append(time.perf_counter() - t0)
    t_adj = float(np.median(ta))
    rng = np.random.default_rng(2024)
    errs, sweep_errs, sweep_h = [], [], []

    def central(d, hh):
        lp = _adj(box, [a + hh * b for a, b in zip(u0, d)], ut, steps, ckpt, False)[0]
        lm = _adj(box, [a - hh * b for a, b in zip(u0, d)], ut, steps, ckpt, False)[0]
        return (lp - lm) / (2 * hh)

    for _ in range(dirs):
        d = rng.standard_normal((3,) + u0[0].shape)
        d /= np.linalg.norm(d)
        fd = central(d, h)
        ad = float(np.dot(g, d.reshape(-1)))
        errs.append(abs(ad - fd) / max(abs(fd), 1e-300))
        if sweep:
            est = [fd if hh == h else central(d, hh) for hh in sweep]
            gaps = [abs(est[m] - est[m + 1]) for m in range(len(est) - 1)]
            m = int(np.argmin(gaps))
            sweep_h.append(sweep[m])
            sweep_errs.append(abs(ad - est[m]) / max(abs(est[m]), 1e-300))
    # tau by central differences of boxes with omega = 1/(tau +- h)
    lt = []
    for s in (1, -1):
        b2 = BGK3D(size, omega=1.0 / (tau_used + s * h), precision=precision, u0=u_rms)
        lt.append(_adj(b2, u0, ut, steps, ckpt, False)[0])
        b2.close()
    fd_tau = (lt[0] - lt[1]) / (2 * h)
    # tangent-linear checks
    tan_errs = []
    for m in range(ntan):
        d = rng.standard_normal((3,) + u0[0].shape)
        dtau = float(rng.standard_normal())
        lo, dl = C.c_double(), C.c_double()
        dd = [np.ascontiguousarray(x) for x in d]
        rc = box._lib.bgk_tangent(box._h, _p(u0[0]), _p(u0[1]), _p(u0[2]), _p(dd[0]), _p(dd[1]), _p(dd[2]), dtau,
                                  _p(ut[0]), _p(ut[1]), _p(ut[2]), steps, C.byref(lo), C.byref(dl))
        if rc:
            raise RuntimeError(box._lib.bgk_last_error().decode())
        pred = float(np.dot(g, d.reshape(-1))) + gtau * dtau
        tan_errs.append(abs(pred - dl.value) / abs(dl.value))
    vs_rec = None
    if mode == "rebuild":
        box._lib.bgk_adjoint_mode(box._h, _abi.BGK_ADJ_RECOMPUTE)
        _, grec, gtrec = _adj(box, u0, ut, steps, ckpt, True)
        vs_rec = {"grad_rel_l2": float(np.linalg.norm(g - grec) / np.linalg.norm(grec)),
                  "grad_tau_rel": abs(gtau - gtrec) / abs(gtrec)}
    box.close()
    vs64 = None
    if precision != "fp64":
        b64 = BGK3D(size, svisc=svisc, u0=u_rms, precision="fp64")
        _, g64, gt64 = _adj(b64, u0, ut, steps, ckpt, True)
        b64.close()
        vs64 = {"grad_rel_l2": float(np.linalg.norm(g - g64) / np.linalg.norm(g64)),
                "grad_tau_rel": abs(gtau - gt64) / abs(gt64)}
    return {
        "config": {"size": size, "steps": steps, "ckpt_every": ckpt, "tau": tau_used, "k0": k0, "u_rms": u_rms,
                   "precision": precision, "h": h, "directions": dirs, "cache_gb": cache_gb, "mode": mode},
        "loss": loss, "loss_in_adjoint_call": loss2, "grad_tau": gtau, "fd_grad_tau": fd_tau,
        "fd": ({"max_rel_err": float(np.max(errs)), "median_rel_err": float(np.median(errs)),
                "p90_rel_err": float(np.percentile(errs, 90)),
                "tau_rel_err": abs(gtau - fd_tau) / abs(fd_tau)} if errs else
               {"tau_rel_err": abs(gtau - fd_tau) / abs(fd_tau)}),
        "fd_sweep": ({"max_rel_err": float(np.max(sweep_errs)), "median_rel_err": float(np.median(sweep_errs)),
                      "p90_rel_err": float(np.percentile(sweep_errs, 90)),
                      "h_chosen": {str(x): sweep_h.count(x) for x in sorted(set(sweep_h))}} if sweep_errs else None),
        "tangent": {"max_rel_err": float(np.max(tan_errs)) if tan_errs else None, "directions": ntan},
        "cost": {"forward_s": t_fwd, "adjoint_s": t_adj, "adjoint_over_forward": t_adj / t_fwd},
        "vs_fp64": vs64,
        "vs_recompute": vs_rec,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--ckpt", type=int, default=32)
    ap.add_argument("--tau", type=float, default=0.51)
    ap.add_argument("--k0", type=float, default=4.0)
    ap.add_argument("--dirs", type=int, default=64)
    ap.add_argument("--h", type=float, default=1e-6)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--cache-gb", type=float, default=0.0)
    ap.add_argument("--mode", default="recompute", choices=["recompute", "rebuild"])
    ap.add_argument("--ntan", type=int, default=4)
    a = ap.parse_args()
    print(json.dumps(run(a.size, a.steps, a.ckpt, a.tau, a.k0, dirs=a.dirs, h=a.h, precision=a.precision,
                         cache_gb=a.cache_gb, mode=a.mode, ntan=a.ntan)))


if __name__ == "__main__":
    main()
