"""Accuracy of the FP32 and FP16 storage forms against FP64 on decaying HIT.

    python -m bgk3d_hit_b200.precision_study [--size 512] [--steps 5000] [--every 100]
        [--k0 6] [--tau 0.503] [--scheme two_lattice] [--les-cs 0] [--out results.json]

Runs the same seeded HIT initial condition (random-phase solenoidal field,
E(k) ~ k^4 exp(-2 (k/k0)^2), u_rms = 0.03) in the three storage forms side by
side on one GPU, through the public API, and reports against the FP64 run:
- E(t): mean kinetic energy 0.5|u|^2 of the local velocity (diagno column),
- eps(t): strain-rate dissipation 2 nu <S:S>, S = -3 omega Pi_neq / (2 rho),
- E(k): shell spectrum of the final velocity field,
as maximum relative errors over the run (E, eps) and over the shells that hold
at least 1e-6 of the peak energy (E(k)). Prints one JSON object.

Plain BGK is unstable when the flow becomes under-resolved at low viscosity
(tau close to 1/2): a form whose diagnostics turn non-finite is stopped, its
blow-up step is reported, and the errors are taken over the steps at which
every form was still finite (the spectrum then at the last such record).
With --les-cs C > 0 every form runs the Smagorinsky collision (cteS = C,
SRC/col_MC.F90:221-309), which keeps such runs finite; eps then still uses
the molecular viscosity.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import _abi
from .hit import hit_velocity
from .solver import BGK3D

FORMS = ("fp64", "fp32", "fp16")


def run(size=512, steps=5000, every=100, k0=6.0, tau=0.503, u_rms=0.03, seed=1234, scheme="two_lattice",
        forms=FORMS, device=0, les_cs=0.0, device_ic=None):
    """device_ic: make the initial field on the GPU (hit_velocity_device) and
    initialise from device memory; default for boxes of 512^3 cells and more."""
    svisc = (tau - 0.5) / 3.0
    if device_ic is None:
        device_ic = size ** 3 >= 512 ** 3
    t0 = time.time()
    if device_ic:
        from .hit import hit_velocity_device

        u, v, w = hit_velocity_device(size, k0, u_rms, seed, device=device)
    else:
        u, v, w = hit_velocity(size, k0, u_rms, seed)
    t_ic = time.time() - t0
    boxes = {}
    for f in forms:
        b = BGK3D(size, svisc=svisc, u0=u_rms, precision=f, scheme=scheme, icheck=every, device=device,
                  les_cs=les_cs)
        if device_ic:
            b.init_velocity_device(u, v, w)
        else:
            b.init_velocity(u, v, w)
        boxes[f] = b
    del u, v, w
    if device_ic:
        import torch

        torch.cuda.empty_cache()
    series = {f: {"step": [], "E": [], "eps": [], "diss": [], "rho": []} for f in forms}
    blowup = {f: None for f in forms}
    spec = {}
    nb = size // 2 + 1

    def record(it):
        for f, b in boxes.items():
            if blowup[f] is not None:
                continue
            try:
                if it == 0:
                    dg, ds = b.diagno(0), b.dissipation(0)
                    d = {"ke_mean": dg[4], "rho_mean": dg[0], "diss": ds[2], "eps_strain": float("nan")}
                else:
                    d = b.diagnostic(it)
            except _abi.BgkError as e:
                if e.code != _abi.BGK_ERR_NONFINITE:
                    raise
                blowup[f] = it
                continue
            if d is None:
                continue
            s_ = series[f]
            s_["step"].append(it)
            s_["E"].append(d["ke_mean"])
            s_["eps"].append(d["eps_strain"])
            s_["diss"].append(d["diss"])
            s_["rho"].append(d["rho_mean"])
        if all(v is None for v in blowup.values()):
            for f, b in boxes.items():
                spec[f] = (it, b.spectrum(nb))

    record(0)
    t0 = time.time()
    for it in range(1, steps + 1):
        if all(v is not None for v in blowup.values()):
            break
        for f, b in boxes.items():
            if blowup[f] is None:
                b.boundaries(it)
                b.col_MC(it)
        if it % every == 0 or it == steps:
            record(it)
    t_run = time.time() - t0
    for b in boxes.values():
        b.close()

    ref = series["fp64"] if "fp64" in series else None
    common = min(len(series[f]["step"]) for f in forms)  # records where every form was finite
    out = {"config": {"size": size, "steps": steps, "every": every, "k0": k0, "tau": tau, "u_rms": u_rms,
                      "seed": seed, "scheme": scheme, "les_cs": les_cs},
           "seconds": {"initial_condition": t_ic, "run": t_run},
           "compared_up_to_step": series[forms[0]]["step"][common - 1],
           "spectrum_step": next(iter(spec.values()))[0] if spec else None, "forms": {}}
    for f in forms:
        s_ = series[f]
        rec = {"blowup_step": blowup[f], "E_initial": s_["E"][0], "E_last": s_["E"][common - 1],
               "eps_last": s_["eps"][common - 1]}
        if ref is not None and f != "fp64" and common > 1:
            E, Er = np.array(s_["E"][:common]), np.array(ref["E"][:common])
            ep, epr = np.array(s_["eps"][1:common]), np.array(ref["eps"][1:common])
            di, dir_ = np.array(s_["diss"][1:common]), np.array(ref["diss"][1:common])
            rec["E_max_rel_err"] = float(np.max(np.abs(E - Er) / np.abs(Er)))
            rec["eps_max_rel_err"] = float(np.max(np.abs(ep - epr) / np.abs(epr)))
            rec["diss_max_rel_err"] = float(np.max(np.abs(di - dir_) / np.abs(dir_)))
            if spec:
                ek, ekr = spec[f][1], spec["fp64"][1]
                mask = ekr >= 1e-6 * ekr.max()
                rec["Ek_max_rel_err"] = float(np.max(np.abs(ek[mask] - ekr[mask]) / ekr[mask]))
                rec["Ek_shells"] = int(mask.sum())
            rec["rho_mean_drift"] = float(abs(s_["rho"][common - 1] - s_["rho"][0]))
        out["forms"][f] = rec
    out["series"] = {f: {k: list(map(float, v)) for k, v in series[f].items()} for f in forms}
    out["spectrum"] = {f: list(map(float, spec[f][1])) for f in spec}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--k0", type=float, default=6.0)
    ap.add_argument("--tau", type=float, default=0.503)
    ap.add_argument("--scheme", default="two_lattice")
    ap.add_argument("--les-cs", type=float, default=0.0, help="Smagorinsky constant (0: BGK)")
    ap.add_argument("--out", default=None, help="write the full series and spectra here (JSON)")
    a = ap.parse_args()
    res = run(a.size, a.steps, a.every, a.k0, a.tau, scheme=a.scheme, les_cs=a.les_cs)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f)
    print(json.dumps({k: v for k, v in res.items() if k not in ("series", "spectrum")}))


if __name__ == "__main__":
    main()
