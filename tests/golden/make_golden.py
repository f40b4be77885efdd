"""Generates the golden fixtures of tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py [case ...]

The reference ships no golden vectors and its Fortran/MPI build cannot be
compiled here, so these fixtures pin the oracle's own output (small boxes,
seeded inputs); tests compare the oracle and the GPU path against them.
Each case is a function oracle_module -> dict of arrays.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def tgv_f64_5x7x9(O):
    """Faithful Taylor-Green (SRC/init.F90) on 5x7x9, FP64, 10 reference steps
    (boundaries + col_MC), svisc 0.01, u0 0.05."""
    L = O.OracleLattice(5, 7, 9, form="f64")
    L.init_tgv(0.05, faithful=True)
    out = {"pops0": L.get_pops()}
    L.step(0.01)
    out["pops1"] = L.get_pops()
    for _ in range(9):
        L.step(0.01)
    out["pops10"] = L.get_pops()
    out["diagno10"] = L.diagno(False)
    out["diss10"] = L.dissipation(0.01, 0.05, 10, False)
    return out


def tgv_f32_6x5x4(O):
    """Same, single precision (the reference's default build), 6x5x4."""
    L = O.OracleLattice(6, 5, 4, form="f32")
    L.init_tgv(0.05, faithful=True)
    for _ in range(10):
        L.step(0.01)
    return {"pops10": L.get_pops(), "diagno10": L.diagno(False)}


def hit_f16_8(O):
    """Seeded random velocity (not the HIT spectrum: uniform noise, seed 11),
    FP16 scaled-deviation storage with scale 2^16, 8^3, 5 steps, svisc 0.005."""
    rng = np.random.default_rng(11)
    u, v, w = (rng.uniform(-0.03, 0.03, 512) for _ in range(3))
    L = O.OracleLattice(8, 8, 8, form="f16", scale=2.0**16)
    L.init_velocity(u, v, w, 1.0)
    out = {"pops0": L.get_pops()}
    for _ in range(5):
        L.step(0.005, periodic=True)
    out["pops5"] = L.get_pops()
    return out


def les_tgv_f64_6x5x4(O):
    """The Smagorinsky collision (SRC/col_MC.F90:221-309, cteS = 0.3) on the
    faithful Taylor-Green state, FP64, 6x5x4, svisc 0.001, 6 periodic steps."""
    L = O.OracleLattice(6, 5, 4, form="f64")
    L.init_tgv(0.05, faithful=True)
    L.set_les(0.3)
    out = {"pops0": L.get_pops()}
    for _ in range(6):
        L.step(0.001, periodic=True)
    out["pops6"] = L.get_pops()
    return out


def les_f16_8(O):
    """The FP16 form's Smagorinsky collision (cteS = 0.17) from the seeded
    random velocity of hit_f16_8, scale 2^16, 8^3, 5 steps, svisc 1e-4."""
    rng = np.random.default_rng(11)
    u, v, w = (rng.uniform(-0.03, 0.03, 512) for _ in range(3))
    L = O.OracleLattice(8, 8, 8, form="f16", scale=2.0**16)
    L.init_velocity(u, v, w, 1.0)
    L.set_les(0.17)
    out = {"pops0": L.get_pops()}
    for _ in range(5):
        L.step(1e-4, periodic=True)
    out["pops5"] = L.get_pops()
    return out


CASES = {"tgv_f64_5x7x9": tgv_f64_5x7x9, "tgv_f32_6x5x4": tgv_f32_6x5x4, "hit_f16_8": hit_f16_8,
         "les_tgv_f64_6x5x4": les_tgv_f64_6x5x4, "les_f16_8": les_f16_8}


def main(names=None):
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle import oracle as O

    for name, fn in CASES.items():
        if names and name not in names:
            continue
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **fn(O))
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1:])
