"""The reference's own shipped run, end to end through the program driver.

RUN/bgk.input of the reference: Taylor-Green 180^3 on one rank, u0 = 0.1,
svisc = 0.0014317, icheck = isignal = 85, itsave = ivtim = 2812, run here for
itfin = 170 steps (two diagnostic records) with a restart written at the end.
The namelist is read as the reference ships it (proc_x/y/z and isignal
included). The C++ driver bgk3d_hit runs it in the reference's default
single-precision build (FP32) and its DOUBLE_P build (FP64), faithful mode
(TGV init with single-precision coordinates and pi, SRC/init.F90:42,84-95).
The oracle starts from the driver's initial populations (the same library
call, bgk_init_tgv, deterministic) and steps in its ghost-fill form: the loop
body boundaries (bcond_comm_step3, SRC/bcond.comm.step3.F90:77-297) + col_MC
on the ghosted lattice, SRC/bgk3d_HIT.F90:127-146. Checked:
- the populations in restart.00000170.bin equal the oracle's bit for bit;
- every number of diagno.dat (itime, xtot, ytot, ztot, rtot, stot;
  SRC/diagno.F90:137,152) and dissipation.dat (itime, t, tke_norm, diss;
  SRC/dissipation.F90:265-278, read after the pointer swap, so border cells
  pull stale ghosts as in the reference) equals the oracle's value to the
  printed precision of E14.6: within half a unit of the sixth digit, plus
  1e-15 absolute for the means that are zero up to rounding. The library
  sums in compensated FP64 in both modes, where the reference's diagno sums
  in the build's precision cell by cell (in single precision a 180^3 sum
  of rho loses digits); so the expected record is the oracle's compensated
  one, with faithful mode's ztot = ytot + zj (SRC/diagno.F90:110): the y
  mean plus the last cell's zj over the cell count.
"""
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAMELIST = """&parameters
lx = 180
ly = 180
lz = 180
proc_x = 1
proc_y = 1
proc_z = 1
u0     = 0.1
svisc  = 0.0014317
itfin  = 170
itsave = 170
isignal= 85
ivtim  = 2812
icheck = 85 /
"""


def _records(path):
    out = []
    for line in open(path).read().splitlines():
        it = int(line[:8])
        toks = re.findall(r"-?0\.\d{6}E[+-]\d\d", line[8:])
        out.append((it, toks))
    return out


def _zj_last(pops, precision):
    """zj of the box's last cell (i = l, j = m, k = n) in the storage form's
    arithmetic, summed in the reference's order (SRC/diagno.F90:100-104)."""
    t = np.float64 if precision == "fp64" else np.float32
    x = pops[:, -1, -1, -1].astype(t)
    rho = x[0]
    for q in range(1, 19):
        rho = t(rho + x[q])
    rho = t(rho + t(1))
    s = x[3]
    for q in (5, 6, 12, 17):
        s = t(s + x[q])
    for q in (1, 8, 10, 14, 15):
        s = t(s - x[q])
    return float(t(s * t(t(1) / rho)))


def _close(tok, ref):
    exp = int(tok[-3:])
    half_unit = 0.5 * 10.0 ** (exp - 6)
    return abs(float(tok) - ref) <= half_unit * (1 + 1e-9) + 1e-15


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_reference_run_configuration_through_the_driver(bgk, oracle_mod, tmp_path, precision):
    from bgk3d_hit_b200 import build as B

    exe = B.build_driver()
    nl = tmp_path / "bgk.input"
    nl.write_text(NAMELIST)
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([exe, str(nl), "--precision", precision, "--out", str(out)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    svisc, u0 = 0.0014317, 0.1
    box = bgk.BGK3D.from_input(str(nl), mode="faithful", precision=precision)
    orc = oracle_mod.OracleLattice(180, 180, 180, form={"fp32": "f32", "fp64": "f64"}[precision])
    try:
        box.init()
        orc.put_pops(box.populations())
        exp_diag, exp_diss = {}, {}
        for it in range(1, 171):
            orc.step(svisc)
            if it % 85 == 0:
                dg = orc.diagno(False)  # rho, ux, uy, uz, ke (compensated sums)
                dg[3] = dg[2] + _zj_last(orc.get_pops(), precision) / 180 ** 3
                exp_diag[it] = dg
                exp_diss[it] = orc.dissipation(svisc, u0, it, 2)  # t, tke_norm, diss, tke
        box.load(str(out / "restart.00000170.bin"))
        assert np.array_equal(box.populations().view(np.uint8), orc.get_pops().view(np.uint8))
    finally:
        orc.close()
        box.close()
    diag = _records(out / "diagno.dat")
    diss = _records(out / "dissipation.dat")
    assert [it for it, _ in diag] == [85, 170] and [it for it, _ in diss] == [85, 170]
    for it, toks in diag:
        rho, ux, uy, uz, ke = exp_diag[it]
        assert len(toks) == 5
        for tok, ref in zip(toks, (ux, uy, uz, rho, ke)):
            assert _close(tok, ref), (it, tok, ref)
    for it, toks in diss:
        t, tke_norm, dss = exp_diss[it][:3]
        assert len(toks) == 3
        for tok, ref in zip(toks, (t, tke_norm, dss)):
            assert _close(tok, ref), (it, tok, ref)
