"""CPU tests of the C-ABI library (no GPU needed): it loads, exports every
entry point of include/bgk3d.h with the declared struct layouts, validates
parameters before touching a device, and the host helpers behave."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bgk3d.h")


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(bgk_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(bgk):
    lib = bgk.load()
    names = header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", bgk._abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (bgk_\w+)", out))
    assert set(names) <= exported
    # the ctypes prototypes cover exactly the header
    assert sorted(n for n, _, _ in bgk._abi.PROTOTYPES) == names


def test_struct_layout_matches_header(bgk, tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stddef.h>\n#include <stdio.h>\n#include "bgk3d.h"\n'
        "#define P(T, f) printf(\"%s.%s %zu\\n\", #T, #f, offsetof(T, f));\n"
        "int main(void) {\n"
        'printf("bgk_params %zu\\nbgk_diag %zu\\n", sizeof(bgk_params), sizeof(bgk_diag));\n'
        + "".join(f"P(bgk_params, {f})\n" for f, _ in bgk._abi.BgkParams._fields_)
        + "".join(f"P(bgk_diag, {f})\n" for f, _ in bgk._abi.BgkDiag._fields_)
        + "return 0; }\n")
    exe = tmp_path / "layout"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    lines = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    assert int(lines["bgk_params"]) == C.sizeof(bgk._abi.BgkParams)
    assert int(lines["bgk_diag"]) == C.sizeof(bgk._abi.BgkDiag)
    for T, S in (("bgk_params", bgk._abi.BgkParams), ("bgk_diag", bgk._abi.BgkDiag)):
        for f, _ in S._fields_:
            assert int(lines[f"{T}.{f}"]) == getattr(S, f).offset, (T, f)


def _params(bgk, **kw):
    p = bgk._abi.BgkParams()
    assert bgk.load().bgk_params_default(C.byref(p)) == 0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def test_defaults(bgk):
    p = _params(bgk)
    assert (p.lx, p.ly, p.lz, p.precision, p.scheme, p.icheck, p.mode) == (64, 64, 64, 0, 0, 10, 0)
    assert p.svisc == 0.01 and p.u0 == 0.05 and p.extras == 1


@pytest.mark.parametrize("bad", [
    dict(lx=0), dict(lz=-3), dict(precision=7), dict(scheme=2), dict(mode=5), dict(icheck=0),
    dict(svisc=0.0), dict(svisc=-1.0), dict(svisc=float("nan")), dict(use_omega=1, omega=2.5),
    dict(fp16_scale=3.0), dict(fp16_scale=-2.0), dict(u0=float("inf")), dict(lx=4096, ly=4096, lz=4096),
    dict(kernel=3), dict(kernel=-1), dict(kernel=16),
    dict(les_cs=-0.1), dict(les_cs=float("nan")), dict(les_cs=11.0),
    dict(proc_z=0), dict(proc_z=2, coord_z=2), dict(proc_z=2, coord_z=-1), dict(proc_z=3),
    dict(proc_z=2, scheme=1), dict(proc_z=2, mode=1), dict(proc_z=2, precision=2),
])
def test_create_rejects_bad_parameters_before_touching_a_device(bgk, bad):
    lib = bgk.load()
    h = C.c_void_p()
    rc = lib.bgk_create(C.byref(_params(bgk, **bad)), C.byref(h))
    assert rc == bgk._abi.BGK_ERR_INVALID
    assert not h.value
    assert lib.bgk_last_error()


def test_null_arguments(bgk):
    lib = bgk.load()
    assert lib.bgk_create(None, None) == bgk._abi.BGK_ERR_INVALID
    assert lib.bgk_col_mc(None, 1) == bgk._abi.BGK_ERR_INVALID
    assert lib.bgk_boundaries(None, 1) == bgk._abi.BGK_ERR_INVALID
    assert lib.bgk_diagnostic(None, 1, None) == bgk._abi.BGK_ERR_INVALID
    assert lib.bgk_destroy(None) == 0
    assert lib.bgk_get_stream(None) is None
    assert lib.bgk_shift3(None, None, None, None, None, None, 1, 1, 1, 8, 0, None) == bgk._abi.BGK_ERR_INVALID


def test_strerror_and_version(bgk):
    lib = bgk.load()
    assert b"sm_100a" in lib.bgk_version()
    for code in (0, 1, -1, -2, -3, -4, -5):
        assert lib.bgk_strerror(code) != b"unknown error"


def test_namelist_reader(tmp_path):
    from bgk3d_hit_b200 import read_namelist

    f = tmp_path / "bgk.input"
    f.write_text("&parameters\nlx = 48\nly = 40\nlz = 32\nproc_x = 1\nproc_y = 1\nproc_z = 1\n"
                 "u0 = 0.05\nsvisc = 1.0d-2\nitfin = 500\nicheck = 10 /\n")
    nl = read_namelist(str(f))
    assert (nl["lx"], nl["ly"], nl["lz"], nl["itfin"], nl["icheck"]) == (48, 40, 32, 500, 10)
    assert nl["svisc"] == 0.01 and nl["u0"] == 0.05


def test_hit_generator_properties():
    from bgk3d_hit_b200.hit import divergence_spectral, hit_velocity

    u, v, w = hit_velocity(32, k0=4, u_rms=0.03, seed=1234)
    assert u.shape == (32, 32, 32)
    assert np.sqrt((u * u + v * v + w * w).mean() / 3) == pytest.approx(0.03, rel=1e-12)
    assert divergence_spectral(u, v, w) < 1e-14
    u2, _, _ = hit_velocity(32, k0=4, u_rms=0.03, seed=1234)
    assert np.array_equal(u, u2)
    u3, _, _ = hit_velocity(32, k0=4, u_rms=0.03, seed=1235)
    assert not np.array_equal(u, u3)
    # shell spectrum peaks near k0 (E ~ k^4 exp(-2 (k/k0)^2) peaks at k0)
    k = np.sqrt(sum(g ** 2 for g in np.meshgrid(*[np.fft.fftfreq(32, 1 / 32)] * 3, indexing="ij")))
    e = sum(np.abs(np.fft.fftn(a)) ** 2 for a in (u, v, w))
    shells = np.bincount(np.rint(k).astype(int).ravel(), e.ravel())
    assert abs(int(np.argmax(shells)) - 4) <= 1


def test_fortran_e14_6_format():
    """diagno.dat / dissipation.dat numbers are written as Fortran E14.6."""
    from bgk3d_hit_b200.solver import fortran_e

    assert fortran_e(0.0123456) == "  0.123456E-01"
    assert fortran_e(-1.5) == " -0.150000E+01"
    assert fortran_e(1.0) == "  0.100000E+01"
    assert fortran_e(0.0) == "  0.000000E+00"
    assert fortran_e(0.0099999996) == "  0.100000E-01"
    assert fortran_e(123456789.0) == "  0.123457E+09"
    assert fortran_e(float("nan")).strip() == "NaN"
    assert all(len(fortran_e(x)) == 14 for x in (1e-30, -3.3e7, 2.5))


def test_driver_builds_and_rejects_bad_input(tmp_path):
    """The C++ program driver (the reference's main loop over the C-ABI)
    builds with g++ and reports a missing or inconsistent namelist before it
    touches a device."""
    import subprocess

    from bgk3d_hit_b200 import build as B

    exe = B.build_driver()
    r = subprocess.run([exe, str(tmp_path / "missing.input")], capture_output=True, text=True)
    assert r.returncode == 2 and "cannot open" in r.stderr
    nl = tmp_path / "bgk.input"
    nl.write_text("&parameters\nlx = 16\nproc_z = 2 /\n")
    r = subprocess.run([exe, str(nl)], capture_output=True, text=True)
    assert r.returncode == 2 and "one box per process" in r.stderr
    r = subprocess.run([exe, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "usage" in r.stdout


def test_bench_reference_arm_line_on_cpu():
    """bench.py --impl reference times the oracle's restatement of the
    reference on the host and prints one JSON line with the contract's keys
    (it needs no GPU)."""
    import json
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--size", "16",
                        "--steps", "3", "--warmup", "1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "GLUPS" and line["value"] > 0
    for k in ("metric", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]


def test_bench_kernel_names_and_shared_config():
    """The bench names the stream-collide kernel each run launches (the key of
    its ncu traffic table) and both arms print the same config dict."""
    import argparse
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    assert bench.kernel_key("fp64", "two_lattice", 256) == "k_two_fp64"
    assert bench.kernel_key("fp16", "two_lattice", 256) == "k_two_f16v"
    assert bench.kernel_key("fp16", "two_lattice", 256, kernel=2) == "k_two_f16v2"
    assert bench.kernel_key("fp16", "aa", 1024) == "k_aa_f16w"  # odd step on eight cells per thread
    assert bench.kernel_key("fp16", "aa", 1024, kernel=4) == "k_aa_f16v"
    assert bench.kernel_key("fp16", "aa", 12) == "k_aa_fp16"  # neither 8 nor 4 cells fit a row of 12
    assert bench.kernel_key("fp16", "two_lattice", 256, les=True) == "k_two_f16v_les"
    assert bench.kernel_key("fp16", "aa", 256, les=True) == "k_aa_f16v_les"
    assert bench.kernel_key("fp16", "two_lattice", 256, kernel=1) == "k_two_fp16"
    assert bench.kernel_key("fp16", "two_lattice", 6) == "k_two_fp16"  # rows too short for four cells per thread
    assert bench.kernel_key("fp32", "two_lattice", 256) == "k_two_f32v"
    assert bench.kernel_key("fp32", "aa", 1024) == "k_aa_f32w"  # odd step on four cells per thread
    assert bench.kernel_key("fp32", "aa", 1024, kernel=2) == "k_aa_f32v"
    assert bench.kernel_key("fp32", "aa", 256, les=True) == "k_aa_f32w_les"
    assert bench.kernel_key("fp32", "aa", 256, kernel=2, les=True) == "k_aa_f32v_les"
    assert bench.kernel_key("fp32", "aa", 256, kernel=1) == "k_aa_fp32"
    assert bench.kernel_key("fp32", "two_lattice", 24) == "k_two_fp32"  # 12 threads per row: not a power of two
    a = argparse.Namespace(size=256, precision="fp64", scheme="two_lattice", tau=0.505, k0=4.0, kernel=0, les_cs=0.0,
                           decomp="replicas", local_slabs=2)
    c1 = bench.config_of(a, 1)
    assert c1["box"] == 256 and c1["cells_per_gpu"] == 256 ** 3 and "replica" in c1["parallelism"]
    a.decomp = "slabs"
    c4 = bench.config_of(a, 4)
    assert c4["box"] == [256, 256, 1024] and c4["slabs"] == 4


def test_header_constants_match_the_binding(bgk):
    txt = open(HEADER).read()
    defs = {k: int(v) for k, v in re.findall(r"#define (BGK_\w+) \(?(-?\d+)\)?", txt)}
    assert len(defs) >= 15
    for k, v in defs.items():
        assert getattr(bgk._abi, k) == v, k


def test_adjoint_rebuild_rule(bgk):
    """BGK_ADJ_REBUILD applies while A = |1 - omega|^-(K-1) <= 64 and, in the
    FP32 form, K * A <= 160: host-only query."""
    lib = bgk.load()
    F64, F32, F16 = bgk._abi.BGK_FP64, bgk._abi.BGK_FP32DEV, bgk._abi.BGK_FP16DEV
    for f in (F64, F32):
        assert lib.bgk_adjoint_rebuilds(f, 1.0 / 0.51, 32) == 1  # A = 1.041^31 = 3.5, K A = 111
        assert lib.bgk_adjoint_rebuilds(f, 1.0 / 0.6, 32) == 0  # A = 1.5^31
        assert lib.bgk_adjoint_rebuilds(f, 1.0 / 0.6, 8) == 1  # A = 1.5^7 = 17, K A = 137
        assert lib.bgk_adjoint_rebuilds(f, 1.0, 2) == 0  # omega = 1: the collision forgets g
        assert lib.bgk_adjoint_rebuilds(f, 1.25, 1) == 1  # one step per segment: nothing rebuilt twice
        assert lib.bgk_adjoint_rebuilds(f, 1.9, 0) == 0
    assert lib.bgk_adjoint_rebuilds(F64, 1.0 / 0.505, 200) == 1  # A = 1.02^199 = 52
    assert lib.bgk_adjoint_rebuilds(F64, 1.0 / 0.505, 250) == 0  # A = 145
    assert lib.bgk_adjoint_rebuilds(F32, 1.0 / 0.505, 200) == 0  # K A = 10400
    assert lib.bgk_adjoint_rebuilds(F32, 1.0 / 0.505, 60) == 0  # A = 3.3, K A = 195
    assert lib.bgk_adjoint_rebuilds(F32, 1.0 / 0.505, 50) == 1  # A = 2.7, K A = 133
    assert lib.bgk_adjoint_rebuilds(F16, 1.0 / 0.51, 32) == 0  # no adjoint in FP16
