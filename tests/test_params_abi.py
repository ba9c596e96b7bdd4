"""Host logic that needs no GPU: the C ABI loads and exports every declared
entry point, parameters parse with the reference's defaults, precedence and
error texts, the output axis resolves like parse_output_axis, and the CLI
rejects bad command lines before touching the device."""
import os
import re
import subprocess

import numpy as np
import pytest

import _cases
import kirch_datuming_b200 as kd
from kirch_datuming_b200 import rsf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "kcig.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(kcig_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 14
    out = subprocess.run(["nm", "-D", "--defined-only", kd.library_path], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (kcig_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    L = kd.lib()
    for n in names:
        assert getattr(L, n) is not None


def test_defaults_match_reference():
    p = kd.params()
    assert (p.adj, p.cig, p.cig_is_angle, p.cmp, p.half_angle, p.isdiff) == (1, 0, 0, 1, 0, 0)
    assert chr(p.interp_type) == "h"
    assert (p.angle_interp, p.angle_grad_radius, p.angle_smooth) == (1, 2, 2)
    assert (p.aperture_trace, p.aperture_trace_taper, p.direct_mute) == (-1, 20, 0)
    assert p.aperture == 90 and p.aperture_taper == 10 and p.aperture_rmin == 0
    assert p.aperture_rtaper == np.float32(0.05) and p.antialias == 1 and p.tau == 0
    assert (p.oazmin, p.oazmax, p.oaztaper) == (80, 50, 10)
    assert p.angle_taper_start == -1 and p.angle_taper_end == -1
    h = kd.params("half_angle=1")
    assert (h.oazmin, h.oazmax) == (40, 25)
    m = kd.params("mode=ANGLE")
    assert m.cig == 1 and m.cig_is_angle == 1


def test_precedence_and_par_file(tmp_path):
    f = tmp_path / "p.txt"
    f.write_text("angle_n=11 # comment\nangle_min=5\n")
    g = kd.geometry(nt=10, nh=3, ns=2, dt=0.01, dh=0.1, ds=0.1, nz=5, nx=5, dz=1, dx=1, sny=2, sdy=1, rny=2, rdy=1)
    ax = lambda *t: kd.output_axis(kd.params("mode=angle", *t), g)  # noqa: E731
    assert ax("angle_n=61", "angle_n=31") == (31, 0.0, 1.0)
    assert ax("angle_n=31.9") == (31, 0.0, 1.0)
    assert ax("par=%s" % f) == (11, 5.0, 1.0)
    assert ax("par=%s" % f, "angle_n=7") == (7, 5.0, 1.0)
    assert ax("angle_n=7", "par=%s" % f) == (11, 5.0, 1.0)
    assert ax('angle_n="21"')[0] == 21
    assert ax() == (181, 0.0, 1.0)
    assert kd.output_axis(kd.params("mode=angle", "half_angle=1"), g) == (91, 0.0, 1.0)
    assert kd.output_axis(kd.params("cig=0"), g) == (1, 0.0, 1.0)
    assert kd.output_axis(kd.params("mode=offset"), g) == (3, 0.0, pytest.approx(0.1))
    assert kd.params("aperture=abc").aperture == 0.0  # strtod semantics, as the reference


@pytest.mark.parametrize("tokens,msg", [
    (["mode=foo"], "Unknown CIG mode: foo. Supported modes are offset and angle."),
    (["direct_mute=1", "direct_mute_taper=0"], "direct_mute_taper must be finite and positive to avoid a hard cutoff."),
    (["direct_mute=1", "direct_mute_slope=-1"], "direct_mute_slope must be finite and non-negative."),
    (["direct_mute=1", "direct_mute_invert=2"], "direct_mute_invert must be 0 or 1."),
    (["direct_mute=1", "direct_mute_qc_shot=-2"],
     "direct_mute_qc_shot must be -1 (disabled) or a zero-based shot index."),
    (["type=cubic"], "Unknown interpolation type: cubic. Supported types are linear (l), partial (p), and hermite (h)"),
])
def test_param_errors(tokens, msg):
    with pytest.raises(kd.KcigError) as e:
        kd.params(*tokens)
    assert e.value.msg == msg
    assert e.value.code == -1


@pytest.mark.parametrize("case", _cases.Golden().cases)
def test_output_axis_matches_reference_log(golden, case):
    kp = kd.params(*golden.tokens(case))
    ng, g0, dg = kd.output_axis(kp, kd.geometry(**golden.geometry_dict(case)))
    info = golden.meta["cases"][case]["info"][0]
    m = re.search(r"n3 = (\d+), o3 = (\S+), d3 = (\S+)", info)
    assert ng == int(m.group(1))
    assert "%g" % g0 == m.group(2) and "%g" % dg == m.group(3)


def _cli(args, cwd):
    return subprocess.run([kd.cli_path] + args, cwd=cwd, capture_output=True, text=True)


def test_cli_errors_without_gpu(tmp_path):
    r = _cli(["migration=m.rsf"], tmp_path)
    assert r.returncode == 1 and "ERROR:Need seismic_data=" in r.stderr
    r = _cli(["seismic_data=d.rsf", "migration=m.rsf", "stable=t.rsf", "sderiv=t.rsf", "rtable=t.rsf"], tmp_path)
    assert r.returncode == 1 and "ERROR:Need rderiv=" in r.stderr
    r = _cli(["seismic_data=nope.rsf", "migration=m.rsf", "stable=t.rsf", "sderiv=t.rsf", "rtable=t.rsf",
              "rderiv=t.rsf"], tmp_path)
    assert r.returncode == 1 and "Cannot open SEP file '%s': current dir is %s, error code is 2 - " % (
        os.path.join(os.path.realpath(tmp_path), "nope.rsf"), os.path.realpath(tmp_path)) in r.stderr
    rsf.write(str(tmp_path / "d2.rsf"), np.zeros((4, 3), np.float32), [4, 3])
    r = _cli(["seismic_data=d2.rsf", "migration=m.rsf", "stable=t.rsf", "sderiv=t.rsf", "rtable=t.rsf",
              "rderiv=t.rsf"], tmp_path)
    assert r.returncode == 1 and "Need 3D data volume for seismic_data= (t,h/r,s)" in r.stderr
    rsf.write(str(tmp_path / "d.rsf"), np.zeros((2, 3, 4), np.float32), [4, 3, 2])
    rsf.write(str(tmp_path / "t.rsf"), np.zeros((2, 5, 5), np.float32), [5, 5, 2])
    rsf.write(str(tmp_path / "t3.rsf"), np.zeros((2, 5, 6), np.float32), [6, 5, 2])
    r = _cli(["seismic_data=d.rsf", "migration=m.rsf", "stable=t.rsf", "sderiv=t3.rsf", "rtable=t.rsf",
              "rderiv=t.rsf"], tmp_path)
    assert r.returncode == 1 and "Dimension mismatch between stable= and sderiv=" in r.stderr
    r = _cli(["seismic_data=d.rsf", "migration=m.rsf", "stable=t.rsf", "sderiv=t.rsf", "rtable=t.rsf",
              "rderiv=t.rsf", "mode=angle", "sgradx=t.rsf"], tmp_path)
    assert r.returncode == 1 and "please provide all of sgradx=" in r.stderr
    r = _cli(["seismic_data=d.rsf", "migration=m.rsf", "stable=t.rsf", "sderiv=t.rsf", "rtable=t.rsf",
              "rderiv=t.rsf", "direct_mute=1", "direct_mute_qc_shot=5"], tmp_path)
    assert r.returncode == 1 and "direct_mute_qc_shot=5 is outside the input shot range [0,1]." in r.stderr
    # truncated binary
    with open(tmp_path / "d.rsf@", "r+b") as f:
        f.truncate(16)
    r = _cli(["seismic_data=d.rsf", "migration=m.rsf", "stable=t.rsf", "sderiv=t.rsf", "rtable=t.rsf",
              "rderiv=t.rsf"], tmp_path)
    assert r.returncode == 1 and "truncated" in r.stderr


def test_rsf_roundtrip_xdr_and_native(tmp_path):
    a = np.arange(24, dtype=np.float32).reshape(2, 3, 4)
    rsf.write(str(tmp_path / "a.rsf"), a, [4, 3, 2], [0.5, 0, 1], [0.01, 2, 3], extra={"label1": "Time"})
    h, b = rsf.read(str(tmp_path / "a.rsf"))
    assert h.n[:3] == [4, 3, 2] and h.native and h.extra["label1"] == "Time"
    assert np.array_equal(b, a.ravel())
    # a big-endian (xdr) file without data_format is read as xdr
    (tmp_path / "x.rsf").write_text('n1=4 n2=6 in="x.rsf@" esize=4\n')
    a.astype(">f4").tofile(tmp_path / "x.rsf@")
    h, b = rsf.read(str(tmp_path / "x.rsf"))
    assert not h.native and np.array_equal(b, a.ravel())
    assert rsf.format_double(np.float32(0.01)) == "0.009999999776"
    assert rsf.format_double(3.0) == "3"
