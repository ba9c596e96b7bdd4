"""greensol_auto and kirchdat2d_freq drop-ins against the reference tools on
the CPU: failing runs give the reference's exit status and ERROR text (every
such case fails before any device work), and greensol_auto, whose work is a
gather of table samples, writes the reference's output bit for bit with the
same header."""
import json
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from kirch_datuming_b200 import rsf

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BIN = os.path.join(ROOT, "kirch_datuming_b200", "bin")
GOLD = np.load(os.path.join(HERE, "golden", "golden_datum.npz"))
with open(os.path.join(HERE, "golden", "cases.json")) as f:
    META = json.load(f)["datum"]


def _errors(stderr):
    return [l.split("ERROR:", 1)[1] for l in stderr.splitlines() if "ERROR:" in l]


def _infos(stderr):
    return [l.split("INFO:", 1)[1] for l in stderr.splitlines() if "INFO:" in l]


def _body(header):
    """header lines after the history line, but the data file's name"""
    return [l for l in header.splitlines()[2:] if l.strip() and not l.strip().startswith("in=")]


@pytest.fixture(scope="module")
def workdir():
    wd = tempfile.mkdtemp()
    t = META["table"]
    v = GOLD["vel"]
    nz, nx, d = META["nz"], META["nx"], META["d"]
    rsf.write(f"{wd}/vel.rsf", v, [nz, nx], [0, 0], [d, d], extra={"should_datum": str(META["should_datum"])})
    rsf.write(f"{wd}/vel_nodatum.rsf", v, [nz, nx], [0, 0], [d, d])
    rsf.write(f"{wd}/vel_deep.rsf", v, [nz, nx], [0, 0], [d, d], extra={"should_datum": "60"})
    rsf.write(f"{wd}/time.rsf", GOLD["table"], t["n"], t["o"], t["d"])
    g = GOLD["green"]
    rsf.write(f"{wd}/green.rsf", g, [g.shape[0], g.shape[1]], [t["o"][2], t["o"][2]], [t["d"][2], t["d"][2]])
    for name, dd in META["data"].items():
        x = GOLD["data_" + name]
        rsf.write(f"{wd}/d_{name}.rsf", x, [META["nt"], dd["nh"], dd["ns"]], [0, dd["h0"], dd["s0"]],
                  [META["dt"], dd["dh"], dd["ds"]])
    rsf.write(f"{wd}/d_wide.rsf", np.zeros((4, 8, META["nt"]), np.float32), [META["nt"], 8, 4], [0, 0.7, 0.2],
              [META["dt"], 0.02, 0.02])
    rsf.write(f"{wd}/d_2d.rsf", np.zeros((8, META["nt"]), np.float32), [META["nt"], 8], [0, 0.1], [META["dt"], 0.02])
    yield wd
    shutil.rmtree(wd)


def _run(tool, args, wd):
    return subprocess.run([os.path.join(BIN, tool)] + args, cwd=wd, capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("case", sorted(META["errors"]))
def test_kirchdat2d_freq_errors(case, workdir):
    want = META["errors"][case]
    r = _run("kirchdat2d_freq", want["args"], workdir)
    assert r.returncode == want["returncode"], r.stderr
    assert _errors(r.stderr) == want["error"]


@pytest.mark.parametrize("case", sorted(META["green_errors"]))
def test_greensol_auto_errors(case, workdir):
    want = META["green_errors"][case]
    r = _run("greensol_auto", want["args"], workdir)
    assert r.returncode == want["returncode"], r.stderr
    assert _errors(r.stderr) == want["error"]


def test_greensol_auto_output(workdir):
    r = _run("greensol_auto", ["ttabel_file=time.rsf", "tgreen_file=g_out.rsf", "model_file=vel.rsf"], workdir)
    assert r.returncode == 0, r.stderr
    assert _infos(r.stderr) == META["green_info"]
    h, g = rsf.read(os.path.join(workdir, "g_out.rsf"), count=GOLD["green"].size)
    assert np.array_equal(g.reshape(GOLD["green"].shape), GOLD["green"])
    with open(os.path.join(workdir, "g_out.rsf")) as f:
        assert _body(f.read()) == _body(META["green_header"])


def test_greensol_auto_xdr_table(workdir):
    """an xdr (big-endian) table gives the same slice"""
    t = META["table"]
    hdr = os.path.join(workdir, "time_xdr.rsf")
    GOLD["table"].astype(">f4").tofile(hdr + "@")
    with open(hdr, "w") as f:
        f.write('in="time_xdr.rsf@"\ndata_format="xdr_float"\nesize=4\n' +
                "".join("n%d=%d\no%d=%r\nd%d=%r\n" % (i + 1, t["n"][i], i + 1, t["o"][i], i + 1, t["d"][i])
                        for i in range(3)))
    r = _run("greensol_auto", ["ttabel_file=time_xdr.rsf", "tgreen_file=g_xdr.rsf", "model_file=vel.rsf"], workdir)
    assert r.returncode == 0, r.stderr
    _, g = rsf.read(os.path.join(workdir, "g_xdr.rsf"), count=GOLD["green"].size)
    assert np.array_equal(g.reshape(GOLD["green"].shape), GOLD["green"])
