"""The eikods2d drop-in against the reference binary (oracle/_ref/eikods2d,
built from its source) on bad inputs: the same exit code and ERROR text (the
reference's log lines also carry a process id and a time stamp, which are not
compared).  Every case fails before any device work, so this runs without a
GPU."""
import os
import subprocess

import numpy as np
import pytest

import kirch_datuming_b200 as kd
from kirch_datuming_b200 import rsf

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "eikods2d")

pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="reference tool not built (make -C oracle ref)")

OUTS = ["out=time.rsf", "tdl1=tdl.rsf", "tds1=tds.rsf"]
CASES = {
    "no_out": ["in=vel.rsf"],
    "missing_velocity": ["in=nope.rsf", "shotfile=sht.rsf"] + OUTS,
    "shotfile_n1": ["in=vel.rsf", "shotfile=sht2.rsf"] + OUTS,
}
# The reference crashes (SIGSEGV) on these after its first log line; the
# drop-in reports the error its source intends (src/eikods2d.cpp:358-363).
OWN = {
    "no_tdl1": (["in=vel.rsf", "shotfile=sht.rsf", "out=time.rsf", "tds1=tds.rsf"], "Output derivative tdl1= missing."),
    "no_tds1": (["in=vel.rsf", "shotfile=sht.rsf", "out=time.rsf", "tdl1=tdl.rsf"], "Output derivative tds1= missing."),
}


def _error_text(stderr):
    lines = [ln for ln in stderr.splitlines() if "ERROR:" in ln]
    return lines[-1].split("ERROR:", 1)[1] if lines else None


def _files(wd):
    rsf.write(str(wd / "vel.rsf"), np.full((12, 10), 2.0, np.float32), [10, 12], [0.0, 0.0], [0.01, 0.01])
    rsf.write(str(wd / "sht.rsf"), np.array([[0.0, 0.05, 0.0]], np.float32), [3, 1])
    rsf.write(str(wd / "sht2.rsf"), np.array([[0.0, 0.05]], np.float32), [2, 1])


@pytest.mark.parametrize("name", sorted(OWN))
def test_error_where_the_reference_crashes(tmp_path, name):
    _files(tmp_path)
    args, msg = OWN[name]
    r = subprocess.run([kd.eikods_cli_path] + args, cwd=tmp_path, capture_output=True, text=True)
    assert (r.returncode, _error_text(r.stderr)) == (1, msg)


def test_usage_without_arguments(tmp_path):
    # both print their usage to stdout and exit 1 (the texts differ)
    for exe in (REF, kd.eikods_cli_path):
        r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True)
        assert r.returncode == 1 and "in=" in r.stdout and "out=" in r.stdout


@pytest.mark.parametrize("name", sorted(CASES))
def test_same_error_as_reference(tmp_path, name):
    _files(tmp_path)
    out = []
    for exe in (REF, kd.eikods_cli_path):
        r = subprocess.run([exe] + CASES[name], cwd=tmp_path, capture_output=True, text=True)
        out.append((r.returncode, _error_text(r.stderr)))
    assert out[0][0] != 0 and out[0][1]
    assert out[1] == out[0]
