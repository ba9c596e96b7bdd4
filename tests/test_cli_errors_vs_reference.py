"""The kirchmig2d_cig drop-in against the reference binary (oracle/_ref/
kirchmig2d_cig, built from its source) on bad inputs: the same exit code and
the same ERROR text (the reference's log lines also carry a process id and a
time stamp, which are not compared).  Every case fails before any device
work, so this runs without a GPU."""
import os
import subprocess

import numpy as np
import pytest

import kirch_datuming_b200 as kd
from kirch_datuming_b200 import rsf

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "kirchmig2d_cig")

pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="reference tool not built (make -C oracle ref)")

BASE = ["seismic_data=d.rsf", "migration=m.rsf", "stable=t.rsf", "sderiv=t.rsf", "rtable=t.rsf", "rderiv=t.rsf"]
CASES = {
    "no_data": ["migration=m.rsf"],
    "no_rderiv": BASE[:5],
    "missing_file": ["seismic_data=nope.rsf"] + BASE[1:],
    "missing_file_subdir": ["seismic_data=./sub/../nope.rsf"] + BASE[1:],
    "data_2d": ["seismic_data=d2.rsf"] + BASE[1:],
    "sderiv_dims": BASE[:3] + ["sderiv=t3.rsf"] + BASE[4:],
    "mode": BASE + ["mode=foo"],
    "one_grad": BASE + ["mode=angle", "sgradx=t.rsf"],
    "qc_shot": BASE + ["direct_mute=1", "direct_mute_qc_shot=5"],
    "interp_type": BASE + ["type=cubic"],
    "mute_taper": BASE + ["direct_mute=1", "direct_mute_taper=0"],
    "mute_slope": BASE + ["direct_mute=1", "direct_mute_slope=-1"],
    "mute_invert": BASE + ["direct_mute=1", "direct_mute_invert=2"],
}


def _error_text(stderr):
    lines = [ln for ln in stderr.splitlines() if "ERROR:" in ln]
    return lines[-1].split("ERROR:", 1)[1] if lines else None


@pytest.mark.parametrize("name", sorted(CASES))
def test_same_error_as_reference(tmp_path, name):
    rsf.write(str(tmp_path / "d.rsf"), np.zeros((2, 3, 4), np.float32), [4, 3, 2])
    rsf.write(str(tmp_path / "d2.rsf"), np.zeros((4, 3), np.float32), [4, 3])
    rsf.write(str(tmp_path / "t.rsf"), np.zeros((2, 5, 5), np.float32), [5, 5, 2])
    rsf.write(str(tmp_path / "t3.rsf"), np.zeros((2, 5, 6), np.float32), [6, 5, 2])
    (tmp_path / "sub").mkdir()
    out = []
    for exe in (REF, kd.cli_path):
        r = subprocess.run([exe] + CASES[name], cwd=tmp_path, capture_output=True, text=True)
        out.append((r.returncode, _error_text(r.stderr)))
    assert out[0][0] != 0 and out[0][1]
    assert out[1] == out[0]


K2D_REF = os.path.join(os.path.dirname(REF), "kirchmig2d")
K2D_CASES = {k: CASES[k] for k in ("no_data", "no_rderiv", "missing_file", "data_2d")}
K2D_CASES["interp_type"] = BASE + ["type=cubic"]


@pytest.mark.skipif(not os.path.exists(K2D_REF), reason="reference kirchmig2d not built")
@pytest.mark.parametrize("name", sorted(K2D_CASES))
def test_kirchmig2d_same_error_as_reference(tmp_path, name):
    rsf.write(str(tmp_path / "d.rsf"), np.zeros((2, 3, 4), np.float32), [4, 3, 2])
    rsf.write(str(tmp_path / "d2.rsf"), np.zeros((4, 3), np.float32), [4, 3])
    rsf.write(str(tmp_path / "t.rsf"), np.zeros((2, 5, 5), np.float32), [5, 5, 2])
    out = []
    for exe in (K2D_REF, kd.kirchmig2d_cli_path):
        r = subprocess.run([exe] + K2D_CASES[name], cwd=tmp_path, capture_output=True, text=True)
        out.append((r.returncode, _error_text(r.stderr)))
    assert out[0][0] != 0 and out[0][1]
    assert out[1] == out[0]
