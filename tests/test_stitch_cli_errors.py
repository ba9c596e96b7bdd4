"""layercom_cig drop-in against the reference tool (oracle/_ref/layercom_cig,
built from its source) on malformed inputs: exit code, INFO lines and ERROR
text must be the same.  Every case fails before any device work, so this runs
without a GPU."""
import os
import subprocess

import numpy as np
import pytest

from test_stitch_oracle import CLI, COMMON, META, _inputs

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "layercom_cig")

pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="reference tool not built (make -C oracle ref)")


def _layers(text):
    def setup(wd):
        with open(os.path.join(wd, "layers.txt"), "w", encoding="utf-8") as f:
            f.write(text)
    return setup


def _model_header(text):
    def setup(wd):
        with open(os.path.join(wd, "model.rsf"), "w") as f:
            f.write(text)
    return setup


def _first_window_n2(wd):
    from kirch_datuming_b200 import rsf
    m, a = META["model"], META["angles"]
    rsf.write(os.path.join(wd, "adcig_1.rsf"), np.zeros((a["n"], 20, 26), np.float32), [26, 20, a["n"]],
              [0.0, m["o"][1], a["o"]], [m["d"][0], m["d"][1], a["d"]])


CASES = {
    "first_not_zero": (_layers("5,25\n18,45\n40,END\n"), []),
    "no_overlap": (_layers("START,25\n30,45\n40,END\n"), []),
    "not_deeper": (_layers("START,25\n18,20\n40,END\n"), []),
    "last_not_end": (_layers("START,25\n18,45\n"), []),
    "needs_two": (_layers("START\n"), []),
    "bad_start": (_layers("abc,25\n"), []),
    "bad_end": (_layers("START,xyz\n"), []),
    "bad_datum": (_layers("START,25,q\n18,45\n40,END\n"), []),
    "empty_layers": (_layers("# nothing\n\n"), []),
    "range": (_layers("START,70\n"), []),
    "no_layer_file": (None, ["layer_txt=nope.txt"]),
    "no_model": (None, ["full_model=none.rsf"]),
    "model_no_n1": (_model_header('in="model.rsf@"\nn2=24\n'), []),
    "model_format": (_model_header('in="model.rsf@"\nn1=60\nn2=24\ndata_format="xdr_float"\n'), []),
    "model_bad_int": (_model_header('in="model.rsf@"\nn1=6o\nn2=24\n'), []),
    "model_no_in": (_model_header("n1=60\nn2=24\n"), []),
    "lateral_size": (_first_window_n2, []),
    "int_arg": (None, ["nlayers=3x"]),
    "real_arg": (None, ["scalex_scale=nan"]),
    "scale_value": (None, ["scale=1,abc,2"]),
    "nangle": (None, ["nangle=5"]),
    "aper": (None, ["scalex_aper=-1"]),
    "positional": (None, ["=3"]),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_same_failure_as_reference(tmp_path, name):
    setup, extra = CASES[name]
    results = []
    for tag, exe in (("ref", REF), ("kcig", CLI)):
        wd = tmp_path / tag
        wd.mkdir()
        _inputs(str(wd))
        if setup:
            setup(str(wd))
        r = subprocess.run([exe] + COMMON + extra, cwd=wd, capture_output=True, text=True)
        results.append((r.returncode, r.stdout, r.stderr, (wd / "out.rsf").exists()))
    ref, got = results
    assert ref[0] != 0 and ref[2].startswith("ERROR: ")
    assert got == ref
