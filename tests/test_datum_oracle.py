"""The datuming oracle (oracle/datum.py) against the reference tools' own
outputs (tests/golden/golden_datum.npz, made by tests/golden/make_golden.py
--datum from oracle/_ref/{greensol_auto,kirchdat2d_freq}), on the CPU.

greensol_auto is a gather: bit for bit.  kirchdat2d_freq computes in FP32
(the reference) against FP64 (the oracle): within 3e-5 relL2 on every case,
the butterfly cases included (at these sizes the butterfly's leaf stage is
exact)."""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import datum as D  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "golden_datum.npz"))
with open(os.path.join(HERE, "golden", "cases.json")) as f:
    META = json.load(f)["datum"]

f32 = np.float32


def rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def kw_of(args):
    kv = dict(a.split("=", 1) for a in args)
    out = dict(aperture=int(kv.get("aperture", 50)), taper=int(kv.get("taper", 10)),
               data_taper=int(kv.get("data_taper", 0)), cmp=int(kv.get("cmp", 1)),
               antialias=float(kv.get("antialias", 1.0)), length=float(kv.get("length", 0.025)))
    if kv.get("auto_datum", "1") == "0":
        sd, rd = f32(float(kv["sdatum"])), f32(float(kv["rdatum"]))
    else:
        sd = rd = f32(0.0 + META["should_datum"] * META["d"])
    return out, sd, rd


def make(case):
    c = META["cases"][case]
    d = META["data"][c["data"]]
    t = META["table"]
    kw, sd, rd = kw_of(c["args"])
    G = GOLD["green"]
    return D.Datum(META["nt"], d["nh"], d["ns"], META["dt"], d["h0"], d["dh"], d["s0"], d["ds"], G, t["o"][2],
                   t["d"][2], G, t["o"][2], t["d"][2], sd, rd, **kw), GOLD["data_" + c["data"]]


def test_greensol_bit_exact():
    t = META["table"]
    nz, nx, ngx = t["n"]
    datum = f32(0.0 + META["should_datum"] * META["d"])
    g = D.greensol(GOLD["table"], nz, nx, t["o"][0], t["o"][1], t["d"][0], t["d"][1], ngx, t["o"][2], t["d"][2],
                   datum)
    assert np.array_equal(g, GOLD["green"])


def test_greensol_errors():
    t = META["table"]
    nz, nx, ngx = t["n"]
    with pytest.raises(ValueError, match="Datum out of range."):
        D.greensol(GOLD["table"], nz, nx, t["o"][0], t["o"][1], t["d"][0], t["d"][1], ngx, t["o"][2], t["d"][2],
                   f32(0.6))


@pytest.mark.parametrize("case", sorted(META["cases"]))
def test_kirchdat2d_freq_vs_reference(case):
    o, data = make(case)
    want_interm = META["cases"][case]["interm"]
    got = o.run(data, interm=want_interm)
    out, im = (got if want_interm else (got, None))
    assert rel(out, GOLD["out_" + case]) < 3e-5
    if want_interm:
        assert rel(im, GOLD["interm_" + case]) < 3e-5


def test_nfft_and_nsam():
    o, _ = make("cmp0")
    # max tau 0.36 s = 90 samples: 128 + 90 + 12 + 2 -> 256
    assert o.nsam == 14 and o.nfft == 256 and o.nw == 129
    # length / dt in float32: 0.025 / 0.004 = 6.25 -> 6 + 2
    assert D.nsam_of(0.025, 0.004) == 8


def test_filter_matches_direct_sum():
    """H(tau, w) of the oracle (exact phase reduction) against the textbook
    double sum of the reference's unfactorised form (:130-139)."""
    dt, nsam, nfft = 0.004, 14, 512
    tau = np.array([0.0331, 0.21, 0.5123])
    iw = np.array([0, 1, 7, 100, 256])
    H = D.filter_H(tau, dt, nsam, nfft, iw)
    F = D.filter_F(tau, dt, nsam) / dt
    for a, t in enumerate(tau):
        q = t / dt
        m = np.ceil(q)
        delta = m - q
        for b, w in enumerate(iw):
            om = 2 * np.pi * w / nfft
            ref = sum(F[a, k] * ((1 - delta) * np.exp(-1j * om * (m + k)) + delta * np.exp(-1j * om * (m + k - 1)))
                      for k in range(nsam - 1))
            assert abs(H[a, b] - ref) <= 1e-12 * max(1.0, abs(ref))


def test_linearity_and_zero():
    o, data = make("cmp1")
    x = data.astype(np.float64)
    y = np.random.default_rng(3).standard_normal(x.shape)
    a = o.run(x)
    b = o.run(y)
    c = o.run(2.0 * x - 0.5 * y)
    assert rel(c, 2.0 * a - 0.5 * b) < 1e-12
    assert not np.any(o.run(np.zeros_like(x)))
