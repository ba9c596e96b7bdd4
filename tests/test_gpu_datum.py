"""Datuming on the GPU (kcig_datum_freq, kcig_green_slice, the drop-in
kirchdat2d_freq) against the FP64 oracle (oracle/datum.py) and the reference
tool's outputs (tests/golden/golden_datum.npz).

Tolerances (relative L2): 1e-5 against the FP64 oracle (FP32 spectra and
sums on the device, the filter H in FP64); 3e-5 against the reference's own
FP32 output, which is itself ~3e-6 from the FP64 oracle.  The butterfly
cases (use_bf=1) are exact at these sizes, so the same bound holds."""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest
import torch

import kirch_datuming_b200 as kd
from kirch_datuming_b200 import rsf

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)
import datum as D  # noqa: E402
from test_datum_oracle import GOLD, META, kw_of, rel  # noqa: E402

pytestmark = pytest.mark.gpu


def params_of(case):
    c = META["cases"][case]
    d = META["data"][c["data"]]
    t = META["table"]
    kw, sd, rd = kw_of(c["args"])
    kv = dict(a.split("=", 1) for a in c["args"])
    ng = GOLD["green"].shape[0]
    p = kd.datum_params(nt=META["nt"], nh=d["nh"], ns=d["ns"], dt=META["dt"], h0=d["h0"], dh=d["dh"], s0=d["s0"],
                        ds=d["ds"], nsg=ng, nrg=ng, sg0=t["o"][2], dsg=t["d"][2], rg0=t["o"][2], drg=t["d"][2],
                        sdatum=float(sd), rdatum=float(rd), **kw)
    p.use_bf = int(kv.get("use_bf", 1))
    return p, GOLD["data_" + c["data"]], c


def oracle_of(case):
    c = META["cases"][case]
    d = META["data"][c["data"]]
    t = META["table"]
    kw, sd, rd = kw_of(c["args"])
    G = GOLD["green"]
    return D.Datum(META["nt"], d["nh"], d["ns"], META["dt"], d["h0"], d["dh"], d["s0"], d["ds"], G, t["o"][2],
                   t["d"][2], G, t["o"][2], t["d"][2], sd, rd, **kw)


@pytest.mark.parametrize("case", sorted(META["cases"]))
def test_datum_freq_host_memory(case):
    p, data, c = params_of(case)
    G = np.ascontiguousarray(GOLD["green"])
    out = np.empty_like(data)
    im = np.empty_like(data) if c["interm"] else None
    kd.datum_freq(p, G, G, np.ascontiguousarray(data), out, im)
    o = oracle_of(case)
    want = o.run(data, interm=c["interm"])
    ref_out, ref_im = (want if c["interm"] else (want, None))
    assert rel(out, ref_out) < 1e-5, rel(out, ref_out)
    assert rel(out, GOLD["out_" + case]) < 3e-5
    if c["interm"]:
        assert rel(im, ref_im) < 1e-5
        assert rel(im, GOLD["interm_" + case]) < 3e-5


@pytest.mark.parametrize("case", ["cmp0", "cmp1_jump"])
def test_datum_freq_device_memory_equals_host(case):
    p, data, c = params_of(case)
    G = np.ascontiguousarray(GOLD["green"])
    out_h = np.empty_like(data)
    kd.datum_freq(p, G, G, np.ascontiguousarray(data), out_h)
    Gd = torch.from_numpy(G).cuda()
    dd = torch.from_numpy(np.ascontiguousarray(data)).cuda()
    out_d = torch.empty_like(dd)
    kd.datum_freq(p, Gd, Gd, dd, out_d)
    torch.cuda.synchronize()
    assert np.array_equal(out_d.cpu().numpy(), out_h)
    ms, launches = kd.datum_last_timing()
    assert launches > 0 and all(m >= 0 for m in ms)


def test_datum_linearity_and_zero():
    p, data, _ = params_of("cmp1")
    G = np.ascontiguousarray(GOLD["green"])
    x = np.ascontiguousarray(data)
    y = np.ascontiguousarray(np.random.default_rng(4).standard_normal(x.shape).astype(np.float32))
    z = np.ascontiguousarray((2.0 * x - 0.5 * y).astype(np.float32))
    outs = []
    for v in (x, y, z):
        o = np.empty_like(v)
        kd.datum_freq(p, G, G, v, o)
        outs.append(o.astype(np.float64))
    assert rel(outs[2], 2.0 * outs[0] - 0.5 * outs[1]) < 1e-5
    zero = np.zeros_like(x)
    o = np.empty_like(x)
    kd.datum_freq(p, G, G, zero, o)
    assert not np.any(o)


def test_datum_larger_survey_vs_oracle():
    """40 shots x 70 fixed receivers (cmp=0, the aperture covering the whole
    spread, the workflow's settings) on the salt fixture's tables, shots off
    the table grid."""
    t = META["table"]
    G = np.ascontiguousarray(GOLD["green"])
    ns, nh, nt, dt = 40, 70, 128, 0.004
    x = np.random.default_rng(9).standard_normal((ns, nh, nt)).astype(np.float32)
    p = kd.datum_params(nt=nt, nh=nh, ns=ns, dt=dt, h0=0.05, dh=0.01, s0=0.1, ds=0.015, nsg=G.shape[0],
                        nrg=G.shape[0], sg0=t["o"][2], dsg=t["d"][2], rg0=t["o"][2], drg=t["d"][2], sdatum=0.1,
                        rdatum=0.1, aperture=200, taper=0, data_taper=20, cmp=0, antialias=1.0, length=0.05)
    out = np.empty_like(x)
    kd.datum_freq(p, G, G, x, out)
    o = D.Datum(nt, nh, ns, dt, 0.05, 0.01, 0.1, 0.015, G, t["o"][2], t["d"][2], G, t["o"][2], t["d"][2],
                np.float32(0.1), np.float32(0.1), aperture=200, taper=0, data_taper=20, cmp=0, antialias=1.0,
                length=0.05)
    assert rel(out, o.run(x)) < 1e-5


def test_datum_receiver_table_too_small():
    p, data, _ = params_of("cmp0")
    p.h0 = 0.7  # receivers past the table's last position
    G = np.ascontiguousarray(GOLD["green"])
    with pytest.raises(kd.KcigError, match="Receiver table too small."):
        kd.datum_freq(p, G, G, np.ascontiguousarray(data), np.empty_like(data))


def test_green_slice_device():
    t = META["table"]
    nz, nx, ngx = t["n"]
    table = torch.from_numpy(np.ascontiguousarray(GOLD["table"])).cuda()
    out = torch.empty((ngx, ngx), dtype=torch.float32, device="cuda")
    datum = float(np.float32(0.0 + META["should_datum"] * META["d"]))
    kd.green_slice(table, nz, nx, ngx, t["o"][0], t["o"][1], t["d"][0], t["d"][1], t["o"][2], t["d"][2], datum, out)
    assert np.array_equal(out.cpu().numpy(), GOLD["green"])


@pytest.mark.parametrize("case", ["cmp0", "cmp1", "defaults"])
def test_kirchdat2d_freq_cli(case):
    c = META["cases"][case]
    d = META["data"][c["data"]]
    t = META["table"]
    with tempfile.TemporaryDirectory() as wd:
        nz, nx, dz = META["nz"], META["nx"], META["d"]
        rsf.write(f"{wd}/vel.rsf", GOLD["vel"], [nz, nx], [0, 0], [dz, dz],
                  extra={"should_datum": str(META["should_datum"])})
        G = GOLD["green"]
        rsf.write(f"{wd}/green.rsf", G, [G.shape[0], G.shape[1]], [t["o"][2], t["o"][2]], [t["d"][2], t["d"][2]])
        rsf.write(f"{wd}/d.rsf", GOLD["data_" + c["data"]], [META["nt"], d["nh"], d["ns"]], [0, d["h0"], d["s0"]],
                  [META["dt"], d["dh"], d["ds"]])
        args = ["input_file=d.rsf", "output_file=out.rsf", "sgreen_file=green.rsf", "rgreen_file=green.rsf",
                "model_file=vel.rsf"] + c["args"] + (["interm=interm.rsf"] if c["interm"] else [])
        r = subprocess.run([os.path.join(ROOT, "kirch_datuming_b200", "bin", "kirchdat2d_freq")] + args, cwd=wd,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        infos = [l.split("INFO:", 1)[1] for l in r.stderr.splitlines() if "INFO:" in l and "Elapsed" not in l]
        assert infos == c["info"]
        _, o = rsf.read(f"{wd}/out.rsf")
        assert rel(o, GOLD["out_" + case]) < 3e-5
        body = lambda h: [l for l in h.splitlines()[2:] if l.strip() and not l.strip().startswith("in=")]
        with open(f"{wd}/out.rsf") as f:
            assert body(f.read()) == body(c["header"])
        if c["interm"]:
            _, im = rsf.read(f"{wd}/interm.rsf", count=o.size)
            assert rel(im, GOLD["interm_" + case]) < 3e-5
            with open(f"{wd}/interm.rsf") as f:
                assert body(f.read()) == body(c["interm_header"])


def _survey(ns, nh, aperture, seed, cmp=0):
    t = META["table"]
    G = np.ascontiguousarray(GOLD["green"])
    nt, dt = 128, 0.004
    x = np.random.default_rng(seed).standard_normal((ns, nh, nt)).astype(np.float32)
    geo = dict(h0=0.05, dh=0.005, s0=0.02, ds=0.005)
    p = kd.datum_params(nt=nt, nh=nh, ns=ns, dt=dt, nsg=G.shape[0], nrg=G.shape[0], sg0=t["o"][2], dsg=t["d"][2],
                        rg0=t["o"][2], drg=t["d"][2], sdatum=0.1, rdatum=0.1, aperture=aperture, taper=3,
                        data_taper=5, cmp=cmp, antialias=1.0, length=0.05, **geo)
    o = D.Datum(nt, nh, ns, dt, geo["h0"], geo["dh"], geo["s0"], geo["ds"], G, t["o"][2], t["d"][2], G, t["o"][2],
                t["d"][2], np.float32(0.1), np.float32(0.1), aperture=aperture, taper=3, data_taper=5, cmp=cmp,
                antialias=1.0, length=0.05)
    return p, G, x, o


def test_datum_tiles_and_band_vs_oracle():
    """150 shots x 140 receivers, aperture 20: two 128-row and two
    128-column tiles per side, K ranges clipped by the aperture band at
    offsets that are not multiples of the K chunk."""
    p, G, x, o = _survey(150, 140, 20, 11)
    out = np.empty_like(x)
    kd.datum_freq(p, G, G, x, out)
    assert rel(out, o.run(x)) < 1e-5


def test_datum_tensor_cores_match_cuda_cores():
    """the tcgen05 GEMM (three TF32 products) against the FP32 CUDA-core
    kernel on the same inputs"""
    p, G, x, _ = _survey(150, 140, 20, 12)
    a = np.empty_like(x)
    kd.datum_freq(p, G, G, x, a)
    os.environ["KCIG_DATUM_GEMM"] = "simt"
    try:
        b = np.empty_like(x)
        kd.datum_freq(p, G, G, x, b)
    finally:
        del os.environ["KCIG_DATUM_GEMM"]
    assert rel(a, b) < 2e-6


def test_datum_shared_operator_vs_oracle():
    """shots and receivers on the same positions, one table, one datum: the
    source operator is the receiver operator transposed term for term, built
    once and read transposed by the source-side GEMM"""
    t = META["table"]
    G = np.ascontiguousarray(GOLD["green"])
    n, nt, dt = 140, 128, 0.004
    x = np.random.default_rng(13).standard_normal((n, n, nt)).astype(np.float32)
    p = kd.datum_params(nt=nt, nh=n, ns=n, dt=dt, h0=0.05, dh=0.005, s0=0.05, ds=0.005, nsg=G.shape[0],
                        nrg=G.shape[0], sg0=t["o"][2], dsg=t["d"][2], rg0=t["o"][2], drg=t["d"][2], sdatum=0.1,
                        rdatum=0.1, aperture=30, taper=4, data_taper=3, cmp=0, antialias=1.0, length=0.05)
    out = np.empty_like(x)
    kd.datum_freq(p, G, G, x, out)
    o = D.Datum(nt, n, n, dt, 0.05, 0.005, 0.05, 0.005, G, t["o"][2], t["d"][2], G, t["o"][2], t["d"][2],
                np.float32(0.1), np.float32(0.1), aperture=30, taper=4, data_taper=3, cmp=0, antialias=1.0,
                length=0.05)
    assert rel(out, o.run(x)) < 1e-5
    ms, _ = kd.datum_last_timing()
    os.environ["KCIG_DATUM_GEMM"] = "simt"
    try:
        b = np.empty_like(x)
        kd.datum_freq(p, G, G, x, b)
        ms_simt, _ = kd.datum_last_timing()
    finally:
        del os.environ["KCIG_DATUM_GEMM"]
    assert rel(out, b) < 2e-6
    assert ms[1] < ms_simt[1]   # one operator built instead of two


def test_datum_buffers_kept_between_calls():
    """the device buffers and cuFFT plans kept between calls: a survey run
    on fresh buffers, after a larger survey (larger buffers, other plans),
    after a cmp = 1 host-memory call with interm, and after datum_release
    gives the same traces bit for bit; so does the larger one run again"""
    ps, G, xs, o = _survey(40, 30, 20, 21)
    pl, _, xl, _ = _survey(150, 140, 20, 22)
    p1, d1, c1 = params_of("cmp1_jump")

    def run(p, x, im=None):
        out = np.empty_like(x)
        kd.datum_freq(p, G, G, np.ascontiguousarray(x), out, im)
        return out

    kd.datum_release()
    first = run(ps, xs)
    big = run(pl, xl)
    after_big = run(ps, xs)
    im = np.empty_like(d1)
    run(p1, d1, im)
    after_cmp1 = run(ps, xs)
    kd.datum_release()
    after_release = run(ps, xs)
    big_again = run(pl, xl)
    for got in (after_big, after_cmp1, after_release):
        assert np.array_equal(got, first)
    assert np.array_equal(big_again, big)
    assert rel(first, o.run(xs)) < 1e-5


def test_datum_calls_from_two_threads():
    """two threads calling at once (one device, so one after the other
    inside the library) get what one thread gets"""
    import threading
    pa, G, xa, _ = _survey(60, 50, 20, 23)
    pb, _, xb, _ = _survey(90, 40, 10, 24, cmp=1)
    want = []
    for p, x in ((pa, xa), (pb, xb)):
        out = np.empty_like(x)
        kd.datum_freq(p, G, G, x, out)
        want.append(out)
    got = [np.empty_like(xa), np.empty_like(xb)]
    errors = []

    def work(i, p, x):
        try:
            for _ in range(3):
                kd.datum_freq(p, G, G, x, got[i])
        except Exception as e:  # noqa: BLE001
            errors.append(e)

    th = [threading.Thread(target=work, args=(0, pa, xa)), threading.Thread(target=work, args=(1, pb, xb))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


@pytest.mark.parametrize("memory", ["host", "device"])
def test_datum_transform_batches(memory):
    """traces transformed in batches of 500 (three batches, the last one of
    200 traces on its own plan; the host-memory cube copied batch by batch
    beside the transforms) give the one-batch result within FP32 rounding,
    the oracle's within 1e-5, and host and device memory agree bit for bit"""
    p, G, x, o = _survey(40, 30, 20, 25, cmp=1)
    one = np.empty_like(x)
    kd.datum_freq(p, G, G, x, one)
    os.environ["KCIG_DATUM_BATCH"] = "500"
    try:
        if memory == "host":
            got = np.empty_like(x)
            im = np.empty_like(x)
            kd.datum_freq(p, G, G, x, got, im)
        else:
            Gd = torch.from_numpy(G).cuda()
            out_d = torch.empty((40, 30, 128), device="cuda")
            im_d = torch.empty_like(out_d)
            kd.datum_freq(p, Gd, Gd, torch.from_numpy(x).cuda(), out_d, im_d)
            torch.cuda.synchronize()
            got, im = out_d.cpu().numpy(), im_d.cpu().numpy()
        other = np.empty_like(x)
        kd.datum_freq(p, G, G, x, other)
    finally:
        del os.environ["KCIG_DATUM_BATCH"]
    assert rel(got, one) < 1e-6
    assert rel(got, o.run(x)) < 1e-5
    assert np.array_equal(other, got)
    want = o.run(x, interm=True)[1]
    assert rel(im, want) < 1e-5
