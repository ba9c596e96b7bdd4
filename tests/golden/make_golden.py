"""Generate the golden fixtures of the parity tests.

Runs the UNMODIFIED reference tools built from their sources by
``make -C oracle ref`` (oracle/_ref/{shotgen,eikods2d,kirchmig2d_cig}) on a
small seeded workload and stores inputs and reference images in
tests/golden/golden.npz, with the parameter tokens of each case in
tests/golden/cases.json.  Needs the reference tree (only in the build
container); the tests only read the committed outputs.

    python tests/golden/make_golden.py            # everything
    python tests/golden/make_golden.py --forward  # only the adj=0 fixtures
    python tests/golden/make_golden.py --eikods   # only the table-generator fixtures
    python tests/golden/make_golden.py --kirchmig2d  # only the plain-tool fixtures
    python tests/golden/make_golden.py --stitch   # only the ADCIG stitching fixtures
    python tests/golden/make_golden.py --datum    # only the datuming fixtures
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from kirch_datuming_b200 import rsf, synth  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")

# small model: v(z) = 1.5 + 0.6 z on a 41 x 81 grid of 10 m, tables every 20 m
NZ, NX, DZ = 41, 81, 0.01
NPOS_EVERY = 2
NT, DT = 301, 0.002

COMMON = ["adj=1"]
MUTE = ["direct_mute=1", "direct_mute_slope=0.5", "direct_mute_intercept=0", "direct_mute_taper=0.05"]
CASES = {
    "base": dict(data="cmp0", tokens=["cig=1", "mode=angle", "cmp=0", "angle_min=0", "angle_max=60",
                                      "angle_step=1", "angle_n=61"] + MUTE),
    "cmp1_half": dict(data="cmp1", tokens=["cig=1", "mode=angle", "cmp=1", "half_angle=1", "angle_min=0",
                                           "angle_max=45", "angle_step=1.5", "angle_n=31"] + MUTE),
    "options": dict(data="cmp0", tokens=["cig=1", "mode=angle", "cmp=0", "angle_interp=0", "diff=1",
                                         "type=linear", "tau=0.01", "antialias=0.5", "aperture=60",
                                         "aperture_taper=5", "aperture_rmin=0.1", "aperture_rtaper=0.05",
                                         "angle_taper_start=30", "angle_taper_end=50", "oazmin=70",
                                         "oazmax=40", "oaztaper=5", "angle_min=0", "angle_max=60",
                                         "angle_step=2", "angle_n=31"] + MUTE),
    "trace_aperture": dict(data="cmp0", tokens=["cig=1", "mode=angle", "cmp=0", "aperture_trace=8",
                                                "aperture_trace_taper=4", "type=partial",
                                                "angle_grad_radius=1", "angle_smooth=0", "direct_mute=1",
                                                "direct_mute_invert=1", "direct_mute_slope=0.3",
                                                "direct_mute_intercept=0.3", "direct_mute_taper=0.04",
                                                "angle_min=0", "angle_max=60", "angle_step=1",
                                                "angle_n=61"]),
    "offset": dict(data="cmp1", tokens=["cig=1", "mode=offset", "cmp=1"] + MUTE),
    "stack": dict(data="cmp0", tokens=["cig=0", "cmp=0"] + MUTE),
    "grads": dict(data="cmp0", grads=True, tokens=["cig=1", "mode=angle", "cmp=0", "angle_smooth=1",
                                                   "angle_min=0", "angle_max=60", "angle_step=1",
                                                   "angle_n=61"] + MUTE),
    "default_axis": dict(data="cmp0", tokens=["cig=1", "mode=angle", "cmp=0", "oazmin=180", "oazmax=180"]),
}

DATA = {
    # shots off the 20 m table grid, receivers on it (fixed spread)
    "cmp0": dict(ns=5, s0=0.05, ds=0.17, nh=21, h0=0.2, dh=0.02, cmp=0),
    # receivers move with the shot: r = s + h, split spread
    "cmp1": dict(ns=4, s0=0.23, ds=0.11, nh=17, h0=-0.16, dh=0.02, cmp=1),
}


# Forward modelling (adj=0, oracle/_ref/kirchmig2d_cig_fwd: the reference tool
# with its model-read helper fixed, oracle/ref_fixes.cpp) of the adjoint images:
# model = the reference's
# image of the named case, data geometry = that case's input data.  Run with
# one OpenMP thread (the reference sums per-thread trace buffers in thread
# order, so the thread count changes the FP32 rounding).
FWD = {
    "fwd_base": dict(image="base", tokens=["cig=1", "mode=angle", "cmp=0", "angle_min=0", "angle_max=60",
                                          "angle_step=1", "angle_n=61"]),
    "fwd_cmp1_half": dict(image="cmp1_half", tokens=["cig=1", "mode=angle", "cmp=1", "half_angle=1",
                                                     "angle_min=0", "angle_max=45", "angle_step=1.5",
                                                     "angle_n=31"]),
    "fwd_options": dict(image="options", tokens=["cig=1", "mode=angle", "cmp=0", "angle_interp=0", "type=linear",
                                                 "tau=0.01", "antialias=0.5", "aperture=60", "aperture_taper=5",
                                                 "aperture_rmin=0.1", "aperture_rtaper=0.05",
                                                 "angle_taper_start=30", "angle_taper_end=50", "oazmin=70",
                                                 "oazmax=40", "oaztaper=5", "angle_min=0", "angle_max=60",
                                                 "angle_step=2", "angle_n=31", "aperture_trace=8",
                                                 "aperture_trace_taper=4"]),
    "fwd_offset": dict(image="offset", tokens=["cig=1", "mode=offset", "cmp=1"]),
    "fwd_stack": dict(image="stack", tokens=["cig=0", "cmp=0"]),
}


def run(cmd, cwd, env=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError("%s failed:\n%s\n%s" % (cmd, r.stdout[-3000:], r.stderr[-3000:]))
    return r.stdout + r.stderr


def main():
    out = {}
    meta = {"nz": NZ, "nx": NX, "dz": DZ, "nt": NT, "dt": DT, "cases": {}, "data": {}}
    with tempfile.TemporaryDirectory() as wd:
        v = synth.velocity_linear_vz(NZ, NX, DZ)
        rsf.write(f"{wd}/vel.rsf", v, [NZ, NX], [0, 0], [DZ, DZ])
        npos = (NX - 1) // NPOS_EVERY + 1
        run([f"{REF}/shotgen", "shotfile=sht.rsf", f"nshot={npos}", "oy=0", f"dy={DZ * NPOS_EVERY}"], wd)
        run([f"{REF}/eikods2d", "in=vel.rsf", "out=time.rsf", "shotfile=sht.rsf", "tdl1=tdl.rsf",
             "tds1=tds.rsf", "gradz=gz.rsf", "gradx=gx.rsf", "b1=2", "b2=2"], wd)
        hT, T = rsf.read(f"{wd}/time.rsf")
        _, D = rsf.read(f"{wd}/tds.rsf")
        _, GX = rsf.read(f"{wd}/gx.rsf")
        _, GZ = rsf.read(f"{wd}/gz.rsf")
        meta["table"] = dict(n=hT.n[:3], o=hT.o[:3], d=hT.d[:3])
        out["T"], out["tds"], out["gradx"], out["gradz"] = T, D, GX, GZ
        tabs = torch.from_numpy(T.reshape(hT.n[2], NX, NZ))
        refl_rows = [(np.full(NX, r), a) for r, a in zip((12, 22, 33), synth.reflectivities(3, 11))]
        for name, d in DATA.items():
            g = synth.Geometry(nz=NZ, nx=NX, dz=DZ, dx=DZ, z0=0, x0=0, nt=NT, dt=DT, t0=0, npos=hT.n[2],
                               p0=hT.o[2], dp=hT.d[2], **d)
            data = synth.shot_gathers(tabs, g, refl_rows, 20.0, seed=5).numpy()
            out["data_" + name] = data
            meta["data"][name] = d
            rsf.write(f"{wd}/data_{name}.rsf", data, [NT, d["nh"], d["ns"]], [0, d["h0"], d["s0"]],
                      [DT, d["dh"], d["ds"]], extra={"unit1": "s"})
        for cname, c in CASES.items():
            args = [f"seismic_data=data_{c['data']}.rsf", f"migration=mig_{cname}.rsf", "stable=time.rsf",
                    "sderiv=tds.rsf", "rtable=time.rsf", "rderiv=tds.rsf"] + COMMON + c["tokens"]
            if c.get("grads"):
                args += ["sgradx=gx.rsf", "sgradz=gz.rsf", "rgradx=gx.rsf", "rgradz=gz.rsf"]
            log = run([f"{REF}/kirchmig2d_cig"] + args, wd)
            h, img = rsf.read(f"{wd}/mig_{cname}.rsf")
            with open(f"{wd}/mig_{cname}.rsf") as f:
                header = f.read()
            out["img_" + cname] = img
            meta["cases"][cname] = dict(data=c["data"], tokens=COMMON + c["tokens"], grads=bool(c.get("grads")),
                                        n=h.n[:3], o=h.o[:3], d=h.d[:3], extra=h.extra,
                                        sha256=hashlib.sha256(img.tobytes()).hexdigest(),
                                        info=[l.split("INFO:", 1)[1] for l in log.splitlines()
                                              if "INFO:cig =" in l])
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "golden.npz"))
    forward()


def forward():
    """adj=0 fixtures (golden_fwd.npz, cases.json "fwd") from the committed
    tables and images."""
    gz = np.load(os.path.join(HERE, "golden.npz"))
    with open(os.path.join(HERE, "cases.json")) as f:
        meta = json.load(f)
    t = meta["table"]
    out = {}
    meta["fwd"] = {}
    env = dict(os.environ, OMP_NUM_THREADS="1")
    with tempfile.TemporaryDirectory() as wd:
        rsf.write(f"{wd}/time.rsf", gz["T"], t["n"], t["o"], t["d"])
        rsf.write(f"{wd}/tds.rsf", gz["tds"], t["n"], t["o"], t["d"])
        for name, c in FWD.items():
            ic = meta["cases"][c["image"]]
            d = meta["data"][ic["data"]]
            img = gz["img_" + c["image"]]
            rsf.write(f"{wd}/img.rsf", img, ic["n"], ic["o"], ic["d"])
            args = ["migration=img.rsf", f"seismic_data=fwd_{name}.rsf", "stable=time.rsf", "sderiv=tds.rsf",
                    "rtable=time.rsf", "rderiv=tds.rsf", "adj=0", f"nt={meta['nt']}", f"nh={d['nh']}",
                    f"ns={d['ns']}", "t0=0", f"dt={meta['dt']}", f"h0={d['h0']}", f"dh={d['dh']}",
                    f"s0={d['s0']}", f"ds={d['ds']}"] + c["tokens"]
            run([f"{REF}/kirchmig2d_cig_fwd"] + args, wd, env=env)
            # the reference writes the adj=0 data header without its second and
            # third axes (dat->headers->ndim is left unset, src/kirchmig2d_cig.cpp:
            # 906-920); the binary holds every trace, read with the parameters' shape
            dat = np.fromfile(f"{wd}/fwd_{name}.rsf@", dtype="<f4")
            assert dat.size == d["ns"] * d["nh"] * meta["nt"], (name, dat.size)
            dat = dat.reshape(d["ns"], d["nh"], meta["nt"])
            out[name] = dat
            meta["fwd"][name] = dict(image=c["image"], data=ic["data"], tokens=["adj=0"] + c["tokens"],
                                     n=[meta["nt"], d["nh"], d["ns"]],
                                     sha256=hashlib.sha256(dat.tobytes()).hexdigest())
    np.savez_compressed(os.path.join(HERE, "golden_fwd.npz"), **out)
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "golden_fwd.npz"))


# table generator: the five-layer salt model on a 31 x 61 grid of 10 m, shots
# off the grid nodes and below the surface, three parameter sets
EIK_NZ, EIK_NX = 31, 61
EIK_SHOTS = [(0.0, 0.05, 0.0), (0.0, 0.2345, 0.0), (0.1, 0.4, 0.0), (0.0, 0.595, 0.0), (0.25, 0.31, 0.0)]
EIK_RUNS = {"o2": ["order=2"], "o1": ["order=1"], "o2_l0": ["order=2", "l=0"]}


def eikods():
    """eikods2d fixtures (golden_eikods.npz, cases.json "eikods")."""
    with open(os.path.join(HERE, "cases.json")) as f:
        meta = json.load(f)
    v, _ = synth.five_layer_salt(EIK_NZ, EIK_NX, DZ, DZ)
    shots = np.asarray(EIK_SHOTS, np.float32)
    out = {"vel": v, "shots": shots}
    meta["eikods"] = {"nz": EIK_NZ, "nx": EIK_NX, "d": DZ, "b1": 2, "b2": 2, "runs": EIK_RUNS}
    env = dict(os.environ, OMP_NUM_THREADS="1")
    with tempfile.TemporaryDirectory() as wd:
        rsf.write(f"{wd}/vel.rsf", v, [EIK_NZ, EIK_NX], [0, 0], [DZ, DZ])
        rsf.write(f"{wd}/sht.rsf", shots, [3, len(EIK_SHOTS)], [0, 0], [1, 1])
        for name, toks in EIK_RUNS.items():
            run([f"{REF}/eikods2d", "in=vel.rsf", "out=time.rsf", "shotfile=sht.rsf", "tdl1=tdl.rsf",
                 "tds1=tds.rsf", "gradz=gz.rsf", "gradx=gx.rsf", "b1=2", "b2=2"] + toks, wd, env=env)
            for f, k in (("time", "time"), ("tdl", "tdl1"), ("tds", "tds1"), ("gz", "gradz"), ("gx", "gradx")):
                if name == "o2_l0" and k not in ("tdl1", "tds1"):
                    continue  # l only changes the derivatives
                h, a = rsf.read(f"{wd}/{f}.rsf")
                out[f"{name}_{k}"] = a.reshape(len(EIK_SHOTS), EIK_NX, EIK_NZ)
                if name == "o2" and k == "time":
                    meta["eikods"]["header"] = dict(n=h.n[:3], o=h.o[:3], d=h.d[:3])
    np.savez_compressed(os.path.join(HERE, "golden_eikods.npz"), **out)
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "golden_eikods.npz"))


# the plain tool kirchmig2d on the same inputs (oracle/_ref/kirchmig2d), one
# OpenMP thread
K2D = {
    "k2d_default": dict(data="cmp1", tokens=["cmp=1"]),
    "k2d_cig_cmp0": dict(data="cmp0", tokens=["cmp=0", "cig=1", "aperture=40", "antialias=0.5", "tau=0.004",
                                              "diff=1", "type=linear"]),
    "k2d_trace_ap": dict(data="cmp1", tokens=["cmp=1", "cig=1", "aperture=60", "aperture_trace=6",
                                              "type=partial"]),
    "k2d_stack_cmp0": dict(data="cmp0", tokens=["cmp=0", "aperture=25"]),
}


def kirchmig2d():
    """kirchmig2d fixtures (golden_k2d.npz, cases.json "k2d")."""
    gz = np.load(os.path.join(HERE, "golden.npz"))
    with open(os.path.join(HERE, "cases.json")) as f:
        meta = json.load(f)
    t = meta["table"]
    out = {}
    meta["k2d"] = {}
    env = dict(os.environ, OMP_NUM_THREADS="1")
    with tempfile.TemporaryDirectory() as wd:
        rsf.write(f"{wd}/time.rsf", gz["T"], t["n"], t["o"], t["d"])
        rsf.write(f"{wd}/tds.rsf", gz["tds"], t["n"], t["o"], t["d"])
        for name, d in DATA.items():
            rsf.write(f"{wd}/data_{name}.rsf", gz["data_" + name], [NT, d["nh"], d["ns"]], [0, d["h0"], d["s0"]],
                      [DT, d["dh"], d["ds"]], extra={"unit1": "s"})
        for name, c in K2D.items():
            args = [f"seismic_data=data_{c['data']}.rsf", "migration=img.rsf", "stable=time.rsf", "sderiv=tds.rsf",
                    "rtable=time.rsf", "rderiv=tds.rsf"] + c["tokens"]
            run([f"{REF}/kirchmig2d"] + args, wd, env=env)
            h, img = rsf.read(f"{wd}/img.rsf")
            out[name] = img.reshape(h.n[2], h.n[1], h.n[0])
            meta["k2d"][name] = dict(data=c["data"], tokens=c["tokens"], n=h.n[:3], o=h.o[:3], d=h.d[:3],
                                     extra={k: v for k, v in h.extra.items() if k.startswith(("label", "unit"))})
    np.savez_compressed(os.path.join(HERE, "golden_k2d.npz"), **out)
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "golden_k2d.npz"))


# ADCIG stitching (layercom_cig): three depth windows of a 60 x 24 model with
# 7 angles; the layer file mixes every separator the tool accepts
STITCH_MODEL = dict(n=[60, 24], o=[0.0, 0.5], d=[0.01, 0.02])
STITCH_ANGLES = dict(n=7, o=0.0, d=10.0)
STITCH_LAYERS = "# depth windows of the test model\nSTART,25\n18\uff0c45   # middle\n\n40;END\n"
STITCH_WINDOWS = [(0, 25), (18, 45), (40, 59)]
STITCH = {
    "default": [],
    "blend3_scales": ["stitch_blend=3", "scale=1.5,0.5;2"],
    "keep_upper": ["stitch_blend=0"],
    "full_overlap": ["stitch_blend=-1", "nlayers=3", "nangle=7"],
    "lateral": ["scalex_aper=5", "scalex_scale=2.5", "scale=0.8"],
    "blend1_lateral1": ["stitch_blend=1", "scalex_aper=1", "scalex_scale=0.5"],
}
STITCH_ERRORS = {
    "nonfinite": ["layer_image_base=bad.rsf"],
    "nlayers": ["nlayers=4"],
    "scale_count": ["scale=1,2"],
    "blend": ["stitch_blend=-2"],
    "bad_argument": ["foo"],
    "missing_key": ["layer_txt="],
}


def stitch():
    """layercom_cig fixtures (golden_stitch.npz, cases.json "stitch")."""
    with open(os.path.join(HERE, "cases.json")) as f:
        meta = json.load(f)
    rng = np.random.default_rng(2024)
    m, a = STITCH_MODEL, STITCH_ANGLES
    out = {}
    vols = []
    for k, (s0, s1) in enumerate(STITCH_WINDOWS):
        v = rng.standard_normal((a["n"], m["n"][1], s1 - s0 + 1)).astype(np.float32)
        vols.append(v)
        out["window_%d" % (k + 1)] = v
    labels = {"label1": "Depth", "label2": "Lateral", "label3": "Scattering angle", "unit1": "km",
              "unit3": "degree"}
    info = dict(model=m, angles=a, layers=STITCH_LAYERS, windows=STITCH_WINDOWS, labels=labels, cases={},
                errors={})
    with tempfile.TemporaryDirectory() as wd:
        rsf.write(f"{wd}/model.rsf", np.zeros(m["n"][::-1], np.float32), m["n"], m["o"], m["d"])
        with open(f"{wd}/layers.txt", "w", encoding="utf-8") as f:
            f.write(STITCH_LAYERS)
        for base in ("adcig", "bad"):
            for k, ((s0, s1), v) in enumerate(zip(STITCH_WINDOWS, vols)):
                v = v.copy()
                if base == "bad" and k == 1:
                    v[3, 5, 2] = np.inf
                rsf.write(f"{wd}/{base}_{k + 1}.rsf", v, [s1 - s0 + 1, m["n"][1], a["n"]],
                          [m["o"][0] + s0 * m["d"][0], m["o"][1], a["o"]], [m["d"][0], m["d"][1], a["d"]],
                          extra=labels)
        common = ["full_model=model.rsf", "layer_image_base=adcig.rsf", "layer_txt=layers.txt",
                  "output_file=out.rsf"]
        for name, extra in STITCH.items():
            r = subprocess.run([f"{REF}/layercom_cig"] + common + extra, cwd=wd, capture_output=True, text=True)
            assert r.returncode == 0, r.stderr
            h, img = rsf.read(f"{wd}/out.rsf")
            out["out_" + name] = img.reshape(h.n[2], h.n[1], h.n[0])
            with open(f"{wd}/out.rsf") as f:
                header = f.read()
            info["cases"][name] = dict(args=extra, header=header, stdout=r.stdout)
        for name, extra in STITCH_ERRORS.items():
            r = subprocess.run([f"{REF}/layercom_cig"] + common + extra, cwd=wd, capture_output=True, text=True)
            assert r.returncode != 0
            info["errors"][name] = dict(args=extra, stderr=r.stderr, returncode=r.returncode)
    meta["stitch"] = info
    np.savez_compressed(os.path.join(HERE, "golden_stitch.npz"), **out)
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "golden_stitch.npz"))


# Datuming between depth levels: greensol_auto and kirchdat2d_freq
# (oracle/_ref/kirchdat2d_freq is the reference tool linked against
# oracle/fftw_dft.c), on the small five-layer salt model with tables every 10 m.
DAT_NZ, DAT_NX, DAT_DATUM = 41, 81, 10
DAT_NT, DAT_DT = 128, 0.004
DAT_DATA = {
    "cmp0": dict(ns=12, s0=0.2, ds=0.02, nh=24, h0=0.1, dh=0.02),
    "cmp1": dict(ns=12, s0=0.25, ds=0.02, nh=16, h0=-0.12, dh=0.02),
    "cmp1_jump": dict(ns=16, s0=0.25, ds=0.01, nh=12, h0=-0.1, dh=0.02),
}
DAT_CASES = {
    "cmp0": dict(data="cmp0", interm=True, args=["cmp=0", "aperture=10", "taper=3", "data_taper=2", "antialias=1",
                                                  "length=0.05", "use_bf=0"]),
    "cmp0_workflow_bf": dict(data="cmp0", args=["aperture=200", "data_taper=20", "taper=0", "length=0.05", "cmp=0",
                                                "antialias=1", "use_bf=1"]),
    "cmp1": dict(data="cmp1", interm=True, args=["cmp=1", "aperture=5", "taper=2", "use_bf=0"]),
    "cmp1_jump": dict(data="cmp1_jump", args=["cmp=1", "aperture=6", "taper=0", "data_taper=1", "use_bf=0"]),
    "manual_datum": dict(data="cmp0", args=["cmp=0", "auto_datum=0", "sdatum=0.08", "rdatum=0.12",
                                            "antialias=0.5", "length=0.03", "aperture=8", "taper=0", "use_bf=0"]),
    "defaults": dict(data="cmp1", args=[]),
}
# (setup, arguments) of failing runs: exit code and ERROR text must match
DAT_ERRORS = {
    "no_input": ["output_file=o.rsf"],
    "cmp": ["cmp=2"],
    "auto_datum": ["auto_datum=2"],
    "no_sdatum": ["auto_datum=0", "rdatum=0.1"],
    "bf_p": ["bf_p=16", "bf_n_leaf=16"],
    "bf_zero": ["bf_p=0"],
    "data_taper": ["data_taper=-1"],
    "antialias": ["antialias=-0.5"],
    "small_table": ["input_file=d_wide.rsf"],
    "no_should_datum": ["model_file=vel_nodatum.rsf"],
    "input_2d": ["input_file=d_2d.rsf"],
}
GREEN_ERRORS = {
    "no_ttabel": ["tgreen_file=g.rsf", "model_file=vel.rsf"],
    "no_should_datum": ["ttabel_file=time.rsf", "tgreen_file=g.rsf", "model_file=vel_nodatum.rsf"],
    "datum_range": ["ttabel_file=time.rsf", "tgreen_file=g.rsf", "model_file=vel_deep.rsf"],
    "table_2d": ["ttabel_file=vel.rsf", "tgreen_file=g.rsf", "model_file=vel.rsf"],
}


def datum():
    """greensol_auto + kirchdat2d_freq fixtures (golden_datum.npz, cases.json "datum")."""
    with open(os.path.join(HERE, "cases.json")) as f:
        meta = json.load(f)
    v, _ = synth.five_layer_salt(DAT_NZ, DAT_NX, DZ, DZ)
    out = {}
    info = dict(nz=DAT_NZ, nx=DAT_NX, d=DZ, should_datum=DAT_DATUM, nt=DAT_NT, dt=DAT_DT, data=DAT_DATA,
                cases={}, errors={}, green_errors={})
    rng = np.random.default_rng(77)
    with tempfile.TemporaryDirectory() as wd:
        rsf.write(f"{wd}/vel.rsf", v, [DAT_NZ, DAT_NX], [0, 0], [DZ, DZ], extra={"should_datum": str(DAT_DATUM)})
        rsf.write(f"{wd}/vel_nodatum.rsf", v, [DAT_NZ, DAT_NX], [0, 0], [DZ, DZ])
        rsf.write(f"{wd}/vel_deep.rsf", v, [DAT_NZ, DAT_NX], [0, 0], [DZ, DZ], extra={"should_datum": "60"})
        run([f"{REF}/shotgen", "shotfile=sht.rsf", f"nshot={DAT_NX}", "oy=0", f"dy={DZ}"], wd)
        run([f"{REF}/eikods2d", "in=vel.rsf", "out=time.rsf", "shotfile=sht.rsf", "tdl1=tdl.rsf", "tds1=tds.rsf",
             "b1=2", "b2=2"], wd)
        h, t = rsf.read(f"{wd}/time.rsf")
        out["vel"], out["table"] = v, t.reshape(h.n[2], h.n[1], h.n[0])
        info["table"] = dict(n=h.n[:3], o=h.o[:3], d=h.d[:3])
        log = run([f"{REF}/greensol_auto", "ttabel_file=time.rsf", "tgreen_file=green.rsf", "model_file=vel.rsf"], wd)
        hg, g = rsf.read(f"{wd}/green.rsf", count=h.n[2] * h.n[2])
        out["green"] = g.reshape(h.n[2], h.n[2])
        with open(f"{wd}/green.rsf") as f:
            info["green_header"] = f.read()
        info["green_info"] = [l.split("INFO:", 1)[1] for l in log.splitlines()
                              if "INFO:" in l and "INFO:greensol_auto " not in l]
        for name, d in DAT_DATA.items():
            x = rng.standard_normal((d["ns"], d["nh"], DAT_NT)).astype(np.float32)
            x[d["ns"] // 2, d["nh"] // 3, DAT_NT // 2] += 25.0
            out["data_" + name] = x
            rsf.write(f"{wd}/d_{name}.rsf", x, [DAT_NT, d["nh"], d["ns"]], [0, d["h0"], d["s0"]],
                      [DAT_DT, d["dh"], d["ds"]], extra={"label1": "Time", "unit1": "s"})
        common = ["sgreen_file=green.rsf", "rgreen_file=green.rsf", "model_file=vel.rsf"]
        for name, c in DAT_CASES.items():
            args = [f"input_file=d_{c['data']}.rsf", "output_file=out.rsf"] + common + c["args"]
            if c.get("interm"):
                args.append("interm=interm.rsf")
            log = run([f"{REF}/kirchdat2d_freq"] + args, wd)
            d = DAT_DATA[c["data"]]
            ho, o = rsf.read(f"{wd}/out.rsf")
            out["out_" + name] = o.reshape(d["ns"], d["nh"], DAT_NT)
            with open(f"{wd}/out.rsf") as f:
                header = f.read()
            rec = dict(data=c["data"], args=c["args"], header=header, interm=bool(c.get("interm")),
                       info=[l.split("INFO:", 1)[1] for l in log.splitlines() if "INFO:" in l
                             and "INFO:Processing " not in l and "Elapsed" not in l
                             and "INFO:kirchdat2d_freq " not in l])
            if c.get("interm"):
                _, im = rsf.read(f"{wd}/interm.rsf", count=d["ns"] * d["nh"] * DAT_NT)
                out["interm_" + name] = im.reshape(d["ns"], d["nh"], DAT_NT)
                with open(f"{wd}/interm.rsf") as f:
                    rec["interm_header"] = f.read()
            info["cases"][name] = rec
        # failing runs
        wide = DAT_DATA["cmp0"]
        rsf.write(f"{wd}/d_wide.rsf", np.zeros((4, 8, DAT_NT), np.float32), [DAT_NT, 8, 4], [0, 0.7, 0.2],
                  [DAT_DT, 0.02, 0.02])
        rsf.write(f"{wd}/d_2d.rsf", np.zeros((8, DAT_NT), np.float32), [DAT_NT, 8], [0, 0.1], [DAT_DT, 0.02])
        base = ["input_file=d_cmp0.rsf", "output_file=o.rsf"] + common
        for name, extra in DAT_ERRORS.items():
            args = (base if name != "no_input" else common) + extra
            r = subprocess.run([f"{REF}/kirchdat2d_freq"] + args, cwd=wd, capture_output=True, text=True)
            assert r.returncode != 0, name
            info["errors"][name] = dict(args=args, returncode=r.returncode,
                                        error=[l.split("ERROR:", 1)[1] for l in r.stderr.splitlines()
                                               if "ERROR:" in l])
        for name, args in GREEN_ERRORS.items():
            r = subprocess.run([f"{REF}/greensol_auto"] + args, cwd=wd, capture_output=True, text=True)
            assert r.returncode != 0, name
            info["green_errors"][name] = dict(args=args, returncode=r.returncode,
                                              error=[l.split("ERROR:", 1)[1] for l in r.stderr.splitlines()
                                                     if "ERROR:" in l])
    meta["datum"] = info
    np.savez_compressed(os.path.join(HERE, "golden_datum.npz"), **out)
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "golden_datum.npz"))


if __name__ == "__main__":
    if "--datum" in sys.argv:
        datum()
    elif "--stitch" in sys.argv:
        stitch()
    elif "--forward" in sys.argv:
        forward()
    elif "--kirchmig2d" in sys.argv:
        kirchmig2d()
    elif "--eikods" in sys.argv:
        eikods()
    else:
        main()
