"""Golden fixture access shared by the tests: inputs, reference images and the
parameter blocks of each case for the library and for the oracle."""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


class Golden:
    def __init__(self):
        self.npz = np.load(os.path.join(GOLDEN, "golden.npz"))
        with open(os.path.join(GOLDEN, "cases.json")) as f:
            self.meta = json.load(f)
        self.nz, self.nx = self.meta["nz"], self.meta["nx"]

    @property
    def cases(self):
        return sorted(self.meta["cases"])

    def tables(self):
        return self.npz["T"], self.npz["tds"]

    def grads(self):
        return self.npz["gradx"], self.npz["gradz"]

    @property
    def fwd_cases(self):
        return sorted(self.meta.get("fwd", {}))

    def fwd_data(self, name):
        return np.load(os.path.join(GOLDEN, "golden_fwd.npz"))[name]

    def data(self, case):
        return self.npz["data_" + self.meta["cases"][case]["data"]]

    def image(self, case):
        c = self.meta["cases"][case]
        return self.npz["img_" + case].reshape(c["n"][2], c["n"][1], c["n"][0])

    def tokens(self, case):
        return list(self.meta["cases"][case]["tokens"])

    @property
    def k2d_cases(self):
        return sorted(self.meta.get("k2d", {}))

    def k2d_image(self, name):
        c = self.meta["k2d"][name]
        return np.load(os.path.join(GOLDEN, "golden_k2d.npz"))[name].reshape(c["n"][2], c["n"][1], c["n"][0])

    def geometry_dict(self, case, data_key=None):
        d = self.meta["data"][data_key or self.meta["cases"][case]["data"]]
        t = self.meta["table"]
        f = lambda v: float(np.float32(v))  # header values are read as float  # noqa: E731
        return dict(nt=self.meta["nt"], nh=d["nh"], ns=d["ns"], t0=0.0, dt=f(self.meta["dt"]), h0=f(d["h0"]),
                    dh=f(d["dh"]), s0=f(d["s0"]), ds=f(d["ds"]), nz=t["n"][0], nx=t["n"][1], z0=f(t["o"][0]),
                    dz=f(t["d"][0]), x0=f(t["o"][1]), dx=f(t["d"][1]), sny=t["n"][2], sy0=f(t["o"][2]),
                    sdy=f(t["d"][2]), rny=t["n"][2], ry0=f(t["o"][2]), rdy=f(t["d"][2]))


def oracle_params(kp, geom: dict, axis, use_grad=False):
    """Oracle parameter block from a library parameter block (same meaning)."""
    import oracle
    ng, g0, dg = axis
    g = dict(geom)
    if g["nh"] == 1:
        g["dh"] = 0.0
    if g["ns"] == 1:
        g["ds"] = 0.0
    return oracle.make_params(
        nt=g["nt"], nh=g["nh"], ns=g["ns"], t0=g["t0"], dt=g["dt"], h0=g["h0"], dh=g["dh"], s0=g["s0"],
        ds=g["ds"], nz=g["nz"], nx=g["nx"], z0=g["z0"], dz=g["dz"], x0=g["x0"], dx=g["dx"], sny=g["sny"],
        sy0=g["sy0"], sdy=g["sdy"], rny=g["rny"], ry0=g["ry0"], rdy=g["rdy"], ng=ng, g0=g0, dg=dg,
        cig=kp.cig, cig_is_angle=kp.cig_is_angle, cmp=kp.cmp, half_angle=kp.half_angle, isdiff=kp.isdiff,
        interp_type=kp.interp_type, use_input_grad=int(use_grad), angle_interp=kp.angle_interp,
        angle_grad_radius=kp.angle_grad_radius, angle_smooth=kp.angle_smooth, aperture_trace=kp.aperture_trace,
        aperture_trace_taper=kp.aperture_trace_taper, direct_mute=kp.direct_mute,
        direct_mute_invert=kp.direct_mute_invert, tau=kp.tau, aper=kp.aperture, aperture_taper=kp.aperture_taper,
        aperture_rmin=kp.aperture_rmin, aperture_rtaper=kp.aperture_rtaper, aal=kp.antialias,
        angle_taper_start=kp.angle_taper_start, angle_taper_end=kp.angle_taper_end, oazmin=kp.oazmin,
        oazmax=kp.oazmax, oaztaper=kp.oaztaper, direct_mute_slope=kp.direct_mute_slope,
        direct_mute_intercept=kp.direct_mute_intercept, direct_mute_taper=kp.direct_mute_taper)


def case_setup(gd: Golden, case: str):
    """(library params, geometry dict, axis, oracle params, use_grad)."""
    import kirch_datuming_b200 as kd
    kp = kd.params(*gd.tokens(case))
    geom = gd.geometry_dict(case)
    axis = kd.output_axis(kp, kd.geometry(**geom))
    use_grad = bool(gd.meta["cases"][case].get("grads"))
    return kp, geom, axis, oracle_params(kp, geom, axis, use_grad), use_grad


def k2d_setup(gd: Golden, name: str):
    """kirchmig2d fixture: (library params, geometry dict, axis, oracle params)."""
    import kirch_datuming_b200 as kd
    c = gd.meta["k2d"][name]
    kp = kd.params_kirchmig2d(*c["tokens"])
    geom = gd.geometry_dict(None, data_key=c["data"])
    axis = kd.output_axis(kp, kd.geometry(**geom))
    return kp, geom, axis, oracle_params(kp, geom, axis)


def fwd_setup(gd: Golden, name: str):
    """adj=0 fixture: (library params, geometry dict, axis, oracle params,
    model image [ng][nx][nz])."""
    import kirch_datuming_b200 as kd
    f = gd.meta["fwd"][name]
    kp = kd.params(*f["tokens"])
    geom = gd.geometry_dict(f["image"])
    axis = kd.output_axis(kp, kd.geometry(**geom))
    return kp, geom, axis, oracle_params(kp, geom, axis), gd.image(f["image"])


def oracle_image(gd: Golden, case: str, fp64=True):
    import oracle
    _, _, _, op, use_grad = case_setup(gd, case)
    T, D = gd.tables()
    grads = None
    if use_grad:
        gx, gz = gd.grads()
        grads = (gx, gz, gx, gz)
    return oracle.migrate_adj(op, gd.data(case), T, D, T, D, grads=grads, fp64=fp64)


def ub_columns(gd: Golden, case: str) -> int:
    """Leading lateral columns where the reference's type=partial derivative
    reads outside its table slice (tinterpsr.cpp:119-124): its image there is
    undefined and is not compared."""
    toks = gd.meta["k2d"][case]["tokens"] if case in gd.meta.get("k2d", {}) else gd.tokens(case)
    return 3 if any(t.startswith("type=p") for t in toks) else 0
