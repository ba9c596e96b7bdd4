"""ctypes binding of the C oracle (kcig_oracle.c).  TEST INFRASTRUCTURE ONLY:
imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg,
never by the library.  Build with ``make -C oracle``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_INT_FIELDS_A = ["nt", "nh", "ns"]
_FLT_FIELDS_A = ["t0", "dt", "h0", "dh", "s0", "ds"]


class OracleParams(ctypes.Structure):
    _fields_ = (
        [(n, ctypes.c_int) for n in ("nt", "nh", "ns")]
        + [(n, ctypes.c_float) for n in ("t0", "dt", "h0", "dh", "s0", "ds")]
        + [(n, ctypes.c_int) for n in ("nz", "nx")]
        + [(n, ctypes.c_float) for n in ("z0", "dz", "x0", "dx")]
        + [("sny", ctypes.c_int)]
        + [(n, ctypes.c_float) for n in ("sy0", "sdy")]
        + [("rny", ctypes.c_int)]
        + [(n, ctypes.c_float) for n in ("ry0", "rdy")]
        + [("ng", ctypes.c_int)]
        + [(n, ctypes.c_float) for n in ("g0", "dg")]
        + [(n, ctypes.c_int) for n in (
            "cig", "cig_is_angle", "cmp", "half_angle", "isdiff", "interp_type",
            "use_input_grad", "angle_interp", "angle_grad_radius", "angle_smooth",
            "aperture_trace", "aperture_trace_taper", "direct_mute", "direct_mute_invert")]
        + [(n, ctypes.c_float) for n in (
            "tau", "aper", "aperture_taper", "aperture_rmin", "aperture_rtaper", "aal",
            "angle_taper_start", "angle_taper_end", "oazmin", "oazmax", "oaztaper",
            "direct_mute_slope", "direct_mute_intercept", "direct_mute_taper")]
    )


def make_params(**kw) -> OracleParams:
    p = OracleParams()
    names = {f[0] for f in OracleParams._fields_}
    for k, v in kw.items():
        if k not in names:
            raise KeyError(k)
        if k == "interp_type" and isinstance(v, str):
            v = ord(v[0])
        setattr(p, k, v)
    return p


_libs: dict = {}


def lib(fp64: bool = True):
    key = "64" if fp64 else "32"
    if key not in _libs:
        path = os.path.join(HERE, "liboracle%s.so" % key)
        if not os.path.exists(path):
            raise FileNotFoundError("oracle not built: run `make -C oracle` (%s)" % path)
        L = ctypes.CDLL(path)
        fp = ctypes.POINTER(ctypes.c_float)
        dp = ctypes.POINTER(ctypes.c_double)
        L.oracle_migrate_adj.argtypes = [ctypes.POINTER(OracleParams), fp, fp, fp, fp, fp,
                                         fp, fp, fp, fp, dp]
        L.oracle_migrate_adj.restype = ctypes.c_int
        L.oracle_kirchmig2d_adj.argtypes = [ctypes.POINTER(OracleParams), fp, fp, fp, fp, fp, dp]
        L.oracle_kirchmig2d_adj.restype = ctypes.c_int
        L.oracle_model_fwd.argtypes = [ctypes.POINTER(OracleParams), fp, fp, fp, fp, fp, fp, fp, fp, fp, dp]
        L.oracle_model_fwd.restype = ctypes.c_int
        L.oracle_doubint.argtypes = [ctypes.c_int, fp, dp, ctypes.c_int, ctypes.c_float]
        L.oracle_mute.argtypes = [ctypes.c_int, fp] + [ctypes.c_float] * 7 + [ctypes.c_int]
        L.oracle_pick.argtypes = [ctypes.c_double, ctypes.c_double, dp, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_double]
        L.oracle_pick.restype = ctypes.c_double
        L.oracle_leg_fields.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_int, fp, fp, fp, fp,
                                        ctypes.c_float, dp, dp, dp, dp]
        L.oracle_leg_fields.restype = ctypes.c_int
        _libs[key] = L
    return _libs[key]


def _fptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def migrate_adj(p: OracleParams, data, stable, sderiv, rtable, rderiv, grads=None,
                fp64: bool = True) -> np.ndarray:
    """Image [ng][nx][nz] as float64 (FP32 values for the mirror build)."""
    L = lib(fp64)
    data, stable, sderiv, rtable, rderiv = map(_f32, (data, stable, sderiv, rtable, rderiv))
    g = [None] * 4 if grads is None else [_f32(x) for x in grads]
    img = np.zeros(p.ng * p.nx * p.nz, dtype=np.float64)
    rc = L.oracle_migrate_adj(ctypes.byref(p), _fptr(data), _fptr(stable), _fptr(sderiv),
                              _fptr(rtable), _fptr(rderiv), *[_fptr(x) for x in g],
                              img.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    if rc != 0:
        raise RuntimeError("oracle_migrate_adj failed: %d" % rc)
    return img.reshape(p.ng, p.nx, p.nz)


def migrate_kirchmig2d(p: OracleParams, data, stable, sderiv, rtable, rderiv, fp64: bool = True) -> np.ndarray:
    """kirchmig2d adj=1 (src/kirchmig2d.cpp:366-540): image [ng][nx][nz],
    ng = nh for cig=1 else 1 (p.ng must say so)."""
    L = lib(fp64)
    data, stable, sderiv, rtable, rderiv = map(_f32, (data, stable, sderiv, rtable, rderiv))
    img = np.zeros(p.ng * p.nx * p.nz, dtype=np.float64)
    rc = L.oracle_kirchmig2d_adj(ctypes.byref(p), _fptr(data), _fptr(stable), _fptr(sderiv), _fptr(rtable),
                                 _fptr(rderiv), img.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    if rc != 0:
        raise RuntimeError("oracle_kirchmig2d_adj failed: %d" % rc)
    return img.reshape(p.ng, p.nx, p.nz)


def model_fwd(p: OracleParams, image, stable, sderiv, rtable, rderiv, grads=None, fp64: bool = True) -> np.ndarray:
    """Forward-modelled data [ns][nh][nt] (float64) from image [ng][nx][nz]
    (kirchmig2d_cig adj=0)."""
    L = lib(fp64)
    image, stable, sderiv, rtable, rderiv = map(_f32, (image, stable, sderiv, rtable, rderiv))
    g = [None] * 4 if grads is None else [_f32(x) for x in grads]
    out = np.zeros(p.ns * p.nh * p.nt, dtype=np.float64)
    rc = L.oracle_model_fwd(ctypes.byref(p), _fptr(image), _fptr(stable), _fptr(sderiv), _fptr(rtable),
                            _fptr(rderiv), *[_fptr(x) for x in g],
                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    if rc != 0:
        raise RuntimeError("oracle_model_fwd failed: %d" % rc)
    return out.reshape(p.ns, p.nh, p.nt)


def doubint(trace, isdiff=0, dt=1.0, fp64=True) -> np.ndarray:
    tr = _f32(trace)
    out = np.zeros(tr.size, dtype=np.float64)
    lib(fp64).oracle_doubint(tr.size, _fptr(tr), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                             int(isdiff), float(dt))
    return out


def mute(trace, t0, dt, sx, rx, slope, intercept, taper, inverted=0, fp64=True) -> np.ndarray:
    tr = _f32(trace).copy()
    lib(fp64).oracle_mute(tr.size, _fptr(tr), t0, dt, sx, rx, slope, intercept, taper, int(inverted))
    return tr


def pick(ti, deltat, dtrace, dt, t0, fp64=True) -> float:
    d = np.ascontiguousarray(dtrace, dtype=np.float64)
    return lib(fp64).oracle_pick(float(ti), float(deltat),
                                 d.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), d.size,
                                 float(dt), float(t0))


def leg_fields(p: OracleParams, is_source: int, tab, der, pos, grads=(None, None), fp64=True):
    nzx = p.nz * p.nx
    outs = [np.zeros(nzx, dtype=np.float64) for _ in range(4)]
    tab, der = _f32(tab), _f32(der)
    gx, gz = (_f32(grads[0]), _f32(grads[1]))
    rc = lib(fp64).oracle_leg_fields(ctypes.byref(p), int(is_source), _fptr(tab), _fptr(der),
                                     _fptr(gx), _fptr(gz), float(pos),
                                     *[o.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for o in outs])
    if rc != 0:
        raise RuntimeError("oracle_leg_fields failed")
    return outs


_eik = None


def eikods(vel, d1, d2, shots, o1=0.0, o2=0.0, o3=0.0, d3=1.0, b1=2, b2=2, order=2, l=1, method=0,
           vel_is_s2=False, max_iter=256, grads=False):
    """eikods2d's tables on the CPU (kcig_eikods_oracle.c).  vel [nx][nz];
    shots [nshot][3] (depth, lateral, third axis).  method 0: the marching
    solver eikods2d runs; 1: sweeps to the fixed point of the same update.
    Returns a dict of float32 arrays [nshot][nx][nz] (time, tdl1, tds1 and,
    with grads, gradz/gradx) plus 'sweeps' [nshot]."""
    global _eik
    if _eik is None:
        path = os.path.join(HERE, "libeikods_oracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError("oracle not built: run `make -C oracle` (%s)" % path)
        _eik = ctypes.CDLL(path)
        fp = ctypes.POINTER(ctypes.c_float)
        ip = ctypes.POINTER(ctypes.c_int)
        _eik.oracle_eikods.argtypes = ([ctypes.c_int] * 3 + [ctypes.c_float] * 6 + [fp, ctypes.c_int, fp]
                                       + [ctypes.c_int] * 6 + [fp] * 5 + [ip])
        _eik.oracle_eikods.restype = ctypes.c_int
    vel = _f32(vel)
    nx, nz = vel.shape
    shots = _f32(np.asarray(shots, np.float32).reshape(-1, 3))
    ns = shots.shape[0]
    out = {k: np.zeros((ns, nx, nz), np.float32) for k in ("time", "tdl1", "tds1")}
    if grads:
        out["gradz"] = np.zeros((ns, nx, nz), np.float32)
        out["gradx"] = np.zeros((ns, nx, nz), np.float32)
    sweeps = np.zeros(ns, np.int32)
    rc = _eik.oracle_eikods(int(method), nz, nx, o1, o2, d1, d2, o3, d3, _fptr(vel), int(vel_is_s2), _fptr(shots),
                            ns, b1, b2, order, l, max_iter, _fptr(out["time"]), _fptr(out["tdl1"]),
                            _fptr(out["tds1"]), _fptr(out.get("gradz")), _fptr(out.get("gradx")),
                            sweeps.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    if rc != 0:
        raise RuntimeError("oracle_eikods failed: %d" % rc)
    out["sweeps"] = sweeps
    return out


def rel_l2(a, b) -> float:
    """||a-b|| / ||b|| in double, the reference comparator (src/rsf_l2cmp.cpp:9-10)."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    num = np.sum((a - b) ** 2)
    den = np.sum(b * b)
    return float(np.sqrt(num / (den + 1e-30)))
