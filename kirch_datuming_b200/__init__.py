"""B200-native adjoint angle-domain Kirchhoff CIG migration (kirchmig2d_cig adj=1).

The compute path is the in-tree CUDA library ``libkcig.so`` (C ABI declared in
include/kcig.h).  This module is its thin Python face, mirroring the
reference's interface: parameters are the tool's own ``key=value`` strings,
arrays use the reference layouts (data [ns][nh][nt], tables [npos][nx][nz],
image [ng][nx][nz]).  There is no CPU implementation behind it: if the
library is missing or no GPU is present, calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = ["lib", "KcigError", "Params", "Geometry", "params", "geometry", "output_axis", "Plan",
           "run_cli", "doubint_device", "leg_fields_device", "shot_positions", "stitch_windows", "eikonal_tables", "eikods", "library_path",
           "cli_path", "eikods_cli_path", "kirchmig2d_cli_path", "layercom_cig_cli_path", "params_kirchmig2d",
           "stitch_window"]

_HERE = os.path.dirname(os.path.abspath(__file__))
library_path = os.path.join(_HERE, "libkcig.so")
cli_path = os.path.join(_HERE, "bin", "kirchmig2d_cig")
kirchmig2d_cli_path = os.path.join(_HERE, "bin", "kirchmig2d")
eikods_cli_path = os.path.join(_HERE, "bin", "eikods2d")
layercom_cig_cli_path = os.path.join(_HERE, "bin", "layercom_cig")
greensol_auto_cli_path = os.path.join(_HERE, "bin", "greensol_auto")
kirchdat2d_freq_cli_path = os.path.join(_HERE, "bin", "kirchdat2d_freq")

MEM_HOST = 0
MEM_DEVICE = 1
MEM_HOST_STREAM = 2


class KcigError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("kcig error %d: %s" % (code, msg))
        self.code = code
        self.msg = msg


class SurrogateConfig(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_float * 3), ("hi", ctypes.c_float * 3), ("fmax", ctypes.c_float),
                ("vref", ctypes.c_float), ("zsrc", ctypes.c_float), ("vgrad", ctypes.c_float),
                ("residual_ms", ctypes.c_float)]


class EikodsOpts(ctypes.Structure):
    """kcig_eikods_opts (include/kcig.h)."""
    _fields_ = [("order", ctypes.c_int), ("b1", ctypes.c_int), ("b2", ctypes.c_int), ("l", ctypes.c_int),
                ("vel_is_slowness2", ctypes.c_int), ("max_iter", ctypes.c_int)]


class Shot(ctypes.Structure):
    _fields_ = [("sx", ctypes.c_float), ("nh", ctypes.c_int), ("h0", ctypes.c_float), ("dh", ctypes.c_float),
                ("nt", ctypes.c_int), ("data", ctypes.c_void_p), ("h", ctypes.c_void_p)]


class Params(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "adj", "cig", "cig_is_angle", "cmp", "half_angle", "isdiff", "interp_type", "angle_interp",
        "angle_grad_radius", "angle_smooth", "aperture_trace", "aperture_trace_taper", "direct_mute",
        "direct_mute_invert", "direct_mute_qc_shot")] + [(n, ctypes.c_float) for n in (
        "tau", "aperture", "aperture_taper", "aperture_rmin", "aperture_rtaper", "antialias",
        "angle_taper_start", "angle_taper_end", "oazmin", "oazmax", "oaztaper", "direct_mute_slope",
        "direct_mute_intercept", "direct_mute_taper")] + [(n, ctypes.c_int) for n in (
        "axis_min_given", "axis_max_given", "axis_step_given", "axis_n_given")] + [
        (n, ctypes.c_float) for n in ("axis_min", "axis_max", "axis_step")] + [("axis_n", ctypes.c_int),
                                                                             ("tool", ctypes.c_int)]


class Geometry(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("nt", "nh", "ns")] + \
               [(n, ctypes.c_float) for n in ("t0", "dt", "h0", "dh", "s0", "ds")] + \
               [(n, ctypes.c_int) for n in ("nz", "nx")] + \
               [(n, ctypes.c_float) for n in ("z0", "dz", "x0", "dx")] + \
               [("sny", ctypes.c_int)] + [(n, ctypes.c_float) for n in ("sy0", "sdy")] + \
               [("rny", ctypes.c_int)] + [(n, ctypes.c_float) for n in ("ry0", "rdy")]


_lib = None


def lib():
    """Load libkcig.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(library_path):
            raise ImportError("libkcig.so is missing: build it with `python -m kirch_datuming_b200.build` (%s)"
                              % library_path)
        L = ctypes.CDLL(library_path)
        P, G = ctypes.POINTER(Params), ctypes.POINTER(Geometry)
        vp, fp, dp = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p
        L.kcig_last_error.restype = ctypes.c_char_p
        L.kcig_params_init.argtypes = [P]
        L.kcig_params_parse.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), P]
        L.kcig_params_parse_kirchmig2d.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), P]
        L.kcig_run_kirchmig2d_cli.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]
        L.kcig_output_axis.argtypes = [P, G, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float),
                                       ctypes.POINTER(ctypes.c_float)]
        L.kcig_plan_create.argtypes = [P, G, ctypes.c_ulonglong, ctypes.POINTER(vp)]
        L.kcig_plan_destroy.argtypes = [vp]
        L.kcig_plan_set_stream.argtypes = [vp, vp]
        L.kcig_plan_set_tables.argtypes = [vp, fp, fp, fp, fp, ctypes.c_int]
        L.kcig_plan_set_gradients.argtypes = [vp, fp, fp, fp, fp, ctypes.c_int]
        L.kcig_migrate.argtypes = [vp, fp, fp, ctypes.c_int]
        L.kcig_model.argtypes = [vp, fp, fp, ctypes.c_int]
        L.kcig_plan_last_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float),
                                           ctypes.POINTER(ctypes.c_int)]
        L.kcig_run_cli.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]
        L.kcig_doubint_device.argtypes = [fp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, vp]
        L.kcig_leg_fields_device.argtypes = [vp, ctypes.c_int, ctypes.c_double, dp, fp, dp, fp]
        L.kcig_eikonal_tables.argtypes = [fp, ctypes.c_int, ctypes.c_int] + [ctypes.c_float] * 4 + [
            ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            fp, fp, vp]
        L.kcig_eikods.argtypes = ([fp, ctypes.c_int, ctypes.c_int] + [ctypes.c_float] * 6
                                  + [fp, ctypes.c_int, ctypes.POINTER(EikodsOpts)] + [fp] * 5
                                  + [ctypes.POINTER(ctypes.c_int), vp])
        L.kcig_tc_selftest.argtypes = [vp, vp, fp, vp, vp]
        SC = ctypes.POINTER(SurrogateConfig)
        L.kcig_surrogate_create.argtypes = [SC, ctypes.c_ulonglong, ctypes.POINTER(vp)]
        L.kcig_surrogate_destroy.argtypes = [vp]
        L.kcig_surrogate_destroy.restype = None
        L.kcig_surrogate_set_params.argtypes = [vp, fp]
        L.kcig_surrogate_get_params.argtypes = [vp, fp]
        L.kcig_surrogate_eval.argtypes = [vp, ctypes.c_int] + [fp] * 7 + [vp]
        L.kcig_surrogate_eval_stages.argtypes = [vp, ctypes.c_int] + [fp] * 4 + [vp]
        L.kcig_surrogate_loss_grad.argtypes = [vp, ctypes.c_int] + [fp] * 6 + [vp]
        L.kcig_surrogate_train.argtypes = ([vp, fp, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                            ctypes.c_int] + [ctypes.c_float] * 4 +
                                           [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                            ctypes.c_ulonglong, fp, vp])
        L.kcig_plan_set_surrogate.argtypes = [vp, vp, vp]
        L.kcig_plan_set_shot_range.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.kcig_shot_positions.argtypes = [ctypes.POINTER(Geometry), ctypes.c_int, ctypes.c_int, vp, vp]
        L.kcig_plan_set_surrogate_options.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.kcig_shots_prepare.argtypes = [vp, ctypes.c_int, ctypes.POINTER(Shot), ctypes.c_int]
        L.kcig_migrate_prepared.argtypes = [vp, fp, ctypes.c_int]
        L.kcig_migrate_shots.argtypes = [vp, ctypes.c_int, ctypes.POINTER(Shot), fp, ctypes.c_int]
        L.kcig_plan_set_graph.argtypes = [vp, ctypes.c_int]
        L.kcig_plan_autotune.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)]
        L.kcig_graph_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp)]
        L.kcig_graph_launch.argtypes = [vp, vp]
        L.kcig_graph_destroy.argtypes = [vp]
        L.kcig_graph_destroy.restype = None
        L.kcig_shots_pairs.argtypes = [vp]
        L.kcig_shots_pairs.restype = ctypes.c_longlong
        L.kcig_stitch_windows.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp,
                                          ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, vp, vp]
        L.kcig_stitch_window.argtypes = ([fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, fp, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, ctypes.POINTER(ctypes.c_longlong), vp])
        L.kcig_run_layercom_cig_cli.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]
        L.kcig_plan_last_timing.argtypes = [vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
        L.kcig_plan_last_prelude_ms.argtypes = [vp]
        L.kcig_plan_last_prelude_ms.restype = ctypes.c_float
        DP = ctypes.POINTER(DatumParams)
        L.kcig_datum_params_init.argtypes = [DP]
        L.kcig_datum_sizes.argtypes = [DP, fp, fp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.kcig_datum_freq.argtypes = [DP, vp, vp, vp, vp, vp, ctypes.c_int, vp]
        L.kcig_datum_last_timing.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)]
        L.kcig_datum_release.argtypes = []
        L.kcig_green_slice.argtypes = ([vp, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_float] * 7
                                       + [vp, ctypes.c_int, vp])
        L.kcig_run_greensol_auto_cli.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]
        L.kcig_run_kirchdat2d_freq_cli.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]
        _lib = L
    return _lib


class DatumParams(ctypes.Structure):
    """kcig_datum_params (include/kcig.h): the settings of kirchdat2d_freq."""
    _fields_ = [("nt", ctypes.c_int), ("nh", ctypes.c_int), ("ns", ctypes.c_int), ("dt", ctypes.c_float),
                ("h0", ctypes.c_float), ("dh", ctypes.c_float), ("s0", ctypes.c_float), ("ds", ctypes.c_float),
                ("nsg", ctypes.c_int), ("nrg", ctypes.c_int), ("sg0", ctypes.c_float), ("dsg", ctypes.c_float),
                ("rg0", ctypes.c_float), ("drg", ctypes.c_float), ("sdatum", ctypes.c_float),
                ("rdatum", ctypes.c_float), ("aperture", ctypes.c_int), ("taper", ctypes.c_int),
                ("data_taper", ctypes.c_int), ("cmp", ctypes.c_int), ("antialias", ctypes.c_float),
                ("length", ctypes.c_float), ("use_bf", ctypes.c_int), ("bf_p", ctypes.c_int),
                ("bf_n_leaf", ctypes.c_int), ("bf_panel_levels", ctypes.c_int), ("bf_amp_eps", ctypes.c_float),
                ("bf_phase_tol", ctypes.c_float)]


def _check(rc: int):
    if rc != 0:
        raise KcigError(rc, lib().kcig_last_error().decode())


def _argv(tokens):
    toks = ["kirchmig2d_cig"] + [str(t) for t in tokens]
    arr = (ctypes.c_char_p * len(toks))(*[t.encode() for t in toks])
    return len(toks), arr


def params(*tokens, **kw) -> Params:
    """kcig_params from kirchmig2d_cig key=value tokens (and/or keywords)."""
    toks = list(tokens) + ["%s=%s" % (k, v) for k, v in kw.items()]
    p = Params()
    argc, argv = _argv(toks)
    _check(lib().kcig_params_parse(argc, argv, ctypes.byref(p)))
    return p


def params_kirchmig2d(*tokens, **kw) -> Params:
    """kcig_params from kirchmig2d key=value tokens (tool = 1)."""
    toks = list(tokens) + ["%s=%s" % (k, v) for k, v in kw.items()]
    p = Params()
    argc, argv = _argv(toks)
    _check(lib().kcig_params_parse_kirchmig2d(argc, argv, ctypes.byref(p)))
    return p


def geometry(**kw) -> Geometry:
    g = Geometry()
    for k, v in kw.items():
        setattr(g, k, v)
    return g


def output_axis(p: Params, g: Geometry):
    ng, g0, dg = ctypes.c_int(), ctypes.c_float(), ctypes.c_float()
    _check(lib().kcig_output_axis(ctypes.byref(p), ctypes.byref(g), ctypes.byref(ng), ctypes.byref(g0),
                                  ctypes.byref(dg)))
    return ng.value, g0.value, dg.value


def _ptr(a):
    """(pointer, memory kind) of a numpy array or a CUDA torch tensor."""
    if a is None:
        return None, MEM_HOST
    if isinstance(a, np.ndarray):
        return a.ctypes.data, MEM_HOST
    if hasattr(a, "data_ptr"):
        return a.data_ptr(), (MEM_DEVICE if a.is_cuda else MEM_HOST)
    raise TypeError(type(a))


class Plan:
    """One migration set-up: kcig_plan_create + tables, then migrate() calls."""

    def __init__(self, p: Params, g: Geometry, scratch_bytes: int = 0, stream=None):
        self._h = ctypes.c_void_p()
        _check(lib().kcig_plan_create(ctypes.byref(p), ctypes.byref(g), scratch_bytes, ctypes.byref(self._h)))
        self.params, self.geometry = p, g
        self.ng, self.g0, self.dg = output_axis(p, g)
        self._keep = []
        if stream is not None:
            _check(lib().kcig_plan_set_stream(self._h, ctypes.c_void_p(stream)))

    def set_tables(self, stable, sderiv, rtable=None, rderiv=None, stream=False):
        """stream=True (host arrays only): the tables stay in host memory and
        each leg batch copies the slices it needs (KCIG_MEM_HOST_STREAM)."""
        rtable = stable if rtable is None else rtable
        rderiv = sderiv if rderiv is None else rderiv
        ptrs = [_ptr(x) for x in (stable, sderiv, rtable, rderiv)]
        mem = {m for _, m in ptrs}
        if len(mem) != 1:
            raise ValueError("tables must all be host or all be device arrays")
        mem = mem.pop()
        if stream:
            if mem != MEM_HOST:
                raise ValueError("stream=True needs host tables")
            mem = MEM_HOST_STREAM
        self._keep += [stable, sderiv, rtable, rderiv]
        _check(lib().kcig_plan_set_tables(self._h, *[p for p, _ in ptrs], mem))

    def set_shot_range(self, first: int = 0, count: int = -1):
        """Migrate only shots first .. first + count - 1 of the survey, at
        their positions in the whole survey (kcig_plan_set_shot_range); the
        data passed to migrate() then holds just those shots."""
        _check(lib().kcig_plan_set_shot_range(self._h, int(first), int(count)))

    def set_gradients(self, sgradx, sgradz, rgradx, rgradz):
        ptrs = [_ptr(x) for x in (sgradx, sgradz, rgradx, rgradz)]
        self._keep += [sgradx, sgradz, rgradx, rgradz]
        _check(lib().kcig_plan_set_gradients(self._h, *[p for p, _ in ptrs], ptrs[0][1]))

    def set_surrogate(self, src=None, rcv=None, angle: str = "fd", tx: str = "network"):
        """Leg fields of the source / receiver legs from Surrogate objects
        instead of the tables (None: that side uses its tables).  angle:
        "fd" (the tables' finite-difference gradient of the surrogate's
        traveltime) or "network" (its input gradient); tx: the antialias
        derivative from the "network" or from the "table"
        (kcig_plan_set_surrogate_options)."""
        self._keep += [src, rcv]
        _check(lib().kcig_plan_set_surrogate(self._h, src.handle if src else None, rcv.handle if rcv else None))
        a = {"fd": 0, "network": 1}[angle]
        t = {"network": 0, "table": 1}[tx]
        _check(lib().kcig_plan_set_surrogate_options(self._h, a, t))

    def prepare_shots(self, shots):
        """Upload ragged shots (include/kcig.h kcig_shot): a list of dicts with
        sx, h0, dh (or h: the receiver axis values) and data [nh][nt] (numpy
        float32 or CUDA float32 tensor)."""
        arr = (Shot * max(1, len(shots)))()
        mems = set()
        keep = []
        for i, s in enumerate(shots):
            d = s["data"]
            if hasattr(d, "is_cuda"):
                d = d.contiguous()
            else:
                import numpy as np
                d = np.ascontiguousarray(d, dtype=np.float32)
            keep.append(d)
            p, m = _ptr(d)
            mems.add(m)
            nh, nt = d.shape
            hp = None
            if s.get("h") is not None:
                import numpy as np
                hv = np.ascontiguousarray(s["h"], dtype=np.float32)
                if hv.size != nh:
                    raise ValueError("shot %d: h has %d values for %d receivers" % (i, hv.size, nh))
                keep.append(hv)
                hp = hv.ctypes.data
            arr[i] = Shot(float(s["sx"]), int(nh), float(s.get("h0", 0.0)), float(s.get("dh", 0.0)), int(nt),
                          ctypes.c_void_p(p), ctypes.c_void_p(hp))
        if len(mems) > 1:
            raise ValueError("shots must all be host or all be device arrays")
        _check(lib().kcig_shots_prepare(self._h, len(shots), arr, mems.pop() if mems else 0))
        return int(lib().kcig_shots_pairs(self._h))

    def migrate_prepared(self, image):
        ip, m = _ptr(image)
        _check(lib().kcig_migrate_prepared(self._h, ip, m))
        return image

    def autotune(self):
        """Pick the summation's tile variant for the prepared shots; returns
        (variant, {variant: ms})."""
        c = ctypes.c_int()
        ms = (ctypes.c_float * 5)()
        _check(lib().kcig_plan_autotune(self._h, ctypes.byref(c), ms))
        return c.value, {i: ms[i] for i in range(1, 5)}

    def set_graph(self, enable=True):
        _check(lib().kcig_plan_set_graph(self._h, 1 if enable else 0))

    def model(self, image, data):
        """Forward modelling (adj=0): data [ns][nh][nt] from image [ng][nx][nz]."""
        (ip, m1), (dp_, m2) = _ptr(image), _ptr(data)
        if m1 != m2:
            raise ValueError("image and data must both be host or both be device arrays")
        _check(lib().kcig_model(self._h, ip, dp_, m1))
        return data

    def migrate(self, data, image):
        (dp_, m1), (ip, m2) = _ptr(data), _ptr(image)
        if m1 != m2:
            raise ValueError("data and image must both be host or both be device arrays")
        _check(lib().kcig_migrate(self._h, dp_, ip, m1))
        return image

    def timing(self):
        """Device ms of the last migration in leg fields and in the summation."""
        f, m = ctypes.c_float(), ctypes.c_float()
        _check(lib().kcig_plan_last_timing(self._h, ctypes.byref(f), ctypes.byref(m)))
        return {"fields_ms": f.value, "sum_ms": m.value, "prelude_ms": float(lib().kcig_plan_last_prelude_ms(self._h))}

    def stats(self):
        a, b, c = ctypes.c_int(), ctypes.c_float(), ctypes.c_int()
        _check(lib().kcig_plan_last_stats(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return {"sum_launches": a.value, "sum_ms": b.value, "launches": c.value}

    def close(self):
        if self._h:
            lib().kcig_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_cli(args) -> int:
    """In-process kirchmig2d_cig; returns 0 or the negative KCIG_ERR_* code."""
    argc, argv = _argv(args)
    return lib().kcig_run_cli(argc, argv)


def doubint_device(traces, isdiff: int = 0, dt: float = 1.0, stream=None):
    """doubint (+diff2) of a CUDA float32 tensor [ntr][nt] -> float64 tensor."""
    import torch
    if not (traces.is_cuda and traces.dtype == torch.float32 and traces.is_contiguous()):
        raise ValueError("expects a contiguous CUDA float32 tensor")
    ntr, nt = traces.shape
    out = torch.empty((ntr, nt), dtype=torch.float64, device=traces.device)
    st = torch.cuda.current_stream().cuda_stream if stream is None else stream
    _check(lib().kcig_doubint_device(traces.data_ptr(), out.data_ptr(), ntr, nt, int(isdiff), float(dt),
                                     ctypes.c_void_p(st)))
    torch.cuda.current_stream().synchronize()
    return out


def stitch_window(out, layer, start: int, end: int, previous_end: int = -1, stitch_blend: int = 15,
                  layer_scale: float = 1.0, use_lateral: bool = False, scalex_aper: int = 0,
                  scalex_scale: float = 1.0, stream=None) -> int:
    """One depth window of layercom_cig's stitching on the device
    (kcig_stitch_window): out [n3][n2][n1] and layer [n3][n2][end-start+1],
    contiguous CUDA float32 tensors; out is updated in place.  Returns the
    number of non-finite scaled samples (written as 0)."""
    import torch
    for t in (out, layer):
        if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous() and t.dim() == 3):
            raise ValueError("expects contiguous 3-D CUDA float32 tensors")
    n3, n2, n1 = out.shape
    if tuple(layer.shape) != (n3, n2, end - start + 1):
        raise ValueError("layer shape %s does not match rows %d..%d" % (tuple(layer.shape), start, end))
    st = torch.cuda.current_stream().cuda_stream if stream is None else stream
    bad = ctypes.c_longlong()
    _check(lib().kcig_stitch_window(out.data_ptr(), n1, n2, n3, layer.data_ptr(), int(start), int(end),
                                    int(previous_end), int(stitch_blend), float(layer_scale), int(bool(use_lateral)),
                                    int(scalex_aper), float(scalex_scale), ctypes.byref(bad), ctypes.c_void_p(st)))
    return bad.value


def stitch_windows(out, layers, windows, stitch_blend: int = 15, scales=None, use_lateral: bool = False,
                   scalex_aper: int = 0, scalex_scale: float = 1.0, stream=None):
    """Every depth window of one stitch in a single device pass
    (kcig_stitch_windows): out [n3][n2][n1] (overwritten; rows no window
    covers become 0), layers[k] [n3][n2][e-s+1] for windows[k] = (s, e),
    contiguous CUDA float32 tensors.  Returns the non-finite count per window."""
    import torch
    n3, n2, n1 = out.shape
    nw = len(windows)
    if len(layers) != nw or nw < 1:
        raise ValueError("one layer per window")
    for t, (s0, e0) in zip([out] + list(layers), [(0, n1 - 1)] + list(windows)):
        if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous() and t.dim() == 3):
            raise ValueError("expects contiguous 3-D CUDA float32 tensors")
        if tuple(t.shape) != (n3, n2, e0 - s0 + 1):
            raise ValueError("layer shape %s does not match rows %d..%d" % (tuple(t.shape), s0, e0))
    scales = [1.0] * nw if scales is None else list(scales)
    ptrs = (ctypes.c_void_p * nw)(*[t.data_ptr() for t in layers])
    starts = (ctypes.c_int * nw)(*[int(w[0]) for w in windows])
    ends = (ctypes.c_int * nw)(*[int(w[1]) for w in windows])
    sc = (ctypes.c_float * nw)(*[float(x) for x in scales])
    bad = (ctypes.c_longlong * nw)()
    st = torch.cuda.current_stream().cuda_stream if stream is None else stream
    _check(lib().kcig_stitch_windows(out.data_ptr(), n1, n2, n3, nw, ptrs, starts, ends, int(stitch_blend), sc,
                                     int(bool(use_lateral)), int(scalex_aper), float(scalex_scale), bad,
                                     ctypes.c_void_p(st)))
    return [int(b) for b in bad]


def shot_positions(g: Geometry, first: int = 0, count: int = None):
    """(FP64, FP32) shot positions of the survey axis as the migration uses
    them (kcig_shot_positions); host-only."""
    import numpy as np
    count = g.ns - first if count is None else count
    pos, posf = np.empty(count, np.float64), np.empty(count, np.float32)
    _check(lib().kcig_shot_positions(ctypes.byref(g), int(first), int(count), pos.ctypes.data, posf.ctypes.data))
    return pos, posf


def leg_fields_device(plan: Plan, is_source: int, pos: float):
    """(T float64, Tx float32, phi float64, w float32) device tensors [nx*nz] of one leg."""
    import torch
    g = plan.geometry
    n = g.nz * g.nx
    T, phi = (torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(2))
    Tx, w = (torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(2))
    _check(lib().kcig_leg_fields_device(plan._h, int(is_source), float(pos), T.data_ptr(), Tx.data_ptr(),
                                        phi.data_ptr(), w.data_ptr()))
    return T, Tx, phi, w


def eikods(vel, d1: float, d2: float, shots, o1: float = 0.0, o2: float = 0.0, o3: float = 0.0, d3: float = 1.0,
           order: int = 2, b1: int = 2, b2: int = 2, l: int = 1, vel_is_slowness2: bool = False,
           max_iter: int = 0, derivs: bool = True, grads: bool = False):
    """eikods2d's tables on the GPU (kcig_eikods).

    vel: CUDA float32 tensor [nx][nz] (velocity, or slowness squared with
    vel_is_slowness2); shots: [nshot][3] (depth, lateral, third axis) as in
    an eikods2d shot file.  Returns a dict of CUDA tensors [nshot][nx][nz]:
    'time', and 'tdl1'/'tds1' (derivs), 'gradz'/'gradx' (grads), plus
    'sweeps' (numpy [nshot], the sweeps each source took)."""
    import numpy as np
    import torch
    if not (vel.is_cuda and vel.dtype == torch.float32 and vel.is_contiguous() and vel.dim() == 2):
        raise ValueError("vel must be a contiguous CUDA float32 tensor [nx][nz]")
    nx, nz = vel.shape
    sh = np.ascontiguousarray(np.asarray(shots, dtype=np.float32).reshape(-1, 3))
    ns = sh.shape[0]
    new = lambda: torch.empty((ns, nx, nz), dtype=torch.float32, device=vel.device)  # noqa: E731
    out = {"time": new()}
    if derivs:
        out["tdl1"], out["tds1"] = new(), new()
    if grads:
        out["gradz"], out["gradx"] = new(), new()
    o = EikodsOpts(order, b1, b2, l, 1 if vel_is_slowness2 else 0, max_iter)
    sweeps = np.zeros(ns, np.int32)
    ptr = lambda k: out[k].data_ptr() if k in out else None  # noqa: E731
    st = torch.cuda.current_stream().cuda_stream
    _check(lib().kcig_eikods(vel.data_ptr(), nz, nx, o1, o2, d1, d2, o3, d3, sh.ctypes.data, ns, ctypes.byref(o),
                             ptr("time"), ptr("tdl1"), ptr("tds1"), ptr("gradz"), ptr("gradx"),
                             sweeps.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.c_void_p(st)))
    out["sweeps"] = sweeps
    return out


def eikonal_tables(vel, dz: float, dx: float, npos: int, p0: float, dp: float, z0: float = 0.0,
                   x0: float = 0.0, zsrc: float = 0.0, b1: int = 2, b2: int = 2, iterations: int = 0,
                   deriv: bool = True):
    """Traveltime tables on the GPU for sources at depth zsrc and lateral
    positions p0 + k*dp (k < npos): eikods with order 2 (the eikods2d
    default); deriv is tds1.  iterations bounds the sweep iterations (0 =
    the library default).

    vel: CUDA float32 tensor [nx][nz] (km/s).  Returns (time, deriv) CUDA
    tensors [npos][nx][nz] (deriv None when not requested)."""
    import torch
    if not (vel.is_cuda and vel.dtype == torch.float32 and vel.is_contiguous()):
        raise ValueError("vel must be a contiguous CUDA float32 tensor [nx][nz]")
    nx, nz = vel.shape
    t = torch.empty((npos, nx, nz), dtype=torch.float32, device=vel.device)
    d = torch.empty_like(t) if deriv else None
    st = torch.cuda.current_stream().cuda_stream
    _check(lib().kcig_eikonal_tables(vel.data_ptr(), nz, nx, dz, dx, z0, x0, npos, p0, dp, zsrc, b1, b2,
                                     iterations, t.data_ptr(), d.data_ptr() if deriv else None,
                                     ctypes.c_void_p(st)))
    return t, d


def tc_selftest(X, W):
    """Tensor-core layout self-test: for 128x128 CUDA bfloat16 tensors X, W
    returns the CUDA float32 tensor [3][128][128] of X W^T, X W and X^T W as
    computed by the surrogate's tcgen05 operand views."""
    import torch
    for t in (X, W):
        if not (t.is_cuda and t.dtype == torch.bfloat16 and t.shape == (128, 128) and t.is_contiguous()):
            raise ValueError("X and W must be contiguous 128x128 CUDA bfloat16 tensors")
    D = torch.empty((3, 128, 128), dtype=torch.float32, device=X.device)
    status = torch.zeros(1, dtype=torch.int32, device=X.device)
    st = torch.cuda.current_stream().cuda_stream
    _check(lib().kcig_tc_selftest(X.data_ptr(), W.data_ptr(), D.data_ptr(), status.data_ptr(), ctypes.c_void_p(st)))
    if int(status.item()) != 0:
        raise KcigError(-6, "tensor-core self-test: the MMA did not complete")
    return D


class Surrogate:
    """Learned traveltime surrogate T(xs, z, x) = Tb + residual_ms * 1e-3 * out
    (or Tb * (1 + out) with residual_ms = 0), Tb the first arrival of the
    background medium vref + vgrad * (z - zsrc) (include/kcig.h,
    kcig_surrogate_*): trained and evaluated by the library's tensor-core
    kernels on the current CUDA device.  lo/hi: domain of (xs, z, x) in km."""

    def __init__(self, lo, hi, fmax: float = 8.0, vref: float = 1.5, zsrc: float = 0.0, seed: int = 0,
                 vgrad: float = 0.0, residual_ms: float = 0.0):
        c = SurrogateConfig()
        for i in range(3):
            c.lo[i], c.hi[i] = float(lo[i]), float(hi[i])
        c.fmax, c.vref, c.zsrc = float(fmax), float(vref), float(zsrc)
        c.vgrad, c.residual_ms = float(vgrad), float(residual_ms)
        self.config = c
        h = ctypes.c_void_p()
        _check(lib().kcig_surrogate_create(ctypes.byref(c), int(seed), ctypes.byref(h)))
        self._h = h
        self.nparams = int(lib().kcig_surrogate_nparams())

    @property
    def handle(self):
        return self._h

    def get_params(self):
        import numpy as np
        p = np.empty(self.nparams, np.float32)
        _check(lib().kcig_surrogate_get_params(self._h, p.ctypes.data))
        return p

    def set_params(self, params):
        import numpy as np
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.nparams:
            raise ValueError("expected %d parameters" % self.nparams)
        _check(lib().kcig_surrogate_set_params(self._h, p.ctypes.data))

    @staticmethod
    def _dev(a, n=None):
        import torch
        t = torch.as_tensor(a, dtype=torch.float32).cuda().contiguous()
        if n is not None and t.numel() != n:
            raise ValueError("length mismatch")
        return t

    def eval(self, xs, z, x):
        """(T, dT/dxs, dT/dz, dT/dx) at the points, as CUDA float32 tensors."""
        import torch
        xs = self._dev(xs)
        n = xs.numel()
        z, x = self._dev(z, n), self._dev(x, n)
        out = [torch.empty(n, dtype=torch.float32, device=xs.device) for _ in range(4)]
        st = torch.cuda.current_stream().cuda_stream
        _check(lib().kcig_surrogate_eval(self._h, n, xs.data_ptr(), z.data_ptr(), x.data_ptr(),
                                         *[o.data_ptr() for o in out], ctypes.c_void_p(st)))
        return tuple(out)

    def eval_stages(self, xs, z, x):
        """FP32 accumulators of the first 128-point tile, [5][128][128]
        (kcig_surrogate_eval_stages)."""
        import torch
        xs = self._dev(xs)
        n = xs.numel()
        z, x = self._dev(z, n), self._dev(x, n)
        out = torch.zeros((8, 128, 128), dtype=torch.float32, device=xs.device)
        st = torch.cuda.current_stream().cuda_stream
        _check(lib().kcig_surrogate_eval_stages(self._h, n, xs.data_ptr(), z.data_ptr(), x.data_ptr(),
                                                out.data_ptr(), ctypes.c_void_p(st)))
        return out

    def loss_grad(self, xs, z, x, Ttrue):
        """Loss of the batch (ms^2) and its parameter gradient (CUDA tensor)."""
        import torch
        xs = self._dev(xs)
        n = xs.numel()
        z, x, Tt = self._dev(z, n), self._dev(x, n), self._dev(Ttrue, n)
        loss = torch.empty(1, dtype=torch.float32, device=xs.device)
        grad = torch.empty(self.nparams, dtype=torch.float32, device=xs.device)
        st = torch.cuda.current_stream().cuda_stream
        _check(lib().kcig_surrogate_loss_grad(self._h, n, xs.data_ptr(), z.data_ptr(), x.data_ptr(), Tt.data_ptr(),
                                              loss.data_ptr(), grad.data_ptr(), ctypes.c_void_p(st)))
        return float(loss.item()), grad

    def train(self, table, p0: float, dp: float, z0: float, dz: float, x0: float, dx: float, steps: int,
              batch: int = 16384, lr: float = 2e-3, lr_final: float = 2e-5, seed: int = 1):
        """Adam on uniform samples of a CUDA table volume [npos][nx][nz];
        returns the per-step losses (ms^2) as a numpy array."""
        import numpy as np
        import torch
        if not (table.is_cuda and table.dtype == torch.float32 and table.is_contiguous() and table.dim() == 3):
            raise ValueError("table must be a contiguous CUDA float32 tensor [npos][nx][nz]")
        npos, nx, nz = table.shape
        losses = np.zeros(max(steps, 1), np.float32)
        st = torch.cuda.current_stream().cuda_stream
        _check(lib().kcig_surrogate_train(self._h, table.data_ptr(), npos, p0, dp, nz, nx, z0, dz, x0, dx, steps,
                                          batch, lr, lr_final, int(seed), losses.ctypes.data, ctypes.c_void_p(st)))
        return losses[:steps]

    def close(self):
        if getattr(self, "_h", None):
            lib().kcig_surrogate_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    """One CUDA graph over several prepared plans (kcig_graph_*): replaying it
    migrates every plan's prepared shots into that plan's device image."""

    def __init__(self, plans, images):
        n = len(plans)
        ps = (ctypes.c_void_p * n)(*[p._h.value for p in plans])
        ims = (ctypes.c_void_p * n)(*[_ptr(im)[0] for im in images])
        self._keep = (list(plans), list(images))
        self._h = ctypes.c_void_p()
        _check(lib().kcig_graph_create(n, ps, ims, ctypes.byref(self._h)))

    def launch(self, stream=None):
        import torch
        st = torch.cuda.current_stream().cuda_stream if stream is None else stream
        _check(lib().kcig_graph_launch(self._h, ctypes.c_void_p(st)))

    def close(self):
        if getattr(self, "_h", None):
            lib().kcig_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------ datuming between depth levels

def datum_params(**kw) -> DatumParams:
    """kcig_datum_params with the reference's defaults, then the given fields."""
    p = DatumParams()
    _check(lib().kcig_datum_params_init(ctypes.byref(p)))
    for k, v in kw.items():
        if not any(f[0] == k for f in DatumParams._fields_):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def datum_sizes(p: DatumParams, stable, rtable):
    """(nsam, nfft) of a run (kcig_datum_sizes); host float32 tables."""
    st = np.ascontiguousarray(stable, np.float32)
    rt = np.ascontiguousarray(rtable, np.float32)
    nsam, nfft = ctypes.c_int(), ctypes.c_int()
    _check(lib().kcig_datum_sizes(ctypes.byref(p), st.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                  rt.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(nsam),
                                  ctypes.byref(nfft)))
    return nsam.value, nfft.value


def datum_freq(p: DatumParams, stable, rtable, data, out, interm=None, stream=None):
    """kcig_datum_freq: data [ns][nh][nt] -> out (and interm) of the same shape.
    All arrays host (contiguous float32 numpy) or all CUDA float32 tensors."""
    ptrs = [_ptr(a) for a in (stable, rtable, data, out)]
    kinds = {k for _, k in ptrs}
    if interm is not None:
        kinds.add(_ptr(interm)[1])
    if len(kinds) != 1:
        raise ValueError("datum_freq: all arrays host or all device")
    for a in (stable, rtable, data, out) + ((interm,) if interm is not None else ()):
        if isinstance(a, np.ndarray) and (a.dtype != np.float32 or not a.flags.c_contiguous):
            raise ValueError("datum_freq: contiguous float32 arrays")
    st = stream
    if st is None and kinds == {MEM_DEVICE}:
        import torch
        st = torch.cuda.current_stream().cuda_stream
    _check(lib().kcig_datum_freq(ctypes.byref(p), ptrs[0][0], ptrs[1][0], ptrs[2][0], ptrs[3][0],
                                 _ptr(interm)[0] if interm is not None else None, kinds.pop(),
                                 ctypes.c_void_p(st) if st else None))
    return out


def datum_last_timing():
    """(forward, operators, receiver side, source side, inverse) ms and the
    kernel launches of the last datum_freq call on this thread."""
    ms = (ctypes.c_float * 5)()
    n = ctypes.c_int()
    _check(lib().kcig_datum_last_timing(ms, ctypes.byref(n)))
    return list(ms), n.value


def datum_release():
    """Free the device buffers and cuFFT plans datum_freq keeps between calls
    on the current device (kcig_datum_release)."""
    _check(lib().kcig_datum_release())


def green_slice(table, nz: int, nx: int, ngx: int, oz: float, ox: float, dz: float, dx: float, ogx: float,
                dgx: float, datum: float, out, stream=None):
    """kcig_green_slice: tgreen [ngx][ngx] from a table [ngx][nx][nz] (both
    host numpy or both CUDA tensors)."""
    (tp, tk), (op, ok) = _ptr(table), _ptr(out)
    if tk != ok:
        raise ValueError("green_slice: table and output in the same memory")
    st = stream
    if st is None and tk == MEM_DEVICE:
        import torch
        st = torch.cuda.current_stream().cuda_stream
    _check(lib().kcig_green_slice(tp, nz, nx, ngx, oz, ox, dz, dx, ogx, dgx, datum, op, tk,
                                  ctypes.c_void_p(st) if st else None))
    return out
