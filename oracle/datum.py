"""TEST INFRASTRUCTURE -- the checker of the datuming path, never the product.

FP64 NumPy restatement of the reference's recursive-layer datuming tools:

* ``greensol``      -- src/greensol_auto.cpp:48-95 (the datum-depth slice of a
  traveltime table: tgreen[gx1][gx2] = T(gx1; x = gx2, z = datum));
* ``kirchdat2d_freq`` -- src/kirchdat2d_frequency_cs.cpp:1177-1413 with the direct
  (``use_bf=0``) receiver and source operators (:493-672): time reversal, data
  edge taper (:255-279), real FFT of length nfft (:82-96), per frequency the
  receiver-side then the source-side Kirchhoff summation with the filter
  H(tau, w) (:98-182), the aperture taper (:229-240), the operator
  anti-aliasing weight (:197-226), inverse FFT, 1/nfft, time reversal
  (:470-491).

Every value is carried in float64.  Integer decisions that the reference makes
in float32 (table indices, nsam, the common-receiver walk of cmp=1) are
evaluated in float32 exactly as the reference evaluates them, so that the
oracle sums the same terms; the weights, filters and phases then follow in
float64.  The butterfly (``use_bf=1``, SERECKIRCH/src/bf1d.cpp) approximates
this same operator and is not restated: its outputs are checked against this
direct operator with the butterfly's own approximation error.

Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU baseline use this
module.
"""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32


def _i(x) -> int:
    """C's float -> int conversion (truncation toward zero)."""
    return int(math.trunc(float(x)))


# ------------------------------------------------------------------ greensol --

def greensol(table: np.ndarray, nz: int, nx: int, oz: float, ox: float, dz: float, dx: float,
             ngx: int, ogx: float, dgx: float, datum: float) -> np.ndarray:
    """tgreen[igx1, igx2] = table[igx1, ix2, idatum] (src/greensol_auto.cpp:71-93).

    ``table`` is the (ngx, nx, nz) float32 cube of eikods2d; ``datum`` is
    (float)(o1 + should_datum * d1) of the layer model.  Raises ValueError with
    the reference's error text where it stops."""
    table = np.asarray(table, np.float32).reshape(ngx, nx, nz)
    datum, oz, dz, ox, dx, ogx, dgx = (f32(v) for v in (datum, oz, dz, ox, dx, ogx, dgx))
    idatum = _i(float((datum - oz) / dz) + 0.5)
    if idatum < 0 or idatum >= nz:
        raise ValueError("Datum out of range.")
    out = np.empty((ngx, ngx), np.float32)
    for i1 in range(ngx):
        gx1 = ogx + f32(i1) * dgx
        ix1 = _i(float((gx1 - ox) / dx) + 0.5)
        for i2 in range(ngx):
            gx2 = ogx + f32(i2) * dgx
            ix2 = _i(float((gx2 - ox) / dx) + 0.5)
            if ix1 < 0 or ix1 >= nx or ix2 < 0 or ix2 >= nx:
                raise ValueError("Receiver table too small.")
            out[i1, i2] = table[i1, ix2, idatum]
    return out


# ----------------------------------------------------------- kirchdat2d_freq --

def nsam_of(length: float, dt: float) -> int:
    """ctx.nsam = (int)(length / dt) + 2 in float32 (:1343)."""
    return _i(f32(length) / f32(dt)) + 2


def choose_nfft(nt: int, nsam: int, dt: float, rtable: np.ndarray, stable: np.ndarray) -> int:
    """:82-96: the next power of two above nt + the longest shift + the filter."""
    max_tau = f32(0.0)
    for t in (rtable, stable):
        m = f32(np.max(t)) if t.size else f32(0.0)
        if m > max_tau:
            max_tau = m
    pmax = int(math.ceil(float(f32(max_tau / f32(dt))))) + (nsam - 2)
    n, p = nt + pmax + 2, 1
    while p < n:
        p <<= 1
    return p


def filter_F(tau: np.ndarray, dt: float, nsam: int) -> np.ndarray:
    """build_filter_F (:98-116): F[k], k = 0..nsam-2, second differences of
    sqrt(t^2 - 1), t = (tau + (k+1) dt) / tau.  ``tau`` any shape; returns
    (..., nsam-1) float64."""
    tau = np.asarray(tau, np.float64)
    k = np.arange(1, nsam, dtype=np.float64)
    t = (tau[..., None] + k * dt) / tau[..., None]
    c = np.sqrt(t * t - 1.0)                       # curr at k = 0..nsam-2
    prev1 = np.concatenate([np.zeros_like(c[..., :1]), c[..., :-1]], axis=-1)
    prev2 = np.concatenate([np.zeros_like(c[..., :2]), c[..., :-2]], axis=-1)[..., :c.shape[-1]]
    return c - 2.0 * prev1 + prev2


def filter_H(tau: np.ndarray, dt: float, nsam: int, nfft: int, iw: np.ndarray) -> np.ndarray:
    """build_H_iw (:118-182) in float64 for every tau (shape T) and frequency
    index iw (shape W): H[..., w] = lin * sum_k F[k]/dt exp(-i w k),
    lin = (1-delta) exp(-i w m) + delta exp(-i w (m-1)), m = ceil(tau/dt),
    delta = m - tau/dt, w = 2 pi iw / nfft.  tau <= 0 or non-finite -> 0."""
    tau = np.asarray(tau, np.float64)
    iw = np.asarray(iw, np.int64)
    if nsam < 2:   # no filter samples: the sum is empty
        return np.zeros(tau.shape + iw.shape, np.complex128)
    ok = np.isfinite(tau) & (tau > 0.0)
    ts = np.where(ok, tau, 1.0)
    F = filter_F(ts, dt, nsam) / dt                               # (..., K)
    K = F.shape[-1]
    k = np.arange(K, dtype=np.int64)
    # exact phase reduction: exp(-2 pi i (iw k mod nfft) / nfft)
    ph = -2.0 * np.pi * ((iw[:, None] * k[None, :]) % nfft) / nfft    # (W, K)
    S = F @ np.exp(1j * ph).T                                      # (..., W)
    q = ts / dt
    m = np.ceil(q)
    delta = m - q
    mi = m.astype(np.int64)
    pm = -2.0 * np.pi * ((iw * mi[..., None]) % nfft) / nfft
    pm1 = -2.0 * np.pi * ((iw * (mi[..., None] - 1)) % nfft) / nfft
    lin = (1.0 - delta[..., None]) * np.exp(1j * pm) + delta[..., None] * np.exp(1j * pm1)
    return np.where(ok[..., None], lin * S, 0.0)


def antialias_w(antialias: float, iw: np.ndarray, dtau: np.ndarray, nfft: int, dt: float) -> np.ndarray:
    """antialias_weight_iw (:197-226): 1 below 0.8 fmax, a raised-cosine roll-off
    to 0 at fmax = 0.5 / (|dtau| antialias), 1 when fmax reaches Nyquist.
    Shapes broadcast: dtau (...), iw (W) -> (..., W)."""
    iw = np.asarray(iw, np.float64)
    dtau = np.abs(np.asarray(dtau, np.float64)) * antialias
    out = np.ones(dtau.shape + iw.shape)
    if antialias <= 0.0:
        return out
    freq = iw / (nfft * dt)
    fnyq = 0.5 / dt
    with np.errstate(divide="ignore", invalid="ignore"):
        fmax = 0.5 / dtau
    act = (dtau > 1e-12) & np.isfinite(dtau) & (fmax < fnyq)
    fmax_b = np.where(act, fmax, 1.0)[..., None]
    fpass = 0.8 * fmax_b
    x = (freq - fpass) / (fmax_b - fpass)
    w = np.where(freq <= fpass, 1.0, np.where(freq >= fmax_b, 0.0, 0.5 * (1.0 + np.cos(np.pi * x))))
    w = np.where(iw <= 0, 1.0, w)
    return np.where(act[..., None], w, 1.0)


def taper_w(left: int, center: int, right: int, tap: int, stride: int) -> float:
    """taper_weight (:229-240)."""
    if center < left or center > right:
        return 0.0
    if tap <= 0:
        return 1.0
    stride = max(stride, 1)
    width = float(tap) * float(stride)
    ul = min(1.0, max(0.0, (center - left) / width))
    ur = min(1.0, max(0.0, (right - center) / width))
    return 0.5 * (1.0 - math.cos(math.pi * ul)) * 0.5 * (1.0 - math.cos(math.pi * ur))


def edge_w(i: int, n: int, tap: int) -> float:
    """data_edge_taper_weight (:255-279)."""
    if tap <= 0 or n <= 1:
        return 1.0
    ntap = min(tap, (n - 1) // 2)
    if ntap <= 0:
        return 1.0
    if i < ntap:
        return 0.5 * (1.0 - math.cos(math.pi * i / ntap))
    if i > n - 1 - ntap:
        return 0.5 * (1.0 - math.cos(math.pi * (n - 1 - i) / ntap))
    return 1.0


def slope_of(table: np.ndarray, row: int, col: int, dcoord: float) -> float:
    """table_slope_first_index (:184-194): d tau / d row (centred inside)."""
    n = table.shape[0]
    if n <= 1 or dcoord == 0.0:
        return 0.0
    t = table.astype(np.float64)
    if row <= 0:
        return (t[1, col] - t[0, col]) / dcoord
    if row >= n - 1:
        return (t[n - 1, col] - t[n - 2, col]) / dcoord
    return 0.5 * (t[row + 1, col] - t[row - 1, col]) / dcoord


class Datum:
    """Geometry and parameters of one kirchdat2d_freq run (the FreqContext of
    :37-52).  Arrays: ``stable`` (nsg, nsg) and ``rtable`` (nrg, nrg) float32,
    indexed [cc][c] as the reference does."""

    def __init__(self, nt, nh, ns, dt, h0, dh, s0, ds, stable, sg0, dsg, rtable, rg0, drg, sdatum, rdatum,
                 aperture=50, taper=10, data_taper=0, cmp=1, antialias=1.0, length=0.025):
        self.nt, self.nh, self.ns = int(nt), int(nh), int(ns)
        self.dt, self.h0, self.dh, self.s0, self.ds = (f32(v) for v in (dt, h0, dh, s0, ds))
        self.stable = np.asarray(stable, np.float32)
        self.rtable = np.asarray(rtable, np.float32)
        self.nsg, self.nrg = self.stable.shape[0], self.rtable.shape[0]
        self.sg0, self.dsg, self.rg0, self.drg = (f32(v) for v in (sg0, dsg, rg0, drg))
        self.sdatum, self.rdatum = f32(sdatum), f32(rdatum)
        self.aper, self.tap, self.data_tap, self.cmp = int(aperture), int(taper), int(data_taper), int(cmp)
        self.antialias = float(f32(antialias))
        self.nsam = nsam_of(length, dt)
        self.nfft = choose_nfft(self.nt, self.nsam, self.dt, self.rtable, self.stable)
        self.nw = self.nfft // 2 + 1

    # float32 index helpers, written as the reference writes them
    def rcv_index(self, is_: int, ih: int) -> int:
        """(int)((((cmp ? s0 + is ds : 0) + h0 + ih dh - rg0) / drg) + 0.5f) (:502,:507)."""
        s = (self.s0 + f32(is_) * self.ds) if self.cmp else f32(0.0)
        return _i(((s + self.h0 + f32(ih) * self.dh) - self.rg0) / self.drg + f32(0.5))

    def src_index(self, is_: int) -> int:
        """(int)((s0 + is ds - sg0) / dsg + 0.5f) (:583, :638)."""
        return _i((self.s0 + f32(is_) * self.ds - self.sg0) / self.dsg + f32(0.5))

    def _H(self, table, cc, c, iw):
        return filter_H(np.float64(table[cc, c]), float(self.dt), self.nsam, self.nfft, iw)

    def receiver_terms(self, is_: int):
        """The receiver operator's terms for one shot: list of (ih, ic, w, tau,
        slope) with w the weight before anti-aliasing (:493-546)."""
        out = []
        nh, aper = self.nh, self.aper
        for ih in range(nh):
            c = self.rcv_index(is_, ih)
            left, right = max(0, ih - aper), min(nh - 1, ih + aper)
            for ic in range(left, right + 1):
                cc = self.rcv_index(is_, ic)
                if c < 0 or c >= self.nrg or cc < 0 or cc >= self.nrg:
                    raise ValueError("Receiver table too small.")
                coef = taper_w(left, ic, right, self.tap, 1)
                tau = float(self.rtable[cc, c])
                dist = float(self.rdatum) ** 2 + (ic - ih) ** 2 * float(self.dh) ** 2
                w = coef / math.pi * float(self.dh) * float(self.rdatum) * tau / dist
                slope = slope_of(self.rtable, cc, c, float(self.drg))
                out.append((ih, ic, w, tau, slope))
        return out

    def source_terms_noncmp(self):
        """(is, ic, w, tau, slope) of the cmp=0 source operator (:621-666)."""
        out = []
        ns, aper = self.ns, self.aper
        for is_ in range(ns):
            c = self.src_index(is_)
            if c < 0 or c >= self.nsg:
                raise ValueError("Source table too small.")
            left, right = max(0, is_ - aper), min(ns - 1, is_ + aper)
            for ic in range(left, right + 1):
                cc = self.src_index(ic)
                if cc < 0 or cc >= self.nsg:
                    raise ValueError("Source table too small.")
                coef = taper_w(left, ic, right, self.tap, 1)
                tau = float(self.stable[cc, c])
                dist = float(self.sdatum) ** 2 + (ic - is_) ** 2 * float(self.ds) ** 2
                w = coef / math.pi * float(self.ds) * float(self.sdatum) * tau / dist
                slope = slope_of(self.stable, cc, c, float(self.dsg))
                out.append((is_, ic, w, tau, slope))
        return out

    def source_terms_cmp(self):
        """(is, ih, ic, hh, w, tau, slope, jump) of the cmp=1 source operator:
        common-receiver gathers r, sources is of the gather, neighbours ic
        (:556-619).  Terms whose offset index falls outside the spread are
        skipped, as the butterfly variant of the same walk does (:1006-1036)."""
        ns, nh, ds, dh = self.ns, self.nh, self.ds, self.dh
        s = f32(abs(f32(ns - 1) * ds))
        h = f32(abs(f32(nh - 1) * dh))
        wide = abs(ds) >= abs(dh)
        jump = 1 if wide else _i(dh / ds + f32(0.5))
        dr = f32(abs(dh)) if wide else f32(abs(ds))
        nr = _i((s + h) / dr + f32(1.5))
        a_s = f32(-1.0) if ds <= 0 else f32(0.0)
        a_h = f32(-1.0) if dh <= 0 else f32(0.0)
        b_l = f32(0.0) if ds <= 0 else f32(-1.0)
        out = []
        for ir in range(nr):
            r = f32(ir) * dr + a_s * s + a_h * h
            sleft = _i((f32(ir) * dr + a_s * s + b_l * h) / ds + f32(0.5))
            sright = _i((f32(ir) * dr + a_s * s + a_s * h) / ds + f32(0.5))
            sleft = max(sleft, 0)
            sright = min(sright, ns - 1)
            lft = _i((r - f32(sleft) * ds) / dh + f32(0.5))
            if lft < 0 or lft > nh - 1:
                sleft += 1
            rgt = _i((r - f32(sright) * ds) / dh + f32(0.5))
            if rgt < 0 or rgt > nh - 1:
                sright -= 1
            for is_ in range(sleft, sright + 1, jump):
                c = self.src_index(is_)
                if c < 0 or c >= self.nsg:
                    raise ValueError("Source table too small.")
                ih = _i((r - f32(is_) * ds) / dh + f32(0.5))
                left = max(sleft, is_ - jump * self.aper)
                right = min(sright, is_ + jump * self.aper)
                for ic in range(left, right + 1, jump):
                    cc = self.src_index(ic)
                    if cc < 0 or cc >= self.nsg:
                        raise ValueError("Source table too small.")
                    hh = _i((r - f32(ic) * ds) / dh + f32(0.5))
                    if ih < 0 or ih >= nh or hh < 0 or hh >= nh:
                        continue
                    coef = taper_w(left, ic, right, self.tap, jump)
                    tau = float(self.stable[cc, c])
                    dist = float(self.sdatum) ** 2 + (ic - is_) ** 2 * float(ds) ** 2
                    w = coef / math.pi * float(ds) * float(self.sdatum) * tau / dist
                    slope = slope_of(self.stable, cc, c, float(self.dsg))
                    out.append((is_, ih, ic, hh, w, tau, slope, jump))
        return out

    # -------------------------------------------------------------- pipeline
    def to_freq(self, data: np.ndarray) -> np.ndarray:
        """read_traces_to_freq (:281-313): reverse, edge taper, pad, r2c."""
        d = np.asarray(data, np.float64).reshape(self.ns, self.nh, self.nt)[..., ::-1]
        ws = np.array([edge_w(i, self.ns, self.data_tap) for i in range(self.ns)])
        wh = np.array([edge_w(i, self.nh, self.data_tap) for i in range(self.nh)])
        d = d * (ws[:, None, None] * wh[None, :, None])
        return np.fft.rfft(d, n=self.nfft, axis=-1)              # (ns, nh, nw)

    def from_freq(self, U: np.ndarray, reverse: bool) -> np.ndarray:
        """write_traces_from_freq (:470-491): c2r, / nfft, optional reversal."""
        x = np.fft.irfft(U, n=self.nfft, axis=-1)[..., :self.nt]   # irfft already divides by nfft
        return x[..., ::-1].copy() if reverse else x

    def receiver(self, Uin: np.ndarray) -> np.ndarray:
        iw = np.arange(self.nw)
        Utmp = np.zeros_like(Uin)
        shots = [0] if self.cmp == 0 else range(self.ns)
        for is0 in shots:
            terms = self.receiver_terms(is0)
            if not terms:
                continue
            ih = np.array([t[0] for t in terms])
            ic = np.array([t[1] for t in terms])
            w = np.array([t[2] for t in terms])
            tau = np.array([t[3] for t in terms])
            slope = np.array([t[4] for t in terms])
            aa = antialias_w(self.antialias, iw, slope * abs(float(self.dh)), self.nfft, float(self.dt))
            coef = w[:, None] * aa
            keep = np.abs(coef) >= 1e-20
            K = np.where(keep, coef * filter_H(tau, float(self.dt), self.nsam, self.nfft, iw), 0.0)
            if self.cmp == 0:
                Kd = np.zeros((self.nh, self.nh, self.nw), np.complex128)
                np.add.at(Kd, (ih, ic), K)
                Utmp += np.einsum("hcw,scw->shw", Kd, Uin)
            else:
                np.add.at(Utmp[is0], ih, K * Uin[is0, ic])
        return Utmp

    def source(self, Utmp: np.ndarray) -> np.ndarray:
        iw = np.arange(self.nw)
        Uout = np.zeros_like(Utmp)
        if self.cmp == 0:
            terms = self.source_terms_noncmp()
            if not terms:
                return Uout
            is_ = np.array([t[0] for t in terms])
            ic = np.array([t[1] for t in terms])
            w = np.array([t[2] for t in terms])
            tau = np.array([t[3] for t in terms])
            slope = np.array([t[4] for t in terms])
            aa = antialias_w(self.antialias, iw, slope * abs(float(self.ds)), self.nfft, float(self.dt))
            coef = w[:, None] * aa
            K = np.where(np.abs(coef) >= 1e-20, coef * filter_H(tau, float(self.dt), self.nsam, self.nfft, iw), 0.0)
            Kd = np.zeros((self.ns, self.ns, self.nw), np.complex128)
            np.add.at(Kd, (is_, ic), K)
            return np.einsum("scw,chw->shw", Kd, Utmp)
        terms = self.source_terms_cmp()
        if not terms:
            return Uout
        is_ = np.array([t[0] for t in terms])
        ih = np.array([t[1] for t in terms])
        ic = np.array([t[2] for t in terms])
        hh = np.array([t[3] for t in terms])
        w = np.array([t[4] for t in terms])
        tau = np.array([t[5] for t in terms])
        slope = np.array([t[6] for t in terms])
        jump = terms[0][7]
        aa = antialias_w(self.antialias, iw, slope * abs(float(f32(jump) * self.ds)), self.nfft, float(self.dt))
        coef = w[:, None] * aa
        K = np.where(np.abs(coef) >= 1e-20, coef * filter_H(tau, float(self.dt), self.nsam, self.nfft, iw), 0.0)
        np.add.at(Uout, (is_, ih), K * Utmp[ic, hh])
        return Uout

    def run(self, data: np.ndarray, interm: bool = False):
        """The whole tool: returns the datumed cube (ns, nh, nt) float64 and,
        with ``interm``, the receiver-side intermediate (not reversed)."""
        Uin = self.to_freq(data)
        Utmp = self.receiver(Uin)
        out = self.from_freq(self.source(Utmp), reverse=True)
        if interm:
            return out, self.from_freq(Utmp, reverse=False)
        return out
