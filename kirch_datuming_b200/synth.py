"""Seeded synthetic workloads with the shapes of the migration benchmarks.

Nothing here is on the migration path: these builders make velocity models,
acquisition geometry and Ricker shot gathers that stand in for field data.
Shot gathers follow the recipe of the benchmark description: for each
reflector (one depth index per lateral grid column), the reflection time of a
source/receiver pair is the Fermat minimum over the reflector points of
``Ts + Tr`` read from the traveltime tables, a Ricker wavelet of the stated
peak frequency is placed there with amplitude equal to the reflector's
reflectivity, and Gaussian noise at ``rms(signal) / 10`` (20 dB) is added.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
import torch


@dataclasses.dataclass
class Geometry:
    """Grid, acquisition and table-position axes of one workload.

    Data layout [ns][nh][nt] (time fastest); tables [npos][nx][nz] (depth
    fastest, index ix*nz+iz); image [ng][nx][nz].
    """
    nz: int
    nx: int
    dz: float
    dx: float
    z0: float
    x0: float
    ns: int
    s0: float
    ds: float
    nh: int
    h0: float
    dh: float
    cmp: int
    nt: int
    dt: float
    t0: float
    npos: int
    p0: float
    dp: float

    @property
    def nzx(self) -> int:
        return self.nz * self.nx

    def shot_x(self) -> np.ndarray:
        s = np.float32(self.s0) + np.arange(self.ns, dtype=np.float32) * np.float32(self.ds if self.ns > 1 else 0.0)
        return s.astype(np.float32)

    def receiver_x(self, ishot: int) -> np.ndarray:
        h = np.float32(self.h0) + np.arange(self.nh, dtype=np.float32) * np.float32(self.dh if self.nh > 1 else 0.0)
        if self.cmp:
            return (self.shot_x()[ishot] + h).astype(np.float32)
        return h.astype(np.float32)

    def pairs(self) -> int:
        return self.ns * self.nh * self.nz * self.nx


def velocity_linear_vz(nz: int, nx: int, dz: float, v0: float = 1.5, grad: float = 0.6) -> np.ndarray:
    """v(z) = v0 + grad*z km/s, layout [nx][nz]."""
    z = np.arange(nz, dtype=np.float64) * dz
    v = (v0 + grad * z).astype(np.float32)
    return np.tile(v[None, :], (nx, 1))


def five_layer_salt(nz: int, nx: int, dz: float, dx: float, seed: int = 7):
    """Five-layer model with a salt-like lens whose top is a Gaussian bump.

    Velocities 1.5 / 2.0 / 2.6 / 4.5 (lens) / 3.2 km/s.  Returns the velocity
    [nx][nz] and a dict of interface depth indices per column (the reflectors
    used to synthesise data).
    """
    rng = np.random.default_rng(seed)
    zmax = (nz - 1) * dz
    xmax = (nx - 1) * dx
    x = np.arange(nx) * dx
    z = np.arange(nz) * dz
    z1 = 0.20 * zmax
    z2 = 0.40 * zmax
    base = 0.62 * zmax
    xc = xmax * (0.5 + 0.1 * (rng.random() - 0.5))
    width = xmax * (0.10 + 0.04 * rng.random())
    bump = np.exp(-((x - xc) / width) ** 2)
    top = base - 0.16 * zmax * bump
    bot = base + 0.08 * zmax * bump
    zz = np.broadcast_to(z[None, :], (nx, nz))
    v = np.full((nx, nz), 1.5, dtype=np.float32)
    v[zz >= z1] = 2.0
    v[zz >= z2] = 2.6
    v[zz >= base] = 3.2
    v[(zz >= top[:, None]) & (zz < bot[:, None])] = 4.5
    deep = 0.85 * zmax
    refl = {
        "z1": np.full(nx, int(round(z1 / dz))),
        "z2": np.full(nx, int(round(z2 / dz))),
        "salt_top": np.clip(np.round(top / dz).astype(int), 0, nz - 1),
        "deep": np.full(nx, int(round(deep / dz))),
    }
    return v, refl


def ricker(t: torch.Tensor, f: float) -> torch.Tensor:
    a = (math.pi * f * t) ** 2
    return (1.0 - 2.0 * a) * torch.exp(-a)


def _rows_at(tables: torch.Tensor, g: Geometry, xs: np.ndarray, rows: torch.Tensor) -> torch.Tensor:
    """Traveltime on one reflector row for lateral positions xs: [len(xs), nx],
    linear interpolation between table positions (clamped)."""
    f = (torch.as_tensor(xs, dtype=torch.float64, device=tables.device) - g.p0) / g.dp
    f = f.clamp(0, g.npos - 1)
    i0 = f.floor().long().clamp(max=g.npos - 1)
    i1 = (i0 + 1).clamp(max=g.npos - 1)
    w = (f - i0.double()).float()[:, None]
    ix = torch.arange(g.nx, device=tables.device)[None, :]
    r0 = tables[i0[:, None], ix, rows[None, :]]
    r1 = tables[i1[:, None], ix, rows[None, :]]
    return (1 - w) * r0 + w * r1


def shot_gathers(tables: torch.Tensor, g: Geometry, reflectors: list, freq: float,
                 seed: int, snr_amp: float = 10.0, shot_chunk: int = 8, noise_on_device: bool = False) -> torch.Tensor:
    """FP32 gathers [ns][nh][nt] on tables.device.

    tables: [npos][nx][nz] source/receiver traveltime table (shared).
    reflectors: list of (depth index per column [nx], reflectivity).
    noise_on_device: draw the noise with a device generator (fast for
    multi-GB cubes; a different seeded realisation than the host draw).
    """
    dev = tables.device
    gen = torch.Generator(device="cpu").manual_seed(seed)
    t = g.t0 + torch.arange(g.nt, device=dev, dtype=torch.float32) * g.dt
    out = torch.zeros(g.ns, g.nh, g.nt, dtype=torch.float32, device=dev)
    sx = g.shot_x()
    for r_rows, refl in reflectors:
        rows = torch.as_tensor(np.asarray(r_rows), device=dev, dtype=torch.long)
        ts_all = _rows_at(tables, g, sx, rows)  # [ns][nx]
        rcv_static = None
        if not g.cmp:
            rcv_static = _rows_at(tables, g, g.receiver_x(0), rows)  # [nh][nx]
        for a in range(0, g.ns, shot_chunk):
            b = min(g.ns, a + shot_chunk)
            ts = ts_all[a:b]
            if rcv_static is not None:
                tr = rcv_static[None].expand(b - a, -1, -1)
            else:
                tr = torch.stack([_rows_at(tables, g, g.receiver_x(i), rows) for i in range(a, b)])
            tref = (ts[:, None, :] + tr).amin(dim=2)  # [chunk][nh]
            out[a:b] += refl * ricker(t[None, None, :] - tref[:, :, None], freq)
    rms = out.square().mean().sqrt()
    if noise_on_device:
        dgen = torch.Generator(device=dev).manual_seed(seed)
        out += torch.randn(out.shape, generator=dgen, dtype=torch.float32, device=dev) * (rms / snr_amp)
    else:
        noise = torch.randn(out.shape, generator=gen, dtype=torch.float32).to(dev)
        out += noise * (rms / snr_amp)
    return out


def reflectivities(n: int, seed: int) -> list:
    rng = np.random.default_rng(seed)
    mag = rng.uniform(0.05, 0.2, size=n)
    sign = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    return [float(s * m) for s, m in zip(sign, mag)]


def vz_small_workload(seed: int = 4, device: str = "cuda"):
    """The small survey the reference can migrate on a CPU: v(z) = 1.5 + 0.6 z km/s on a
    201 x 401 grid of 10 m; flat reflectors at 0.6 / 1.2 / 1.7 km with
    reflectivity +-U(0.05, 0.2); 64 shots evenly spaced over 0..4 km, 201
    receivers every 10 m from 1.0 to 3.0 km (cmp=0); nt=1001, dt=2 ms; 20 Hz
    Ricker; traveltime tables from the GPU eikonal solver at the 401 grid
    columns.  Returns (vel, tables, deriv, data, geometry)."""
    import kirch_datuming_b200 as kd
    nz, nx, dz = 201, 401, 0.01
    vel = torch.from_numpy(velocity_linear_vz(nz, nx, dz)).to(device)
    T, D = kd.eikonal_tables(vel, dz, dz, nx, 0.0, dz)
    g = Geometry(nz=nz, nx=nx, dz=dz, dx=dz, z0=0.0, x0=0.0, ns=64, s0=0.0, ds=4.0 / 63, nh=201, h0=1.0, dh=dz,
                 cmp=0, nt=1001, dt=0.002, t0=0.0, npos=nx, p0=0.0, dp=dz)
    amps = reflectivities(3, seed)
    refl = [(np.full(nx, int(round(zr / dz))), a) for zr, a in zip((0.6, 1.2, 1.7), amps)]
    data = shot_gathers(T, g, refl, 20.0, seed=seed)
    return vel, T, D, data, g
