"""Benchmark of the adjoint angle-domain Kirchhoff CIG migration (kirchmig2d_cig adj=1).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl kcig|reference]

Workload (the production-size table-path configuration): five-layer 2-D model
with a salt-like lens, nz=601 x nx=1601 at 10 m; 400 shots x 400 receivers on
a fixed spread (cmp=0) every 40 m; nt=3001 at 1 ms; 15 Hz Ricker gathers from
the model's traveltime tables plus 20 dB noise (seeded, synthetic); FP32
tables at the 400 source/receiver positions; 61 angle bins over 0-60 degrees.
One step = one migration of all 160,000 traces: 1.54e11 image-point x trace
pairs.  Every step reads inputs far larger than L2 (1.9 GB of traces, 3.1 GB
of tables), so L2 holds nothing between steps.

Prints one JSON line (rank 0).  Multi-GPU (torchrun): the one 400-shot survey
is partitioned by shots over the ranks (each rank migrates its block at the
shots' positions in the whole survey, kcig_plan_set_shot_range) and the
ranks' images are summed with one NCCL all-reduce inside the timed region:
the total work is fixed (strong scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# ------------------------------------------------------------------ workload --
NZ, NX, DZ = 601, 1601, 0.01
NPOS, DP = 400, 0.04          # source/receiver positions 0 .. 15.96 km
SIZES = {"full": (400, 0.04), "small": (64, 0.24)}  # small: the same grid, 64 x 64 positions (profiling)
NT, DT = 3001, 0.001
FREQ = 15.0
TOKENS = ["cig=1", "mode=angle", "cmp=0", "angle_min=0", "angle_max=60", "angle_step=1", "angle_n=61",
          "direct_mute=1", "direct_mute_slope=0.5", "direct_mute_intercept=0", "direct_mute_taper=0.05"]
WORKLOAD = "five-layer salt 601x1601@10m, 400 shots x 400 receivers (cmp=0, 40 m), nt=3001 dt=1ms, 61 angle bins"
B_PAIR = 16  # algorithmic HBM bytes per pair: the receiver leg's T, dT/dr, gx, gz in FP32


def geometry_dict(ns=None, nh=None):
    ns = NPOS if ns is None else ns
    nh = NPOS if nh is None else nh
    f = lambda v: float(np.float32(v))  # noqa: E731
    return dict(nt=NT, nh=nh, ns=ns, t0=0.0, dt=f(DT), h0=0.0, dh=f(DP), s0=0.0, ds=f(DP), nz=NZ, nx=NX, z0=0.0,
                dz=f(DZ), x0=0.0, dx=f(DZ), sny=NPOS, sy0=0.0, sdy=f(DP), rny=NPOS, ry0=0.0, rdy=f(DP))


def make_workload(seed: int):
    """Velocity, tables and gathers on the current CUDA device."""
    import torch
    import kirch_datuming_b200 as kd
    from kirch_datuming_b200 import synth
    v, refl = synth.five_layer_salt(NZ, NX, DZ, DZ, seed=7)
    vel = torch.from_numpy(v).cuda()
    T, D = kd.eikonal_tables(vel, DZ, DZ, NPOS, 0.0, DP)
    g = synth.Geometry(nz=NZ, nx=NX, dz=DZ, dx=DZ, z0=0, x0=0, ns=NPOS, s0=0.0, ds=DP, nh=NPOS, h0=0.0, dh=DP,
                       cmp=0, nt=NT, dt=DT, t0=0.0, npos=NPOS, p0=0.0, dp=DP)
    amps = synth.reflectivities(len(refl), seed)
    data = synth.shot_gathers(T, g, [(rows, a) for rows, a in zip(refl.values(), amps)], FREQ, seed=seed)
    torch.cuda.synchronize()
    return v, T, D, data


# ------------------------------------------------------------------ clocks ---
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                     stderr=subprocess.DEVNULL, text=True)
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, val in zip(names, p[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks(kind: str = "hbm"):
    """(peak, source) of the HBM copy bandwidth (GB/s) or, kind="tensor", the
    dense BF16 tensor throughput of a burst (TFLOP/s)."""
    key, fallback = ("hbm_gbs", 6650.0) if kind == "hbm" else ("bf16_tflops", 1590.0)
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m[key]), "of measured"
    except Exception:
        return fallback, "of fallback"


def profiled_traffic():
    """DRAM bytes per pair of the summation kernel from the committed ncu
    summary (profiles/k_sum_traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "k_sum_traffic.json")) as f:
            return float(json.load(f)["dram_bytes_per_pair"])
    except Exception:
        return None


def issue_ceiling(pairs_per_s: float, sm_mhz):
    """The summation's instruction-issue ceiling next to its HBM roofline:
    148 SMs x 4 schedulers x one warp instruction per cycle, divided by the
    thread instructions per pair of the committed ncu summary; with that
    summary's L2 hit rate.  None without the summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "k_sum_traffic.json")) as f:
            p = json.load(f)
        ipp = float(p["thread_instructions_per_pair"])
        mhz = float(sm_mhz) if sm_mhz else 1965.0
        ceiling = 148 * 4 * 32 * mhz * 1e6 / ipp / 1e9
        return {"thread_instructions_per_pair": ipp, "sm_mhz": mhz, "ceiling_gpairs": ceiling,
                "frac": pairs_per_s / 1e9 / ceiling, "issue_active_pct_ncu": p.get("issue_active_pct"),
                "l2_sector_hit_rate_pct_ncu": p.get("l2_sector_hit_rate_pct")}
    except Exception:
        return None


# ----------------------------------------------------------- reference (CPU) --
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "kirchmig2d_cig")
REF_EIK = os.path.join(ROOT, "oracle", "_ref", "eikods2d")
SAMPLE_SHOT = 200          # shot at 8.0 km
SAMPLE_RCV = (176, 48)     # 48 receivers, 7.04 .. 8.92 km


def prepare_sample(wd: str, threads: int, tables=None):
    """Write the inputs of a bounded sample of the workload: one shot x 48
    receivers over the full 601x1601 image (4.62e7 pairs).  Tables are cut
    from the GPU workload's tables when given, else made by the reference's
    own eikods2d for the positions the sample uses."""
    from kirch_datuming_b200 import rsf, synth
    import torch
    r0, nr = SAMPLE_RCV
    p_lo, p_hi = min(r0, SAMPLE_SHOT) - 1, max(r0 + nr, SAMPLE_SHOT + 1) + 1
    npos = p_hi - p_lo
    v, refl = synth.five_layer_salt(NZ, NX, DZ, DZ, seed=7)
    if tables is not None:
        T = np.ascontiguousarray(tables[0][p_lo:p_hi]).ravel()
        D = np.ascontiguousarray(tables[1][p_lo:p_hi]).ravel()
        src = "the GPU workload"
    elif os.path.exists(REF_EIK):
        rsf.write(f"{wd}/vel.rsf", v, [NZ, NX], [0, 0], [DZ, DZ])
        rsf.write(f"{wd}/sht.rsf", np.array([[0.0, (p_lo + k) * DP, 0.0] for k in range(npos)], np.float32),
                  [3, npos], [0, 0], [DP, 1])
        subprocess.run([REF_EIK, "in=vel.rsf", "out=time.rsf", "shotfile=sht.rsf", "tdl1=tdl.rsf", "tds1=tds.rsf",
                        "b1=2", "b2=2"], cwd=wd, check=True, capture_output=True,
                       env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
        _, T = rsf.read(f"{wd}/time.rsf")
        _, D = rsf.read(f"{wd}/tds.rsf")
        src = "eikods2d"
    else:
        raise RuntimeError("no tables for the CPU sample")
    rsf.write(f"{wd}/time.rsf", T, [NZ, NX, npos], [0, 0, p_lo * DP], [DZ, DZ, DP])
    rsf.write(f"{wd}/tds.rsf", D, [NZ, NX, npos], [0, 0, p_lo * DP], [DZ, DZ, DP])
    g = synth.Geometry(nz=NZ, nx=NX, dz=DZ, dx=DZ, z0=0, x0=0, ns=1, s0=SAMPLE_SHOT * DP, ds=DP, nh=nr,
                       h0=r0 * DP, dh=DP, cmp=0, nt=NT, dt=DT, t0=0.0, npos=npos, p0=p_lo * DP, dp=DP)
    amps = synth.reflectivities(len(refl), 1)
    data = synth.shot_gathers(torch.from_numpy(np.asarray(T).reshape(npos, NX, NZ)), g,
                              [(rows, a) for rows, a in zip(refl.values(), amps)], FREQ, seed=1).numpy()
    rsf.write(f"{wd}/data.rsf", data, [NT, nr, 1], [0, r0 * DP, SAMPLE_SHOT * DP], [DT, DP, DP],
              extra={"unit1": "s"})
    return {"npos": npos, "p_lo": p_lo, "pairs": nr * NZ * NX, "tables": src,
            "sample": "1 shot (x=8.0 km) x 48 receivers (7.04-8.92 km) over the full 601x1601 image: "
                      "%.3g pairs, same parameters; tables from %s" % (nr * NZ * NX, src)}


def run_sample(wd: str, threads: int, meta: dict):
    """Time the reference tool (or, without it, the oracle port) on the
    prepared sample; returns a cpu_baseline dict."""
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    kind = "reference" if os.path.exists(REF_BIN) else "port"
    if kind == "reference":
        t = time.perf_counter()
        r = subprocess.run([REF_BIN, "seismic_data=data.rsf", "migration=mig.rsf", "stable=time.rsf",
                            "sderiv=tds.rsf", "rtable=time.rsf", "rderiv=tds.rsf", "adj=1"] + TOKENS,
                           cwd=wd, capture_output=True, text=True, env=env)
        wall = time.perf_counter() - t
        if r.returncode != 0:
            raise RuntimeError("reference failed: " + r.stderr[-2000:])
        m = re.search(r"Done\. Elapsed time: ([0-9.]+) s", r.stdout + r.stderr)
        el = float(m.group(1)) if m else wall
    else:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle
        import _cases
        import kirch_datuming_b200 as kd
        from kirch_datuming_b200 import rsf
        _, data = rsf.read(f"{wd}/data.rsf")
        _, T = rsf.read(f"{wd}/time.rsf")
        _, D = rsf.read(f"{wd}/tds.rsf")
        geom = sample_geometry(meta)
        kp = kd.params(*TOKENS)
        axis = kd.output_axis(kp, kd.geometry(**geom))
        os.environ["OMP_NUM_THREADS"] = str(threads)
        t = time.perf_counter()
        oracle.migrate_adj(_cases.oracle_params(kp, geom, axis), data, T, D, T, D, fp64=False)
        el = time.perf_counter() - t
    return {"value": meta["pairs"] / el / 1e9, "unit": "Gpairs/s", "cores": threads, "kind": kind,
            "seconds": round(el, 3), "sample": meta["sample"]}


def sample_geometry(meta: dict) -> dict:
    """Geometry of the bounded sample (one shot, 48 receivers, the table
    positions it uses) as the library's geometry keys."""
    r0, nr = SAMPLE_RCV
    f = lambda x: float(np.float32(x))  # noqa: E731
    return dict(geometry_dict(1, nr), s0=f(SAMPLE_SHOT * DP), h0=f(r0 * DP), sny=meta["npos"],
                rny=meta["npos"], sy0=f(meta["p_lo"] * DP), ry0=f(meta["p_lo"] * DP))


def sample_parity(wd: str, meta: dict, threads: int) -> dict:
    """Image errors on the bounded sample of the production workload (one
    shot x 48 receivers over the full 601x1601 grid): the GPU image against
    the FP64 oracle and against the reference binary's own FP32 image, and
    the reference against the FP64 oracle (relative L2 in double, as
    src/rsf_l2cmp.cpp:9-10)."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    import _cases
    import kirch_datuming_b200 as kd
    from kirch_datuming_b200 import rsf
    _, data = rsf.read(f"{wd}/data.rsf")
    _, T = rsf.read(f"{wd}/time.rsf")
    _, D = rsf.read(f"{wd}/tds.rsf")
    geom = sample_geometry(meta)
    kp = kd.params(*TOKENS)
    axis = kd.output_axis(kp, kd.geometry(**geom))
    plan = kd.Plan(kp, kd.geometry(**geom))
    dT = torch.from_numpy(np.ascontiguousarray(T, dtype=np.float32)).cuda()
    dD = torch.from_numpy(np.ascontiguousarray(D, dtype=np.float32)).cuda()
    plan.set_tables(dT, dD, dT, dD)
    img = torch.zeros((plan.ng, NX, NZ), dtype=torch.float32, device="cuda")
    plan.migrate(torch.from_numpy(np.ascontiguousarray(data, dtype=np.float32)).cuda(), img)
    plan.close()
    gpu = img.cpu().numpy().astype(np.float64)
    os.environ["OMP_NUM_THREADS"] = str(threads)
    o64 = oracle.migrate_adj(_cases.oracle_params(kp, geom, axis), data, T, D, T, D, fp64=True)
    out = {"sample": meta["sample"], "relL2_vs_fp64_oracle": oracle.rel_l2(gpu, o64),
           "relL2_vs_reference": None, "reference_vs_fp64": None}
    if os.path.exists(f"{wd}/mig.rsf"):
        _, ref = rsf.read(f"{wd}/mig.rsf")
        ref = np.asarray(ref, dtype=np.float64).reshape(o64.shape)
        out["relL2_vs_reference"] = oracle.rel_l2(gpu, ref)
        out["reference_vs_fp64"] = oracle.rel_l2(ref, o64)
    return out


def cpu_sample(threads: int, tables=None, parity: bool = False):
    """cpu_baseline of the bounded sample; with parity=True also the image
    errors of the same sample (sample_parity), as (baseline, parity)."""
    wd = tempfile.mkdtemp(prefix="kcig_cpu_")
    try:
        meta = prepare_sample(wd, threads, tables)
        base = run_sample(wd, threads, meta)
        if not parity:
            return base
        try:
            par = sample_parity(wd, meta, threads)
        except Exception as e:  # noqa: BLE001 -- reported, never required
            par = {"error": str(e)[-300:]}
        return base, par
    finally:
        shutil.rmtree(wd, ignore_errors=True)


# ---------------------------------------------------------- tables section ---
def tables_section(steps: int, warmup: int, threads: int):
    """The table generator on the migration's grid: kcig_eikods (order 2,
    time + tdl1 + tds1, the eikods2d outputs the migration reads) for the
    400 surface positions, device time per call with CUDA events; beside it
    the reference eikods2d on a bounded sample of the same positions with all
    host threads, and the deviation of the GPU tables from the reference's on
    that sample (order 2: the marching result depends on the heap's
    acceptance order, see kcig_eikods)."""
    import torch
    import kirch_datuming_b200 as kd
    from kirch_datuming_b200 import rsf, synth
    v, _ = synth.five_layer_salt(NZ, NX, DZ, DZ, seed=7)
    vel = torch.from_numpy(v).cuda()
    shots = np.zeros((NPOS, 3), np.float32)
    shots[:, 1] = np.arange(NPOS, dtype=np.float32) * np.float32(DP)
    for _ in range(max(1, min(warmup, 1))):
        r = kd.eikods(vel, DZ, DZ, shots)
    del r
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = max(1, min(steps, 3))
    e0.record()
    for _ in range(n):
        r = kd.eikods(vel, DZ, DZ, shots)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / n
    sweeps = r["sweeps"]
    out = {"workload": "five-layer salt 601x1601@10m, %d surface sources every %g km: time, tdl1, tds1" % (NPOS, DP),
           "value": NPOS / (ms / 1e3), "unit": "tables/s", "ms_per_call": ms,
           "sweeps": {"min": int(sweeps.min()), "mean": float(sweeps.mean()), "max": int(sweeps.max())}}
    if os.path.exists(REF_EIK):
        nsmp = max(8, threads)
        idx = np.linspace(0, NPOS - 1, nsmp).round().astype(int)
        wd = tempfile.mkdtemp(prefix="kcig_eik_")
        try:
            rsf.write(f"{wd}/vel.rsf", v, [NZ, NX], [0, 0], [DZ, DZ])
            rsf.write(f"{wd}/sht.rsf", shots[idx], [3, nsmp], [0, 0], [1, 1])
            t = time.perf_counter()
            subprocess.run([REF_EIK, "in=vel.rsf", "out=time.rsf", "shotfile=sht.rsf", "tdl1=tdl.rsf",
                            "tds1=tds.rsf", "b1=2", "b2=2"], cwd=wd, check=True, capture_output=True,
                           env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
            el = time.perf_counter() - t
            _, Tr = rsf.read(f"{wd}/time.rsf")
            _, Dr = rsf.read(f"{wd}/tds.rsf")
        finally:
            shutil.rmtree(wd, ignore_errors=True)
        Tg = r["time"][torch.from_numpy(idx).cuda()].cpu().numpy().ravel()
        Dg = r["tds1"][torch.from_numpy(idx).cuda()].cpu().numpy().ravel()
        dT, dD = np.abs(Tg - Tr), np.abs(Dg - Dr)
        out["cpu_baseline"] = {"value": nsmp / el, "unit": "tables/s", "cores": threads, "kind": "reference",
                               "seconds": round(el, 3),
                               "sample": "%d of the %d positions, eikods2d b1=2 b2=2 (order 2)" % (nsmp, NPOS)}
        out["vs_reference_sample"] = {
            "time_exact_frac": float((dT == 0).mean()), "time_max_abs_s": float(dT.max()),
            "time_p99_abs_s": float(np.percentile(dT, 99)), "tds1_exact_frac": float((dD == 0).mean()),
            "tds1_p99_abs": float(np.percentile(dD, 99))}
    del r
    torch.cuda.empty_cache()
    return out


# -------------------------------------------------------------------- main ---
# ------------------------------------------- 1201x4001 grid sample ---
BIG_NZ, BIG_NX, BIG_NT, BIG_NPOS, BIG_NS = 1201, 4001, 4001, 800, 8
BIG_TOKENS = ["cig=1", "mode=angle", "cmp=0", "angle_min=0", "angle_max=90", "angle_step=1", "angle_n=91",
             "direct_mute=1", "direct_mute_slope=0.5", "direct_mute_intercept=0", "direct_mute_taper=0.05"]


def large_grid_sample_section():
    """The 1201 x 4001 grid at 10 m (nt=4001 at 1 ms, 91 angle bins)
    with its tables kept in pinned host memory (KCIG_MEM_HOST_STREAM), on a
    sample of the survey: 8 shots x 800 receivers on a fixed spread, tables at
    the 800 receiver positions (the full 1000 x 800 survey needs 4001 positions,
    154 GB of host tables; this sample needs 31 GB).  Tables from kcig_eikods
    on the device, copied to pinned host memory, freed on the device; then
    one untimed and one timed migration through the C ABI with host data.
    Beside it the surrogate path on the same sample: a network trained on the
    sample's own tables (on the device, before they leave it) supplies every
    leg's traveltime and source-position derivative (angle from the
    finite-difference gradient of its traveltime), with no table read; its
    image is compared with the streamed-table image."""
    import psutil
    import torch
    import kirch_datuming_b200 as kd
    from kirch_datuming_b200 import synth
    nzx = BIG_NZ * BIG_NX
    host_bytes = 2 * BIG_NPOS * nzx * 4
    avail = psutil.virtual_memory().available
    if avail < 2.5 * host_bytes:
        return {"skipped": "host memory: %.0f GB available, %.0f GB of host tables" % (avail / 1e9, host_bytes / 1e9)}
    dz = 0.01
    x_lo = 16.0
    v, refl = synth.five_layer_salt(BIG_NZ, BIG_NX, dz, dz, seed=11)
    vel = torch.from_numpy(v).cuda()
    pos = np.float32(x_lo) + np.arange(BIG_NPOS, dtype=np.float32) * np.float32(dz)
    shots = np.zeros((BIG_NPOS, 3), np.float32)
    shots[:, 1] = pos
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = kd.eikods(vel, dz, dz, shots)
    torch.cuda.synchronize()
    t_tables = time.perf_counter() - t0
    T, D = r["time"], r["tds1"]
    del r["tdl1"]
    # the surrogate: background gradient fitted to the model's mean velocity
    # profile (v = 1.5 + g z), trained on the sample's tables
    zs = np.arange(BIG_NZ) * dz
    vbar = v.mean(axis=0).astype(np.float64)
    vgrad = float(np.sum((vbar - 1.5) * zs) / np.sum(zs * zs))
    sg_cfg = dict(lo=(float(pos[0]), 0.0, 0.0), hi=(float(pos[-1]) + dz, (BIG_NZ - 1) * dz, (BIG_NX - 1) * dz),
                  fmax=6.0, vref=1.5, zsrc=0.0, vgrad=vgrad, residual_ms=20.0)
    net = kd.Surrogate(seed=1, **sg_cfg)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = net.train(T, float(pos[0]), dz, 0.0, dz, 0.0, dz, 40000, batch=16384, lr=3e-3, lr_final=3e-5, seed=3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    rng = np.random.default_rng(0)
    ip, iz, ix = rng.integers(0, BIG_NPOS, 200000), rng.integers(0, BIG_NZ, 200000), rng.integers(0, BIG_NX, 200000)
    Tt = T[torch.from_numpy(ip).cuda(), torch.from_numpy(ix).cuda(), torch.from_numpy(iz).cuda()].cpu().numpy()
    Tg = net.eval(pos[ip], (iz * dz).astype(np.float32), (ix * dz).astype(np.float32))[0].cpu().numpy()
    tt_err = 1000.0 * np.abs(Tg - Tt)
    ds_km = 1.0  # shots every 100 receivers
    g = synth.Geometry(nz=BIG_NZ, nx=BIG_NX, dz=dz, dx=dz, z0=0, x0=0, ns=BIG_NS, s0=float(pos[0]), ds=ds_km,
                       nh=BIG_NPOS, h0=float(pos[0]), dh=dz, cmp=0, nt=BIG_NT, dt=0.001, t0=0.0, npos=BIG_NPOS,
                       p0=float(pos[0]), dp=dz)
    amps = synth.reflectivities(len(refl), 5)
    data = synth.shot_gathers(T, g, [(rows, a) for rows, a in zip(refl.values(), amps)], 15.0, seed=5,
                              noise_on_device=True)
    hT = torch.empty(T.shape, dtype=torch.float32, pin_memory=True)
    hD = torch.empty(D.shape, dtype=torch.float32, pin_memory=True)
    hT.copy_(T)
    hD.copy_(D)
    hdata = data.cpu().pin_memory()
    del T, D, r, data, vel
    torch.cuda.empty_cache()
    f = lambda x: float(np.float32(x))  # noqa: E731
    geom = dict(nt=BIG_NT, nh=BIG_NPOS, ns=BIG_NS, t0=0.0, dt=f(0.001), h0=f(pos[0]), dh=f(dz), s0=f(pos[0]),
                ds=f(ds_km), nz=BIG_NZ, nx=BIG_NX, z0=0.0, dz=f(dz), x0=0.0, dx=f(dz), sny=BIG_NPOS, sy0=f(pos[0]),
                sdy=f(dz), rny=BIG_NPOS, ry0=f(pos[0]), rdy=f(dz))
    kp = kd.params(*BIG_TOKENS)
    plan = kd.Plan(kp, kd.geometry(**geom))
    ng = plan.ng
    himg = torch.zeros((ng, BIG_NX, BIG_NZ), dtype=torch.float32).pin_memory()
    free0, total = torch.cuda.mem_get_info()
    ts = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        plan.set_tables(hT, hD, hT, hD, stream=True)
        plan.migrate(hdata, himg)
        ts.append(time.perf_counter() - t0)
    free1, _ = torch.cuda.mem_get_info()
    plan.close()
    img_table = himg.clone()
    splan = kd.Plan(kp, kd.geometry(**geom))
    splan.set_surrogate(net, net, angle="fd", tx="network")
    sts = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        splan.migrate(hdata, himg)
        sts.append(time.perf_counter() - t0)
    sfields = splan.timing()["fields_ms"]
    splan.close()
    net.close()
    a_, b_ = himg.double(), img_table.double()
    sg_rel = float((a_ - b_).norm() / b_.norm())
    pairs = BIG_NS * BIG_NPOS * nzx
    out = {"workload": "1201x4001@10m grid (five-layer salt), nt=4001 dt=1ms, 91 angle bins; sample of "
                       "8 shots x 800 receivers (cmp=0, 10 m); tables at the 800 receiver positions in pinned "
                       "host memory (KCIG_MEM_HOST_STREAM)",
           "value": pairs / ts[-1] / 1e9, "unit": "Gpairs/s", "pairs": pairs, "seconds": ts[-1],
           "host_tables_gb": host_bytes / 1e9, "tables_seconds": t_tables,
           "device_used_gb_during_migration": (total - free1) / 1e9,
           "image_finite": bool(torch.isfinite(img_table).all().item()),
           "image_rms": float(img_table.double().pow(2).mean().sqrt().item()),
           "surrogate": {"value": pairs / sts[-1] / 1e9, "unit": "Gpairs/s", "seconds": sts[-1],
                         "fields_ms": sfields, "host_tables_gb": 0.0,
                         "relL2_vs_streamed_table_image": sg_rel,
                         "config": {k: list(v_) if isinstance(v_, tuple) else v_ for k, v_ in sg_cfg.items()},
                         "training": {"steps": 40000, "batch": 16384, "seconds": t_train,
                                      "final_loss_ms2": float(np.mean(losses[-50:])),
                                      "traveltime_err_ms": {"rms": float(np.sqrt(np.mean(tt_err ** 2))),
                                                            "p99": float(np.percentile(tt_err, 99)),
                                                            "max": float(tt_err.max())}}}}
    del hT, hD, hdata, himg, img_table
    return out


# ------------------------------------------------------- surrogate section ---
# tensor FLOPs per (leg, point) of k_sg_fields by what the network supplies
# (the xs features folded into a per-leg bias): the traveltime only (layer 1
# on the z and x features, layers 2-4), plus its source-position derivative
# (the backward pass through layers 4-2), plus the depth and lateral input
# gradient for the angle (the backward pass through layer 1)
SG_FLOPS = {"t": 2 * 128 * (256 + 3 * 128), "tx": 2 * 128 * (256 + 3 * 128 + 3 * 128),
            "all": 2 * 128 * (256 + 3 * 128 + 3 * 128 + 256)}
SG_CONFIG = dict(lo=(0.0, 0.0, 0.0), hi=(4.0, 2.0, 4.0), fmax=3.0, vref=1.5, zsrc=0.0, vgrad=0.6, residual_ms=1.0)
SG_LR = (1e-3, 1e-5)  # Adam learning rate, cosine-decayed to the second value
SG_WORKLOAD = ("v(z)=1.5+0.6z 201x401@10m, 64 shots x 201 receivers (cmp=0, 10 m), nt=1001 dt=2ms, 61 angle bins, "
               "3 flat reflectors, 20 Hz; network trained on the 401-position GPU eikonal tables")


STITCH_WINDOWS = [(0, 130), (110, 250), (230, 370), (350, 490), (470, 600)]
STITCH_WORKLOAD = ("ADCIG stitching (layercom_cig): five depth windows, rows 0-130 / 110-250 / 230-370 / "
                   "350-490 / 470-600, of a 601 x 1601 image with 61 angle bins (235 MB out), stitch_blend=15, "
                   "lateral taper scalex_aper=50 scalex_scale=1.5")


def stitch_section(steps: int, warmup: int, threads: int):
    """ADCIG stitching: the device calls (kcig_stitch_window) timed with CUDA
    events against the HBM peak, and the drop-in CLI and the reference tool
    (oracle/_ref/layercom_cig, all host threads) timed on the same RSF files
    (wall time: both read and write the files)."""
    import torch
    import kirch_datuming_b200 as kd
    from kirch_datuming_b200 import rsf
    n1, n2, n3 = NZ, NX, 61
    g = torch.Generator(device="cuda").manual_seed(5)
    vols = [torch.randn((n3, n2, e - s + 1), device="cuda", generator=g) for s, e in STITCH_WINDOWS]
    scales = [1.0, 1.1, 0.9, 1.2, 0.8]
    out = torch.empty((n3, n2, n1), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream()

    def once():
        out.zero_()
        prev = -1
        for k, ((s, e), v) in enumerate(zip(STITCH_WINDOWS, vols)):
            kd.stitch_window(out, v, s, e, prev, 15, scales[k], k > 0, 50, 1.5)
            prev = e

    for _ in range(max(1, warmup)):
        once()
    ms = []
    for _ in range(max(1, steps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        once()
        e1.record(st)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    t = statistics.median(ms)
    # algorithmic bytes: every window sample read once and written once, the
    # blended rows' output read once more, the zeroed output written once
    win = sum((e - s + 1) for s, e in STITCH_WINDOWS) * n2 * n3
    blend = sum(min(15, STITCH_WINDOWS[k - 1][1] - STITCH_WINDOWS[k][0] + 1) for k in range(1, 5)) * n2 * n3
    algo = 4 * (2 * win + blend + n1 * n2 * n3)
    peak, peak_src = measured_peaks()
    # the same stitch as one call over all windows (kcig_stitch_windows): one
    # pass, every window sample read once and every output sample written once
    ref_out = out.clone()

    def once_all():
        kd.stitch_windows(out, vols, STITCH_WINDOWS, 15, scales, True, 50, 1.5)

    for _ in range(max(1, warmup)):
        once_all()
    same_all = bool(torch.equal(out.view(torch.int32), ref_out.view(torch.int32)))
    ms_all = []
    for _ in range(max(1, steps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        once_all()
        e1.record(st)
        torch.cuda.synchronize()
        ms_all.append(e0.elapsed_time(e1))
    t_all = statistics.median(ms_all)
    algo_all = 4 * (win + n1 * n2 * n3)
    res = {"workload": STITCH_WORKLOAD, "device_ms": t_all, "samples_out": n1 * n2 * n3,
           "roofline": {"bound": "hbm", "achieved": algo_all / (t_all / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": algo_all / (t_all / 1e3) / 1e9 / peak, "peak_source": peak_src,
                        "kernel": "k_stitch_all",
                        "note": "one kcig_stitch_windows call: the weight upload, one kernel, the counters' "
                                "read-back and the synchronisation"},
           "one_pass_equals_window_calls": same_all,
           "window_calls": {"device_ms": t, "achieved_gbs": algo / (t / 1e3) / 1e9,
                            "note": "five kcig_stitch_window calls with the zeroing of the output; each call "
                                    "also copies its blend weights in and its non-finite count out and "
                                    "synchronises"}}
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "layercom_cig")
    with tempfile.TemporaryDirectory() as wd:
        rsf.write(f"{wd}/model.rsf", np.zeros((n2, n1), np.float32), [n1, n2], [0.0, 0.0], [DZ, DZ])
        with open(f"{wd}/layers.txt", "w") as f:
            f.write("".join("%d %d\n" % w for w in STITCH_WINDOWS))
        for k, ((s, e), v) in enumerate(zip(STITCH_WINDOWS, vols)):
            rsf.write(f"{wd}/adcig_{k + 1}.rsf", v.cpu().numpy(), [e - s + 1, n2, n3], [s * DZ, 0.0, 0.0],
                      [DZ, DZ, 1.0])
        args = ["full_model=model.rsf", "layer_image_base=adcig.rsf", "layer_txt=layers.txt", "stitch_blend=15",
                "scale=1,1.1,0.9,1.2,0.8", "scalex_aper=50", "scalex_scale=1.5"]
        walls = {}
        for name, exe in (("kcig", kd.layercom_cig_cli_path), ("reference", ref_bin)):
            if not os.path.exists(exe):
                continue
            env = dict(os.environ, OMP_NUM_THREADS=str(threads))
            wall = []
            for _ in range(2):
                t0 = time.perf_counter()
                r = subprocess.run([exe] + args + ["output_file=out_%s.rsf" % name], cwd=wd, env=env,
                                   capture_output=True, text=True, timeout=120)
                wall.append((time.perf_counter() - t0) * 1e3)
                if r.returncode != 0:
                    raise RuntimeError(r.stderr)
            walls[name] = min(wall)
        same = None
        if len(walls) == 2:
            a = np.fromfile(f"{wd}/out_kcig.rsf@", dtype="<f4")
            b = np.fromfile(f"{wd}/out_reference.rsf@", dtype="<f4")
            same = bool(np.array_equal(a.view(np.uint32), b.view(np.uint32)))
    res["cli_wall_ms"] = walls
    res["cli_outputs_identical"] = same
    res["reference_threads"] = threads
    return res


DAT_ROW = 120         # datum depth row (1.2 km) of the migration workload's tables
DAT_ARGS = dict(aperture=200, taper=0, data_taper=20, length=0.05, antialias=1.0, cmp=0)  # the workflow's settings
DAT_WORKLOAD = ("kirchdat2d_freq on the migration workload: five-layer salt 601x1601@10m, Green's tables sliced "
                "at row 120 (1.2 km) from the 400-position eikods2d tables, 400 shots x 400 receivers (cmp=0, 40 m), "
                "nt=3001 dt=1ms; aperture=200 taper=0 data_taper=20 length=0.05 antialias=1")
DAT_SAMPLE = 100      # the CPU reference's bounded sample: the first 100 shots x 100 receivers


def datum_terms(nh: int, ns: int, aper: int) -> int:
    """Terms of the exact operator per frequency, both sides, cmp=0: every
    (output trace, input trace) pair inside the aperture."""
    r = sum(min(nh - 1, i + aper) - max(0, i - aper) + 1 for i in range(nh)) * ns
    s = sum(min(ns - 1, i + aper) - max(0, i - aper) + 1 for i in range(ns)) * nh
    return r + s


def datum_section(steps: int, warmup: int, threads: int, T=None, data=None):
    """Frequency-domain datuming (the recursive workflow's step between depth
    windows) on the migration workload: device time with the cube in HBM,
    end to end through the C ABI with host arrays, the stage split, the
    reference tool on a bounded sample and the FP64 oracle on a smaller one."""
    import torch
    import kirch_datuming_b200 as kd
    from kirch_datuming_b200 import rsf, synth
    f = lambda x: float(np.float32(x))  # noqa: E731
    if T is None or data is None:
        v, refl = synth.five_layer_salt(NZ, NX, DZ, DZ, seed=7)
        T, _ = kd.eikonal_tables(torch.from_numpy(v).cuda(), DZ, DZ, NPOS, 0.0, DP, deriv=False)
        g = synth.Geometry(nz=NZ, nx=NX, dz=DZ, dx=DZ, z0=0, x0=0, ns=NPOS, s0=0.0, ds=DP, nh=NPOS, h0=0.0, dh=DP,
                           cmp=0, nt=NT, dt=DT, t0=0.0, npos=NPOS, p0=0.0, dp=DP)
        data = synth.shot_gathers(T, g, [(rows, a) for rows, a in zip(refl.values(), synth.reflectivities(len(refl), 3))],
                                  FREQ, seed=3)
    datum = f(DAT_ROW * DZ)
    green = torch.empty((NPOS, NPOS), dtype=torch.float32, device="cuda")
    kd.green_slice(T, NZ, NX, NPOS, 0.0, 0.0, DZ, DZ, 0.0, DP, datum, green)
    gh = green.cpu().numpy()

    def params(ns, nh, ng):
        return kd.datum_params(nt=NT, nh=nh, ns=ns, dt=f(DT), h0=0.0, dh=f(DP), s0=0.0, ds=f(DP), nsg=ng, nrg=ng,
                               sg0=0.0, dsg=f(DP), rg0=0.0, drg=f(DP), sdatum=datum, rdatum=datum, **DAT_ARGS)

    p = params(NPOS, NPOS, NPOS)
    nsam, nfft = kd.datum_sizes(p, gh, gh)
    nw = nfft // 2 + 1
    out = torch.empty_like(data)
    st = torch.cuda.current_stream()
    for _ in range(max(1, warmup)):
        kd.datum_freq(p, green, green, data, out)
    ms, stages = [], []
    for _ in range(max(1, steps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        kd.datum_freq(p, green, green, data, out)
        e1.record(st)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
        stages.append(kd.datum_last_timing())
    t = statistics.median(ms)
    st_ms, launches = stages[len(stages) // 2]
    terms = datum_terms(NPOS, NPOS, DAT_ARGS["aperture"]) * nw
    # end to end: pinned host arrays through kcig_datum_freq (the cube in and out over PCIe)
    hdata_t = torch.empty(tuple(data.shape), dtype=torch.float32, pin_memory=True)
    hdata_t.copy_(data)
    hout_t = torch.empty(tuple(data.shape), dtype=torch.float32, pin_memory=True)
    hdata, hout = hdata_t.numpy(), hout_t.numpy()
    e2e = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        kd.datum_freq(p, gh, gh, hdata, hout)
        e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = min(e2e)
    same = bool(np.array_equal(hout, out.cpu().numpy()))
    gemm_ms = st_ms[2] + st_ms[3]
    # executed tensor work of k_cgemm_tc: per side and frequency ceil(400/128) x ceil(400/208) tiles of
    # 128 rows x 208 complex columns, four real products (Ar.Br, Ai.Bi, Ar.Bi, Ai.Br) over 400 k, three TF32
    # products each
    tiles = math.ceil(NPOS / 128) * math.ceil(NPOS / 208)
    tensor_flops = 2 * nw * tiles * (128 * 208 * NPOS) * 2.0 * 4 * 3
    peak_bf16, peak_src = measured_peaks(kind="tensor")
    tf32_peak = peak_bf16 / 2
    res = {"workload": DAT_WORKLOAD, "nfft": nfft, "frequencies": nw, "nsam": nsam,
           "value": terms / (t / 1e3) / 1e9, "unit": "Gterms/s", "ms": t,
           "stages_ms": {"forward_fft": st_ms[0], "operators": st_ms[1], "receiver_side": st_ms[2],
                         "source_side": st_ms[3], "inverse_fft": st_ms[4]},
           "gpu_launches": launches,
           "e2e": {"value": terms / (e2e_ms / 1e3) / 1e9, "unit": "Gterms/s", "ms": e2e_ms,
                   "h2d_bytes": hdata.nbytes + 2 * gh.nbytes, "d2h_bytes": hout.nbytes,
                   "equals_device_run": same},
           "roofline": {"bound": "tensor", "kernel": "k_cgemm_tc (both sides)",
                        "achieved": tensor_flops / (gemm_ms / 1e3) / 1e12, "peak": tf32_peak, "unit": "TFLOP/s",
                        "frac": tensor_flops / (gemm_ms / 1e3) / 1e12 / tf32_peak,
                        "peak_source": "dense TF32 = half the BF16 figure " + peak_src,
                        "useful_frac": datum_terms(NPOS, NPOS, DAT_ARGS["aperture"]) * 8.0 * 3 * nw
                                       / tensor_flops,
                        "note": "executed TF32 tensor flops (3 products per FP32 product, padded 128-row / "
                                "208-column tiles); useful_frac = the exact operator's terms over the executed "
                                "products"},
           "unit_note": "a term is one (output trace, input trace, frequency) product of the exact operator, "
                        "receiver and source sides; the reference's butterfly approximates these sums"}
    # the reference tool (use_bf=1, its default) on the bounded sample, and the GPU on the same sample
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "kirchdat2d_freq")
    n = DAT_SAMPLE
    sub = np.ascontiguousarray(hdata[:n, :n, :])
    gsub = np.ascontiguousarray(gh[:n, :n])
    ps = params(n, n, n)
    gpu_sub = np.empty_like(sub)
    kd.datum_freq(ps, gsub, gsub, sub, gpu_sub)
    nfft_s = kd.datum_sizes(ps, gsub, gsub)[1]
    terms_s = datum_terms(n, n, DAT_ARGS["aperture"]) * (nfft_s // 2 + 1)
    if os.path.exists(ref_bin):
        with tempfile.TemporaryDirectory() as wd:
            rsf.write(f"{wd}/vel.rsf", np.zeros((4, 4), np.float32), [4, 4], [0, 0], [DZ, DZ],
                      extra={"should_datum": str(DAT_ROW)})
            rsf.write(f"{wd}/green.rsf", gsub, [n, n], [0.0, 0.0], [f(DP), f(DP)])
            rsf.write(f"{wd}/d.rsf", sub, [NT, n, n], [0, 0, 0], [f(DT), f(DP), f(DP)])
            args = ["input_file=d.rsf", "output_file=o.rsf", "sgreen_file=green.rsf", "rgreen_file=green.rsf",
                    "model_file=vel.rsf", "aperture=200", "taper=0", "data_taper=20", "length=0.05", "cmp=0",
                    "antialias=1", "use_bf=1"]
            env = dict(os.environ, OMP_NUM_THREADS=str(threads))
            t0 = time.perf_counter()
            r = subprocess.run([ref_bin] + args, cwd=wd, env=env, capture_output=True, text=True, timeout=900)
            sec = time.perf_counter() - t0
            if r.returncode == 0:
                _, ro = rsf.read(f"{wd}/o.rsf")
                ro = ro.astype(np.float64).reshape(gpu_sub.shape)
                res["cpu_baseline"] = {"value": terms_s / sec / 1e9, "unit": "Gterms/s", "cores": threads,
                                       "kind": "reference", "seconds": sec,
                                       "sample": "oracle/_ref/kirchdat2d_freq (use_bf=1, the default) on the first "
                                                 "%d shots x %d receivers, nt=%d, %d frequencies, wall time incl. "
                                                 "file I/O" % (n, n, NT, nfft_s // 2 + 1)}
                res["parity"] = {"relL2_gpu_vs_reference_bf": float(np.linalg.norm(gpu_sub - ro) / np.linalg.norm(ro)),
                                 "note": "the reference's default applies the butterfly approximation of the "
                                         "operator; the GPU applies the exact operator"}
            else:
                res["cpu_baseline"] = {"value": None, "error": r.stderr[-300:]}
    # the FP64 oracle on a smaller sample (12 shots x 24 receivers, full nt)
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import datum as D
        ns_o, nh_o = 12, 24
        so = np.ascontiguousarray(hdata[:ns_o, :nh_o, :])
        ng = max(ns_o, nh_o)
        go = np.ascontiguousarray(gh[:ng, :ng])
        po = params(ns_o, nh_o, ng)
        gpu_o = np.empty_like(so)
        kd.datum_freq(po, go, go, so, gpu_o)
        o = D.Datum(NT, nh_o, ns_o, f(DT), 0.0, f(DP), 0.0, f(DP), go, 0.0, f(DP), go, 0.0, f(DP), np.float32(datum),
                    np.float32(datum), **DAT_ARGS).run(so)
        res.setdefault("parity", {})["relL2_gpu_vs_fp64_oracle"] = float(np.linalg.norm(gpu_o - o) / np.linalg.norm(o))
        res["parity"]["oracle_sample"] = "first %d shots x %d receivers, nt=%d" % (ns_o, nh_o, NT)
    except Exception as e:  # noqa: BLE001
        res.setdefault("parity", {})["oracle_error"] = str(e)[-300:]
    kd.datum_release()  # the spectra buffers kept between calls (10.5 GB here)
    return res


def surrogate_section(train_steps: int, steps: int, warmup: int, threads: int):
    """Table path vs learned-surrogate path on the same v(z) 201x401 gathers,
    every image judged against the FP64 oracle of the table path (run on the
    host cores): throughput of each (device time per migration), the
    surrogate's training time and traveltime error on the tables, the image
    error of each way the surrogate can supply the leg fields, of the
    background alone (the method without the network), and the floor any
    surrogate that supplies its own source-position derivative meets."""
    import torch
    import kirch_datuming_b200 as kd
    from kirch_datuming_b200 import synth
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    import _cases
    import surrogate as sgo
    vel, T1, D1, data1, g = synth.vz_small_workload(seed=4)
    f = lambda v: float(np.float32(v))  # noqa: E731
    gd = dict(nt=g.nt, nh=g.nh, ns=g.ns, t0=0.0, dt=f(g.dt), h0=f(g.h0), dh=f(g.dh), s0=0.0, ds=f(g.ds), nz=g.nz,
              nx=g.nx, z0=0.0, dz=f(g.dz), x0=0.0, dx=f(g.dx), sny=g.npos, sy0=0.0, sdy=f(g.dp), rny=g.npos, ry0=0.0,
              rdy=f(g.dp))
    geom = kd.geometry(**gd)
    kp = kd.params(*TOKENS)
    pairs = g.nz * g.nx * g.ns * g.nh
    st = torch.cuda.current_stream()
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
    os.environ["OMP_NUM_THREADS"] = str(threads)
    Th, Dh, dh_ = T1.cpu().numpy(), D1.cpu().numpy(), data1.cpu().numpy()
    op = _cases.oracle_params(kp, gd, kd.output_axis(kp, geom))
    t0 = time.perf_counter()
    o64 = oracle.migrate_adj(op, dh_, Th, Dh, Th, Dh, fp64=True)
    oracle_s = time.perf_counter() - t0

    def run(sur=None, angle="fd", tx="network"):
        plan = kd.Plan(kp, geom, stream=st.cuda_stream)
        plan.set_tables(T1, D1, T1, D1)
        if sur is not None:
            plan.set_surrogate(sur, sur, angle=angle, tx=tx)
        img = torch.zeros((plan.ng, g.nx, g.nz), dtype=torch.float32, device="cuda")
        for _ in range(warmup):
            plan.migrate(data1, img)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fields, summ = [], []
        e0.record(st)
        for _ in range(steps):
            plan.migrate(data1, img)
            t = plan.timing()
            fields.append(t["fields_ms"])
            summ.append(t["sum_ms"])
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        plan.close()
        im = img.cpu().double().numpy()
        return {"value": pairs / (ms / 1e3) / 1e9, "unit": "Gpairs/s", "ms_per_step": ms,
                "fields_ms": statistics.median(fields), "k_sum_ms": statistics.median(summ),
                "relL2_vs_fp64_oracle": rel(im, o64)}, im

    table, img_t = run()
    net = kd.Surrogate(seed=1, **SG_CONFIG)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = net.train(T1, 0.0, g.dp, 0.0, g.dz, 0.0, g.dx, train_steps, batch=16384, lr=SG_LR[0], lr_final=SG_LR[1],
                       seed=3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    rng = np.random.default_rng(0)
    n = 200000
    ip, iz, ix = rng.integers(0, g.npos, n), rng.integers(0, g.nz, n), rng.integers(0, g.nx, n)
    Tt = T1[torch.from_numpy(ip).cuda(), torch.from_numpy(ix).cuda(), torch.from_numpy(iz).cuda()].cpu().numpy()
    pts = ((ip * g.dp).astype(np.float32), (iz * g.dz).astype(np.float32), (ix * g.dx).astype(np.float32))

    def tt_err(sur):
        e = 1000.0 * np.abs(sur.eval(*pts)[0].cpu().numpy() - Tt)
        return {"rms": float(np.sqrt(np.mean(e ** 2))), "p99": float(np.percentile(e, 99)), "max": float(e.max())}

    variants = {}
    for name, angle, tx in (("fd_angle_network_tx", "fd", "network"), ("fd_angle_table_tx", "fd", "table"),
                            ("network_angle_network_tx", "network", "network")):
        r, im = run(net, angle, tx)
        r["relL2_vs_table_path"] = rel(im, img_t)
        variants[name] = r
    background = kd.Surrogate(seed=1, **SG_CONFIG)
    p = background.get_params()
    p[sgo.OFF_WO:] = 0.0  # output weights and bias: T = the background alone
    background.set_params(p)
    bg_err = tt_err(background)
    bg_fd, _ = run(background, "fd", "network")
    bg_tab, _ = run(background, "fd", "table")
    # the floor of a surrogate that supplies its own source-position
    # derivative: the table path with dT/dxs replaced by the exact derivative
    # of the table traveltime itself (central difference across the table
    # positions) instead of eikods2d's tds1 -- 8 of the 64 shots (FP64 oracle)
    sel = np.arange(0, g.ns, 8)
    gd8 = dict(gd, ns=len(sel), ds=f(8 * g.ds))
    op8 = _cases.oracle_params(kp, gd8, kd.output_axis(kp, kd.geometry(**gd8)))
    sub = np.ascontiguousarray(dh_[sel])
    Dfd = np.empty_like(Th)
    Dfd[1:-1] = (Th[2:].astype(np.float64) - Th[:-2]) / (2 * g.dp)
    Dfd[0], Dfd[-1] = (Th[1] - Th[0]) / g.dp, (Th[-1] - Th[-2]) / g.dp
    ref8 = oracle.migrate_adj(op8, sub, Th, Dh, Th, Dh, fp64=True)
    fd8 = oracle.migrate_adj(op8, sub, Th, Dfd, Th, Dfd, fp64=True)
    evals = (g.ns + g.nh) * g.nz * g.nx  # legs x points per migration
    fl = variants["fd_angle_network_tx"]["fields_ms"]
    achieved = evals * SG_FLOPS["tx"] / (fl / 1e3) / 1e12
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak, peak_src = float(json.load(fh)["bf16_tflops"]), "of measured"
    except Exception:
        peak, peak_src = 1590.0, "of fallback"
    out = {
        "workload": SG_WORKLOAD, "pairs_per_step": pairs,
        "oracle": {"seconds": oracle_s, "threads": threads},
        "network": {"config": {k: list(v) if isinstance(v, tuple) else v for k, v in SG_CONFIG.items()},
                    "layers": "3 inputs, 64 Fourier frequencies each, 4 x 128 SiLU, BF16 operands, FP32 accumulation"},
        "table_path": table,
        "surrogate_path": variants,
        "background_only": {"traveltime_err_ms": bg_err, "fd_angle_network_tx": bg_fd, "fd_angle_table_tx": bg_tab},
        "derivative_floor": {
            "what": "table path with dT/dxs = central difference of the table traveltime across positions instead "
                    "of tds1 (the derivative a traveltime-only surrogate converges to); 8 of 64 shots, FP64 oracle",
            "relL2_vs_fp64_oracle": rel(fd8, ref8)},
        "meets_rel_l2_1e-3": {k: v["relL2_vs_fp64_oracle"] <= 1e-3 for k, v in variants.items()},
        "training": {"steps": train_steps, "batch": 16384, "lr": list(SG_LR), "seconds": train_s,
                     "samples_per_s": train_steps * 16384 / train_s, "final_loss_ms2": float(np.mean(losses[-50:])),
                     "traveltime_err_ms": tt_err(net)},
        "roofline": {"bound": "tensor", "kernel": "k_sg_fields (traveltime + source-position derivative)",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "peak_source": peak_src, "flops_per_eval": SG_FLOPS["tx"], "evals_per_step": evals,
                     "note": "fields_ms also holds the finite-difference direction pass"},
    }
    net.close()
    background.close()
    return out


# --------------------------------------------------------- batched section ---
BATCH_WORKLOAD = ("v(z)=1.5+0.6z 201x401@10m in five 0.4 km depth windows (own tables from the window top, own "
                  "mute: slopes 50/40/30/20/10 s/km, tapers 0.05-0.10 s); 512 shots over 0-4 km, receivers "
                  "~U{96..480} every 8 m around the source, nt ~U{1501..4001} at 1 ms; 61 angle bins")
MUTE_SLOPES = (50.0, 40.0, 30.0, 20.0, 10.0)
MUTE_TAPERS = (0.05, 0.06, 0.07, 0.08, 0.10)


def batched_section(steps: int, warmup: int, seed: int = 21, small: bool = False):
    """The uneven-workload configuration: every depth window is a plan of its
    own with ragged shots prepared on the device, the summation tile is
    autotuned per window, and one CUDA graph replays all five windows.
    small: the first window and 64 shots only (a case for profilers)."""
    import torch
    import kirch_datuming_b200 as kd
    from kirch_datuming_b200 import synth
    nz_all, nx, dz, nshot, dh, nrg, nt_max = 201, 401, 0.01, 64 if small else 512, 0.008, 501, 4001
    rng = np.random.default_rng(seed)
    nh = rng.integers(96, 481, nshot)
    nts = rng.integers(1501, 4002, nshot)
    sx = (np.arange(nshot) * (4.0 / (nshot - 1))).astype(np.float32)
    i0 = np.clip(np.round((sx - nh * dh / 2) / dh).astype(int), 0, nrg - nh)
    vel = synth.velocity_linear_vz(nz_all, nx, dz)
    amps = synth.reflectivities(5, seed)
    rows = [(0, 40), (40, 80), (80, 120), (120, 160), (160, 201)][:1 if small else 5]
    f = lambda v: float(np.float32(v))  # noqa: E731
    plans, images, tuned, pairs = [], [], [], 0
    for w, (r0, r1) in enumerate(rows):
        nzw = r1 - r0
        vw = torch.from_numpy(np.ascontiguousarray(vel[:, r0:r1])).cuda()
        T, D = kd.eikonal_tables(vw, dz, dz, nx, 0.0, dz)
        g = synth.Geometry(nz=nzw, nx=nx, dz=dz, dx=dz, z0=0.0, x0=0.0, ns=nshot, s0=0.0, ds=4.0 / (nshot - 1),
                           nh=nrg, h0=0.0, dh=dh, cmp=0, nt=nt_max, dt=0.001, t0=0.0, npos=nx, p0=0.0, dp=dz)
        cube = synth.shot_gathers(T, g, [(np.full(nx, 20), amps[w])], 20.0, seed=seed + w, noise_on_device=True)
        grid = (np.arange(nrg) * dh).astype(np.float32)  # receiver stations shared by every shot
        shots = [dict(sx=float(sx[s]), dh=dh, h=grid[i0[s]:i0[s] + nh[s]],
                      data=cube[s, i0[s]:i0[s] + nh[s], :nts[s]].contiguous()) for s in range(nshot)]
        del cube
        kp = kd.params(*(TOKENS[:7] + ["direct_mute=1", "direct_mute_slope=%g" % MUTE_SLOPES[w],
                                      "direct_mute_intercept=0", "direct_mute_taper=%g" % MUTE_TAPERS[w]]))
        geom = kd.geometry(nt=nt_max, nh=1, ns=1, t0=0.0, dt=f(0.001), h0=0.0, dh=f(dh), s0=0.0, ds=0.0, nz=nzw,
                           nx=nx, z0=0.0, dz=f(dz), x0=0.0, dx=f(dz), sny=nx, sy0=0.0, sdy=f(dz), rny=nx, ry0=0.0,
                           rdy=f(dz))
        plan = kd.Plan(kp, geom)
        plan.set_tables(T, D, T, D)
        pairs += plan.prepare_shots(shots)
        del shots
        choice, ms = plan.autotune()
        tuned.append({"window": w, "tile": choice, "ms": ms})
        plans.append(plan)
        images.append(torch.zeros((plan.ng, nx, nzw), dtype=torch.float32, device="cuda"))
        torch.cuda.synchronize()
    st = torch.cuda.current_stream()

    def timed(step_fn):
        for _ in range(warmup):
            step_fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            step_fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    ms_direct = timed(lambda: [p.migrate_prepared(im) for p, im in zip(plans, images)])
    stages = [p.timing() for p in plans]  # of the last direct run
    ref = [im.clone() for im in images]
    graph = kd.Graph(plans, images)
    ms_graph = timed(lambda: graph.launch(st.cuda_stream))
    same = all(torch.equal(a, b) for a, b in zip(images, ref))
    graph.close()
    for p in plans:
        p.close()
    return {"workload": BATCH_WORKLOAD if not small else "first window of: " + BATCH_WORKLOAD.replace("512", "64"),
            "pairs_per_step": pairs,
            "value": pairs / (ms_graph / 1e3) / 1e9, "unit": "Gpairs/s", "ms_per_step": ms_graph,
            "direct": {"value": pairs / (ms_direct / 1e3) / 1e9, "ms_per_step": ms_direct,
                       "stage_ms_per_window": stages},
            "graph_equals_direct": same, "autotune": tuned,
            "launch": "one CUDA graph replaying the five window plans (kcig_graph_launch)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="kcig", choices=["kcig", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-batched", action="store_true", help="skip the uneven five-window workload")
    ap.add_argument("--no-stitch", action="store_true", help="skip the ADCIG stitching section")
    ap.add_argument("--only-stitch", action="store_true", help="only the ADCIG stitching section (one JSON object)")
    ap.add_argument("--no-datum", action="store_true", help="skip the datuming section")
    ap.add_argument("--only-datum", action="store_true", help="only the datuming section (one JSON object)")
    ap.add_argument("--no-tables", action="store_true", help="skip the table-generator section")
    ap.add_argument("--no-stream", action="store_true", help="skip the host-resident-tables measurement")
    ap.add_argument("--large-grid-sample", action="store_true",
                    help="only the 1201x4001 grid sample with host-resident tables (one JSON object)")
    ap.add_argument("--only-surrogate", action="store_true",
                    help="run only the traveltime-surrogate section and print its object (profiling)")
    ap.add_argument("--only-batched", action="store_true",
                    help="run only the uneven five-window workload and print its object (profiling)")
    ap.add_argument("--surrogate-steps", type=int, default=160000,
                    help="training steps of the traveltime surrogate (0: skip the surrogate section)")
    ap.add_argument("--size", default="full", choices=sorted(SIZES),
                    help="small: 64 shots x 64 receivers every 240 m on the same grid (ncu captures)")
    args = ap.parse_args()
    global NPOS, DP, WORKLOAD
    NPOS, DP = SIZES[args.size]
    if args.size != "full":
        WORKLOAD = WORKLOAD.replace("400 shots x 400 receivers (cmp=0, 40 m)",
                                    "%d shots x %d receivers (cmp=0, %g m)" % (NPOS, NPOS, DP * 1000))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    metric = "Gpairs/s (image pt×trace) on 1 B200, surrogate vs table path, relL2≤1e-3"

    if args.impl == "reference":
        if rank != 0:
            return 0
        vals = []
        wd = tempfile.mkdtemp(prefix="kcig_ref_")
        try:
            meta = prepare_sample(wd, threads)
            for _ in range(min(args.warmup, 1)):  # one untimed run warms the page cache
                run_sample(wd, threads, meta)
            for _ in range(max(1, args.steps)):
                vals.append(run_sample(wd, threads, meta))
        finally:
            shutil.rmtree(wd, ignore_errors=True)
        base = vals[0]
        v = statistics.median([x["value"] for x in vals])
        sec = statistics.median([x["seconds"] for x in vals])
        line = {"metric": metric, "value": v, "unit": "Gpairs/s", "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD + "; reference timed on a bounded sample per step",
                           "sample": base["sample"]},
                "cpu_baseline": {"value": v, "unit": "Gpairs/s", "cores": threads, "kind": base["kind"],
                                 "sample": base["sample"]},
                "e2e": {"value": v, "unit": "Gpairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    import kirch_datuming_b200 as kd
    torch.cuda.set_device(local)
    if args.large_grid_sample:
        print(json.dumps({"large_grid_sample": large_grid_sample_section()}), flush=True)
        return 0
    if args.only_stitch:
        threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
        print(json.dumps({"stitch": stitch_section(args.steps, args.warmup, threads)}), flush=True)
        return 0
    if args.only_datum:
        threads = len(os.sched_getaffinity(0))
        print(json.dumps({"datum": datum_section(args.steps, args.warmup, threads)}), flush=True)
        return 0
    if args.only_surrogate:
        threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
        print(json.dumps({"surrogate": surrogate_section(args.surrogate_steps, args.steps, args.warmup, threads)}),
              flush=True)
        return 0
    if args.only_batched:
        print(json.dumps({"batched": batched_section(args.steps, args.warmup, small=args.size == "small")}),
              flush=True)
        return 0
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    from kirch_datuming_b200 import shard
    v, T, D, data_all = make_workload(seed=11)  # the same survey on every rank
    kp = kd.params(*TOKENS)
    geom = geometry_dict()
    st = torch.cuda.current_stream()
    plan = kd.Plan(kp, kd.geometry(**geom), stream=st.cuda_stream)
    plan.set_tables(T, D, T, D)
    # this rank's block of shots, at their positions in the whole survey
    first, count = shard.shot_range(NPOS, rank, world)
    if world > 1:
        plan.set_shot_range(first, count)
        data = data_all[first:first + count].contiguous()
        del data_all
    else:
        data = data_all
    ng = plan.ng
    image = torch.zeros((ng, NX, NZ), dtype=torch.float32, device="cuda")
    pairs = NPOS * NPOS * NZ * NX  # the whole survey: every rank's share together

    def step():
        plan.migrate(data, image)
        shard.reduce_image(image)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sum_ms, launches = [], 0
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(args.steps):
        step()
        s = plan.stats()
        sum_ms.append(s["sum_ms"] / max(1, s["sum_launches"]))
        launches += s["launches"]
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop()
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()

    # end to end through the public C ABI with pinned host buffers: every
    # step copies the tables and this rank's traces in and the image out; with
    # several ranks the images are summed on the devices in between (device
    # time on the plan's stream, the max over ranks)
    hT, hD = T.cpu().pin_memory(), D.cpu().pin_memory()
    hdata = data.cpu().pin_memory()
    himg = torch.zeros((ng, NX, NZ), dtype=torch.float32).pin_memory()
    eplan = kd.Plan(kp, kd.geometry(**geom), stream=st.cuda_stream)
    if world > 1:
        eplan.set_shot_range(first, count)
    e2e_ms = []
    for i in range(args.e2e_steps + 1):
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(st)
        eplan.set_tables(hT, hD, hT, hD)
        eplan.migrate(hdata, himg)
        if dist is not None:
            image.copy_(himg, non_blocking=True)
            shard.reduce_image(image)
            himg.copy_(image, non_blocking=True)
        a1.record(st)
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) * 1e3
        e2e_ms.append(max(wall, a0.elapsed_time(a1)))
    e2e_ms = statistics.median(e2e_ms[1:]) if len(e2e_ms) > 1 else e2e_ms[0]
    if dist is not None:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    eplan.close()
    # the same call with the tables left in host memory (KCIG_MEM_HOST_STREAM):
    # only the slices each leg batch interpolates cross PCIe -- the mode for
    # tables larger than the device memory
    stream_ms = None
    if dist is None and not args.no_stream:
        splan = kd.Plan(kp, kd.geometry(**geom))
        ts = []
        for i in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            splan.set_tables(hT, hD, hT, hD, stream=True)
            splan.migrate(hdata, himg)
            ts.append((time.perf_counter() - t0) * 1e3)
        stream_ms = ts[-1]
        splan.close()
    h2d = hT.numel() * 4 + hD.numel() * 4 + hdata.numel() * 4
    d2h = himg.numel() * 4

    ksum_ms = statistics.median(sum_ms)
    peak, peak_src = measured_peaks()
    pairs_rank = count * NPOS * NZ * NX  # the summation kernel's own share
    achieved = pairs_rank * B_PAIR / (ksum_ms / 1e3) / 1e9
    tpp = profiled_traffic()
    line = {
        "metric": metric, "value": pairs / (ms / 1e3) / 1e9, "unit": "Gpairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "pairs_per_step": pairs,
                   "parallelism": ("dp%d (one survey, shots %d..%d on rank 0 of %d, image all-reduce)"
                                   % (world, first, first + count - 1, world)) if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (1.9 GB traces, 3.1 GB tables per step)",
                   "tables": "GPU eikods2d tables (kcig_eikods: order 2, tds1), 400 positions"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src, "kernel": "k_sum", "kernel_ms": ksum_ms,
                     "algorithmic_bytes_per_pair": B_PAIR,
                     "traffic": (tpp * pairs_rank) if tpp is not None else None,
                     "issue": issue_ceiling(pairs_rank / (ksum_ms / 1e3), (clk or {}).get("sm_mhz")),
                     "note": "16 B/pair counts the receiver leg's fields once per pair; k_sum loads each "
                             "receiver leg once per block of 4 shots, so its DRAM traffic (ncu, 'traffic') is "
                             "below the algorithmic bytes and frac can pass 1: the kernel is issue-bound"},
        "e2e": {"value": pairs / (e2e_ms / 1e3) / 1e9, "unit": "Gpairs/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
        "streamed_tables": None if stream_ms is None else {
            "value": pairs / (stream_ms / 1e3) / 1e9, "unit": "Gpairs/s", "ms_per_step": stream_ms,
            "note": "end to end as e2e, tables kept in pinned host memory (KCIG_MEM_HOST_STREAM)"},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if rank == 0 and not args.no_cpu_baseline and args.size == "full":
        try:
            line["cpu_baseline"], line["parity"] = cpu_sample(threads, tables=(T.cpu().numpy(), D.cpu().numpy()),
                                                              parity=True)
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "error": str(e)[:300]}
    if dist is None and not args.no_tables and args.size == "full":
        line["tables"] = tables_section(args.steps, args.warmup, threads)
    if dist is None and args.surrogate_steps > 0:
        try:  # an extra object: its failure is recorded, the line still prints
            line["surrogate"] = surrogate_section(args.surrogate_steps, args.steps, args.warmup, threads)
        except Exception as e:  # noqa: BLE001
            line["surrogate"] = {"workload": SG_WORKLOAD, "error": str(e)[-400:]}
    if dist is None and not args.no_datum and args.size == "full":
        try:  # an extra object: its failure is recorded, the line still prints
            line["datum"] = datum_section(args.steps, args.warmup, threads, T=T, data=data)
        except Exception as e:  # noqa: BLE001
            line["datum"] = {"workload": DAT_WORKLOAD, "error": str(e)[-400:]}
        torch.cuda.empty_cache()
    if dist is None and not args.no_batched:
        plan.close()
        del T, D, data, image
        torch.cuda.empty_cache()
        line["batched"] = batched_section(args.steps, args.warmup, small=args.size == "small")
    if dist is None and not args.no_stitch and args.size == "full":
        torch.cuda.empty_cache()
        try:  # an extra object: its failure is recorded, the line still prints
            line["stitch"] = stitch_section(args.steps, args.warmup, threads)
        except Exception as e:  # noqa: BLE001
            line["stitch"] = {"workload": STITCH_WORKLOAD, "error": str(e)[-400:]}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None or args.no_batched:
        plan.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
