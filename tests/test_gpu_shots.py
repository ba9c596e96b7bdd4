"""Shots of uneven receiver count and trace length through the prepared
(graph-capturable) path: the image equals the sum of one-shot migrations,
each a file the reference would migrate with ns = 1."""
import numpy as np
import pytest

import _cases
import kirch_datuming_b200 as kd
import oracle

pytestmark = pytest.mark.gpu


def _ragged(gd, case):
    """Shots built from a golden gather: shot i keeps a different window of
    receivers and a different trace length."""
    d = gd.data(case)
    geom = gd.geometry_dict(case)
    ns, nh, nt = d.shape
    f32 = np.float32
    out = []
    for i in range(ns):
        a = i % 3
        nhi = nh - 2 * i - a
        nti = nt - 37 * i
        h0 = f32(geom["h0"]) + f32(a) * f32(geom["dh"])
        sx = f32(geom["s0"]) + f32(i) * f32(geom["ds"])
        out.append(dict(sx=float(sx), h0=float(h0), dh=geom["dh"], data=np.ascontiguousarray(d[i, a:a + nhi, :nti])))
    return out


def _one_shot_geom(geom, s):
    g = dict(geom)
    nh, nt = s["data"].shape
    g.update(ns=1, s0=s["sx"], ds=0.0, nh=nh, h0=s["h0"], dh=s["dh"], nt=nt)
    return g


@pytest.mark.parametrize("case", ["base", "cmp1_half", "options", "offset"])
def test_ragged_shots_equal_one_shot_runs(golden, case):
    kp, geom, axis, op, _ = _cases.case_setup(golden, case)
    # one output axis for every run: the one-shot plans would otherwise each
    # derive the offset axis from their own receivers
    kp.axis_n_given, kp.axis_n = 1, axis[0]
    kp.axis_min_given, kp.axis_min = 1, axis[1]
    kp.axis_step_given, kp.axis_step = 1, axis[2]
    kp.axis_max_given = 0
    T, D = golden.tables()
    shots = _ragged(golden, case)
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(T, D, T, D)
    img = np.zeros((axis[0], geom["nx"], geom["nz"]), np.float32)
    pairs = plan.prepare_shots(shots)
    assert pairs == sum(s["data"].shape[0] for s in shots) * geom["nz"] * geom["nx"]
    plan.migrate_prepared(img)
    ref = np.zeros(img.shape, np.float64)
    o64 = np.zeros(img.shape, np.float64)
    for s in shots:
        g1 = _one_shot_geom(geom, s)
        p1 = kd.Plan(kp, kd.geometry(**g1))
        p1.set_tables(T, D, T, D)
        im1 = np.zeros(img.shape, np.float32)
        p1.migrate(s["data"][None], im1)
        p1.close()
        ref += im1
        o64 += oracle.migrate_adj(_cases.oracle_params(kp, g1, axis), s["data"][None], T, D, T, D, fp64=True)
    plan.close()
    assert np.linalg.norm(img - ref) <= 1e-6 * np.linalg.norm(ref)
    assert np.linalg.norm(img - o64) <= 1e-5 * np.linalg.norm(o64)


def test_graph_replay_matches_direct(golden):
    import torch
    kp, geom, axis, op, _ = _cases.case_setup(golden, "base")
    T, D = golden.tables()
    shots = _ragged(golden, "base")
    dev = [dict(s, data=torch.from_numpy(s["data"]).cuda()) for s in shots]
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(torch.from_numpy(T).cuda(), torch.from_numpy(D).cuda(), torch.from_numpy(T).cuda(),
                    torch.from_numpy(D).cuda())
    plan.prepare_shots(dev)
    direct = torch.zeros((axis[0], geom["nx"], geom["nz"]), device="cuda")
    plan.migrate_prepared(direct)
    plan.set_graph(True)
    g1 = torch.full_like(direct, 7.0)
    plan.migrate_prepared(g1)   # direct run, then capture
    g1.fill_(7.0)
    plan.migrate_prepared(g1)   # replay
    plan.migrate_prepared(g1)   # replay again: the image is overwritten, not accumulated
    assert torch.equal(g1, direct)
    plan.close()


def test_prepared_rejects_long_shot(golden):
    kp, geom, axis, op, _ = _cases.case_setup(golden, "base")
    T, D = golden.tables()
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(T, D, T, D)
    bad = [dict(sx=0.1, h0=0.2, dh=0.02, data=np.zeros((3, geom["nt"] + 1), np.float32))]
    with pytest.raises(kd.KcigError):
        plan.prepare_shots(bad)
    plan.close()


def test_autotune_and_multi_plan_graph(golden):
    # two "windows" (two plans with different mute parameters) in one graph;
    # the autotuned tile must not change the image beyond summation order
    import torch
    images, plans, direct = [], [], []
    T, D = golden.tables()
    tT, tD = torch.from_numpy(T).cuda(), torch.from_numpy(D).cuda()
    for slope in (0.5, 0.3):
        kp, geom, axis, op, _ = _cases.case_setup(golden, "base")
        kp.direct_mute_slope = slope
        plan = kd.Plan(kp, kd.geometry(**geom))
        plan.set_tables(tT, tD, tT, tD)
        shots = [dict(s, data=torch.from_numpy(s["data"]).cuda()) for s in _ragged(golden, "base")]
        plan.prepare_shots(shots)
        ref = torch.zeros((axis[0], geom["nx"], geom["nz"]), device="cuda")
        plan.migrate_prepared(ref)
        choice, ms = plan.autotune()
        assert 1 <= choice <= 4 and all(v > 0 for v in ms.values())
        tuned = torch.zeros_like(ref)
        plan.migrate_prepared(tuned)
        assert (tuned - ref).norm() <= 1e-6 * ref.norm()
        plans.append(plan)
        direct.append(tuned)
        images.append(torch.full_like(ref, 3.0))
    g = kd.Graph(plans, images)
    for im in images:
        im.fill_(3.0)
    g.launch()
    g.launch()
    torch.cuda.synchronize()
    for im, ref in zip(images, direct):
        assert torch.equal(im, ref)
    assert not torch.equal(images[0], images[1])  # each window its own mute
    g.close()
    for p in plans:
        p.close()


def test_receiver_stations_given_explicitly(golden):
    # receivers given as an explicit axis (kcig_shot.h): equal values share a
    # leg across shots.  The values are taken as given (FP32), where h0 + k*dh
    # is rebuilt in FP64 for the continuous quantities: the images agree to
    # that rounding (~1e-8 km in position)
    kp, geom, axis, op, _ = _cases.case_setup(golden, "base")
    T, D = golden.tables()
    shots = _ragged(golden, "base")
    f32 = np.float32
    explicit = []
    for s in shots:
        nh = s["data"].shape[0]
        h = f32(s["h0"]) + np.arange(nh, dtype=f32) * f32(s["dh"])
        explicit.append(dict(sx=s["sx"], dh=s["dh"], h=h, data=s["data"]))
    imgs = []
    for ss in (shots, explicit):
        plan = kd.Plan(kp, kd.geometry(**geom))
        plan.set_tables(T, D, T, D)
        im = np.zeros((axis[0], geom["nx"], geom["nz"]), np.float32)
        plan.prepare_shots(ss)
        plan.migrate_prepared(im)
        plan.close()
        imgs.append(im)
    assert np.linalg.norm(imgs[1] - imgs[0]) <= 1e-5 * np.linalg.norm(imgs[0])
