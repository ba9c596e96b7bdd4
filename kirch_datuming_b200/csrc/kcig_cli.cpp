// kcig_run_cli: the drop-in kirchmig2d_cig (adj=1 migration, adj=0 forward modelling), and
// kcig_run_kirchmig2d_cli: the drop-in kirchmig2d (adj=1).  Same argv keys, files,
// defaults, ERROR texts, output header and exit status as
// src/kirchmig2d_cig.cpp:494-1401; the migration itself runs on the GPU.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <unistd.h>

#include <chrono>
#include <string>
#include <vector>

#include "kcig_common.h"
#include "kcig_par.h"
#include "kcig_rsf.h"

namespace kcig {
int params_from_map(const ParMap &m, kcig_params *p);
int params_from_map_kirchmig2d(const ParMap &m, kcig_params *p);
}

using namespace kcig;

static void log_line(const char *lvl, const char *msg)
{
    fprintf(stderr, "%d %s:%s\n", (int)getpid(), lvl, msg);
}

static int fail(int rc)
{
    log_line("ERROR", kcig_last_error());
    return rc;
}

static int open3(const ParMap &m, const char *key, RsfFile *f, const char *need3)
{
    int rc = rsf_open(m.str(key), f);
    if (rc) return rc;
    if (f->ndim < 3) return set_error(KCIG_ERR_ARG, "%s", need3);
    return KCIG_OK;
}

// direct mute in the reference's FP32 (kirchmig2d_cig.cpp:110-129), used only
// to write the QC before/after gathers of one shot (:1070-1080).
static void qc_mute(float *trace, int nt, float t0, float dt, float sx, float rx, const kcig_params &p)
{
    const float offset_time = p.direct_mute_slope * fabsf(rx - sx);
    const float boundary =
        p.direct_mute_invert ? p.direct_mute_intercept - offset_time : p.direct_mute_intercept + offset_time;
    for (int it = 0; it < nt; it++) {
        const float time = t0 + (float)it * dt;
        float w = 0.0f;
        if (time >= boundary + p.direct_mute_taper) w = 1.0f;
        else if (time > boundary) {
            const float u = (time - boundary) / p.direct_mute_taper;
            w = 0.5f * (1.0f - cosf((float)M_PI * u));
        }
        trace[it] *= w;
    }
}

// tool 0: kirchmig2d_cig; tool 1: kirchmig2d (src/kirchmig2d.cpp:35-612),
// whose flow is the same with its own parameter block and no angle, mute or
// gradient-file options
static int run_tool(int argc, char **argv, int tool)
{
    ParMap m;
    int rc = m.parse(argc, argv);
    if (rc) return fail(rc);
    kcig_params p;
    // mode is validated before the file keys (:554-563)
    if (tool == 0) {
        const std::string mode =
            m.have("mode") ? m.str("mode") : (m.have("cig_mode") ? m.str("cig_mode") : "offset");
        std::string lm;
        for (char c : mode) lm.push_back((char)tolower((unsigned char)c));
        if (lm != "offset" && lm != "angle")
            return fail(set_error(KCIG_ERR_ARG, "Unknown CIG mode: %s. Supported modes are offset and angle.",
                                  mode.c_str()));
    }
    static const char *need[6][2] = {{"seismic_data", "Need seismic_data="}, {"migration", "Need migration="},
                                     {"stable", "Need stable="},             {"sderiv", "Need sderiv="},
                                     {"rtable", "Need rtable="},             {"rderiv", "Need rderiv="}};
    for (auto &k : need)
        if (!m.have(k[0])) return fail(set_error(KCIG_ERR_ARG, "%s", k[1]));
    rc = tool == 1 ? params_from_map_kirchmig2d(m, &p) : params_from_map(m, &p);
    if (rc) return fail(rc);
    if (tool == 1 && !p.adj) return fail(set_error(KCIG_ERR_UNSUPPORTED, "kirchmig2d adj=0 is not built"));
    const bool fwd = !p.adj;  // adj=0: migration= is read, seismic_data= written (:643-701)
    const bool angle = p.cig && p.cig_is_angle;
    int use_grad = 0;
    if (angle) {
        const int hg = m.have("sgradx") + m.have("sgradz") + m.have("rgradx") + m.have("rgradz");
        if (hg && hg != 4)
            return fail(set_error(KCIG_ERR_ARG,
                                  "For mode=angle, please provide all of sgradx=, sgradz=, rgradx=, and rgradz=, or "
                                  "provide none of them."));
        use_grad = hg == 4;
    }
    RsfFile dat, stim, sder, rtim, rder;
    kcig_geometry g;
    if (!fwd) {
        if ((rc = open3(m, "seismic_data", &dat, "Need 3D data volume for seismic_data= (t,h/r,s)"))) return fail(rc);
        g.nt = dat.n[0];
        g.nh = dat.n[1];
        g.ns = dat.n[2];
        g.t0 = (float)dat.o[0];
        g.dt = (float)dat.d[0];
        g.h0 = (float)dat.o[1];
        g.dh = (float)dat.d[1];
        g.s0 = (float)dat.o[2];
        g.ds = (float)dat.d[2];
    } else {
        // the data geometry comes from the parameters (:663-701)
        struct { const char *k; int *v; int def; const char *need; } ints[3] = {
            {"nt", &g.nt, 0, "Need nt="}, {"nh", &g.nh, 1, nullptr}, {"ns", &g.ns, 1, nullptr}};
        for (auto &q : ints) {
            if (!m.have(q.k)) {
                if (q.need) return fail(set_error(KCIG_ERR_ARG, "%s", q.need));
                *q.v = q.def;
            } else if ((rc = m.get_int(q.k, q.v))) {
                return fail(rc);
            }
        }
        struct { const char *k; float *v; const char *need; } fls[5] = {
            {"t0", &g.t0, nullptr}, {"dt", &g.dt, "Need dt="}, {"h0", &g.h0, nullptr}, {"dh", &g.dh, "Need dh="},
            {"s0", &g.s0, nullptr}};
        for (auto &q : fls) {
            if (!m.have(q.k)) {
                if (q.need) return fail(set_error(KCIG_ERR_ARG, "%s", q.need));
                *q.v = 0.0f;
            } else if ((rc = m.get_float(q.k, q.v))) {
                return fail(rc);
            }
        }
        if (!m.have("ds")) return fail(set_error(KCIG_ERR_ARG, "Need ds="));
        if ((rc = m.get_float("ds", &g.ds))) return fail(rc);
        if (g.nt < 1 || g.nh < 1 || g.ns < 1) return fail(set_error(KCIG_ERR_ARG, "Need 3D data volume for seismic_data= (t,h/r,s)"));
    }
    if (g.nh == 1) g.dh = 0.0f;
    if (g.ns == 1) g.ds = 0.0f;
    if (p.direct_mute && p.direct_mute_qc_shot >= g.ns)
        return fail(set_error(KCIG_ERR_ARG, "direct_mute_qc_shot=%d is outside the input shot range [0,%d].",
                              p.direct_mute_qc_shot, g.ns - 1));
    const bool qc = p.direct_mute && p.direct_mute_qc_shot >= 0;
    if (qc && (!m.have("direct_mute_qc_before") || !m.have("direct_mute_qc_after")))
        return fail(set_error(KCIG_ERR_ARG,
                              "direct_mute_qc_shot requires direct_mute_qc_before= and direct_mute_qc_after=."));
    if ((rc = open3(m, "stable", &stim, "Need 3D data volume for stable= (z,x,s)"))) return fail(rc);
    if ((rc = open3(m, "sderiv", &sder, "Need 3D data volume for sderiv= (z,x,s)"))) return fail(rc);
    g.nz = stim.n[0];
    g.nx = stim.n[1];
    g.sny = stim.n[2];
    if (sder.n[0] != g.nz || sder.n[1] != g.nx || sder.n[2] != g.sny)
        return fail(set_error(KCIG_ERR_ARG,
                              "Dimension mismatch between stable= and sderiv=. Expected sderiv n1=%d n2=%d n3=%d", g.nz,
                              g.nx, g.sny));
    g.z0 = (float)stim.o[0];
    g.dz = (float)stim.d[0];
    g.x0 = (float)stim.o[1];
    g.dx = (float)stim.d[1];
    g.sy0 = (float)stim.o[2];
    g.sdy = (float)stim.d[2];
    if ((rc = open3(m, "rtable", &rtim, "Need 3D data volume for rtable= (z,x,r)"))) return fail(rc);
    if ((rc = open3(m, "rderiv", &rder, "Need 3D data volume for rderiv= (z,x,r)"))) return fail(rc);
    if (rtim.n[0] != g.nz || rtim.n[1] != g.nx)
        return fail(set_error(KCIG_ERR_ARG, "Dimension mismatch in rtable=. Expected n1=%d n2=%d", g.nz, g.nx));
    g.rny = rtim.n[2];
    if (rder.n[0] != g.nz || rder.n[1] != g.nx || rder.n[2] != g.rny)
        return fail(set_error(KCIG_ERR_ARG,
                              "Dimension mismatch between rtable= and rderiv=. Expected rderiv n1=%d n2=%d n3=%d", g.nz,
                              g.nx, g.rny));
    g.ry0 = (float)rtim.o[2];
    g.rdy = (float)rtim.d[2];
    RsfFile gv[4];
    const char *gk[4] = {"sgradx", "sgradz", "rgradx", "rgradz"};
    if (use_grad) {
        for (int q = 0; q < 4; q++) {
            char need3[128];
            snprintf(need3, sizeof need3, "Need 3D data volume for %s= (z,x,source_or_receiver)", gk[q]);
            if ((rc = open3(m, gk[q], &gv[q], need3))) return fail(rc);
            const int n3 = q < 2 ? g.sny : g.rny;
            if (gv[q].n[0] != g.nz || gv[q].n[1] != g.nx || gv[q].n[2] != n3)
                return fail(set_error(KCIG_ERR_ARG, "Dimension mismatch in %s=. Expected n1=%d n2=%d n3=%d", gk[q], g.nz,
                                      g.nx, n3));
        }
    }
    // read everything (host), migrate on the device
    const size_t nzx = (size_t)g.nz * g.nx;
    std::vector<float> data((size_t)g.nt * g.nh * g.ns);
    std::vector<float> st(nzx * g.sny), sd(nzx * g.sny);
    if (!fwd && (rc = rsf_read(dat, 0, (long long)data.size(), data.data()))) return fail(rc);
    if ((rc = rsf_read(stim, 0, (long long)st.size(), st.data()))) return fail(rc);
    if ((rc = rsf_read(sder, 0, (long long)sd.size(), sd.data()))) return fail(rc);
    const bool same_r = (rtim.binary == stim.binary && rder.binary == sder.binary && g.rny == g.sny);
    std::vector<float> rt, rd;
    if (!same_r) {
        rt.resize(nzx * g.rny);
        rd.resize(nzx * g.rny);
        if ((rc = rsf_read(rtim, 0, (long long)rt.size(), rt.data()))) return fail(rc);
        if ((rc = rsf_read(rder, 0, (long long)rd.size(), rd.data()))) return fail(rc);
    }
    std::vector<float> gvol[4];
    if (use_grad)
        for (int q = 0; q < 4; q++) {
            gvol[q].resize(nzx * (q < 2 ? g.sny : g.rny));
            if ((rc = rsf_read(gv[q], 0, (long long)gvol[q].size(), gvol[q].data()))) return fail(rc);
        }
    if (qc) {
        const int is = p.direct_mute_qc_shot;
        std::vector<float> before(data.begin() + (size_t)is * g.nh * g.nt,
                                  data.begin() + (size_t)(is + 1) * g.nh * g.nt);
        std::vector<float> after(before);
        const float s = g.s0 + (float)is * g.ds;
        for (int ih = 0; ih < g.nh; ih++) {
            const float h = g.h0 + (float)ih * g.dh;
            qc_mute(after.data() + (size_t)ih * g.nt, g.nt, g.t0, g.dt, s, p.cmp ? s + h : h, p);
        }
        const int n2[2] = {g.nt, g.nh};
        const double o2[2] = {g.t0, g.h0}, d2[2] = {g.dt, g.dh};
        std::vector<std::pair<std::string, std::string>> k2 = {
            {"label1", "Time"}, {"unit1", "s"}, {"label2", p.cmp ? "Offset" : "Receiver"}};
        if ((rc = rsf_write(m.str("direct_mute_qc_before"), 2, n2, o2, d2, k2, before.data(), (long long)before.size())))
            return fail(rc);
        if ((rc = rsf_write(m.str("direct_mute_qc_after"), 2, n2, o2, d2, k2, after.data(), (long long)after.size())))
            return fail(rc);
    }
    kcig_plan *plan = nullptr;
    if ((rc = kcig_plan_create(&p, &g, 0, &plan))) return fail(rc);
    int ng;
    float g0, dg;
    kcig_output_axis(&p, &g, &ng, &g0, &dg);
    char msg[256];
    snprintf(msg, sizeof msg, "cig = %d, mode = %s, n3 = %d, o3 = %g, d3 = %g", p.cig, p.cig_is_angle ? "angle" : "offset",
             ng, g0, dg);
    log_line("INFO", msg);
    std::vector<float> img((size_t)ng * nzx);
    auto t_start = std::chrono::steady_clock::now();
    rc = kcig_plan_set_tables(plan, st.data(), sd.data(), same_r ? st.data() : rt.data(), same_r ? sd.data() : rd.data(),
                              KCIG_MEM_HOST);
    if (!rc && use_grad)
        rc = kcig_plan_set_gradients(plan, gvol[0].data(), gvol[1].data(), gvol[2].data(), gvol[3].data(), KCIG_MEM_HOST);
    if (fwd) {
        // the model: nzx * ng floats of migration= (:966), whatever its header says
        RsfFile mig;
        if (!rc) rc = rsf_open(m.str("migration"), &mig);
        if (!rc) rc = rsf_read(mig, 0, (long long)img.size(), img.data());
        if (!rc) rc = kcig_model(plan, img.data(), data.data(), KCIG_MEM_HOST);
    } else if (!rc) {
        rc = kcig_migrate(plan, data.data(), img.data(), KCIG_MEM_HOST);
    }
    kcig_plan_destroy(plan);
    if (rc) return fail(rc);
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    log_line("INFO", "FINISH.");
    snprintf(msg, sizeof msg, "Done. Elapsed time: %.3f s.", el);
    log_line("INFO", msg);
    if (fwd) {
        // the data header of :906-920, with its three axes
        const int n3[3] = {g.nt, g.nh, g.ns};
        const double o3[3] = {g.t0, g.h0, g.s0};
        const double d3[3] = {g.dt, g.dh, g.ds};
        std::vector<std::pair<std::string, std::string>> keys = {
            {"label1", "Time"}, {"unit1", "s"}, {"label2", p.cmp ? "Offset" : "Receiver"}, {"label3", "Shot"}};
        if ((rc = rsf_write(m.str("seismic_data"), 3, n3, o3, d3, keys, data.data(), (long long)data.size())))
            return fail(rc);
        return KCIG_OK;
    }
    // output header (:876-905)
    const int n3[3] = {g.nz, g.nx, p.cig ? ng : 1};
    const double o3[3] = {g.z0, g.x0, p.cig ? (double)g0 : 0.0};
    const double d3[3] = {g.dz, g.dx, p.cig ? (double)dg : 1.0};
    std::vector<std::pair<std::string, std::string>> keys = {{"label1", "Depth"}, {"label2", "Lateral"}};
    auto unit = dat.extra.find("unit1");
    if (unit != dat.extra.end()) keys.push_back({"unit1", unit->second});
    if (p.cig) {
        if (p.cig_is_angle) {
            keys.push_back({"label3", p.half_angle ? "Half-opening angle" : "Scattering angle"});
            keys.push_back({"unit3", "degree"});
        } else {
            keys.push_back({"label3", p.cmp ? "Offset" : "Receiver"});
            if (unit != dat.extra.end()) keys.push_back({"unit3", unit->second});
        }
    }
    if ((rc = rsf_write(m.str("migration"), 3, n3, o3, d3, keys, img.data(), (long long)img.size()))) return fail(rc);
    return KCIG_OK;
}

extern "C" int kcig_run_cli(int argc, char **argv)
{
    rsf_set_program("kirchmig2d_cig");
    return run_tool(argc, argv, 0);
}

extern "C" int kcig_run_kirchmig2d_cli(int argc, char **argv)
{
    rsf_set_program("kirchmig2d");
    return run_tool(argc, argv, 1);
}
