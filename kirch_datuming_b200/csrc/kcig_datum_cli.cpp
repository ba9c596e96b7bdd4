// kcig_run_greensol_auto_cli and kcig_run_kirchdat2d_freq_cli: the drop-in
// greensol_auto (src/greensol_auto.cpp:23-101) and kirchdat2d_freq
// (src/kirchdat2d_frequency_cs.cpp:1177-1413).  Same argv keys, defaults,
// checks in the same order, INFO lines, ERROR texts and output headers; the
// datuming runs on the device (kcig_datum_freq).
#include <errno.h>
#include <limits.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <chrono>
#include <string>
#include <vector>

#include "kcig_common.h"
#include "kcig_par.h"
#include "kcig_rsf.h"

using namespace kcig;

namespace {

void log_line(const char *lvl, const char *msg) { fprintf(stderr, "%d %s:%s\n", (int)getpid(), lvl, msg); }

int fail(int rc)
{
    log_line("ERROR", kcig_last_error());
    return rc;
}

// sep_have_hdr_int / sep_get_hdr_int: a header value that parse_int accepts
// (SEBASIC/src/se_util.cpp:355-384: optional sign, digits only, int range)
bool header_int(const RsfFile &f, const char *key, int *v)
{
    const auto it = f.extra.find(key);
    if (it == f.extra.end()) return false;
    const char *s = it->second.c_str();
    if (*s != '+' && *s != '-' && (*s < '0' || *s > '9')) return false;
    char *e = nullptr;
    errno = 0;
    const long x = strtol(s, &e, 10);
    if (e == s || *e || errno == ERANGE || x < INT_MIN || x > INT_MAX) return false;
    *v = (int)x;
    return true;
}

float from_xdr(float v)
{
    uint32_t u;
    memcpy(&u, &v, 4);
    u = __builtin_bswap32(u);
    memcpy(&v, &u, 4);
    return v;
}

}  // namespace

extern "C" int kcig_run_greensol_auto_cli(int argc, char **argv)
{
    rsf_set_program("greensol_auto");
    ParMap m;
    int rc = m.parse(argc, argv);
    if (rc) return fail(rc);
    if (!m.have("ttabel_file")) return fail(set_error(KCIG_ERR_ARG, "Need ttabel_file="));
    if (!m.have("tgreen_file")) return fail(set_error(KCIG_ERR_ARG, "Need tgreen_file="));
    if (!m.have("model_file")) return fail(set_error(KCIG_ERR_ARG, "Need model_file="));
    RsfFile tt, model;
    if ((rc = rsf_open(m.str("ttabel_file"), &tt))) return fail(rc);
    if ((rc = rsf_open(m.str("model_file"), &model))) return fail(rc);
    if (tt.ndim < 3) return fail(set_error(KCIG_ERR_ARG, "Need 3D data volume for ttabel= (z,x,gx)"));
    const int nz = tt.n[0], nx = tt.n[1], ngx = tt.n[2];
    const float dz = (float)tt.d[0], dx = (float)tt.d[1], oz = (float)tt.o[0], ox = (float)tt.o[1];
    const float dgx = (float)tt.d[2], ogx = (float)tt.o[2];
    int should_datum = 0;
    if (!header_int(model, "should_datum", &should_datum))
        return fail(set_error(KCIG_ERR_ARG, "Need should_datum in model_file header"));
    char msg[512];
    snprintf(msg, sizeof msg, "Read should_datum=%d from %s", should_datum, m.str("model_file").c_str());
    log_line("INFO", msg);
    const float datum = (float)(model.o[0] + should_datum * model.d[0]);
    // only the datum row of every (gx, x) column is needed: read each column's
    // sample where it lies (the reference seeks sample by sample, :84-93)
    const int idatum = (int)((datum - oz) / dz + 0.5);
    if (idatum < 0 || idatum >= nz) return fail(set_error(KCIG_ERR_ARG, "Datum out of range."));
    std::vector<float> slice((size_t)ngx * nx);
    FILE *fp = fopen(tt.binary.c_str(), "rb");
    if (!fp) return fail(set_error(KCIG_ERR_IO, "Cannot open data file '%s' of '%s'", tt.binary.c_str(), tt.path.c_str()));
    for (size_t k = 0; k < slice.size(); k++) {
        if (fseeko(fp, (off_t)((k * (size_t)nz + idatum) * 4), SEEK_SET) != 0 || fread(&slice[k], 4, 1, fp) != 1) {
            fclose(fp);
            return fail(set_error(KCIG_ERR_IO, "Failed to read '%s' (file truncated)", tt.binary.c_str()));
        }
        if (!tt.native) slice[k] = from_xdr(slice[k]);
    }
    fclose(fp);
    // the gather itself, on the (ngx, nx, 1) slice at datum row 0
    std::vector<float> green((size_t)ngx * ngx);
    if ((rc = kcig_green_slice(slice.data(), 1, nx, ngx, 0.0f, ox, 1.0f, dx, ogx, dgx, 0.0f, green.data(),
                               KCIG_MEM_HOST, nullptr)))
        return fail(rc);
    // header of :57-62: two axes, only the first one set
    const int n[2] = {ngx, 1};
    const double o[2] = {ogx, 0.0}, d[2] = {dgx, 1.0};
    if ((rc = rsf_write(m.str("tgreen_file"), 2, n, o, d, {}, green.data(), (long long)green.size()))) return fail(rc);
    return KCIG_OK;
}

extern "C" int kcig_run_kirchdat2d_freq_cli(int argc, char **argv)
{
    rsf_set_program("kirchdat2d_freq");
    ParMap m;
    int rc = m.parse(argc, argv);
    if (rc) return fail(rc);
    static const char *need[5][2] = {{"input_file", "Need input_file="},
                                     {"output_file", "Need output_file="},
                                     {"sgreen_file", "Need sgreen_file="},
                                     {"rgreen_file", "Need rgreen_file="},
                                     {"model_file", "Need model_file="}};
    for (auto &k : need)
        if (!m.have(k[0])) return fail(set_error(KCIG_ERR_ARG, "%s", k[1]));
    RsfFile in, model;
    if ((rc = rsf_open(m.str("input_file"), &in))) return fail(rc);
    if ((rc = rsf_open(m.str("model_file"), &model))) return fail(rc);
    kcig_datum_params p;
    kcig_datum_params_init(&p);
    int verb = 1, auto_datum = 1;
    if (m.have("verb")) m.get_int("verb", &verb);
    if (m.have("cmp")) m.get_int("cmp", &p.cmp);
    if (p.cmp != 0 && p.cmp != 1) return fail(set_error(KCIG_ERR_ARG, "cmp must be 0 or 1."));
    if (m.have("auto_datum")) m.get_int("auto_datum", &auto_datum);
    if (auto_datum != 0 && auto_datum != 1) return fail(set_error(KCIG_ERR_ARG, "auto_datum must be 0 or 1."));
    if (auto_datum) {
        int should_datum = 0;
        if (!header_int(model, "should_datum", &should_datum))
            return fail(set_error(KCIG_ERR_ARG, "Need should_datum in model_file header when auto_datum=1"));
        p.sdatum = (float)(model.o[0] + should_datum * model.d[0]);
        p.rdatum = p.sdatum;
    } else {
        if (!m.have("sdatum")) return fail(set_error(KCIG_ERR_ARG, "Need sdatum= when auto_datum=0"));
        if (!m.have("rdatum")) return fail(set_error(KCIG_ERR_ARG, "Need rdatum= when auto_datum=0"));
        m.get_float("sdatum", &p.sdatum);
        m.get_float("rdatum", &p.rdatum);
    }
    if (m.have("use_bf")) m.get_int("use_bf", &p.use_bf);
    if (m.have("bf_p")) m.get_int("bf_p", &p.bf_p);
    if (m.have("bf_n_leaf")) m.get_int("bf_n_leaf", &p.bf_n_leaf);
    if (m.have("bf_panel_levels")) m.get_int("bf_panel_levels", &p.bf_panel_levels);
    if (m.have("bf_amp_eps")) m.get_float("bf_amp_eps", &p.bf_amp_eps);
    if (m.have("bf_phase_tol")) m.get_float("bf_phase_tol", &p.bf_phase_tol);
    if (p.bf_p <= 0 || p.bf_n_leaf <= 1) return fail(set_error(KCIG_ERR_ARG, "Need bf_p > 0 and bf_n_leaf > 1."));
    if (p.bf_p >= p.bf_n_leaf)
        return fail(set_error(KCIG_ERR_ARG,
                              "Need bf_p < bf_n_leaf for meaningful butterfly interpolation / exact leaf-stage settings."));
    char msg[512];
    snprintf(msg, sizeof msg, "Use butterfly: %s.", p.use_bf ? "yes" : "no");
    log_line("INFO", msg);
    snprintf(msg, sizeof msg,
             "Adaptive segmented butterfly parameters: p = %d, n_leaf = %d, panel_levels = %d, amp_eps = %g, phase_tol = %g.",
             p.bf_p, p.bf_n_leaf, p.bf_panel_levels, (double)p.bf_amp_eps, (double)p.bf_phase_tol);
    log_line("INFO", msg);
    if (m.have("aperture")) m.get_int("aperture", &p.aperture);
    if (m.have("taper")) m.get_int("taper", &p.taper);
    if (m.have("data_taper")) m.get_int("data_taper", &p.data_taper);
    if (p.data_taper < 0) return fail(set_error(KCIG_ERR_ARG, "data_taper must be >= 0."));
    if (m.have("antialias")) m.get_float("antialias", &p.antialias);
    if (p.antialias < 0.0f) return fail(set_error(KCIG_ERR_ARG, "antialias must be >= 0."));
    if (m.have("length")) m.get_float("length", &p.length);
    if (in.ndim < 3) return fail(set_error(KCIG_ERR_ARG, "Input must be 3D."));
    p.nt = in.n[0];
    p.nh = in.n[1];
    p.ns = in.n[2];
    p.dt = (float)in.d[0];
    p.h0 = (float)in.o[1];
    p.dh = (float)in.d[1];
    p.s0 = (float)in.o[2];
    p.ds = (float)in.d[2];
    RsfFile sg, rg;
    if ((rc = rsf_open(m.str("sgreen_file"), &sg))) return fail(rc);
    if (sg.ndim < 2) return fail(set_error(KCIG_ERR_ARG, "Source Green's function must be 2D."));
    p.nsg = sg.n[0];
    p.sg0 = (float)sg.o[0];
    p.dsg = (float)sg.d[0];
    std::vector<float> st((size_t)p.nsg * p.nsg), rt;
    if ((rc = rsf_read(sg, 0, (long long)st.size(), st.data()))) return fail(rc);
    if ((rc = rsf_open(m.str("rgreen_file"), &rg))) return fail(rc);
    if (rg.ndim < 2) return fail(set_error(KCIG_ERR_ARG, "Receiver Green's function must be 2D."));
    p.nrg = rg.n[0];
    p.rg0 = (float)rg.o[0];
    p.drg = (float)rg.d[0];
    rt.resize((size_t)p.nrg * p.nrg);
    if ((rc = rsf_read(rg, 0, (long long)rt.size(), rt.data()))) return fail(rc);
    if (verb) {
        snprintf(msg, sizeof msg,
                 "data_taper = %d traces on both source and receiver/offset edges; set data_taper=0 to disable.",
                 p.data_taper);
        log_line("INFO", msg);
        snprintf(msg, sizeof msg, "antialias = %g; set antialias=0 to disable frequency-domain operator anti-aliasing.",
                 (double)p.antialias);
        log_line("INFO", msg);
    }
    const size_t ntr = (size_t)p.ns * p.nh, total = ntr * (size_t)p.nt;
    std::vector<float> data(total), out(total), interm;
    if ((rc = rsf_read(in, 0, (long long)total, data.data()))) return fail(rc);
    const bool want_interm = m.have("interm");
    if (want_interm) interm.resize(total);
    const auto t0 = std::chrono::steady_clock::now();
    if ((rc = kcig_datum_freq(&p, st.data(), rt.data(), data.data(), out.data(), want_interm ? interm.data() : nullptr,
                              KCIG_MEM_HOST, nullptr)))
        return fail(rc);
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    snprintf(msg, sizeof msg, "Done. Elapsed time: %.3f s.", el);
    log_line("INFO", msg);
    if (want_interm) {  // the reference leaves this header's axes unset (:1331-1335)
        const int n1[1] = {1};
        const double o1[1] = {0.0}, d1[1] = {1.0};
        if ((rc = rsf_write(m.str("interm"), 1, n1, o1, d1, {}, interm.data(), (long long)total))) return fail(rc);
    }
    // output header (:1383-1392)
    const int n[3] = {p.nt, p.nh, p.ns};
    const double o[3] = {0.0, p.h0, p.s0}, d[3] = {p.dt, p.dh, p.ds};
    if ((rc = rsf_write(m.str("output_file"), 3, n, o, d, {}, out.data(), (long long)total))) return fail(rc);
    return KCIG_OK;
}
