// Parameter block of kirchmig2d_cig (src/kirchmig2d_cig.cpp:494-958) and the
// output-axis resolution of parse_output_axis (:323-368).
#include <ctype.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <fstream>
#include <sstream>
#include <string>

#include "kcig_common.h"
#include "kcig_par.h"

namespace kcig {

static thread_local std::string g_err = "no error";

int set_error(int code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_error(cudaError_t e, const char *what)
{
    return set_error(e == cudaErrorMemoryAllocation ? KCIG_ERR_NOMEM : KCIG_ERR_CUDA, "CUDA error %s (%s) in %s",
                     cudaGetErrorName(e), cudaGetErrorString(e), what);
}

// ------------------------------------------------------------------ ParMap --
static std::string unquote(std::string v)
{
    if (v.size() >= 2 && ((v.front() == '"' && v.back() == '"') || (v.front() == '\'' && v.back() == '\'')))
        v = v.substr(1, v.size() - 2);
    return v;
}

void ParMap::add_token(const std::string &tok)
{
    const size_t eq = tok.find('=');
    if (eq == std::string::npos || eq == 0) return;
    std::string k = tok.substr(0, eq);
    while (!k.empty() && isspace((unsigned char)k.back())) k.pop_back();
    while (!k.empty() && isspace((unsigned char)k.front())) k.erase(k.begin());
    if (k.empty()) return;
    kv_[k] = unquote(tok.substr(eq + 1));
}

int ParMap::add_file(const std::string &path)
{
    std::ifstream f(path);
    if (!f) return set_error(KCIG_ERR_IO, "Cannot open parameter file '%s'", path.c_str());
    std::string line;
    while (std::getline(f, line)) {
        const size_t h = line.find('#');
        if (h != std::string::npos) line = line.substr(0, h);
        // split on white space, keeping quoted values together
        size_t i = 0;
        while (i < line.size()) {
            while (i < line.size() && isspace((unsigned char)line[i])) i++;
            if (i >= line.size()) break;
            std::string tok;
            char q = 0;
            while (i < line.size() && (q || !isspace((unsigned char)line[i]))) {
                const char c = line[i++];
                if (q && c == q) q = 0;
                else if (!q && (c == '"' || c == '\'')) q = c;
                tok.push_back(c);
            }
            if (tok.rfind("par=", 0) == 0) {
                int rc = add_file(unquote(tok.substr(4)));
                if (rc) return rc;
            } else {
                add_token(tok);
            }
        }
    }
    return KCIG_OK;
}

int ParMap::parse(int argc, char **argv)
{
    for (int i = 1; i < argc; i++) {
        if (!argv[i]) continue;
        std::string t = argv[i];
        if (t.rfind("par=", 0) == 0) {
            int rc = add_file(t.substr(4));
            if (rc) return rc;
        } else {
            add_token(t);
        }
    }
    return KCIG_OK;
}

int ParMap::get_int(const char *k, int *v) const
{
    *v = (int)strtod(str(k).c_str(), nullptr);
    return KCIG_OK;
}

int ParMap::get_float(const char *k, float *v) const
{
    *v = (float)strtod(str(k).c_str(), nullptr);
    return KCIG_OK;
}

static bool ieq(const char *a, const char *b)
{
    while (*a && *b) {
        if (tolower((unsigned char)*a) != tolower((unsigned char)*b)) return false;
        a++;
        b++;
    }
    return *a == 0 && *b == 0;
}

// Fill p from an already parsed map; the reference's order and validation.
int params_from_map(const ParMap &m, kcig_params *p)
{
    kcig_params_init(p);
    if (m.have("aperture_trace")) m.get_int("aperture_trace", &p->aperture_trace);
    const bool mode_given = m.have("mode") || m.have("cig_mode");
    std::string mode = m.have("mode") ? m.str("mode") : (m.have("cig_mode") ? m.str("cig_mode") : "offset");
    if (ieq(mode.c_str(), "offset")) p->cig_is_angle = 0;
    else if (ieq(mode.c_str(), "angle")) p->cig_is_angle = 1;
    else
        return set_error(KCIG_ERR_ARG, "Unknown CIG mode: %s. Supported modes are offset and angle.", mode.c_str());
    p->adj = 1;
    if (m.have("adj")) m.get_int("adj", &p->adj);
    p->cig = mode_given ? 1 : 0;
    if (m.have("cig")) m.get_int("cig", &p->cig);
    p->cmp = 1;
    if (m.have("cmp")) m.get_int("cmp", &p->cmp);
    if (m.have("half_angle")) m.get_int("half_angle", &p->half_angle);
    if (p->half_angle) {
        p->oazmin = 40.0f;
        p->oazmax = 25.0f;
    }
    if (m.have("oazmin")) m.get_float("oazmin", &p->oazmin);
    if (m.have("oazmax")) m.get_float("oazmax", &p->oazmax);
    if (m.have("oaztaper")) m.get_float("oaztaper", &p->oaztaper);
    if (m.have("diff")) m.get_int("diff", &p->isdiff);
    if (m.have("direct_mute")) m.get_int("direct_mute", &p->direct_mute);
    if (m.have("direct_mute_slope")) m.get_float("direct_mute_slope", &p->direct_mute_slope);
    if (m.have("direct_mute_invert")) m.get_int("direct_mute_invert", &p->direct_mute_invert);
    if (m.have("direct_mute_intercept")) m.get_float("direct_mute_intercept", &p->direct_mute_intercept);
    if (m.have("direct_mute_taper")) m.get_float("direct_mute_taper", &p->direct_mute_taper);
    if (m.have("direct_mute_qc_shot")) m.get_int("direct_mute_qc_shot", &p->direct_mute_qc_shot);
    if (p->direct_mute) {
        // :719-738 (the shot-range check needs ns and lives in the plan/CLI)
        if (!p->adj)
            return set_error(KCIG_ERR_ARG, "direct_mute=1 is an input-data preprocessing option and requires adj=1.");
        if (!isfinite(p->direct_mute_slope) || p->direct_mute_slope < 0.0f)
            return set_error(KCIG_ERR_ARG, "direct_mute_slope must be finite and non-negative.");
        if (!isfinite(p->direct_mute_intercept))
            return set_error(KCIG_ERR_ARG, "direct_mute_intercept must be finite.");
        if (!isfinite(p->direct_mute_taper) || p->direct_mute_taper <= 0.0f)
            return set_error(KCIG_ERR_ARG, "direct_mute_taper must be finite and positive to avoid a hard cutoff.");
        if (p->direct_mute_invert != 0 && p->direct_mute_invert != 1)
            return set_error(KCIG_ERR_ARG, "direct_mute_invert must be 0 or 1.");
        if (p->direct_mute_qc_shot < -1)
            return set_error(KCIG_ERR_ARG, "direct_mute_qc_shot must be -1 (disabled) or a zero-based shot index.");
    }
    if (m.have("tau")) m.get_float("tau", &p->tau);
    if (m.have("aperture")) m.get_float("aperture", &p->aperture);
    if (m.have("aperture_taper")) m.get_float("aperture_taper", &p->aperture_taper);
    if (m.have("aperture_rmin")) m.get_float("aperture_rmin", &p->aperture_rmin);
    if (m.have("aperture_rtaper")) m.get_float("aperture_rtaper", &p->aperture_rtaper);
    if (m.have("antialias")) m.get_float("antialias", &p->antialias);
    if (m.have("angle_interp")) m.get_int("angle_interp", &p->angle_interp);
    if (m.have("angle_taper_start")) m.get_float("angle_taper_start", &p->angle_taper_start);
    if (m.have("angle_taper_end")) m.get_float("angle_taper_end", &p->angle_taper_end);
    if (m.have("angle_grad_radius")) m.get_int("angle_grad_radius", &p->angle_grad_radius);
    if (p->angle_grad_radius < 1) p->angle_grad_radius = 1;
    if (m.have("angle_smooth")) m.get_int("angle_smooth", &p->angle_smooth);
    if (p->angle_smooth < 0) p->angle_smooth = 0;
    if (m.have("aperture_trace_taper")) m.get_int("aperture_trace_taper", &p->aperture_trace_taper);
    if (p->aperture_trace_taper < 0) p->aperture_trace_taper = 0;
    // parse_output_axis (:323-368): cig_* first, then the mode's own keys
    const char *pre[2] = {"cig", p->cig_is_angle ? "angle" : "offset"};
    for (int s = 0; s < 2; s++) {
        char key[64];
        snprintf(key, sizeof key, "%s_min", pre[s]);
        if (m.have(key)) { m.get_float(key, &p->axis_min); p->axis_min_given = 1; }
        snprintf(key, sizeof key, "%s_max", pre[s]);
        if (m.have(key)) { m.get_float(key, &p->axis_max); p->axis_max_given = 1; }
        snprintf(key, sizeof key, "%s_step", pre[s]);
        if (m.have(key)) { m.get_float(key, &p->axis_step); p->axis_step_given = 1; }
        snprintf(key, sizeof key, "%s_n", pre[s]);
        if (m.have(key)) { m.get_int(key, &p->axis_n); p->axis_n_given = 1; }
    }
    std::string type = m.have("type") ? m.str("type") : "hermit";
    if (type.empty() || (type[0] != 'l' && type[0] != 'p' && type[0] != 'h'))
        return set_error(KCIG_ERR_ARG,
                         "Unknown interpolation type: %s. Supported types are linear (l), partial (p), and hermite (h)",
                         type.c_str());
    p->interp_type = type[0];
    return KCIG_OK;
}

// kirchmig2d's parameter block (src/kirchmig2d.cpp:55-340): its own keys
// and defaults; everything it does not have stays off.
int params_from_map_kirchmig2d(const ParMap &m, kcig_params *p)
{
    kcig_params_init(p);
    p->tool = 1;
    p->cig_is_angle = 0;
    p->aperture_trace_taper = 0;  // a hard trace-index cut (:57-60, :423)
    p->aperture_taper = 0.0f;     // a hard cone (:459-486)
    p->aperture_rmin = 0.0f;
    p->direct_mute = 0;
    if (m.have("aperture_trace")) m.get_int("aperture_trace", &p->aperture_trace);
    if (m.have("adj")) m.get_int("adj", &p->adj);
    p->cig = 0;
    if (m.have("cig")) m.get_int("cig", &p->cig);
    p->cmp = 1;
    if (m.have("cmp")) m.get_int("cmp", &p->cmp);
    if (m.have("diff")) m.get_int("diff", &p->isdiff);
    if (m.have("tau")) m.get_float("tau", &p->tau);
    if (m.have("aperture")) m.get_float("aperture", &p->aperture);
    if (m.have("antialias")) m.get_float("antialias", &p->antialias);
    std::string type = m.have("type") ? m.str("type") : "hermit";
    if (type.empty() || (type[0] != 'l' && type[0] != 'p' && type[0] != 'h'))
        return set_error(KCIG_ERR_ARG,
                         "Unknown interpolation type: %s. Supported types are: linear (l), partial (p) and hermite (h)",
                         type.c_str());
    p->interp_type = type[0];
    return KCIG_OK;
}

}  // namespace kcig

using namespace kcig;

extern "C" int kcig_params_parse_kirchmig2d(int argc, char **argv, kcig_params *p)
{
    if (!p) return set_error(KCIG_ERR_ARG, "kcig_params_parse_kirchmig2d: null");
    ParMap m;
    int rc = m.parse(argc, argv);
    if (rc) return rc;
    return params_from_map_kirchmig2d(m, p);
}

extern "C" const char *kcig_last_error(void) { return g_err.c_str(); }

extern "C" int kcig_params_init(kcig_params *p)
{
    if (!p) return set_error(KCIG_ERR_ARG, "kcig_params_init: null");
    memset(p, 0, sizeof *p);
    p->adj = 1;
    p->cig = 0;
    p->cig_is_angle = 0;
    p->cmp = 1;
    p->half_angle = 0;
    p->isdiff = 0;
    p->interp_type = 'h';
    p->angle_interp = 1;
    p->angle_grad_radius = 2;
    p->angle_smooth = 2;
    p->aperture_trace = -1;
    p->aperture_trace_taper = 20;
    p->direct_mute = 0;
    p->direct_mute_invert = 0;
    p->direct_mute_qc_shot = -1;
    p->tau = 0.0f;
    p->aperture = 90.0f;
    p->aperture_taper = 10.0f;
    p->aperture_rmin = 0.0f;
    p->aperture_rtaper = 0.05f;
    p->antialias = 1.0f;
    p->angle_taper_start = -1.0f;
    p->angle_taper_end = -1.0f;
    p->oazmin = 80.0f;
    p->oazmax = 50.0f;
    p->oaztaper = 10.0f;
    p->direct_mute_slope = 0.0f;
    p->direct_mute_intercept = 0.0f;
    p->direct_mute_taper = 0.05f;
    return KCIG_OK;
}

extern "C" int kcig_params_parse(int argc, char **argv, kcig_params *p)
{
    if (!p) return set_error(KCIG_ERR_ARG, "kcig_params_parse: null");
    ParMap m;
    int rc = m.parse(argc, argv);
    if (rc) return rc;
    return params_from_map(m, p);
}

extern "C" int kcig_output_axis(const kcig_params *p, const kcig_geometry *g, int *ng, float *g0, float *dg)
{
    if (!p || !g) return set_error(KCIG_ERR_ARG, "kcig_output_axis: null");
    if (!p->cig) {
        *ng = 1;
        *g0 = 0.0f;
        *dg = 1.0f;
        return KCIG_OK;
    }
    if (p->tool == 1) {  // kirchmig2d: one image per offset index (:243, :283-287)
        *ng = g->nh;
        *g0 = g->h0;
        *dg = g->nh == 1 ? 0.0f : g->dh;
        return KCIG_OK;
    }
    const int is_angle = p->cig_is_angle;
    const int nh = g->nh;
    const float h0 = g->h0;
    const float dh = (g->nh == 1) ? 0.0f : g->dh;
    const float hend = h0 + (float)(nh - 1) * dh;
    float vmin = is_angle ? 0.0f : (h0 < hend ? h0 : hend);
    float vmax = is_angle ? (p->half_angle ? 90.0f : 180.0f) : (h0 > hend ? h0 : hend);
    float vstep = is_angle ? 1.0f : (dh != 0.0f ? fabsf(dh) : 1.0f);
    int nval = is_angle ? (p->half_angle ? 91 : 181) : nh;
    if (p->axis_min_given) vmin = p->axis_min;
    if (p->axis_max_given) vmax = p->axis_max;
    if (p->axis_step_given) vstep = p->axis_step;
    if (p->axis_n_given) nval = p->axis_n;
    if (vstep <= 0.0f) return set_error(KCIG_ERR_ARG, "CIG axis step must be positive.");
    if (!p->axis_n_given) nval = (int)floorf((vmax - vmin) / vstep + 0.5f) + 1;
    if (nval <= 0) return set_error(KCIG_ERR_ARG, "CIG axis sample number must be positive.");
    *g0 = vmin;
    *dg = vstep;
    *ng = nval;
    return KCIG_OK;
}
