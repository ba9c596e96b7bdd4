// kcig_run_eikods_cli: the drop-in eikods2d (src/eikods2d.cpp:149-765) for
// 2-D velocity files.  Same argv keys, defaults, required outputs, ERROR texts
// and output headers (n/o/d of the velocity's first two axes, the shot axis
// with o = first shot's lateral position and d = the spacing of the first two
// shots); the tables are computed on the GPU by kcig_eikods.
//
// Not built (KCIG_ERR_UNSUPPORTED with the key named): efmm=1 (the separate
// efmm.cpp solver), plane-wave sources (plane1/2/3), the second derivatives
// (tdl2=, tds2=) and 3-D velocity volumes (n3 > 1).
#include <cuda_runtime.h>
#include <stdio.h>
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

struct DevPtr {
    void *p = nullptr;
    ~DevPtr()
    {
        if (p) cudaFree(p);
    }
};

}  // namespace

extern "C" int kcig_run_eikods_cli(int argc, char **argv)
{
    rsf_set_program("eikods2d");
    if (argc < 2) {
        printf("eikods2d in=vel.rsf out=time.rsf tdl1=... tds1=... [shotfile= gradz= gradx= order=2 b1= b2= "
               "vel=1 l=1 zshot= yshot=]\n");
        return set_error(KCIG_ERR_ARG, "no parameters");
    }
    ParMap m;
    int rc = m.parse(argc, argv);
    if (rc) return fail(rc);
    if (!m.have("in")) return fail(set_error(KCIG_ERR_ARG, "Need in="));
    if (!m.have("out")) return fail(set_error(KCIG_ERR_ARG, "Need out="));
    RsfFile vel;
    if ((rc = rsf_open(m.str("in"), &vel))) return fail(rc);
    const int n1 = vel.n[0], n2 = vel.n[1], n3 = vel.n[2];
    const float d1 = (float)vel.d[0], d2 = (float)vel.d[1], d3 = (float)vel.d[2];
    const float o1 = (float)vel.o[0], o2 = (float)vel.o[1], o3 = (float)vel.o[2];
    printf("Reading velocity model from %s\nWriting traveltime to %s\nn1=%d, n2=%d, n3=%d\n", m.str("in").c_str(),
           m.str("out").c_str(), n1, n2, n3);

    int isvel = 1, order = 2, efmm = 0, l = 1;
    float br1 = d1, br2 = d2;
    if (m.have("vel") && (rc = m.get_int("vel", &isvel))) return fail(rc);
    if (m.have("order") && (rc = m.get_int("order", &order))) return fail(rc);
    if (m.have("efmm") && (rc = m.get_int("efmm", &efmm))) return fail(rc);
    if (m.have("br1") && (rc = m.get_float("br1", &br1))) return fail(rc);
    if (m.have("br2") && (rc = m.get_float("br2", &br2))) return fail(rc);
    for (const char *k : {"plane1", "plane2", "plane3"}) {
        int v = 0;
        if (m.have(k) && (rc = m.get_int(k, &v))) return fail(rc);
        if (v) return fail(set_error(KCIG_ERR_UNSUPPORTED, "%s=1 (plane-wave source) is not built", k));
    }
    if (efmm) return fail(set_error(KCIG_ERR_UNSUPPORTED, "efmm=1 is not built"));
    // the box in samples: b= wins over br= (physical), at least 1 (:244-263)
    int b1 = (int)(br1 / d1 + 0.5), b2 = (int)(br2 / d2 + 0.5);
    if (m.have("b1") && (rc = m.get_int("b1", &b1))) return fail(rc);
    if (m.have("b2") && (rc = m.get_int("b2", &b2))) return fail(rc);
    if (b1 < 1) b1 = 1;
    if (b2 < 1) b2 = 1;

    std::vector<float> shots;
    int nshot = 1;
    float oshot = 0.0f, dshot = 0.0f;
    if (m.have("shotfile")) {
        RsfFile sf;
        if ((rc = rsf_open(m.str("shotfile"), &sf))) return fail(rc);
        nshot = sf.n[1];
        if (sf.n[0] != 3) return fail(set_error(KCIG_ERR_ARG, "Need n1=3 in shotfile"));
        shots.resize(3 * (size_t)nshot);
        if ((rc = rsf_read(sf, 0, 3LL * nshot, shots.data()))) return fail(rc);
        oshot = shots[1];
        // the spacing of the first two shots (the reference reads past a
        // one-shot file here; 0 is written instead)
        dshot = nshot > 1 ? -shots[1] + shots[4] : 0.0f;
    } else {
        float zs = 0.0f, ys = (float)(o2 + 0.5 * (n2 - 1) * d2), xs = (float)(o3 + 0.5 * (n3 - 1) * d3);
        if (m.have("zshot") && (rc = m.get_float("zshot", &zs))) return fail(rc);
        if (m.have("yshot") && (rc = m.get_float("yshot", &ys))) return fail(rc);
        if (m.have("xshot") && (rc = m.get_float("xshot", &xs))) return fail(rc);
        shots = {zs, ys, xs};
        oshot = ys;
        dshot = (float)(-ys + (o2 + 0.5 * (n2 - 1) * d2));
        char msg[256];
        snprintf(msg, sizeof msg, "Shooting from zshot=%g yshot=%g xshot=%g", zs, ys, xs);
        log_line("INFO", msg);
    }
    if (n1 <= 0 || n2 <= 0 || n3 <= 0)
        return fail(set_error(KCIG_ERR_ARG, "Invalid input dimensions n1=%d n2=%d n3=%d", n1, n2, n3));
    if (n3 > 1) return fail(set_error(KCIG_ERR_UNSUPPORTED, "3-D velocity (n3=%d) is not built", n3));
    if (!m.have("tdl1")) return fail(set_error(KCIG_ERR_ARG, "Output derivative tdl1= missing."));
    if (!m.have("tds1")) return fail(set_error(KCIG_ERR_ARG, "Output derivative tds1= missing."));
    for (const char *k : {"tdl2", "tds2"})
        if (m.have(k)) return fail(set_error(KCIG_ERR_UNSUPPORTED, "%s= (second derivative) is not built", k));
    if (m.have("l") && (rc = m.get_int("l", &l))) return fail(rc);

    const size_t nzx = (size_t)n1 * n2, total = nzx * nshot;
    std::vector<float> hv(nzx);
    if ((rc = rsf_read(vel, 0, (long long)nzx, hv.data()))) return fail(rc);
    const bool gz = m.have("gradz"), gx = m.have("gradx");
    const auto t_start = std::chrono::steady_clock::now();
    DevPtr dv, dt, dl, ds, dgz, dgx;
    if (cudaMalloc(&dv.p, nzx * 4) != cudaSuccess || cudaMalloc(&dt.p, total * 4) != cudaSuccess ||
        cudaMalloc(&dl.p, total * 4) != cudaSuccess || cudaMalloc(&ds.p, total * 4) != cudaSuccess ||
        (gz && cudaMalloc(&dgz.p, total * 4) != cudaSuccess) || (gx && cudaMalloc(&dgx.p, total * 4) != cudaSuccess))
        return fail(set_error(KCIG_ERR_NOMEM, "eikods2d: device allocation of %zu samples failed", total));
    if (cudaMemcpy(dv.p, hv.data(), nzx * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(set_error(KCIG_ERR_CUDA, "eikods2d: velocity upload failed"));
    kcig_eikods_opts opt;
    opt.order = order;
    opt.b1 = b1;
    opt.b2 = b2;
    opt.l = l;
    opt.vel_is_slowness2 = isvel ? 0 : 1;
    opt.max_iter = 0;
    rc = kcig_eikods((const float *)dv.p, n1, n2, o1, o2, d1, d2, o3, d3, shots.data(), nshot, &opt, (float *)dt.p,
                     (float *)dl.p, (float *)ds.p, (float *)dgz.p, (float *)dgx.p, nullptr, nullptr);
    if (rc) return fail(rc);
    const int n[3] = {n1, n2, nshot};
    const double o[3] = {o1, o2, oshot}, d[3] = {d1, d2, dshot};
    std::vector<float> host(total);
    struct {
        const char *key;
        void *dev;
    } outs[5] = {{"out", dt.p}, {"tdl1", dl.p}, {"tds1", ds.p}, {"gradz", dgz.p}, {"gradx", dgx.p}};
    for (auto &q : outs) {
        if (!q.dev) continue;
        if (cudaMemcpy(host.data(), q.dev, total * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail(set_error(KCIG_ERR_CUDA, "eikods2d: download of %s failed", q.key));
        if ((rc = rsf_write(m.str(q.key), 3, n, o, d, {}, host.data(), (long long)total))) return fail(rc);
    }
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    char msg[128];
    snprintf(msg, sizeof msg, "%d shots done. Elapsed time: %.3f s.", nshot, el);
    log_line("INFO", msg);
    return KCIG_OK;
}
