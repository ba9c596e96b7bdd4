// Migration plan: host orchestration of the shot/trace loop of
// src/kirchmig2d_cig.cpp:979-1339 (adj=1) around the K1/K2/K3 kernels.
//
// The host resolves, once per trace and in double precision, everything the
// reference computes per trace with scalar code: source/receiver positions,
// the table slices and interpolation weights (:987-1029, :1148-1180), the
// trace-index aperture (:1082-1099) and the offset bin (:1100-1105).  The GPU
// does all per-sample and per-image-point work.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <tuple>
#include <mutex>
#include <vector>

#include "kcig_common.h"

using namespace kcig;

struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
    int ensure(size_t bytes)
    {
        if (bytes <= n && p) return KCIG_OK;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        if (bytes == 0) return KCIG_OK;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            p = nullptr;
            return cuda_error(e, "cudaMalloc(scratch)");
        }
        n = bytes;
        return KCIG_OK;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    template <class T> T *as() const { return (T *)p; }
};

struct kcig_plan {
    kcig_params p;
    kcig_geometry g;
    int ng = 1;
    float g0 = 0.f, dg = 1.f;
    int device = 0;
    cudaStream_t st = 0;
    unsigned long long budget = 0;
    const float *stab = nullptr, *sder = nullptr, *rtab = nullptr, *rder = nullptr;
    const float *sgx = nullptr, *sgz = nullptr, *rgx = nullptr, *rgz = nullptr;
    DevBuf own_stab, own_sder, own_rtab, own_rder, own_sgx, own_sgz, own_rgx, own_rgz;
    DevBuf d_data, d_image, d_rT, d_rF, d_sT, d_sF, d_work, d_D, d_legs, d_tr;
    DevBuf d_part;  // partial images of a split summation (small grids)
    DevBuf d_status;  // flag of the leg-field kernels' bounded waits (k_leg_tile)
    // tables left in host memory (KCIG_MEM_HOST_STREAM): the slices of each
    // leg batch are copied into d_stage
    int stream_tables = 0;
    const float *h_stab = nullptr, *h_sder = nullptr, *h_rtab = nullptr, *h_rder = nullptr;
    DevBuf d_stage;
    int sum_launches = 0, all_launches = 0;
    float sum_ms = 0.f, fields_ms = 0.f, prelude_ms = 0.f;
    kcig_surrogate *sg_src = nullptr, *sg_rcv = nullptr;  // leg fields from surrogates instead of tables
    int sg_angle = KCIG_SG_ANGLE_FD, sg_tx = KCIG_SG_TX_NETWORK;  // what the surrogates supply
    int shot_first = 0, shot_count = -1;  // kcig_plan_set_shot_range: shots of the survey kcig_migrate takes
    struct ShotsPrepared *shots = nullptr;                 // ragged shots uploaded by kcig_shots_prepare
    int use_graph = 0;                                     // replay kcig_migrate_prepared as a CUDA graph
    int tile = 0;                                          // summation tile variant (kcig_plan_autotune)
    cudaStream_t own_st = nullptr;                         // capture stream when the plan's is the legacy one
    // host traces are copied on their own non-blocking stream while the leg
    // fields compute (it does not synchronise with the legacy stream); the
    // first trace prelude waits for copy_ev
    cudaStream_t copy_st = nullptr;
    cudaEvent_t copy_ev = nullptr, order_ev = nullptr;
};

// Ragged shots on the device, batched (kcig_shots_prepare); the launch
// sequence that migrates them needs no host work, so it can be captured.
struct ShotBatch {
    int ns = 0, nhb = 0, nrl = 0;  // shots, padded receivers per shot, receiver legs
    size_t sleg0 = 0, rleg0 = 0;   // first source / receiver leg in `legs`
    size_t tr0 = 0, shot0 = 0;     // first padded trace, first shot
    int unit_tw = 0;
};
struct ShotsPrepared {
    std::vector<ShotBatch> batches;
    int nshots = 0, ntmax = 0;
    size_t ntr = 0;
    long long pairs = 0;
    DevBuf data, legs, trf, stop, snh;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    float *graph_image = nullptr;
};

static void release_shots(kcig_plan *P)
{
    if (!P->shots) return;
    ShotsPrepared *S = P->shots;
    if (S->exec) cudaGraphExecDestroy(S->exec);
    if (S->graph) cudaGraphDestroy(S->graph);
    S->data.release();
    S->legs.release();
    S->trf.release();
    S->stop.release();
    S->snh.release();
    delete S;
    P->shots = nullptr;
}

namespace {

int upload(DevBuf &b, const void *src, size_t bytes, cudaStream_t st)
{
    KCIG_TRY(b.ensure(bytes));
    KCIG_CUDA(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, st));
    return KCIG_OK;
}

// Slice choice and weights of one leg.  Which slice a position falls in is a
// discrete decision that, for a position on a table node, depends on the
// rounding of the reference's FP32 expression (pos - o)/d; it is therefore
// taken in that same FP32 arithmetic (posf is the position as the reference
// computes it in float).  The in-interval coordinate and all weights are FP64
// (from pos).  Returns the slice index the reference assigns to ist
// (:987-1016) or uses for the receiver (:1148-1180).
int leg_interp(const kcig_plan *P, int is_source, float posf, double pos, LegInterp *L)
{
    const kcig_geometry &g = P->g;
    const int n = is_source ? g.sny : g.rny;
    const float of = is_source ? g.sy0 : g.ry0;
    const float df = is_source ? g.sdy : g.rdy;
    const double o = of, d = df;
    memset(L, 0, sizeof *L);
    L->type = P->p.interp_type;
    L->pos = pos;
    L->posf = posf;
    L->i1 = -1;
    float f = 0.0f;
    bool left;
    int tool1_index = 0;
    if (P->p.tool == 1) {
        // kirchmig2d.cpp:372-395, :413-440: the index is the float quotient
        // truncated; at or below 0 the first slice and at or above n-1 the
        // last are taken unchanged (the first interval is not interpolated,
        // unlike kirchmig2d_cig); the raw index also drives aperture_trace
        tool1_index = (df != 0.0f) ? (int)((posf - of) / df) : 0;
        left = tool1_index <= 0;
        f = left ? 0.0f : (tool1_index >= n - 1 ? (float)(n - 1) : (float)tool1_index);
    } else if (is_source) {
        left = (n <= 1 || df == 0.0f);
        if (!left) f = (posf - of) / df;
        if (!left && f <= 0.0f) left = true;
    } else {
        if (n > 1 && df != 0.0f) f = (posf - of) / df;
        left = (n <= 1 || df == 0.0f || f <= 0.0f);
    }
    int ret;
    if (left) {
        L->i0 = 0;
        ret = 0;
    } else if (f >= (float)(n - 1)) {
        L->i0 = n - 1;
        ret = n - 1;
    } else {
        const int i0 = P->p.tool == 1 ? tool1_index : (int)floorf(f);
        const double x = pos - (o + (double)i0 * d);
        const double t = x / d;
        L->i0 = i0;
        L->i1 = i0 + 1;
        L->t = t;
        L->dxp = d;
        ret = i0;
        if (L->type == 'l') {
            // tinterp_linear / dinterp_linear (tinterpsr.cpp:37-70)
            L->c[0] = 1.0 - t; L->c[2] = t;
            L->e[0] = -1.0 / d; L->e[2] = 1.0 / d;
        } else if (L->type == 'p') {
            L->k1 = (int)(x / (double)g.dx + 0.5);
            L->k2 = (int)((d - x) / (double)g.dx + 0.5);
        } else {
            // tinterp_hermite / dinterp_hermite (tinterpsr.cpp:142-188)
            const double h00 = 2. * t * t * t - 3. * t * t + 1.;
            const double h10 = t * t * t - 2. * t * t + t;
            const double h01 = -2. * t * t * t + 3. * t * t;
            const double h11 = t * t * t - t * t;
            const double g00 = -6. * t * (1. - t);
            const double g10 = (1. - t) * (1. - 3. * t);
            const double g01 = 6. * t * (1. - t);
            const double g11 = 3. * t * t - 2. * t;
            L->c[0] = h00; L->c[1] = h10 * d; L->c[2] = h01; L->c[3] = h11 * d;
            L->e[0] = g00 / d; L->e[1] = g10; L->e[2] = g01 / d; L->e[3] = g11;
        }
    }
    if (P->p.tool == 1) ret = tool1_index;
    // interp_volume_linear_stream (:294-322) for the optional gradient files
    L->gi0 = 0;
    L->gi1 = 0;
    L->gw = 0.0;
    if (n > 1 && df != 0.0f) {
        const float fg = (posf - of) / df;
        if (fg <= 0.0f) L->gi0 = 0;
        else if (fg >= (float)(n - 1)) L->gi0 = n - 1;
        else {
            L->gi0 = (int)floorf(fg);
            L->gi1 = L->gi0 + 1;
            L->gw = (pos - o) / d - (double)L->gi0;
        }
    }
    return ret;
}

// Legs per field launch and the FP64 work planes they need (4 per leg).
int field_batch(const kcig_plan *P, size_t nlegs)
{
    const size_t nzx = (size_t)P->g.nz * P->g.nx;
    return std::max(1, std::min<int>((int)nlegs, (int)std::min<size_t>(64, (256ull << 20) / (nzx * 32) + 1)));
}

// The leg-field kernels' status flag: cleared before a migration's launches,
// read after them (KCIG_ERR_DEVICE when a bounded wait gave up).
int plan_status_reset(kcig_plan *P, cudaStream_t st)
{
    KCIG_TRY(P->d_status.ensure(sizeof(int)));
    KCIG_CUDA(cudaMemsetAsync(P->d_status.p, 0, sizeof(int), st));
    return KCIG_OK;
}

int plan_status_check(kcig_plan *P, cudaStream_t st)
{
    if (!P->d_status.p) return KCIG_OK;
    int h = 0;
    KCIG_CUDA(cudaMemcpyAsync(&h, P->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    KCIG_CUDA(cudaStreamSynchronize(st));
    if (h) return set_error(KCIG_ERR_DEVICE, "leg fields: a staged table copy did not complete");
    return KCIG_OK;
}

// Leg fields of n legs whose LegInterp records are already on the device;
// tab/der (device) replace the plan's tables when given (staged slices).
int compute_fields_dev(kcig_plan *P, int is_source, const LegInterp *d_legs, int n, double2 *TP, float2 *XW,
                       const float *tab = nullptr, const float *der = nullptr)
{
    const kcig_geometry &g = P->g;
    const size_t nzx = (size_t)g.nz * g.nx;
    if (n <= 0) return KCIG_OK;
    const int angle = P->p.cig && P->p.cig_is_angle;
    if (kcig_surrogate *sgt = is_source ? P->sg_src : P->sg_rcv) {
        // the surrogate's traveltime; its source-position derivative from the
        // network or the tables; its direction from the network or, as with
        // tables, from the finite-difference gradient of the traveltime field
        const bool tx_table = P->sg_tx == KCIG_SG_TX_TABLE;
        const bool fd_angle = angle && P->sg_angle == KCIG_SG_ANGLE_FD;
        FieldArgs a;
        memset(&a, 0, sizeof a);
        a.tab = is_source ? P->stab : P->rtab;
        a.der = is_source ? P->sder : P->rder;
        a.nz = g.nz;
        a.nx = g.nx;
        a.dz = g.dz;
        a.dx = g.dx;
        a.x0 = g.x0;
        a.radius = P->p.angle_grad_radius;
        a.smooth = P->p.angle_smooth;
        a.angle = angle;
        a.aper = P->p.aperture;
        a.aper_taper = P->p.aperture_taper;
        a.rmin = P->p.aperture_rmin;
        a.rtaper = P->p.aperture_rtaper;
        a.status = P->d_status.as<int>();
        a.type_p = P->p.interp_type == 'p';
        if (tx_table) {
            if (!a.tab || !a.der || P->stream_tables)
                return set_error(KCIG_ERR_ARG, "surrogate with table derivatives: the plan needs device tables");
            a.legs = d_legs;
            a.n = n;
            int nl = 0;
            KCIG_TRY(launch_leg_interp(a, LegFields{TP, XW}, nullptr, P->st, &nl));
            P->all_launches += nl;
        }
        const int mode = tx_table ? 0 : (angle && !fd_angle ? 2 : 1);
        KCIG_TRY(launch_surrogate_fields(sgt, d_legs, n, g, P->p, LegFields{TP, XW}, mode, P->st));
        P->all_launches += 1;
        if (fd_angle) {
            const int FB = leg_grad_needs_work(a) ? field_batch(P, (size_t)n) : n;
            if (leg_grad_needs_work(a)) KCIG_TRY(P->d_work.ensure((size_t)FB * 4 * nzx * sizeof(double)));
            for (int j0 = 0; j0 < n; j0 += FB) {
                a.legs = d_legs + j0;
                a.n = std::min(FB, n - j0);
                int nl = 0;
                KCIG_TRY(launch_leg_grad(a, LegFields{TP + (size_t)j0 * nzx, XW + (size_t)j0 * nzx},
                                         P->d_work.as<double>(), P->st, &nl));
                P->all_launches += nl;
            }
        }
        return KCIG_OK;
    }
    if (P->stream_tables && !tab)
        return set_error(KCIG_ERR_UNSUPPORTED, "tables kept in host memory need the host-side leg path");
    const int FB = field_batch(P, (size_t)n);
    if (angle) KCIG_TRY(P->d_work.ensure((size_t)FB * 4 * nzx * sizeof(double)));
    for (int j0 = 0; j0 < n; j0 += FB) {
        FieldArgs a;
        a.tab = tab ? tab : (is_source ? P->stab : P->rtab);
        a.der = der ? der : (is_source ? P->sder : P->rder);
        a.gxv = is_source ? P->sgx : P->rgx;
        a.gzv = is_source ? P->sgz : P->rgz;
        a.legs = d_legs + j0;
        a.n = std::min(FB, n - j0);
        a.nz = g.nz;
        a.nx = g.nx;
        a.dz = g.dz;
        a.dx = g.dx;
        a.x0 = g.x0;
        a.radius = P->p.angle_grad_radius;
        a.smooth = P->p.angle_smooth;
        a.angle = angle;
        a.use_grad = P->sgx != nullptr;
        a.aper = P->p.aperture;
        a.aper_taper = P->p.aperture_taper;
        a.rmin = P->p.aperture_rmin;
        a.rtaper = P->p.aperture_rtaper;
        a.cone = P->p.tool == 1;
        a.status = P->d_status.as<int>();
        a.type_p = P->p.interp_type == 'p';
        LegFields out{TP + (size_t)j0 * nzx, XW + (size_t)j0 * nzx};
        int nl = 0;
        KCIG_TRY(launch_leg_fields(a, out, P->d_work.as<double>(), P->st, &nl));
        P->all_launches += nl;
    }
    return KCIG_OK;
}

int compute_fields(kcig_plan *P, int is_source, const std::vector<LegInterp> &legs, double2 *TP, float2 *XW)
{
    KCIG_TRY(P->d_legs.ensure(legs.size() * sizeof(LegInterp)));
    if (legs.empty()) return KCIG_OK;
    if (!P->stream_tables || (is_source ? P->sg_src : P->sg_rcv)) {
        KCIG_CUDA(cudaMemcpyAsync(P->d_legs.p, legs.data(), legs.size() * sizeof(LegInterp), cudaMemcpyHostToDevice,
                                  P->st));
        return compute_fields_dev(P, is_source, P->d_legs.as<LegInterp>(), (int)legs.size(), TP, XW);
    }
    // Tables in host memory: legs go in groups whose slices fit the staging
    // buffer (two per leg of a field launch at most, and a quarter of the
    // plan's budget); each group's slices are copied in stream order, the
    // group's legs renumbered to their staging slots, and its fields
    // computed.  Values are read exactly as from device tables.
    const size_t nzx = (size_t)P->g.nz * P->g.nx, slice = nzx * sizeof(float);
    const float *ht = is_source ? P->h_stab : P->h_rtab, *hd = is_source ? P->h_sder : P->h_rder;
    const int npos = is_source ? P->g.sny : P->g.rny;
    const int FB = field_batch(P, legs.size());
    const size_t by_budget = P->budget / 4 / (2 * slice);
    const int cap = (int)std::max<size_t>(2, std::min<size_t>((size_t)2 * FB, by_budget));
    KCIG_TRY(P->d_stage.ensure((size_t)2 * cap * slice));
    float *sT = P->d_stage.as<float>(), *sD = sT + (size_t)cap * nzx;
    std::vector<LegInterp> grp;
    std::map<int, int> slot;
    size_t j = 0;
    while (j < legs.size()) {
        grp.clear();
        slot.clear();
        size_t k = j;
        for (; k < legs.size(); k++) {
            LegInterp L = legs[k];
            const int need = (slot.count(L.i0) ? 0 : 1) + (L.i1 >= 0 && L.i1 != L.i0 && !slot.count(L.i1) ? 1 : 0);
            if ((int)slot.size() + need > cap) break;
            for (int *ip : {&L.i0, &L.i1}) {
                if (*ip < 0) continue;
                if (*ip >= npos) return set_error(KCIG_ERR_ARG, "table slice %d outside [0,%d)", *ip, npos);
                auto it = slot.find(*ip);
                if (it == slot.end()) {
                    const int q = (int)slot.size();
                    KCIG_CUDA(cudaMemcpyAsync(sT + (size_t)q * nzx, ht + (size_t)*ip * nzx, slice,
                                              cudaMemcpyHostToDevice, P->st));
                    KCIG_CUDA(cudaMemcpyAsync(sD + (size_t)q * nzx, hd + (size_t)*ip * nzx, slice,
                                              cudaMemcpyHostToDevice, P->st));
                    it = slot.emplace(*ip, q).first;
                }
                *ip = it->second;
            }
            grp.push_back(L);
        }
        KCIG_CUDA(cudaMemcpyAsync(P->d_legs.p, grp.data(), grp.size() * sizeof(LegInterp), cudaMemcpyHostToDevice,
                                  P->st));
        KCIG_TRY(compute_fields_dev(P, is_source, P->d_legs.as<LegInterp>(), (int)grp.size(), TP + j * nzx,
                                    XW + j * nzx, sT, sD));
        j = k;
    }
    return KCIG_OK;
}

}  // namespace

// ------------------------------------------------------------------ C ABI --
extern "C" int kcig_plan_create(const kcig_params *p, const kcig_geometry *g, unsigned long long scratch_bytes,
                                kcig_plan **out)
{
    if (!p || !g || !out) return set_error(KCIG_ERR_ARG, "kcig_plan_create: null argument");
    *out = nullptr;
    if (g->nt < 1 || g->nh < 1 || g->ns < 1) return set_error(KCIG_ERR_ARG, "Need 3D data volume for seismic_data= (t,h/r,s)");
    if (g->nz < 1 || g->nx < 1 || g->sny < 1) return set_error(KCIG_ERR_ARG, "Need 3D data volume for stable= (z,x,s)");
    if (g->rny < 1) return set_error(KCIG_ERR_ARG, "Need 3D data volume for rtable= (z,x,r)");
    if (!(g->dt > 0.0f)) return set_error(KCIG_ERR_ARG, "time sampling d1 of seismic_data= must be positive");
    if ((long long)g->nz * g->nx > 0x7fffffffLL) return set_error(KCIG_ERR_ARG, "image grid too large");
    if (p->direct_mute && p->direct_mute_qc_shot >= g->ns)
        return set_error(KCIG_ERR_ARG, "direct_mute_qc_shot=%d is outside the input shot range [0,%d].",
                         p->direct_mute_qc_shot, g->ns - 1);
    kcig_plan *P = new kcig_plan();
    P->p = *p;
    P->g = *g;
    if (P->g.nh == 1) P->g.dh = 0.0f;  // :700-701
    if (P->g.ns == 1) P->g.ds = 0.0f;
    int rc = kcig_output_axis(p, &P->g, &P->ng, &P->g0, &P->dg);
    if (rc) {
        delete P;
        return rc;
    }
    cudaGetDevice(&P->device);
    P->budget = scratch_bytes;
    if (P->budget == 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            delete P;
            return set_error(KCIG_ERR_CUDA, "no CUDA device available");
        }
        P->budget = (unsigned long long)(fr > (6ull << 30) ? (fr - (4ull << 30)) * 0.8 : fr / 2);
        P->budget = std::min<unsigned long long>(P->budget, 96ull << 30);
    }
    *out = P;
    return KCIG_OK;
}

extern "C" int kcig_plan_destroy(kcig_plan *P)
{
    if (!P) return KCIG_OK;
    DevBuf *bufs[] = {&P->own_stab, &P->own_sder, &P->own_rtab, &P->own_rder, &P->own_sgx, &P->own_sgz,
                      &P->own_rgx,  &P->own_rgz,  &P->d_data,   &P->d_image,  &P->d_rT,   &P->d_rF,
                      &P->d_sT,     &P->d_sF,   &P->d_work,   &P->d_D,      &P->d_legs, &P->d_tr,
                      &P->d_part,   &P->d_stage};
    for (DevBuf *b : bufs) b->release();
    release_shots(P);
    if (P->own_st) cudaStreamDestroy(P->own_st);
    if (P->copy_st) cudaStreamDestroy(P->copy_st);
    if (P->copy_ev) cudaEventDestroy(P->copy_ev);
    if (P->order_ev) cudaEventDestroy(P->order_ev);
    delete P;
    return KCIG_OK;
}

extern "C" int kcig_plan_set_stream(kcig_plan *P, void *stream)
{
    if (!P) return set_error(KCIG_ERR_ARG, "null plan");
    P->st = (cudaStream_t)stream;
    return KCIG_OK;
}

static int bind_volume(kcig_plan *P, DevBuf &own, const float *src, int npos, int memory, const float **dst,
                       const float *alias_src, const float *alias_dev)
{
    const size_t bytes = (size_t)npos * P->g.nz * P->g.nx * sizeof(float);
    if (!src) return set_error(KCIG_ERR_ARG, "missing table pointer");
    if (memory == KCIG_MEM_DEVICE) {
        *dst = src;
        return KCIG_OK;
    }
    if (alias_src == src && alias_dev) {
        *dst = alias_dev;
        return KCIG_OK;
    }
    KCIG_TRY(upload(own, src, bytes, P->st));
    *dst = own.as<float>();
    return KCIG_OK;
}

extern "C" int kcig_plan_set_tables(kcig_plan *P, const float *stable, const float *sderiv, const float *rtable,
                                    const float *rderiv, int memory)
{
    if (!P) return set_error(KCIG_ERR_ARG, "null plan");
    P->stream_tables = 0;
    if (memory == KCIG_MEM_HOST_STREAM) {
        if (!stable || !sderiv || !rtable || !rderiv) return set_error(KCIG_ERR_ARG, "missing table pointer");
        for (DevBuf *b : {&P->own_stab, &P->own_sder, &P->own_rtab, &P->own_rder}) b->release();
        P->stream_tables = 1;
        P->h_stab = stable;
        P->h_sder = sderiv;
        P->h_rtab = rtable;
        P->h_rder = rderiv;
        // the device pointers only mark the tables as set; no kernel reads them
        P->stab = stable;
        P->sder = sderiv;
        P->rtab = rtable;
        P->rder = rderiv;
        return KCIG_OK;
    }
    if (memory != KCIG_MEM_HOST && memory != KCIG_MEM_DEVICE)
        return set_error(KCIG_ERR_ARG, "kcig_plan_set_tables: unknown memory kind %d", memory);
    KCIG_TRY(bind_volume(P, P->own_stab, stable, P->g.sny, memory, &P->stab, nullptr, nullptr));
    KCIG_TRY(bind_volume(P, P->own_sder, sderiv, P->g.sny, memory, &P->sder, nullptr, nullptr));
    const bool same = (P->g.rny == P->g.sny);
    KCIG_TRY(bind_volume(P, P->own_rtab, rtable, P->g.rny, memory, &P->rtab, same ? stable : nullptr, P->stab));
    KCIG_TRY(bind_volume(P, P->own_rder, rderiv, P->g.rny, memory, &P->rder, same ? sderiv : nullptr, P->sder));
    KCIG_CUDA(cudaStreamSynchronize(P->st));
    return KCIG_OK;
}

extern "C" int kcig_plan_set_gradients(kcig_plan *P, const float *sgradx, const float *sgradz, const float *rgradx,
                                       const float *rgradz, int memory)
{
    if (!P) return set_error(KCIG_ERR_ARG, "null plan");
    const int n = (sgradx != nullptr) + (sgradz != nullptr) + (rgradx != nullptr) + (rgradz != nullptr);
    if (n == 0) {
        P->sgx = P->sgz = P->rgx = P->rgz = nullptr;
        return KCIG_OK;
    }
    if (n != 4)
        return set_error(KCIG_ERR_ARG,
                         "For mode=angle, please provide all of sgradx=, sgradz=, rgradx=, and rgradz=, or provide none of them.");
    KCIG_TRY(bind_volume(P, P->own_sgx, sgradx, P->g.sny, memory, &P->sgx, nullptr, nullptr));
    KCIG_TRY(bind_volume(P, P->own_sgz, sgradz, P->g.sny, memory, &P->sgz, nullptr, nullptr));
    const bool same = (P->g.rny == P->g.sny);
    KCIG_TRY(bind_volume(P, P->own_rgx, rgradx, P->g.rny, memory, &P->rgx, same ? sgradx : nullptr, P->sgx));
    KCIG_TRY(bind_volume(P, P->own_rgz, rgradz, P->g.rny, memory, &P->rgz, same ? sgradz : nullptr, P->sgz));
    KCIG_CUDA(cudaStreamSynchronize(P->st));
    return KCIG_OK;
}

extern "C" int kcig_plan_last_stats(const kcig_plan *P, int *sum_launches, float *sum_ms, int *all_launches)
{
    if (!P) return set_error(KCIG_ERR_ARG, "null plan");
    if (sum_launches) *sum_launches = P->sum_launches;
    if (sum_ms) *sum_ms = P->sum_ms;
    if (all_launches) *all_launches = P->all_launches;
    return KCIG_OK;
}

extern "C" int kcig_leg_fields_device(kcig_plan *P, int is_source, double pos, double *T, float *Tx, double *phi,
                                      float *w)
{
    if (!P || !(is_source ? (P->sg_src || P->stab) : (P->sg_rcv || P->rtab)))
        return set_error(KCIG_ERR_ARG, "kcig_leg_fields_device: plan without tables");
    const size_t nzx = (size_t)P->g.nz * P->g.nx;
    std::vector<LegInterp> legs(1);
    leg_interp(P, is_source, (float)pos, pos, &legs[0]);
    legs[0].scale = 1.0f;
    DevBuf tp, xw;
    int rc = tp.ensure(nzx * sizeof(double2));
    if (!rc) rc = xw.ensure(nzx * sizeof(float2));
    kcig_surrogate *sgt = is_source ? P->sg_src : P->sg_rcv;
    if (!rc && sgt) rc = sg_reset_status(sgt, P->st);
    if (!rc) rc = plan_status_reset(P, P->st);
    if (!rc) rc = compute_fields(P, is_source, legs, tp.as<double2>(), xw.as<float2>());
    if (!rc && sgt) rc = sg_check_status(sgt, P->st);
    // unpack {T, phi} and {Tx, w} into the caller's planes
    struct Cp { void *dst; const char *src; size_t el, pitch; } cps[4] = {
        {T, tp.as<char>(), sizeof(double), sizeof(double2)},
        {phi, tp.as<char>() + sizeof(double), sizeof(double), sizeof(double2)},
        {Tx, xw.as<char>(), sizeof(float), sizeof(float2)},
        {w, xw.as<char>() + sizeof(float), sizeof(float), sizeof(float2)}};
    for (int q = 0; q < 4 && rc == KCIG_OK; q++) {
        if (!cps[q].dst) continue;
        cudaError_t e = cudaMemcpy2DAsync(cps[q].dst, cps[q].el, cps[q].src, cps[q].pitch, cps[q].el, nzx,
                                          cudaMemcpyDeviceToDevice, P->st);
        if (e != cudaSuccess) rc = cuda_error(e, "cudaMemcpy2DAsync(leg fields)");
    }
    cudaError_t e = cudaStreamSynchronize(P->st);
    if (!rc && e != cudaSuccess) rc = cuda_error(e, "cudaStreamSynchronize(leg fields)");
    if (!rc) rc = plan_status_check(P, P->st);
    tp.release();
    xw.release();
    return rc;
}

extern "C" int kcig_doubint_device(const float *in, double *out, int ntr, int nt, int isdiff, float dt, void *stream)
{
    if (!in || !out || ntr < 0 || nt < 1) return set_error(KCIG_ERR_ARG, "kcig_doubint_device: bad arguments");
    return launch_doubint_plain(in, out, ntr, nt, isdiff, (double)dt, (cudaStream_t)stream);
}

extern "C" int kcig_migrate(kcig_plan *P, const float *data, float *image, int memory)
{
    if (!P || !data || !image) return set_error(KCIG_ERR_ARG, "kcig_migrate: null argument");
    if (!(P->sg_src || P->stab) || !(P->sg_rcv || P->rtab))
        return set_error(KCIG_ERR_ARG, "kcig_migrate: tables not set");
    for (kcig_surrogate *s : {P->sg_src, P->sg_rcv})
        if (s) KCIG_TRY(sg_reset_status(s, P->st));
    const kcig_params &p = P->p;
    const kcig_geometry &g = P->g;
    const size_t nzx = (size_t)g.nz * g.nx;
    const int angle = p.cig && p.cig_is_angle;
    P->sum_launches = 0;
    P->all_launches = 0;
    P->sum_ms = 0.f;
    cudaStream_t st = P->st;
    KCIG_TRY(plan_status_reset(P, st));

    // data and image on the device
    const float *d_data = data;
    float *d_img = image;
    const int ns = P->shot_count > 0 ? P->shot_count : g.ns;  // shots of this call (kcig_plan_set_shot_range)
    const size_t data_bytes = (size_t)ns * g.nh * g.nt * sizeof(float);
    bool data_pending = false;
    if (memory == KCIG_MEM_HOST) {
        if (!P->copy_st) {
            KCIG_CUDA(cudaStreamCreateWithFlags(&P->copy_st, cudaStreamNonBlocking));
            KCIG_CUDA(cudaEventCreateWithFlags(&P->copy_ev, cudaEventDisableTiming));
            KCIG_CUDA(cudaEventCreateWithFlags(&P->order_ev, cudaEventDisableTiming));
        }
        KCIG_TRY(P->d_data.ensure(data_bytes));
        // the copy starts after the plan's earlier work (which may still read
        // the buffer) and overlaps the leg fields computed below
        KCIG_CUDA(cudaEventRecord(P->order_ev, st));
        KCIG_CUDA(cudaStreamWaitEvent(P->copy_st, P->order_ev, 0));
        KCIG_CUDA(cudaMemcpyAsync(P->d_data.p, data, data_bytes, cudaMemcpyHostToDevice, P->copy_st));
        KCIG_CUDA(cudaEventRecord(P->copy_ev, P->copy_st));
        data_pending = true;
        d_data = P->d_data.as<float>();
        KCIG_TRY(P->d_image.ensure((size_t)P->ng * nzx * sizeof(float)));
        d_img = P->d_image.as<float>();
    }

    // per-trace scalars (:1054-1105), all in double
    const double ds = g.ns == 1 ? 0.0 : (double)g.ds, dh = g.nh == 1 ? 0.0 : (double)g.dh;
    // positions in FP64 for every continuous use, and as the reference's
    // float expressions (:980, :1055, :1061) for its discrete decisions; a
    // shot range takes its shots' positions from the whole survey's axis
    std::vector<double> sx(ns), hx(g.nh);
    std::vector<float> sxf(ns), hxf(g.nh);
    kcig_shot_positions(&g, P->shot_first, ns, sx.data(), sxf.data());
    for (int ih = 0; ih < g.nh; ih++) {
        hx[ih] = (double)g.h0 + (double)ih * dh;
        hxf[ih] = g.h0 + (float)ih * (float)dh;
    }
    std::vector<LegInterp> slegs(ns);
    std::vector<int> ist(ns);
    for (int is = 0; is < ns; is++) {
        ist[is] = leg_interp(P, 1, sxf[is], sx[is], &slegs[is]);
        slegs[is].scale = (float)ds;
    }
    const size_t ntr_all = (size_t)ns * g.nh;
    std::vector<float> trw(ntr_all);
    std::vector<int> igo(ntr_all, 0);
    std::vector<double> msx(ntr_all), mrx(ntr_all);
    for (int is = 0; is < ns; is++)
        for (int ih = 0; ih < g.nh; ih++) {
            const size_t t = (size_t)is * g.nh + ih;
            const double rpos = p.cmp ? sx[is] + hx[ih] : hx[ih];
            const float rposf = p.cmp ? sxf[is] + hxf[ih] : hxf[ih];
            msx[t] = sx[is];
            mrx[t] = rpos;
            float rf = 0.0f;
            if (g.rny > 1 && g.rdy != 0.0f) rf = (rposf - g.ry0) / g.rdy;
            int iht = (g.rny > 1 && g.rdy != 0.0f) ? (int)floorf(rf) : 0;
            // kirchmig2d: the truncated quotient (:413)
            if (p.tool == 1) iht = g.rdy != 0.0f ? (int)((rposf - g.ry0) / g.rdy) : 0;
            double w = 1.0;
            if (p.aperture_trace != -1) {
                const double ad = fabs((double)(iht - ist[is]));
                if (ad >= (double)p.aperture_trace) w = 0.0;
                else if (p.aperture_trace_taper > 0) {
                    const double tb = std::max(0.0, (double)(p.aperture_trace - p.aperture_trace_taper));
                    if (ad > tb) {
                        const double den = (double)p.aperture_trace - tb;
                        if (den > 0.0) w = 0.5 * (1.0 + cos(M_PI * ((ad - tb) / den)));
                    }
                }
            }
            if (p.tool == 1) {
                // kirchmig2d: image = offset index (cig=1) or the stack; the
                // weight's sign says whether the source is the left leg of
                // the cone test (:457 cmp: h >= 0; :474 h - s >= 0)
                igo[t] = p.cig ? ih : 0;
                const bool src_left = p.cmp ? (hxf[ih] >= 0.0f) : (hxf[ih] - sxf[is] >= 0.0f);
                if (!src_left) w = -w;
            } else if (p.cig && !p.cig_is_angle) {
                // value_to_nearest_bin(h) (:35-41), a discrete decision in float
                int ig = -1;
                if (P->ng > 0 && P->dg > 0.0f && isfinite(hxf[ih])) {
                    ig = (int)floorf((hxf[ih] - P->g0) / P->dg + 0.5f);
                    if (ig < 0 || ig >= P->ng) ig = -1;
                }
                if (ig < 0) w = 0.0;
                igo[t] = ig < 0 ? 0 : ig;
            }
            trw[t] = (float)w;
        }

    // scratch plan: receivers shared across shots (cmp=0) are computed once
    const bool shared_r = !p.cmp;
    const size_t leg_bytes = nzx * (sizeof(double2) + sizeof(float2));
    const unsigned long long budget = P->budget;
    int nhc = g.nh;
    if (shared_r && (unsigned long long)nhc * leg_bytes > budget / 2)
        nhc = (int)std::max<unsigned long long>(1, (budget / 2) / leg_bytes);
    const size_t work_bytes = angle ? (size_t)std::min<size_t>(64, (256ull << 20) / (nzx * 32) + 1) * 4 * nzx * 8 : 0;
    const size_t per_shot = leg_bytes + (size_t)nhc * g.nt * sizeof(double2) + (size_t)nhc * 32 +
                            (shared_r ? 0 : (size_t)nhc * leg_bytes);
    const unsigned long long fixed = (shared_r ? (unsigned long long)nhc * leg_bytes : 0) + work_bytes;
    long long room = (long long)budget - (long long)fixed;
    int nsb = (int)std::max<long long>(1, room / (long long)per_shot);
    nsb = std::min(nsb, ns);

    if (shared_r) {
        KCIG_TRY(P->d_rT.ensure((size_t)nhc * nzx * sizeof(double2)));
        KCIG_TRY(P->d_rF.ensure((size_t)nhc * nzx * sizeof(float2)));
    } else {
        KCIG_TRY(P->d_rT.ensure((size_t)nsb * g.nh * nzx * sizeof(double2)));
        KCIG_TRY(P->d_rF.ensure((size_t)nsb * g.nh * nzx * sizeof(float2)));
    }
    KCIG_TRY(P->d_sT.ensure((size_t)nsb * nzx * sizeof(double2)));
    KCIG_TRY(P->d_sF.ensure((size_t)nsb * nzx * sizeof(float2)));
    KCIG_TRY(P->d_D.ensure((size_t)nsb * nhc * g.nt * sizeof(double2)));
    const size_t trn = (size_t)nsb * nhc;
    // one allocation: doubles first (8-byte aligned), then floats and ints
    KCIG_TRY(P->d_tr.ensure(trn * (2 * sizeof(double) + sizeof(float) + 2 * sizeof(int))));
    double *d_msx = P->d_tr.as<double>();
    double *d_mrx = d_msx + trn;
    float *d_trw = (float *)(d_mrx + trn);
    int *d_rfi = (int *)(d_trw + trn);
    int *d_igo = d_rfi + trn;

    std::vector<cudaEvent_t> evs, fevs;
    // leg fields of one batch, bracketed by events (the plan's fields time)
    auto fields = [&](int is_source, const std::vector<LegInterp> &legs, double2 *TP, float2 *XW) {
        cudaEvent_t f0, f1;
        cudaEventCreate(&f0);
        cudaEventCreate(&f1);
        fevs.push_back(f0);
        fevs.push_back(f1);
        cudaEventRecord(f0, st);
        const int r = compute_fields(P, is_source, legs, TP, XW);
        cudaEventRecord(f1, st);
        return r;
    };
    bool first = true;
    std::vector<float> h_trw(trn);
    std::vector<int> h_rfi(trn), h_igo(trn);
    std::vector<double> h_msx(trn), h_mrx(trn);
    int rc = KCIG_OK;

    for (int r0 = 0; r0 < g.nh && rc == KCIG_OK; r0 += nhc) {
        const int nhb = std::min(nhc, g.nh - r0);
        if (shared_r) {
            std::vector<LegInterp> rl(nhb);
            for (int r = 0; r < nhb; r++) {
                leg_interp(P, 0, hxf[r0 + r], hx[r0 + r], &rl[r]);
                rl[r].scale = (float)dh;
            }
            rc = fields(0, rl, P->d_rT.as<double2>(), P->d_rF.as<float2>());
            if (rc) break;
        }
        for (int s0 = 0; s0 < ns && rc == KCIG_OK; s0 += nsb) {
            const int nsh = std::min(nsb, ns - s0);
            std::vector<LegInterp> sl(slegs.begin() + s0, slegs.begin() + s0 + nsh);
            rc = fields(1, sl, P->d_sT.as<double2>(), P->d_sF.as<float2>());
            if (rc) break;
            // per-trace arrays of this (shot batch, receiver chunk)
            std::vector<LegInterp> rl;
            // receiver legs by (FP64, float) position; kirchmig2d's cmp=1 cone
            // test also depends on the shot of a leg right of its source
            std::map<std::tuple<double, float, float>, int> seen;
            for (int k = 0; k < nsh; k++)
                for (int r = 0; r < nhb; r++) {
                    const size_t t = (size_t)(s0 + k) * g.nh + (r0 + r);
                    const size_t b = (size_t)k * nhb + r;
                    h_trw[b] = trw[t];
                    h_igo[b] = igo[t];
                    h_msx[b] = msx[t];
                    h_mrx[b] = mrx[t];
                    if (shared_r) {
                        h_rfi[b] = r;
                    } else {
                        const bool cexact = p.tool == 1 && p.cmp && hxf[r0 + r] >= 0.0f;
                        const std::tuple<double, float, float> key(mrx[t], sxf[s0 + k] + hxf[r0 + r],
                                                                   cexact ? sxf[s0 + k] : 0.0f);
                        auto it = seen.find(key);
                        if (it == seen.end()) {
                            LegInterp L;
                            leg_interp(P, 0, std::get<1>(key), std::get<0>(key), &L);
                            L.scale = (float)dh;
                            L.cexact = cexact ? 1 : 0;
                            L.cs = sxf[s0 + k];
                            L.ch = hxf[r0 + r];
                            it = seen.emplace(key, (int)rl.size()).first;
                            rl.push_back(L);
                        }
                        h_rfi[b] = it->second;
                    }
                }
            if (!shared_r) {
                rc = fields(0, rl, P->d_rT.as<double2>(), P->d_rF.as<float2>());
                if (rc) break;
            }
            const size_t nb = (size_t)nsh * nhb;
            {
                const void *srcs[5] = {h_trw.data(), h_rfi.data(), h_igo.data(), h_msx.data(), h_mrx.data()};
                void *dsts[5] = {d_trw, d_rfi, d_igo, d_msx, d_mrx};
                const size_t sz[5] = {sizeof(float), sizeof(int), sizeof(int), sizeof(double), sizeof(double)};
                for (int q = 0; q < 5 && rc == KCIG_OK; q++) {
                    cudaError_t e = cudaMemcpyAsync(dsts[q], srcs[q], nb * sz[q], cudaMemcpyHostToDevice, st);
                    if (e != cudaSuccess) rc = cuda_error(e, "cudaMemcpyAsync(trace tables)");
                }
                if (rc) break;
            }
            PreludeArgs pa;
            memset(&pa, 0, sizeof pa);
            pa.data = d_data;
            pa.D = P->d_D.as<double2>();
            pa.mute_sx = p.direct_mute ? d_msx : nullptr;
            pa.mute_rx = d_mrx;
            pa.ntr = (int)nb;
            pa.nt = g.nt;
            pa.isdiff = p.isdiff;
            pa.invert = p.direct_mute_invert;
            pa.nh = g.nh;
            pa.nhc = nhb;
            pa.shot0 = s0;
            pa.rcv0 = r0;
            pa.t0 = g.t0;
            pa.dt = g.dt;
            pa.slope = p.direct_mute_slope;
            pa.intercept = p.direct_mute_intercept;
            pa.taper = p.direct_mute_taper;
            if (data_pending) {  // the traces have landed before their first use
                cudaError_t e = cudaStreamWaitEvent(st, P->copy_ev, 0);
                if (e != cudaSuccess) {
                    rc = cuda_error(e, "cudaStreamWaitEvent(traces)");
                    break;
                }
                data_pending = false;
            }
            rc = launch_prelude(pa, st);
            if (rc) break;
            P->all_launches++;

            SumArgs sa;
            memset(&sa, 0, sizeof sa);
            sa.STP = P->d_sT.as<double2>();
            sa.SXW = P->d_sF.as<float2>();
            sa.RTP = P->d_rT.as<double2>();
            sa.RXW = P->d_rF.as<float2>();
            sa.D = P->d_D.as<double2>();
            sa.trw = d_trw;
            sa.rfi = d_rfi;
            sa.igo = d_igo;
            sa.image = d_img;
            sa.zero_init = first ? 1 : 0;
            sa.nz = g.nz;
            sa.nx = g.nx;
            sa.nt = g.nt;
            sa.nsb = nsh;
            sa.nh = nhb;
            sa.ng = P->ng;
            sa.mode = p.tool == 1 ? 3 : (angle ? (p.angle_interp ? 0 : 1) : 2);
            // a uniform flag spares the pair loop a dependent load per pair
            sa.unit_tw = std::all_of(h_trw.begin(), h_trw.begin() + nb, [](float v) { return v == 1.0f; }) ? 1 : 0;
            sa.tile = P->tile;
            sa.nsplit = sum_nsplit(g.nz, g.nx, nsh, shared_r);
            if (sa.nsplit > 1) {
                rc = P->d_part.ensure((size_t)sa.nsplit * P->ng * nzx * sizeof(float));
                if (rc) break;
                sa.partial = P->d_part.as<float>();
            }
            sa.shared_r = shared_r ? 1 : 0;
            sa.half = p.half_angle;
            sa.t0 = g.t0;
            sa.dt = g.dt;
            sa.inv_dt = 1.0 / (double)g.dt;
            sa.tau = p.tau;
            sa.deg = (p.half_angle ? 90.0 : 180.0) / M_PI;
            sa.ug0 = P->g0;
            sa.uinv = 1.0 / (double)P->dg;
            sa.dtf = g.dt;
            sa.aal = p.antialias;
            sa.g0 = P->g0;
            sa.dg = P->dg;
            sa.oazmin = p.oazmin;
            sa.oazmax = p.oazmax;
            sa.oaztaper = p.oaztaper;
            sa.ats = p.angle_taper_start;
            sa.ate = p.angle_taper_end;
            cudaEvent_t e0, e1;
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            evs.push_back(e0);
            evs.push_back(e1);
            cudaEventRecord(e0, st);
            int nl = 0;
            rc = launch_sum(sa, st, &nl);
            cudaEventRecord(e1, st);
            if (rc) break;
            P->sum_launches += nl;
            P->all_launches += nl + (sa.nsplit > 1 ? 1 : 0);
            first = false;
            // the host-side arrays are reused by the next batch
            if (s0 + nsb < ns || r0 + nhc < g.nh) {
                cudaError_t e = cudaStreamSynchronize(st);
                if (e != cudaSuccess) {
                    rc = cuda_error(e, "cudaStreamSynchronize(batch)");
                    break;
                }
            }
        }
    }
    if (rc == KCIG_OK && memory == KCIG_MEM_HOST) {
        cudaError_t e = cudaMemcpyAsync(image, d_img, (size_t)P->ng * nzx * sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) rc = cuda_error(e, "cudaMemcpyAsync(image)");
    }
    cudaError_t e = cudaStreamSynchronize(st);
    if (rc == KCIG_OK && e != cudaSuccess) rc = cuda_error(e, "cudaStreamSynchronize(migrate)");
    if (memory == KCIG_MEM_HOST && P->copy_st) {  // the caller's traces are no longer read after this
        e = cudaStreamSynchronize(P->copy_st);
        if (rc == KCIG_OK && e != cudaSuccess) rc = cuda_error(e, "cudaStreamSynchronize(trace copy)");
    }
    for (size_t i = 0; i + 1 < evs.size(); i += 2) {
        float ms = 0.f;
        if (rc == KCIG_OK && cudaEventElapsedTime(&ms, evs[i], evs[i + 1]) == cudaSuccess) P->sum_ms += ms;
        cudaEventDestroy(evs[i]);
        cudaEventDestroy(evs[i + 1]);
    }
    P->fields_ms = 0.f;
    for (size_t i = 0; i + 1 < fevs.size(); i += 2) {
        float ms = 0.f;
        if (rc == KCIG_OK && cudaEventElapsedTime(&ms, fevs[i], fevs[i + 1]) == cudaSuccess) P->fields_ms += ms;
        cudaEventDestroy(fevs[i]);
        cudaEventDestroy(fevs[i + 1]);
    }
    for (kcig_surrogate *s : {P->sg_src, P->sg_rcv})
        if (s && rc == KCIG_OK) rc = sg_check_status(s, st);
    if (rc == KCIG_OK) rc = plan_status_check(P, st);
    return rc;
}

extern "C" int kcig_plan_last_timing(const kcig_plan *P, float *fields_ms, float *sum_ms)
{
    if (!P) return set_error(KCIG_ERR_ARG, "kcig_plan_last_timing: null plan");
    if (fields_ms) *fields_ms = P->fields_ms;
    if (sum_ms) *sum_ms = P->sum_ms;
    return KCIG_OK;
}

extern "C" float kcig_plan_last_prelude_ms(const kcig_plan *P) { return P ? P->prelude_ms : 0.f; }

extern "C" int kcig_plan_set_surrogate(kcig_plan *P, kcig_surrogate *src, kcig_surrogate *rcv)
{
    if (!P) return set_error(KCIG_ERR_ARG, "kcig_plan_set_surrogate: null plan");
    if (P->p.tool == 1 && (src || rcv))
        return set_error(KCIG_ERR_UNSUPPORTED, "kirchmig2d with a traveltime surrogate is not built");
    P->sg_src = src;
    P->sg_rcv = rcv;
    return KCIG_OK;
}

extern "C" int kcig_shot_positions(const kcig_geometry *g, int first, int count, double *pos, float *posf)
{
    if (!g || first < 0 || count < 0 || (long long)first + count > g->ns)
        return set_error(KCIG_ERR_ARG, "kcig_shot_positions: shots [%d, %d) outside the axis of %d shots", first,
                         first + count, g ? g->ns : 0);
    const double ds = g->ns == 1 ? 0.0 : (double)g->ds;
    for (int k = 0; k < count; k++) {
        const int is = first + k;
        if (pos) pos[k] = (double)g->s0 + (double)is * ds;
        if (posf) posf[k] = g->s0 + (float)is * (float)ds;
    }
    return KCIG_OK;
}

extern "C" int kcig_plan_set_shot_range(kcig_plan *P, int first, int count)
{
    if (!P) return set_error(KCIG_ERR_ARG, "kcig_plan_set_shot_range: null plan");
    if (count == -1 && first == 0) {
        P->shot_first = 0;
        P->shot_count = -1;
        return KCIG_OK;
    }
    if (first < 0 || count < 1 || (long long)first + count > P->g.ns)
        return set_error(KCIG_ERR_ARG, "kcig_plan_set_shot_range: shots [%d, %d) outside the survey's %d", first,
                         first + count, P->g.ns);
    P->shot_first = first;
    P->shot_count = count;
    return KCIG_OK;
}

extern "C" int kcig_plan_set_surrogate_options(kcig_plan *P, int angle, int tx)
{
    if (!P) return set_error(KCIG_ERR_ARG, "kcig_plan_set_surrogate_options: null plan");
    if ((angle != KCIG_SG_ANGLE_FD && angle != KCIG_SG_ANGLE_NETWORK) || (tx != KCIG_SG_TX_NETWORK && tx != KCIG_SG_TX_TABLE))
        return set_error(KCIG_ERR_ARG, "kcig_plan_set_surrogate_options: angle %d / tx %d not known", angle, tx);
    P->sg_angle = angle;
    P->sg_tx = tx;
    return KCIG_OK;
}

// ------------------------------------------------------- forward modelling --
// kirchmig2d_cig adj=0: data [ns][nh][nt] from an image [ng][nx][nz] with the
// plan's geometry, the exact adjoint of kcig_migrate without the direct mute
// and diff2 (the reference's forward branch applies neither and rejects
// direct_mute=1).  Same per-trace gates as the migration.
extern "C" int kcig_model(kcig_plan *P, const float *image, float *data, int memory)
{
    if (P && P->shot_count > 0)
        return set_error(KCIG_ERR_UNSUPPORTED, "kcig_model: a shot range is not built for forward modelling");
    if (!P || !image || !data) return set_error(KCIG_ERR_ARG, "kcig_model: null argument");
    if (!(P->sg_src || P->stab) || !(P->sg_rcv || P->rtab)) return set_error(KCIG_ERR_ARG, "kcig_model: tables not set");
    const kcig_params &p = P->p;
    const kcig_geometry &g = P->g;
    if (p.tool == 1) return set_error(KCIG_ERR_UNSUPPORTED, "kirchmig2d adj=0 is not built");
    if (p.direct_mute) return set_error(KCIG_ERR_ARG, "direct_mute=1 is an input-data preprocessing option and requires adj=1.");
    const size_t nzx = (size_t)g.nz * g.nx;
    const int angle = p.cig && p.cig_is_angle;
    cudaStream_t st = P->st;
    P->sum_launches = 0;
    P->all_launches = 0;
    KCIG_TRY(plan_status_reset(P, st));
    const float *d_img = image;
    float *d_dat = data;
    const size_t img_bytes = (size_t)P->ng * nzx * sizeof(float);
    const size_t dat_bytes = (size_t)g.ns * g.nh * g.nt * sizeof(float);
    if (memory == KCIG_MEM_HOST) {
        KCIG_TRY(upload(P->d_image, image, img_bytes, st));
        d_img = P->d_image.as<float>();
        KCIG_TRY(P->d_data.ensure(dat_bytes));
        d_dat = P->d_data.as<float>();
    }
    const double ds = g.ns == 1 ? 0.0 : (double)g.ds, dh = g.nh == 1 ? 0.0 : (double)g.dh;
    std::vector<double> sx(g.ns), hx(g.nh);
    std::vector<float> sxf(g.ns), hxf(g.nh);
    for (int is = 0; is < g.ns; is++) {
        sx[is] = (double)g.s0 + (double)is * ds;
        sxf[is] = g.s0 + (float)is * (float)ds;
    }
    for (int ih = 0; ih < g.nh; ih++) {
        hx[ih] = (double)g.h0 + (double)ih * dh;
        hxf[ih] = g.h0 + (float)ih * (float)dh;
    }
    // batches of shots: source and receiver legs, raw traces
    const size_t leg_bytes = nzx * (sizeof(double2) + sizeof(float2));
    const size_t per_shot = leg_bytes * (1 + (size_t)g.nh) + (size_t)g.nh * g.nt * sizeof(double) + (size_t)g.nh * 16;
    int nsb = (int)std::max<long long>(1, (long long)(P->budget / 2) / (long long)per_shot);
    nsb = std::min(nsb, g.ns);
    int rc = P->d_sT.ensure((size_t)nsb * nzx * sizeof(double2));
    if (!rc) rc = P->d_sF.ensure((size_t)nsb * nzx * sizeof(float2));
    if (!rc) rc = P->d_rT.ensure((size_t)nsb * g.nh * nzx * sizeof(double2));
    if (!rc) rc = P->d_rF.ensure((size_t)nsb * g.nh * nzx * sizeof(float2));
    if (!rc) rc = P->d_D.ensure((size_t)nsb * g.nh * g.nt * sizeof(double));  // raw traces
    if (!rc) rc = P->d_tr.ensure((size_t)nsb * g.nh * (sizeof(float) + 2 * sizeof(int)));
    if (rc) return rc;
    float *d_trw = P->d_tr.as<float>();
    int *d_rfi = (int *)(d_trw + (size_t)nsb * g.nh);
    int *d_igo = d_rfi + (size_t)nsb * g.nh;
    std::vector<float> h_trw((size_t)nsb * g.nh);
    std::vector<int> h_rfi(h_trw.size()), h_igo(h_trw.size());
    for (int s0 = 0; s0 < g.ns && rc == KCIG_OK; s0 += nsb) {
        const int nsh = std::min(nsb, g.ns - s0);
        std::vector<LegInterp> sl(nsh), rl;
        std::map<std::pair<double, float>, int> seen;
        for (int k = 0; k < nsh; k++) {
            const int is = s0 + k;
            const int ist = leg_interp(P, 1, sxf[is], sx[is], &sl[k]);
            sl[k].scale = (float)ds;
            for (int ih = 0; ih < g.nh; ih++) {
                const size_t b = (size_t)k * g.nh + ih;
                const double rpos = p.cmp ? sx[is] + hx[ih] : hx[ih];
                const float rposf = p.cmp ? sxf[is] + hxf[ih] : hxf[ih];
                const std::pair<double, float> key(rpos, rposf);
                auto it = seen.find(key);
                if (it == seen.end()) {
                    LegInterp L;
                    leg_interp(P, 0, rposf, rpos, &L);
                    L.scale = (float)dh;
                    it = seen.emplace(key, (int)rl.size()).first;
                    rl.push_back(L);
                }
                h_rfi[b] = it->second;
                float rf = 0.0f;
                if (g.rny > 1 && g.rdy != 0.0f) rf = (rposf - g.ry0) / g.rdy;
                const int iht = (g.rny > 1 && g.rdy != 0.0f) ? (int)floorf(rf) : 0;
                double w = 1.0;
                if (p.aperture_trace != -1) {
                    const double ad = fabs((double)(iht - ist));
                    if (ad >= (double)p.aperture_trace) w = 0.0;
                    else if (p.aperture_trace_taper > 0) {
                        const double tb = std::max(0.0, (double)(p.aperture_trace - p.aperture_trace_taper));
                        if (ad > tb) {
                            const double den = (double)p.aperture_trace - tb;
                            if (den > 0.0) w = 0.5 * (1.0 + cos(M_PI * ((ad - tb) / den)));
                        }
                    }
                }
                int bin = 0;
                if (p.cig && !p.cig_is_angle) {
                    int b2 = -1;
                    if (P->ng > 0 && P->dg > 0.0f && std::isfinite(hxf[ih])) {
                        b2 = (int)floorf((hxf[ih] - P->g0) / P->dg + 0.5f);
                        if (b2 < 0 || b2 >= P->ng) b2 = -1;
                    }
                    if (b2 < 0) w = 0.0;
                    bin = b2 < 0 ? 0 : b2;
                }
                h_trw[b] = (float)w;
                h_igo[b] = bin;
            }
        }
        rc = compute_fields(P, 1, sl, P->d_sT.as<double2>(), P->d_sF.as<float2>());
        if (!rc) rc = compute_fields(P, 0, rl, P->d_rT.as<double2>(), P->d_rF.as<float2>());
        const size_t nb = (size_t)nsh * g.nh;
        const void *srcs[3] = {h_trw.data(), h_rfi.data(), h_igo.data()};
        void *dsts[3] = {d_trw, d_rfi, d_igo};
        for (int q = 0; q < 3 && rc == KCIG_OK; q++) {
            cudaError_t e = cudaMemcpyAsync(dsts[q], srcs[q], nb * 4, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) rc = cuda_error(e, "cudaMemcpyAsync(trace tables)");
        }
        if (rc) break;
        SprayArgs sa;
        memset(&sa, 0, sizeof sa);
        sa.STP = P->d_sT.as<double2>();
        sa.SXW = P->d_sF.as<float2>();
        sa.RTP = P->d_rT.as<double2>();
        sa.RXW = P->d_rF.as<float2>();
        sa.trw = d_trw;
        sa.rfi = d_rfi;
        sa.igo = d_igo;
        sa.image = d_img;
        sa.raw = P->d_D.as<double>();
        sa.nz = g.nz;
        sa.nx = g.nx;
        sa.nt = g.nt;
        sa.nsb = nsh;
        sa.nh = g.nh;
        sa.ng = P->ng;
        sa.mode = angle ? (p.angle_interp ? 0 : 1) : 2;
        sa.t0 = g.t0;
        sa.inv_dt = 1.0 / (double)g.dt;
        sa.tau = p.tau;
        sa.deg = (p.half_angle ? 90.0 : 180.0) / M_PI;
        sa.ug0 = P->g0;
        sa.uinv = 1.0 / (double)P->dg;
        sa.aal = p.antialias;
        sa.oazmin = p.oazmin;
        sa.oazmax = p.oazmax;
        sa.oaztaper = p.oaztaper;
        sa.ats = p.angle_taper_start;
        sa.ate = p.angle_taper_end;
        rc = launch_spray(sa, st);
        if (!rc) rc = launch_doubint_f32(P->d_D.as<double>(), d_dat + (size_t)s0 * g.nh * g.nt, (int)nb, g.nt, st);
        P->all_launches += 2;
        P->sum_launches += 1;
        if (!rc) {  // the host tables are reused by the next batch
            cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) rc = cuda_error(e, "cudaStreamSynchronize(model)");
        }
    }
    if (!rc && memory == KCIG_MEM_HOST) {
        cudaError_t e = cudaMemcpyAsync(data, d_dat, dat_bytes, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) rc = cuda_error(e, "cudaMemcpyAsync(data)");
    }
    cudaError_t e = cudaStreamSynchronize(st);
    if (!rc && e != cudaSuccess) rc = cuda_error(e, "cudaStreamSynchronize(model)");
    if (!rc) rc = plan_status_check(P, st);
    return rc;
}

// ------------------------------------------------------------ ragged shots --
// Each shot is migrated as the reference migrates a one-shot file (ns = 1:
// the source leg's antialias term uses ds = 0; the receiver leg's uses the
// shot's own dh, 0 for one receiver), so the image equals the sum of the
// per-shot runs.  Shots keep their own receiver positions and trace length.
namespace {

// The trace tables of a prepared batch (views into the per-trace buffer).
struct TraceViews {
    const double *msx, *mrx;
    const long long *toff;
    const float *trw;
    const int *rfi, *igo, *tnt;
};

TraceViews trace_views(const ShotsPrepared *S)
{
    const size_t ntr = S->ntr;
    TraceViews v;
    v.msx = S->trf.as<double>();
    v.mrx = v.msx + ntr;
    v.toff = (const long long *)(v.mrx + ntr);
    v.trw = (const float *)(v.toff + ntr);
    v.rfi = (const int *)(v.trw + ntr);
    v.igo = v.rfi + ntr;
    v.tnt = v.igo + ntr;
    return v;
}

// leg fields of batch b
int batch_fields(kcig_plan *P, size_t b, cudaStream_t st)
{
    const ShotsPrepared *S = P->shots;
    const ShotBatch &B = S->batches[b];
    const LegInterp *legs = S->legs.as<LegInterp>();
    cudaStream_t saved = P->st;
    P->st = st;
    int rc = compute_fields_dev(P, 1, legs + B.sleg0, B.ns, P->d_sT.as<double2>(), P->d_sF.as<float2>());
    if (!rc) rc = compute_fields_dev(P, 0, legs + B.rleg0, B.nrl, P->d_rT.as<double2>(), P->d_rF.as<float2>());
    P->st = saved;
    return rc;
}

// integrated traces of batch b
int batch_prelude(kcig_plan *P, size_t b, cudaStream_t st)
{
    const ShotsPrepared *S = P->shots;
    const ShotBatch &B = S->batches[b];
    const kcig_params &p = P->p;
    const kcig_geometry &g = P->g;
    const TraceViews v = trace_views(S);
    PreludeArgs pa;
    memset(&pa, 0, sizeof pa);
    pa.data = S->data.as<float>();
    pa.D = P->d_D.as<double2>();
    pa.mute_sx = p.direct_mute ? v.msx + B.tr0 : nullptr;
    pa.mute_rx = v.mrx + B.tr0;
    pa.ntr = B.ns * B.nhb;
    pa.nt = S->ntmax;
    pa.isdiff = p.isdiff;
    pa.invert = p.direct_mute_invert;
    pa.nh = B.nhb;
    pa.nhc = B.nhb;
    pa.t0 = g.t0;
    pa.dt = g.dt;
    pa.slope = p.direct_mute_slope;
    pa.intercept = p.direct_mute_intercept;
    pa.taper = p.direct_mute_taper;
    pa.toff = v.toff + B.tr0;
    pa.tnt = v.tnt + B.tr0;
    KCIG_TRY(launch_prelude(pa, st));
    P->all_launches++;
    return KCIG_OK;
}

SumArgs batch_sum_args(const kcig_plan *P, size_t b, float *d_img)
{
    const ShotsPrepared *S = P->shots;
    const ShotBatch &B = S->batches[b];
    const kcig_params &p = P->p;
    const kcig_geometry &g = P->g;
    const TraceViews v = trace_views(S);
    const int angle = p.cig && p.cig_is_angle;
    SumArgs sa;
    memset(&sa, 0, sizeof sa);
    sa.STP = P->d_sT.as<double2>();
    sa.SXW = P->d_sF.as<float2>();
    sa.RTP = P->d_rT.as<double2>();
    sa.RXW = P->d_rF.as<float2>();
    sa.D = P->d_D.as<double2>();
    sa.trw = v.trw + B.tr0;
    sa.rfi = v.rfi + B.tr0;
    sa.igo = v.igo + B.tr0;
    sa.stop = S->stop.as<float>() + B.shot0;
    sa.snh = S->snh.as<int>() + B.shot0;
    sa.tile = P->tile;
    sa.nsplit = sum_nsplit(g.nz, g.nx, B.ns, false);
    if (sa.nsplit > 1) sa.partial = P->d_part.as<float>();  // sized by kcig_shots_prepare
    sa.image = d_img;
    sa.zero_init = b == 0 ? 1 : 0;
    sa.nz = g.nz;
    sa.nx = g.nx;
    sa.nt = S->ntmax;
    sa.nsb = B.ns;
    sa.nh = B.nhb;
    sa.ng = P->ng;
    sa.mode = angle ? (p.angle_interp ? 0 : 1) : 2;
    sa.unit_tw = B.unit_tw;
    sa.shared_r = 0;
    sa.half = p.half_angle;
    sa.t0 = g.t0;
    sa.dt = g.dt;
    sa.inv_dt = 1.0 / (double)g.dt;
    sa.tau = p.tau;
    sa.deg = (p.half_angle ? 90.0 : 180.0) / M_PI;
    sa.ug0 = P->g0;
    sa.uinv = 1.0 / (double)P->dg;
    sa.dtf = g.dt;
    sa.aal = p.antialias;
    sa.g0 = P->g0;
    sa.dg = P->dg;
    sa.oazmin = p.oazmin;
    sa.oazmax = p.oazmax;
    sa.oaztaper = p.oaztaper;
    sa.ats = p.angle_taper_start;
    sa.ate = p.angle_taper_end;
    return sa;
}

int batch_inputs(kcig_plan *P, size_t b, cudaStream_t st)
{
    KCIG_TRY(batch_fields(P, b, st));
    return batch_prelude(P, b, st);
}

// `ev` (4 events per batch, or null): before the fields, after the fields,
// after the prelude, after the summation -- for the stage times of a direct
// (uncaptured) run
int run_prepared(kcig_plan *P, float *d_img, cudaStream_t st, cudaEvent_t *ev = nullptr)
{
    ShotsPrepared *S = P->shots;
    for (size_t b = 0; b < S->batches.size(); b++) {
        if (ev) cudaEventRecord(ev[4 * b], st);
        KCIG_TRY(batch_fields(P, b, st));
        if (ev) cudaEventRecord(ev[4 * b + 1], st);
        KCIG_TRY(batch_prelude(P, b, st));
        if (ev) cudaEventRecord(ev[4 * b + 2], st);
        const SumArgs sa = batch_sum_args(P, b, d_img);
        int nl = 0;
        KCIG_TRY(launch_sum(sa, st, &nl));
        if (ev) cudaEventRecord(ev[4 * b + 3], st);
        P->sum_launches += nl;
        P->all_launches += nl + (sa.nsplit > 1 ? 1 : 0);
    }
    if (S->batches.empty()) {
        const size_t nzx = (size_t)P->g.nz * P->g.nx;
        KCIG_CUDA(cudaMemsetAsync(d_img, 0, (size_t)P->ng * nzx * sizeof(float), st));
    }
    return KCIG_OK;
}

}  // namespace

extern "C" int kcig_shots_prepare(kcig_plan *P, int nshots, const kcig_shot *shots, int memory)
{
    if (!P || nshots < 0 || (nshots > 0 && !shots)) return set_error(KCIG_ERR_ARG, "kcig_shots_prepare: bad arguments");
    if (P->p.tool == 1) return set_error(KCIG_ERR_UNSUPPORTED, "kirchmig2d shots of uneven size are not built");
    const kcig_params &p = P->p;
    const kcig_geometry &g = P->g;
    if (!(P->sg_src || P->stab) || !(P->sg_rcv || P->rtab))
        return set_error(KCIG_ERR_ARG, "kcig_shots_prepare: tables not set");
    const size_t nzx = (size_t)g.nz * g.nx;
    const int angle = p.cig && p.cig_is_angle;
    int ntmax = 1;
    size_t nsamp = 0;
    for (int i = 0; i < nshots; i++) {
        const kcig_shot &sh = shots[i];
        if (sh.nh < 1 || sh.nt < 1 || !sh.data || !std::isfinite(sh.sx))
            return set_error(KCIG_ERR_ARG, "kcig_shots_prepare: shot %d: need nh >= 1, nt >= 1, data", i);
        if (sh.nt > g.nt) return set_error(KCIG_ERR_ARG, "kcig_shots_prepare: shot %d: nt=%d exceeds the plan's nt=%d", i, sh.nt, g.nt);
        ntmax = std::max(ntmax, sh.nt);
        nsamp += (size_t)sh.nh * sh.nt;
    }
    release_shots(P);
    ShotsPrepared *S = new ShotsPrepared();
    P->shots = S;
    S->nshots = nshots;
    S->ntmax = ntmax;
    cudaStream_t st = P->st;

    // all samples in one device buffer, shot after shot
    std::vector<size_t> base(nshots);
    int rc = S->data.ensure(std::max<size_t>(nsamp, 1) * sizeof(float));
    size_t at = 0;
    for (int i = 0; i < nshots && rc == KCIG_OK; i++) {
        base[i] = at;
        const size_t n = (size_t)shots[i].nh * shots[i].nt;
        cudaError_t e = cudaMemcpyAsync(S->data.as<float>() + at, shots[i].data, n * sizeof(float),
                                        memory == KCIG_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) rc = cuda_error(e, "cudaMemcpyAsync(shot data)");
        at += n;
    }
    if (rc) { release_shots(P); return rc; }

    // batches: as many shots as the scratch budget holds, receivers shared
    // within a batch when position and spacing agree
    const size_t leg_bytes = nzx * (sizeof(double2) + sizeof(float2));
    const unsigned long long budget = P->budget;
    const size_t work_bytes = angle ? (size_t)field_batch(P, 64) * 4 * nzx * 8 : 0;
    std::vector<LegInterp> hlegs;
    std::vector<double> h_msx, h_mrx;
    std::vector<long long> h_toff;
    std::vector<float> h_trw, h_stop;
    std::vector<int> h_snh;
    std::vector<int> h_rfi, h_igo, h_tnt;
    size_t max_s = 0, max_r = 0, max_d = 0;
    int i0 = 0;
    while (i0 < nshots) {
        // grow the batch
        std::map<std::tuple<double, float, float>, int> seen;
        int nhb = 0, i1 = i0;
        for (; i1 < nshots; i1++) {
            const kcig_shot &sh = shots[i1];
            const float dhf = sh.nh == 1 ? 0.0f : sh.dh;
            std::map<std::tuple<double, float, float>, int> add;
            for (int k = 0; k < sh.nh; k++) {
                const double hx = sh.h ? (double)sh.h[k] : (double)sh.h0 + (double)k * (double)dhf;
                const float hxf = sh.h ? sh.h[k] : sh.h0 + (float)k * dhf;
                const double rpos = p.cmp ? (double)sh.sx + hx : hx;
                const float rposf = p.cmp ? sh.sx + hxf : hxf;
                const auto key = std::make_tuple(rpos, rposf, dhf);
                if (!seen.count(key)) add.emplace(key, 0);
            }
            const int ns1 = i1 - i0 + 1, nh1 = std::max(nhb, sh.nh);
            const size_t need = (size_t)(ns1 + seen.size() + add.size()) * leg_bytes +
                                (size_t)ns1 * nh1 * ((size_t)ntmax * sizeof(double2) + 48) + work_bytes;
            if (i1 > i0 && need > budget) break;
            for (auto &kv : add) seen.emplace(kv.first, 0);
            nhb = nh1;
        }
        ShotBatch B;
        B.ns = i1 - i0;
        B.nhb = nhb;
        B.sleg0 = hlegs.size();
        B.tr0 = h_trw.size();
        B.shot0 = h_stop.size();
        std::vector<int> ist(B.ns);
        for (int k = 0; k < B.ns; k++) {
            const kcig_shot &sh = shots[i0 + k];
            LegInterp L;
            ist[k] = leg_interp(P, 1, sh.sx, (double)sh.sx, &L);
            L.scale = 0.0f;  // one-shot file: ds = 0
            hlegs.push_back(L);
            h_stop.push_back((float)(sh.nt - 1));
            h_snh.push_back(sh.nh);
        }
        B.rleg0 = hlegs.size();
        std::map<std::tuple<double, float, float>, int> index;
        bool unit = true;
        for (int k = 0; k < B.ns; k++) {
            const kcig_shot &sh = shots[i0 + k];
            const float dhf = sh.nh == 1 ? 0.0f : sh.dh;
            for (int r = 0; r < B.nhb; r++) {
                if (r >= sh.nh) {  // padding: no samples, weight 0
                    h_msx.push_back(0.0);
                    h_mrx.push_back(0.0);
                    h_toff.push_back(-1);
                    h_trw.push_back(0.0f);
                    h_rfi.push_back(0);
                    h_igo.push_back(0);
                    h_tnt.push_back(0);
                    unit = false;
                    continue;
                }
                const double hx = sh.h ? (double)sh.h[r] : (double)sh.h0 + (double)r * (double)dhf;
                const float hxf = sh.h ? sh.h[r] : sh.h0 + (float)r * dhf;
                const double rpos = p.cmp ? (double)sh.sx + hx : hx;
                const float rposf = p.cmp ? sh.sx + hxf : hxf;
                const auto key = std::make_tuple(rpos, rposf, dhf);
                auto it = index.find(key);
                if (it == index.end()) {
                    LegInterp L;
                    leg_interp(P, 0, rposf, rpos, &L);
                    L.scale = dhf;
                    it = index.emplace(key, (int)index.size()).first;
                    hlegs.push_back(L);
                }
                // trace aperture (:1082-1099) and offset bin (:35-41), as the regular path
                float rf = 0.0f;
                if (g.rny > 1 && g.rdy != 0.0f) rf = (rposf - g.ry0) / g.rdy;
                const int iht = (g.rny > 1 && g.rdy != 0.0f) ? (int)floorf(rf) : 0;
                double w = 1.0;
                if (p.aperture_trace != -1) {
                    const double ad = fabs((double)(iht - ist[k]));
                    if (ad >= (double)p.aperture_trace) w = 0.0;
                    else if (p.aperture_trace_taper > 0) {
                        const double tb = std::max(0.0, (double)(p.aperture_trace - p.aperture_trace_taper));
                        if (ad > tb) {
                            const double den = (double)p.aperture_trace - tb;
                            if (den > 0.0) w = 0.5 * (1.0 + cos(M_PI * ((ad - tb) / den)));
                        }
                    }
                }
                int ig = 0;
                if (p.cig && !p.cig_is_angle) {
                    int b = -1;
                    if (P->ng > 0 && P->dg > 0.0f && std::isfinite(hxf)) {
                        b = (int)floorf((hxf - P->g0) / P->dg + 0.5f);
                        if (b < 0 || b >= P->ng) b = -1;
                    }
                    if (b < 0) w = 0.0;
                    ig = b < 0 ? 0 : b;
                }
                if (w != 1.0) unit = false;
                h_msx.push_back((double)sh.sx);
                h_mrx.push_back(rpos);
                h_toff.push_back((long long)(base[i0 + k] + (size_t)r * sh.nt));
                h_trw.push_back((float)w);
                h_rfi.push_back(it->second);
                h_igo.push_back(ig);
                h_tnt.push_back(sh.nt);
                S->pairs += (long long)nzx;
            }
        }
        B.nrl = (int)index.size();
        B.unit_tw = unit ? 1 : 0;
        max_s = std::max<size_t>(max_s, B.ns);
        max_r = std::max<size_t>(max_r, B.nrl);
        max_d = std::max<size_t>(max_d, (size_t)B.ns * B.nhb);
        S->batches.push_back(B);
        i0 = i1;
    }
    const size_t ntr = h_trw.size();
    S->ntr = ntr;
    rc = S->legs.ensure(std::max<size_t>(hlegs.size(), 1) * sizeof(LegInterp));
    if (!rc) rc = S->trf.ensure(std::max<size_t>(ntr, 1) * (3 * 8 + 4 * 4));
    if (!rc) rc = S->stop.ensure(std::max<size_t>(h_stop.size(), 1) * sizeof(float));
    if (!rc) rc = S->snh.ensure(std::max<size_t>(h_snh.size(), 1) * sizeof(int));
    if (!rc) rc = P->d_sT.ensure(std::max<size_t>(max_s, 1) * nzx * sizeof(double2));
    if (!rc) rc = P->d_sF.ensure(std::max<size_t>(max_s, 1) * nzx * sizeof(float2));
    if (!rc) rc = P->d_rT.ensure(std::max<size_t>(max_r, 1) * nzx * sizeof(double2));
    if (!rc) rc = P->d_rF.ensure(std::max<size_t>(max_r, 1) * nzx * sizeof(float2));
    if (!rc) rc = P->d_D.ensure(std::max<size_t>(max_d, 1) * (size_t)ntmax * sizeof(double2));
    if (!rc && angle && !(P->sg_src && P->sg_rcv))
        rc = P->d_work.ensure((size_t)field_batch(P, std::max(max_s, max_r)) * 4 * nzx * sizeof(double));
    int max_split = 1;
    for (const ShotBatch &B : S->batches) max_split = std::max(max_split, sum_nsplit(g.nz, g.nx, B.ns, false));
    if (!rc && max_split > 1) rc = P->d_part.ensure((size_t)max_split * P->ng * nzx * sizeof(float));
    struct Cp { void *dst; const void *src; size_t bytes; } cps[] = {
        {S->legs.p, hlegs.data(), hlegs.size() * sizeof(LegInterp)},
        {S->trf.as<double>(), h_msx.data(), ntr * 8},
        {S->trf.as<double>() + ntr, h_mrx.data(), ntr * 8},
        {S->trf.as<double>() + 2 * ntr, h_toff.data(), ntr * 8},
        {S->trf.as<char>() + 24 * ntr, h_trw.data(), ntr * 4},
        {S->trf.as<char>() + 28 * ntr, h_rfi.data(), ntr * 4},
        {S->trf.as<char>() + 32 * ntr, h_igo.data(), ntr * 4},
        {S->trf.as<char>() + 36 * ntr, h_tnt.data(), ntr * 4},
        {S->stop.p, h_stop.data(), h_stop.size() * 4},
        {S->snh.p, h_snh.data(), h_snh.size() * 4}};
    for (auto &c : cps) {
        if (rc || c.bytes == 0) continue;
        cudaError_t e = cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) rc = cuda_error(e, "cudaMemcpyAsync(shot tables)");
    }
    cudaError_t e = cudaStreamSynchronize(st);  // the host vectors go out of scope
    if (!rc && e != cudaSuccess) rc = cuda_error(e, "cudaStreamSynchronize(shots)");
    if (rc) release_shots(P);
    return rc;
}

extern "C" int kcig_plan_set_graph(kcig_plan *P, int enable)
{
    if (!P) return set_error(KCIG_ERR_ARG, "kcig_plan_set_graph: null plan");
    P->use_graph = enable ? 1 : 0;
    if (P->shots && P->shots->exec) {
        cudaGraphExecDestroy(P->shots->exec);
        cudaGraphDestroy(P->shots->graph);
        P->shots->exec = nullptr;
        P->shots->graph = nullptr;
        P->shots->graph_image = nullptr;
    }
    return KCIG_OK;
}

extern "C" int kcig_migrate_prepared(kcig_plan *P, float *image, int memory)
{
    if (!P || !image) return set_error(KCIG_ERR_ARG, "kcig_migrate_prepared: null argument");
    ShotsPrepared *S = P->shots;
    if (!S) return set_error(KCIG_ERR_ARG, "kcig_migrate_prepared: no shots prepared (kcig_shots_prepare)");
    const size_t nzx = (size_t)P->g.nz * P->g.nx;
    const size_t img_bytes = (size_t)P->ng * nzx * sizeof(float);
    P->sum_launches = 0;
    P->all_launches = 0;
    P->sum_ms = 0.f;
    P->fields_ms = 0.f;
    for (kcig_surrogate *s : {P->sg_src, P->sg_rcv})
        if (s) KCIG_TRY(sg_reset_status(s, P->st));
    KCIG_TRY(plan_status_reset(P, P->st));
    float *d_img = image;
    if (memory == KCIG_MEM_HOST) {
        KCIG_TRY(P->d_image.ensure(img_bytes));
        d_img = P->d_image.as<float>();
    }
    cudaStream_t st = P->st;
    int rc = KCIG_OK;
    if (P->use_graph) {
        if (!st) {  // the legacy stream cannot be captured
            if (!P->own_st) KCIG_CUDA(cudaStreamCreateWithFlags(&P->own_st, cudaStreamNonBlocking));
            st = P->own_st;
            KCIG_CUDA(cudaDeviceSynchronize());  // order against work on the legacy stream
        }
        if (S->exec && S->graph_image == d_img) {
            KCIG_CUDA(cudaGraphLaunch(S->exec, st));
            P->sum_launches = -1;  // inside the graph
        } else {
            // one direct run (it also raises every kernel's shared-memory
            // limit), then capture the same sequence for the next calls
            rc = run_prepared(P, d_img, st);
            if (!rc) {
                if (S->exec) {
                    cudaGraphExecDestroy(S->exec);
                    cudaGraphDestroy(S->graph);
                    S->exec = nullptr;
                    S->graph = nullptr;
                }
                const int sl = P->sum_launches, al = P->all_launches;
                cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
                if (e != cudaSuccess) rc = cuda_error(e, "cudaStreamBeginCapture");
                if (!rc) {
                    const int rc2 = run_prepared(P, d_img, st);
                    cudaGraph_t gr = nullptr;
                    e = cudaStreamEndCapture(st, &gr);
                    if (rc2) rc = rc2;
                    else if (e != cudaSuccess) rc = cuda_error(e, "cudaStreamEndCapture");
                    if (!rc) {
                        e = cudaGraphInstantiate(&S->exec, gr, 0);
                        if (e != cudaSuccess) {
                            rc = cuda_error(e, "cudaGraphInstantiate");
                            cudaGraphDestroy(gr);
                        } else {
                            S->graph = gr;
                            S->graph_image = d_img;
                        }
                    } else if (gr) {
                        cudaGraphDestroy(gr);
                    }
                }
                P->sum_launches = sl;
                P->all_launches = al;
            }
        }
    } else {
        std::vector<cudaEvent_t> ev(4 * S->batches.size());
        for (auto &x : ev) cudaEventCreate(&x);
        rc = run_prepared(P, d_img, st, ev.data());
        if (!rc) {
            cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) rc = cuda_error(e, "cudaStreamSynchronize(prepared)");
        }
        P->prelude_ms = 0.f;
        for (size_t b = 0; b < S->batches.size() && !rc; b++) {
            float f = 0.f, q = 0.f, m = 0.f;
            cudaEventElapsedTime(&f, ev[4 * b], ev[4 * b + 1]);
            cudaEventElapsedTime(&q, ev[4 * b + 1], ev[4 * b + 2]);
            cudaEventElapsedTime(&m, ev[4 * b + 2], ev[4 * b + 3]);
            P->fields_ms += f;
            P->prelude_ms += q;
            P->sum_ms += m;
        }
        for (auto &x : ev) cudaEventDestroy(x);
    }
    if (!rc && memory == KCIG_MEM_HOST) {
        cudaError_t e = cudaMemcpyAsync(image, d_img, img_bytes, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) rc = cuda_error(e, "cudaMemcpyAsync(image)");
    }
    cudaError_t e = cudaStreamSynchronize(st);
    if (!rc && e != cudaSuccess) rc = cuda_error(e, "cudaStreamSynchronize(prepared)");
    for (kcig_surrogate *s : {P->sg_src, P->sg_rcv})
        if (s && rc == KCIG_OK) rc = sg_check_status(s, st);
    if (rc == KCIG_OK) rc = plan_status_check(P, st);
    return rc;
}

extern "C" int kcig_plan_autotune(kcig_plan *P, int *choice, float *ms)
{
    if (!P || !P->shots || P->shots->batches.empty())
        return set_error(KCIG_ERR_ARG, "kcig_plan_autotune: no shots prepared (kcig_shots_prepare)");
    const size_t nzx = (size_t)P->g.nz * P->g.nx;
    KCIG_TRY(P->d_image.ensure((size_t)P->ng * nzx * sizeof(float)));
    cudaStream_t st = P->st;
    KCIG_TRY(batch_inputs(P, 0, st));
    SumArgs sa = batch_sum_args(P, 0, P->d_image.as<float>());
    cudaEvent_t e0, e1;
    KCIG_CUDA(cudaEventCreate(&e0));
    KCIG_CUDA(cudaEventCreate(&e1));
    int best = 0, rc = KCIG_OK;
    float best_ms = 0.f;
    for (int t = 1; t < kSumTiles && rc == KCIG_OK; t++) {
        sa.tile = t;
        rc = launch_sum(sa, st, nullptr);  // warm-up (shared-memory limit, caches)
        float tms = 0.f;
        for (int rep = 0; rep < 3 && rc == KCIG_OK; rep++) {
            cudaEventRecord(e0, st);
            rc = launch_sum(sa, st, nullptr);
            cudaEventRecord(e1, st);
            cudaError_t e = cudaEventSynchronize(e1);
            if (!rc && e != cudaSuccess) rc = cuda_error(e, "cudaEventSynchronize(autotune)");
            float x = 0.f;
            cudaEventElapsedTime(&x, e0, e1);
            tms = rep == 0 ? x : std::min(tms, x);
        }
        if (ms) ms[t] = tms;
        if (!rc && (best == 0 || tms < best_ms)) {
            best = t;
            best_ms = tms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (ms) ms[0] = best_ms;
    P->tile = best;
    if (choice) *choice = best;
    kcig_plan_set_graph(P, P->use_graph);  // a captured graph used the old tile
    return KCIG_OK;
}

// Several prepared plans (the depth windows of the recursive workflow) in one
// CUDA graph: one replay migrates every plan's shots into its image.
struct kcig_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

extern "C" int kcig_graph_create(int n, kcig_plan *const *plans, float *const *images, kcig_graph **out)
{
    if (n < 1 || !plans || !images || !out) return set_error(KCIG_ERR_ARG, "kcig_graph_create: bad arguments");
    *out = nullptr;
    for (int i = 0; i < n; i++)
        if (!plans[i] || !plans[i]->shots || !images[i])
            return set_error(KCIG_ERR_ARG, "kcig_graph_create: plan %d has no prepared shots or image", i);
    cudaStream_t st;
    KCIG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    int rc = KCIG_OK;
    // one direct pass first: kernels' shared-memory limits are raised outside the capture
    for (int i = 0; i < n && rc == KCIG_OK; i++) rc = run_prepared(plans[i], images[i], st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (!rc && e != cudaSuccess) rc = cuda_error(e, "cudaStreamSynchronize(graph warm-up)");
    kcig_graph *G = new kcig_graph();
    if (!rc) {
        e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) rc = cuda_error(e, "cudaStreamBeginCapture");
        if (!rc) {
            int rc2 = KCIG_OK;
            for (int i = 0; i < n && rc2 == KCIG_OK; i++) rc2 = run_prepared(plans[i], images[i], st);
            e = cudaStreamEndCapture(st, &G->graph);
            if (rc2) rc = rc2;
            else if (e != cudaSuccess) rc = cuda_error(e, "cudaStreamEndCapture");
        }
        if (!rc) {
            e = cudaGraphInstantiate(&G->exec, G->graph, 0);
            if (e != cudaSuccess) rc = cuda_error(e, "cudaGraphInstantiate");
        }
    }
    cudaStreamDestroy(st);
    if (rc) {
        kcig_graph_destroy(G);
        return rc;
    }
    *out = G;
    return KCIG_OK;
}

extern "C" int kcig_graph_launch(kcig_graph *G, void *stream)
{
    if (!G || !G->exec) return set_error(KCIG_ERR_ARG, "kcig_graph_launch: no graph");
    KCIG_CUDA(cudaGraphLaunch(G->exec, (cudaStream_t)stream));
    return KCIG_OK;
}

extern "C" void kcig_graph_destroy(kcig_graph *G)
{
    if (!G) return;
    if (G->exec) cudaGraphExecDestroy(G->exec);
    if (G->graph) cudaGraphDestroy(G->graph);
    delete G;
}

extern "C" int kcig_migrate_shots(kcig_plan *P, int nshots, const kcig_shot *shots, float *image, int memory)
{
    KCIG_TRY(kcig_shots_prepare(P, nshots, shots, memory));
    return kcig_migrate_prepared(P, image, memory);
}

extern "C" long long kcig_shots_pairs(const kcig_plan *P)
{
    return (P && P->shots) ? P->shots->pairs : 0;
}

// ------------------------------------------------- allocation-free variant --
// kcig_leg_fields_noalloc computes what kcig_leg_fields_device computes, for
// callers that may not allocate device memory: host applications whose device
// memory is owned by another allocator or budgeted to the byte, and code that
// runs where a cudaMalloc would synchronise or fail.  Its scratch -- the leg
// descriptor, the {T, phi} and {Tx, w} planes and the four FP64 gradient
// planes -- lives in the fixed array below, which every device that loads the
// library holds until the process exits.
#define KCIG_NOALLOC_MAX_POINTS (1 << 18)  // nz*nx limit of the fixed scratch
#define KCIG_NOALLOC_SCRATCH_BYTES (16u << 20)

static __device__ __align__(256) unsigned char g_noalloc_scratch[KCIG_NOALLOC_SCRATCH_BYTES];
static_assert(sizeof(LegInterp) <= 248, "descriptor slot (the last 8 bytes hold the status flag)");
static_assert(256 + (size_t)KCIG_NOALLOC_MAX_POINTS * 56 <= KCIG_NOALLOC_SCRATCH_BYTES, "scratch layout");

namespace {
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[256];  // device address of g_noalloc_scratch, per device ordinal

// Host code cannot use g_noalloc_scratch as an address: the name denotes a
// host-side shadow.  The device address is looked up once per device, with
// that device current.
int noalloc_scratch(void **out)
{
    int dev = 0;
    KCIG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return set_error(KCIG_ERR_ARG, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return KCIG_OK;
}
}  // namespace

extern "C" int kcig_leg_fields_noalloc(const kcig_params *p, const kcig_geometry *g, const float *table,
                                       const float *deriv, const float *gradx, const float *gradz, int is_source,
                                       double pos, double *T, float *Tx, double *phi, float *w, void *stream)
{
    if (!p || !g || !table || !deriv) return set_error(KCIG_ERR_ARG, "kcig_leg_fields_noalloc: null argument");
    if ((gradx == nullptr) != (gradz == nullptr))
        return set_error(KCIG_ERR_ARG, "kcig_leg_fields_noalloc: give both gradient volumes or neither");
    if (g->nz < 1 || g->nx < 1 || (is_source ? g->sny : g->rny) < 1)
        return set_error(KCIG_ERR_ARG, "kcig_leg_fields_noalloc: empty grid or position axis");
    const long long nzx = (long long)g->nz * g->nx;
    if (nzx > KCIG_NOALLOC_MAX_POINTS)
        return set_error(KCIG_ERR_ARG, "kcig_leg_fields_noalloc: nz*nx=%lld exceeds the allocation-free limit %d",
                         nzx, KCIG_NOALLOC_MAX_POINTS);
    void *base = nullptr;
    KCIG_TRY(noalloc_scratch(&base));
    cudaStream_t st = (cudaStream_t)stream;
    // scratch layout: [descriptor | {T,phi} | {Tx,w} | 4 gradient planes]
    char *s = (char *)base;
    LegInterp *d_leg = (LegInterp *)s;
    int *d_status = (int *)(s + 248);  // the kernels' wait flag, in the descriptor slot's tail
    double2 *d_tp = (double2 *)(s + 256);
    float2 *d_xw = (float2 *)((char *)d_tp + (size_t)nzx * sizeof(double2));
    double *d_work = (double *)((char *)d_xw + (size_t)nzx * sizeof(float2));

    kcig_plan view;  // parameter/geometry view for leg_interp; owns no device memory
    view.p = *p;
    view.g = *g;
    LegInterp L;
    leg_interp(&view, is_source, (float)pos, pos, &L);
    L.scale = 1.0f;
    KCIG_CUDA(cudaMemcpyAsync(d_leg, &L, sizeof L, cudaMemcpyHostToDevice, st));
    FieldArgs a;
    a.tab = table;
    a.der = deriv;
    a.gxv = gradx;
    a.gzv = gradz;
    a.legs = d_leg;
    a.n = 1;
    a.nz = g->nz;
    a.nx = g->nx;
    a.dz = g->dz;
    a.dx = g->dx;
    a.x0 = g->x0;
    a.radius = p->angle_grad_radius;
    a.smooth = p->angle_smooth;
    a.angle = p->cig && p->cig_is_angle;
    a.use_grad = gradx != nullptr;
    a.aper = p->aperture;
    a.aper_taper = p->aperture_taper;
    a.rmin = p->aperture_rmin;
    a.rtaper = p->aperture_rtaper;
    a.cone = p->tool == 1;
    a.status = d_status;
    a.type_p = p->interp_type == 'p';
    KCIG_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), st));
    KCIG_TRY(launch_leg_fields(a, LegFields{d_tp, d_xw}, d_work, st));
    struct Cp { void *dst; const char *src; size_t el, pitch; } cps[4] = {
        {T, (const char *)d_tp, sizeof(double), sizeof(double2)},
        {phi, (const char *)d_tp + sizeof(double), sizeof(double), sizeof(double2)},
        {Tx, (const char *)d_xw, sizeof(float), sizeof(float2)},
        {w, (const char *)d_xw + sizeof(float), sizeof(float), sizeof(float2)}};
    for (const Cp &c : cps) {
        if (!c.dst) continue;
        KCIG_CUDA(cudaMemcpy2DAsync(c.dst, c.el, c.src, c.pitch, c.el, (size_t)nzx, cudaMemcpyDeviceToDevice, st));
    }
    int flag = 0;
    KCIG_CUDA(cudaMemcpyAsync(&flag, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    KCIG_CUDA(cudaStreamSynchronize(st));
    if (flag) return set_error(KCIG_ERR_DEVICE, "kcig_leg_fields_noalloc: a staged table copy did not complete");
    return KCIG_OK;
}
