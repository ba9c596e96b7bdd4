/*
 * kcig_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the adjoint (adj=1) summation of kirchmig2d_cig, used
 * exclusively as the checker of the CUDA library (tests, __graft_entry__.smoke
 * and the cpu_baseline leg of bench.py).  Nothing in the shipped library links
 * or calls this file.
 *
 * Two builds come from this one source (see oracle/Makefile):
 *
 *   KCIG_ORACLE_FP64=1  liboracle64.so  every operation in IEEE double: the
 *                       FP64 oracle every image is measured against.
 *   KCIG_ORACLE_FP64=0  liboracle32.so  the reference's own mixed rounding:
 *                       FP32 storage and arithmetic, with the few expressions
 *                       the reference evaluates in double (Hermite weights,
 *                       the kirmig_pick sum) evaluated in double.  This build
 *                       is pinned bit-for-bit against the reference binary
 *                       compiled from its sources (oracle/_ref), which is what
 *                       pins the FP64 build's algorithm.
 *
 * Every routine cites the reference file:line it restates.  Paths are relative
 * to the reference project root.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef KCIG_ORACLE_FP64
#define KCIG_ORACLE_FP64 1
#endif

#if KCIG_ORACLE_FP64
typedef double R; /* working precision of every FP32 variable of the reference */
#define RF(x) ((double)(x))
#define R_FLOOR floor
#define R_FABS fabs
#define R_ATAN atan
#define R_ATAN2 atan2
#define R_COS cos
#define R_SQRT sqrt
#define R_PI 3.14159265358979323846
#else
typedef float R;
#define RF(x) ((float)(x))
#define R_FLOOR floorf
#define R_FABS fabsf
#define R_ATAN atanf
#define R_ATAN2 atan2f
#define R_COS cosf
#define R_SQRT sqrtf
#define R_PI ((float)3.14159265358979323846)
#endif

#define MAXV(a, b) ((a) > (b) ? (a) : (b))
#define MINV(a, b) ((a) < (b) ? (a) : (b))

/* Parameter block.  Field meaning and defaults follow
 * src/kirchmig2d_cig.cpp:494-958 (a1 of the hot path). */
typedef struct {
    int nt, nh, ns;
    float t0, dt, h0, dh, s0, ds;
    int nz, nx;
    float z0, dz, x0, dx;
    int sny;
    float sy0, sdy;
    int rny;
    float ry0, rdy;
    int ng;
    float g0, dg;
    int cig, cig_is_angle, cmp, half_angle, isdiff, interp_type;
    int use_input_grad, angle_interp, angle_grad_radius, angle_smooth;
    int aperture_trace, aperture_trace_taper, direct_mute, direct_mute_invert;
    float tau, aper, aperture_taper, aperture_rmin, aperture_rtaper, aal;
    float angle_taper_start, angle_taper_end, oazmin, oazmax, oaztaper;
    float direct_mute_slope, direct_mute_intercept, direct_mute_taper;
} oracle_params;

static int idx2d(int iz, int ix, int nz) { return ix * nz + iz; }

/* src/kirchmig2d_cig.cpp:35-41 */
static int nearest_bin(R value, R g0, R dg, int ng)
{
    if (ng <= 0 || dg <= RF(0) || !isfinite(value)) return -1;
    int ig = (int)R_FLOOR((value - g0) / dg + RF(0.5));
    if (ig < 0 || ig >= ng) return -1;
    return ig;
}

/* src/kirchmig2d_cig.cpp:54-79 */
static int linear_bins(R value, R g0, R dg, int ng, int *ig0, int *ig1, R *w0, R *w1)
{
    if (ng <= 0 || dg <= RF(0) || !isfinite(value)) return 0;
    const R u = (value - g0) / dg;
    if (u < RF(-1.0e-5) || u > (R)(ng - 1) + RF(1.0e-5)) return 0;
    if (u <= RF(0)) { *ig0 = 0; *ig1 = 0; *w0 = RF(1); *w1 = RF(0); return 1; }
    if (u >= (R)(ng - 1)) { *ig0 = ng - 1; *ig1 = ng - 1; *w0 = RF(1); *w1 = RF(0); return 1; }
    *ig0 = (int)R_FLOOR(u);
    *ig1 = *ig0 + 1;
    *w1 = u - (R)(*ig0);
    *w0 = RF(1) - *w1;
    return 1;
}

/* src/kirchmig2d_cig.cpp:88-96 */
static R angle_taper_weight(R angle, R start, R end)
{
    if (!isfinite(angle)) return RF(0);
    if (start < RF(0) || end <= start) return RF(1);
    if (angle <= start) return RF(1);
    if (angle >= end) return RF(0);
    const R x = (angle - start) / (end - start);
    return RF(0.5) * (RF(1) + R_COS(R_PI * x));
}

/* src/kirchmig2d_cig.cpp:110-129 */
static void direct_mute(R *trace, int nt, R t0, R dt, R sx, R rx, R slope,
                        R intercept, R taper, int inverted)
{
    const R offset_time = slope * R_FABS(rx - sx);
    const R boundary = inverted ? intercept - offset_time : intercept + offset_time;
    for (int it = 0; it < nt; it++) {
        const R time = t0 + (R)it * dt;
        R w = RF(0);
        if (time >= boundary + taper) {
            w = RF(1);
        } else if (time > boundary) {
            const R u = (time - boundary) / taper;
            w = RF(0.5) * (RF(1) - R_COS(R_PI * u));
        }
        trace[it] *= w;
    }
}

/* src/kirchmig2d_cig.cpp:130-152 */
static R fd_x(const R *tab, int nz, int nx, int iz, int ix, R dx, int r)
{
    if (nx <= 1 || dx == RF(0)) return RF(0);
    if (r < 1) r = 1;
    const int il = MAXV(0, ix - r), ir = MINV(nx - 1, ix + r);
    if (ir == il) return RF(0);
    return (tab[idx2d(iz, ir, nz)] - tab[idx2d(iz, il, nz)]) / ((R)(ir - il) * dx);
}
static R fd_z(const R *tab, int nz, int nx, int iz, int ix, R dz, int r)
{
    (void)nx;
    if (nz <= 1 || dz == RF(0)) return RF(0);
    if (r < 1) r = 1;
    const int it = MAXV(0, iz - r), ib = MINV(nz - 1, iz + r);
    if (ib == it) return RF(0);
    return (tab[idx2d(ib, ix, nz)] - tab[idx2d(it, ix, nz)]) / ((R)(ib - it) * dz);
}

/* src/kirchmig2d_cig.cpp:171-187 */
static R angle_from_grad(R sx, R sz, R rx, R rz, int half)
{
    const R ns = R_SQRT(sx * sx + sz * sz);
    const R nr = R_SQRT(rx * rx + rz * rz);
    if (ns <= RF(1.0e-12) || nr <= RF(1.0e-12)) return (R)NAN;
    const R dot = sx * rx + sz * rz;
    const R cross = sx * rz - sz * rx;
    const R opening = R_ATAN2(R_FABS(cross), dot);
    R deg = opening * RF(180.0) / R_PI;
    return half ? RF(0.5) * deg : deg;
}

/* src/kirchmig2d_cig.cpp:200-211 */
static R depth_mute_weight(R angle, int iz, int nz, R amin, R amax, R band)
{
    if (!isfinite(angle)) return RF(0);
    const R zf = (nz > 1) ? (R)iz / (R)(nz - 1) : RF(0);
    const R cutoff = amin + zf * (amax - amin);
    if (band <= RF(0)) return (angle <= cutoff) ? RF(1) : RF(0);
    if (angle <= cutoff) return RF(1);
    if (angle >= cutoff + band) return RF(0);
    const R u = (angle - cutoff) / band;
    return RF(0.5) * (RF(1) + R_COS(R_PI * u));
}

/* src/kirchmig2d_cig.cpp:226-238 */
static R aperture_leg_weight(R leg, R aper, R band)
{
    if (!isfinite(leg)) return RF(0);
    if (band <= RF(0)) return (leg <= aper) ? RF(1) : RF(0);
    const R inner = aper - band;
    if (leg <= inner) return RF(1);
    if (leg >= aper) return RF(0);
    const R u = (leg - inner) / band;
    return RF(0.5) * (RF(1) + R_COS(R_PI * u));
}

/* src/kirchmig2d_cig.cpp:256-269 */
static R aperture_floor_weight(R d, R rmin, R rt)
{
    if (rmin <= RF(0)) return RF(0);
    if (rt <= RF(0)) return (d <= rmin) ? RF(1) : RF(0);
    const R inner = rmin - rt;
    if (inner <= RF(0)) {
        if (d >= rmin) return RF(0);
        const R u = d / rmin;
        return RF(0.5) * (RF(1) + R_COS(R_PI * u));
    }
    if (d <= inner) return RF(1);
    if (d >= rmin) return RF(0);
    const R u = (d - inner) / rt;
    return RF(0.5) * (RF(1) + R_COS(R_PI * u));
}

/* src/kirchmig2d_cig.cpp:381-394 */
static void diff2(R *trace, int n, R d, R *tmp)
{
    for (int i = 0; i < n; i++) tmp[i] = trace[i];
    for (int i = 1; i < n - 1; i++) trace[i] = (tmp[i + 1] - tmp[i - 1]) / (RF(2) * d);
    trace[0] = (tmp[1] - tmp[0]) / d;
    trace[n - 1] = (tmp[n - 1] - tmp[n - 2]) / d;
}

/* SERECKIRCH/src/kirmig.cpp:8-24: causal then anticausal running sum. */
static void doubint(int nt, R *trace)
{
    R tt = trace[0];
    for (int it = 1; it < nt; it++) { tt += trace[it]; trace[it] = tt; }
    tt = trace[nt - 1];
    for (int it = nt - 2; it >= 0; it--) { tt += trace[it]; trace[it] = tt; }
}

/* SERECKIRCH/src/kirmig.cpp:34-58 (adj branch).  The reference sums the
 * six-term expression in double (its literals are double) and rounds once
 * into the FP32 sample; the products ftm*trace[itm+1] and ftp*trace[itp+1]
 * have two float operands and are therefore float products there. */
static R kirmig_pick(R ti, R deltat, const R *trace, int nt, R dt, R t0)
{
    int it, itm, itp;
    R ft, tm, tp, ftm, ftp, imp;
    ft = (ti - t0) / dt; it = (int)R_FLOOR(ft); ft -= (R)it;
    if (it < 0 || it >= nt - 1) return RF(0);
    tm = ti - deltat - dt;
    ftm = (tm - t0) / dt; itm = (int)R_FLOOR(ftm); ftm -= (R)itm;
    if (itm < 0) return RF(0);
    tp = ti + deltat + dt;
    ftp = (tp - t0) / dt; itp = (int)R_FLOOR(ftp); ftp -= (R)itp;
    if (itp >= nt - 1) return RF(0);
    imp = dt / (dt + tp - tm);
    imp *= imp;
#if KCIG_ORACLE_FP64
    return imp * (2. * (1. - ft) * trace[it] + 2. * ft * trace[it + 1] -
                  (1. - ftm) * trace[itm] - ftm * trace[itm + 1] -
                  (1. - ftp) * trace[itp] - ftp * trace[itp + 1]);
#else
    {
        double sum = 2. * (1. - ft) * trace[it] + 2. * ft * trace[it + 1];
        sum -= (1. - ftm) * trace[itm];
        sum -= (double)(ftm * trace[itm + 1]);
        sum -= (1. - ftp) * trace[itp];
        sum -= (double)(ftp * trace[itp + 1]);
        return (float)(0.0 + (double)imp * sum);
    }
#endif
}

/* SERECKIRCH/src/kirmig.cpp:59-68 (the forward branch): the sample, scaled
 * by imp, is spread over the same six trace samples with the same weights
 * (the reference's s = imp*sample is a float product; the six updates are
 * evaluated in double and rounded into the float trace). */
static void kirmig_spray(R ti, R deltat, R sample, R *trace, int nt, R dt, R t0)
{
    int it, itm, itp;
    R ft, tm, tp, ftm, ftp, imp, sv;
    ft = (ti - t0) / dt; it = (int)R_FLOOR(ft); ft -= (R)it;
    if (it < 0 || it >= nt - 1) return;
    tm = ti - deltat - dt;
    ftm = (tm - t0) / dt; itm = (int)R_FLOOR(ftm); ftm -= (R)itm;
    if (itm < 0) return;
    tp = ti + deltat + dt;
    ftp = (tp - t0) / dt; itp = (int)R_FLOOR(ftp); ftp -= (R)itp;
    if (itp >= nt - 1) return;
    imp = dt / (dt + tp - tm);
    imp *= imp;
    sv = imp * sample;
#if KCIG_ORACLE_FP64
    trace[it] += 2. * (1. - ft) * sv;
    trace[it + 1] += 2. * ft * sv;
    trace[itm] -= (1. - ftm) * sv;
    trace[itm + 1] -= ftm * sv;
    trace[itp] -= (1. - ftp) * sv;
    trace[itp + 1] -= ftp * sv;
#else
    /* the reference's operand types: a double literal promotes the update
     * to double before it is added to the float sample; ftm*s and ftp*s are
     * float products subtracted in float */
    trace[it] = (float)((double)trace[it] + 2. * (1. - ft) * sv);
    trace[it + 1] = (float)((double)trace[it + 1] + 2. * ft * sv);
    trace[itm] = (float)((double)trace[itm] - (1. - ftm) * sv);
    trace[itm + 1] = trace[itm + 1] - ftm * sv;
    trace[itp] = (float)((double)trace[itp] - (1. - ftp) * sv);
    trace[itp + 1] = trace[itp + 1] - ftp * sv;
#endif
}

/* SERECKIRCH/src/tinterpsr.cpp:37-70, 142-188, 72-140.  Writes the value
 * field p and the position-derivative field dp between slices (p0,m0) and
 * (p1,m1) at in-interval coordinate x of a position axis with spacing dxp. */
static void interp_slices(int type, R *p, R *dp, R x, R dxp, const R *p0, const R *p1,
                          const R *m0, const R *m1, int n1, int nn, R dd)
{
    int i;
    if (type == 'l') {
        const R t = x / dxp;
#pragma omp parallel for
        for (i = 0; i < nn; i++) {
#if KCIG_ORACLE_FP64
            p[i] = (1. - t) * p0[i] + t * p1[i];
#else
            p[i] = (float)((1. - (double)t) * p0[i] + (double)(t * p1[i]));
#endif
            dp[i] = (-p0[i] + p1[i]) / dxp;
        }
    } else if (type == 'p') {
        /* tinterp_partial / dinterp_partial.  For the first k2 lateral columns
         * the reference's right-slice derivative terms index p1[i - k2*n1]
         * below the start of the slice (tinterpsr.cpp:119-124, undefined
         * behaviour that reads whatever precedes the buffer); P1() clamps
         * such an index to the slice's first column at the same depth. */
        const R t = x / dxp;
        const int k1 = (int)((double)(x / dd) + 0.5);
        const int k2 = (int)((double)((dxp - x) / dd) + 0.5);
#define CLI(j) ((j) < 0 ? i % n1 : ((j) >= nn ? nn - n1 + i % n1 : (j)))
#define P1(j) p1[CLI(j)]
#define P0(j) p0[CLI(j)]
#pragma omp parallel for
        for (i = 0; i < nn; i++) {
            /* the reference stores after every update, so each "-=" rounds; t*(...)
             * has two float operands there and is a float product */
            double v;
            R dv;
            if (i - k1 * n1 >= 0 && i + k2 * n1 < nn) {
                v = (1. - t) * p0[i - k1 * n1] + (double)(t * p1[i + k2 * n1]);
                dv = (-p0[i - k1 * n1] + p1[i + k2 * n1]) / dxp;
                if (i - (k1 + 1) * n1 >= 0 && i - (k1 - 1) * n1 < nn)
                    dv = (R)(dv - (1. - t) * (double)(-p0[i - (k1 + 1) * n1] + p0[i - (k1 - 1) * n1]) / (2. * dd));
                else if (i - (k1 + 1) * n1 < 0)
                    dv = (R)(dv - (1. - t) * (double)(-p0[i - k1 * n1] + P0(i - (k1 - 1) * n1)) / dd);
                else
                    dv = (R)(dv - (1. - t) * (double)(-p0[i - (k1 + 1) * n1] + p0[i - k1 * n1]) / dd);
                if (i - (k2 + 1) * n1 >= 0 && i - (k2 - 1) * n1 < nn)
                    dv = (R)(dv - (double)(t * (-p1[i - (k2 + 1) * n1] + p1[i - (k2 - 1) * n1])) / (2. * dd));
                else if (i - (k2 + 1) * n1 < 0)
                    dv = (R)(dv - (double)(t * (-P1(i - k2 * n1) + P1(i - (k2 - 1) * n1))) / dd);
                else
                    dv = (R)(dv - (double)(t * (-p1[i - (k2 + 1) * n1] + p1[i - k2 * n1])) / dd);
            } else {
                v = (1. - t) * p0[i] + (double)(t * p1[i]);
                dv = (-p0[i] + p1[i]) / dxp;
            }
            p[i] = (R)v;
            dp[i] = dv;
        }
#undef P1
#undef P0
#undef CLI
    } else { /* 'h' cubic Hermite (default) */
        const R t = x / dxp;
        double h00 = 2. * t * t * t - 3. * t * t + 1.;
        double h10 = t * t * t - 2. * t * t + t;
        double h01 = -2. * t * t * t + 3. * t * t;
        double h11 = t * t * t - t * t;
        double g00 = -6. * t * (1. - t);
        double g10 = (1. - t) * (1. - 3. * t);
        double g01 = 6. * t * (1. - t);
        double g11 = 3. * t * t - 2. * t;
#pragma omp parallel for
        for (i = 0; i < nn; i++) {
            p[i] = (R)(h00 * p0[i] + h10 * dxp * m0[i] + h01 * p1[i] + h11 * dxp * m1[i]);
            dp[i] = (R)((g00 * p0[i] + g10 * dxp * m0[i] + g01 * p1[i] + g11 * dxp * m1[i]) / dxp);
        }
    }
}

static void load_slice(R *dst, const float *vol, int index, long nzx)
{
    const float *src = vol + (long)index * nzx;
    for (long i = 0; i < nzx; i++) dst[i] = (R)src[i];
}

/* Which slice(s) a position falls in is a discrete decision, and for a
 * position on a table node it depends on the rounding of the FP32 expression
 * (pos - o)/d.  Both builds therefore take every slice and trace-index
 * decision from the reference's own FP32 arithmetic (posf: the position as
 * the reference computes it in float); only the continuous quantities (the
 * in-interval coordinate and everything after it) run in the build's
 * precision. */

/* Source/receiver table interpolation at coordinate `pos` on the position
 * axis (o, d, n): src/kirchmig2d_cig.cpp:987-1029 (source) and :1148-1180
 * (receiver).  Returns the left slice index as the reference assigns it. */
static int table_at(int is_source, const oracle_params *P, const float *tab, const float *der,
                    float posf, R pos, float of, float df, int n, R *T, R *Tx, R *s0, R *s1, R *m0,
                    R *m1)
{
    const long nzx = (long)P->nz * P->nx;
    int i0;
    int clamp_left;
    float f = 0.0f;
    if (is_source) {
        clamp_left = (n <= 1 || df == 0.0f);
        if (!clamp_left) f = (posf - of) / df;
        if (!clamp_left && f <= 0.0f) clamp_left = 1;
    } else {
        if (n > 1 && df != 0.0f) f = (posf - of) / df;
        clamp_left = (n <= 1 || df == 0.0f || f <= 0.0f);
    }
    if (clamp_left) {
        load_slice(T, tab, 0, nzx);
        load_slice(Tx, der, 0, nzx);
        return 0;
    }
    if (f >= (float)(n - 1)) {
        load_slice(T, tab, n - 1, nzx);
        load_slice(Tx, der, n - 1, nzx);
        return n - 1;
    }
    i0 = (int)floorf(f);
    const R coord = pos - ((R)of + (R)i0 * (R)df);
    load_slice(s0, tab, i0, nzx);
    load_slice(s1, tab, i0 + 1, nzx);
    load_slice(m0, der, i0, nzx);
    load_slice(m1, der, i0 + 1, nzx);
    interp_slices(P->interp_type, T, Tx, coord, (R)df, s0, s1, m0, m1, P->nz, (int)nzx, RF(P->dx));
    return i0;
}

/* src/kirchmig2d_cig.cpp:294-322 */
static void interp_volume_linear(R *out, const float *vol, int npos, long nzx, float coordf, R coord,
                                 float of, float df, R *a, R *b)
{
    if (npos <= 1 || df == 0.0f) { load_slice(out, vol, 0, nzx); return; }
    const float ff = (coordf - of) / df;
    if (ff <= 0.0f) { load_slice(out, vol, 0, nzx); return; }
    if (ff >= (float)(npos - 1)) { load_slice(out, vol, npos - 1, nzx); return; }
    const int i0 = (int)floorf(ff);
    const R w = (coord - (R)of) / (R)df - (R)i0;
    load_slice(a, vol, i0, nzx);
    load_slice(b, vol, i0 + 1, nzx);
    for (long i = 0; i < nzx; i++) out[i] = (RF(1) - w) * a[i] + w * b[i];
}

/* src/kirchmig2d_cig.cpp:424-435 */
static void grad_plane(const R *tab, int nz, int nx, R dz, R dx, int r, R *gx, R *gz)
{
#pragma omp parallel for
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++) {
            const int i = idx2d(iz, ix, nz);
            gx[i] = fd_x(tab, nz, nx, iz, ix, dx, r);
            gz[i] = fd_z(tab, nz, nx, iz, ix, dz, r);
        }
}

/* src/kirchmig2d_cig.cpp:438-492: two separable box passes (z then x). */
static void box_z(const R *in, R *out, int nz, int nx, int r)
{
#pragma omp parallel for
    for (int ix = 0; ix < nx; ix++) {
        const R *c = in + (long)ix * nz;
        R *o = out + (long)ix * nz;
        for (int iz = 0; iz < nz; iz++) {
            const int a = (iz - r < 0) ? 0 : iz - r;
            const int b = (iz + r > nz - 1) ? nz - 1 : iz + r;
            R s = RF(0);
            for (int k = a; k <= b; k++) s += c[k];
            o[iz] = s / (R)(b - a + 1);
        }
    }
}
static void box_x(const R *in, R *out, int nz, int nx, int r)
{
#pragma omp parallel for
    for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nx; ix++) {
            const int a = (ix - r < 0) ? 0 : ix - r;
            const int b = (ix + r > nx - 1) ? nx - 1 : ix + r;
            R s = RF(0);
            for (int k = a; k <= b; k++) s += in[(long)k * nz + iz];
            out[(long)ix * nz + iz] = s / (R)(b - a + 1);
        }
}
static void smooth_pass(const R *src, R *dst, R *work, int nz, int nx, int rz, int rx)
{
    const long n = (long)nz * nx;
    if (rz > 0) box_z(src, work, nz, nx, rz); else memcpy(work, src, n * sizeof(R));
    if (rx > 0) box_x(work, dst, nz, nx, rx); else memcpy(dst, work, n * sizeof(R));
}
static void smooth_component(R *f, int nz, int nx, int rz, int rx, R *t1, R *t2)
{
    if (rz <= 0 && rx <= 0) return;
    smooth_pass(f, t1, t2, nz, nx, rz, rx);
    smooth_pass(t1, f, t2, nz, nx, rz, rx);
}

/* Stabilised gradient field of one leg (src/kirchmig2d_cig.cpp:1041-1052 for
 * the source, :1190-1201 for the receiver). */
static void leg_gradient(const oracle_params *P, const R *T, const R *ingx, const R *ingz,
                         R *gx, R *gz, R *t1, R *t2)
{
    const long nzx = (long)P->nz * P->nx;
    if (P->use_input_grad) {
        memcpy(gx, ingx, nzx * sizeof(R));
        memcpy(gz, ingz, nzx * sizeof(R));
    } else {
        grad_plane(T, P->nz, P->nx, RF(P->dz), RF(P->dx), P->angle_grad_radius, gx, gz);
    }
    if (P->angle_smooth > 0) {
        smooth_component(gx, P->nz, P->nx, P->angle_smooth, P->angle_smooth, t1, t2);
        smooth_component(gz, P->nz, P->nx, P->angle_smooth, P->angle_smooth, t1, t2);
    }
}

/* ---------------------------------------------------------------- exports -- */

void oracle_doubint(int nt, const float *in, double *out, int isdiff, float dt)
{
    R *tr = (R *)malloc(sizeof(R) * (size_t)nt * 2);
    for (int i = 0; i < nt; i++) tr[i] = (R)in[i];
    doubint(nt, tr);
    if (isdiff == 1) diff2(tr, nt, RF(dt), tr + nt);
    for (int i = 0; i < nt; i++) out[i] = (double)tr[i];
    free(tr);
}

void oracle_mute(int nt, float *trace, float t0, float dt, float sx, float rx, float slope,
                 float intercept, float taper, int inverted)
{
    R *tr = (R *)malloc(sizeof(R) * (size_t)nt);
    for (int i = 0; i < nt; i++) tr[i] = (R)trace[i];
    direct_mute(tr, nt, RF(t0), RF(dt), RF(sx), RF(rx), RF(slope), RF(intercept), RF(taper), inverted);
    for (int i = 0; i < nt; i++) trace[i] = (float)tr[i];
    free(tr);
}

double oracle_pick(double ti, double deltat, const double *dtrace, int nt, double dt, double t0)
{
    R *tr = (R *)malloc(sizeof(R) * (size_t)nt);
    for (int i = 0; i < nt; i++) tr[i] = (R)dtrace[i];
    double v = (double)kirmig_pick((R)ti, (R)deltat, tr, nt, (R)dt, (R)t0);
    free(tr);
    return v;
}

/* Leg fields of one source (is_source=1) or receiver position: traveltime T,
 * its position derivative Tx and the stabilised gradient (gx, gz), all [nzx]. */
int oracle_leg_fields(const oracle_params *P, int is_source, const float *tab, const float *der,
                      const float *vgx, const float *vgz, float pos, double *T_out,
                      double *Tx_out, double *gx_out, double *gz_out)
{
    const long nzx = (long)P->nz * P->nx;
    R *buf = (R *)malloc(sizeof(R) * (size_t)nzx * 12);
    if (!buf) return -1;
    R *T = buf, *Tx = buf + nzx, *s0 = buf + 2 * nzx, *s1 = buf + 3 * nzx, *m0 = buf + 4 * nzx,
      *m1 = buf + 5 * nzx, *gx = buf + 6 * nzx, *gz = buf + 7 * nzx, *t1 = buf + 8 * nzx,
      *t2 = buf + 9 * nzx, *ig = buf + 10 * nzx, *ih = buf + 11 * nzx;
    const int n = is_source ? P->sny : P->rny;
    const R o = is_source ? RF(P->sy0) : RF(P->ry0);
    const R d = is_source ? RF(P->sdy) : RF(P->rdy);
    table_at(is_source, P, tab, der, pos, (R)pos, (float)o, (float)d, n, T, Tx, s0, s1, m0, m1);
    if (P->use_input_grad) {
        interp_volume_linear(ig, vgx, n, nzx, pos, (R)pos, (float)o, (float)d, s0, s1);
        interp_volume_linear(ih, vgz, n, nzx, pos, (R)pos, (float)o, (float)d, s0, s1);
    }
    leg_gradient(P, T, ig, ih, gx, gz, t1, t2);
    for (long i = 0; i < nzx; i++) {
        T_out[i] = (double)T[i];
        Tx_out[i] = (double)Tx[i];
        gx_out[i] = (double)gx[i];
        gz_out[i] = (double)gz[i];
    }
    free(buf);
    return 0;
}

/* The whole adjoint migration, src/kirchmig2d_cig.cpp:979-1339 with adj=1.
 * data [ns][nh][nt]; tables [n][nx][nz]; image [ng][nx][nz] (accumulated into
 * the caller's zeroed buffer).  Gradient volumes may be NULL unless
 * P->use_input_grad. */
int oracle_migrate_adj(const oracle_params *P, const float *data, const float *stab,
                       const float *sder, const float *rtab, const float *rder,
                       const float *sgx_v, const float *sgz_v, const float *rgx_v,
                       const float *rgz_v, double *image)
{
    const int nz = P->nz, nx = P->nx, nt = P->nt, ng = P->ng;
    const long nzx = (long)nz * nx;
    const int angle = P->cig && P->cig_is_angle;
    const R ds = RF(P->ns == 1 ? 0.0f : P->ds);
    const R dh = RF(P->nh == 1 ? 0.0f : P->dh);
    R *buf = (R *)malloc(sizeof(R) * (size_t)nzx * 18);
    R *trace = (R *)malloc(sizeof(R) * (size_t)nt * 2);
    R *out = (R *)calloc((size_t)nzx * ng, sizeof(R));
    if (!buf || !trace || !out) { free(buf); free(trace); free(out); return -1; }
    R *ST = buf, *STx = buf + nzx, *RT = buf + 2 * nzx, *RTx = buf + 3 * nzx;
    R *s0 = buf + 4 * nzx, *s1 = buf + 5 * nzx, *m0 = buf + 6 * nzx, *m1 = buf + 7 * nzx;
    R *gsx = buf + 8 * nzx, *gsz = buf + 9 * nzx, *grx = buf + 10 * nzx, *grz = buf + 11 * nzx;
    R *t1 = buf + 12 * nzx, *t2 = buf + 13 * nzx, *sgx = buf + 14 * nzx, *sgz = buf + 15 * nzx;
    R *rgx = buf + 16 * nzx, *rgz = buf + 17 * nzx;
    const R t0 = RF(P->t0), dt = RF(P->dt), tau = RF(P->tau), aal = RF(P->aal);
    const R dz = RF(P->dz), dxg = RF(P->dx), x0 = RF(P->x0);
    const R g0 = RF(P->g0), dg = RF(P->dg);

    for (int is = 0; is < P->ns; is++) {
        const R s = RF(P->s0) + (R)is * ds;
        const float sf = P->s0 + (float)is * (P->ns == 1 ? 0.0f : P->ds); /* reference's float s */
        const int ist = table_at(1, P, stab, sder, sf, s, P->sy0, P->sdy, P->sny, ST, STx,
                                 s0, s1, m0, m1);
        if (angle) {
            if (P->use_input_grad) {
                interp_volume_linear(sgx, sgx_v, P->sny, nzx, sf, s, P->sy0, P->sdy, s0, s1);
                interp_volume_linear(sgz, sgz_v, P->sny, nzx, sf, s, P->sy0, P->sdy, s0, s1);
            }
            leg_gradient(P, ST, sgx, sgz, gsx, gsz, t1, t2);
        }
        for (int ih = 0; ih < P->nh; ih++) {
            const R h = RF(P->h0) + (R)ih * dh;
            const R rpos = P->cmp ? (s + h) : h;
            const float hf = P->h0 + (float)ih * (P->nh == 1 ? 0.0f : P->dh);
            const float rposf = P->cmp ? (sf + hf) : hf;
            float rf = 0.0f;
            if (P->rny > 1 && P->rdy != 0.0f) rf = (rposf - P->ry0) / P->rdy;
            const int iht = (P->rny > 1 && P->rdy != 0.0f) ? (int)floorf(rf) : 0;
            const float *src = data + ((long)is * P->nh + ih) * nt;
            for (int it = 0; it < nt; it++) trace[it] = (R)src[it];
            if (P->direct_mute)
                direct_mute(trace, nt, t0, dt, s, rpos, RF(P->direct_mute_slope),
                            RF(P->direct_mute_intercept), RF(P->direct_mute_taper),
                            P->direct_mute_invert);
            R trace_w = RF(1);
            if (P->aperture_trace != -1) {
                const R ad = R_FABS((R)(iht - ist));
                if (ad >= (R)P->aperture_trace) continue;
                if (P->aperture_trace_taper > 0) {
                    const R tb = MAXV(RF(0), (R)(P->aperture_trace - P->aperture_trace_taper));
                    if (ad > tb) {
                        const R den = (R)P->aperture_trace - tb;
                        if (den > RF(0)) trace_w = RF(0.5) * (RF(1) + R_COS(R_PI * ((ad - tb) / den)));
                    }
                }
            }
            int ig_offset = 0;
            if (P->cig && !P->cig_is_angle) {
                /* a discrete decision: taken in the reference's float */
                {
                    const float u = (hf - P->g0) / P->dg + 0.5f;
                    ig_offset = (ng <= 0 || P->dg <= 0.0f || !isfinite(hf)) ? -1 : (int)floorf(u);
                    if (ig_offset >= ng) ig_offset = -1;
                }
                if (ig_offset < 0) continue;
            }
            doubint(nt, trace);
            if (P->isdiff == 1) diff2(trace, nt, dt, trace + nt);
            table_at(0, P, rtab, rder, rposf, rpos, P->ry0, P->rdy, P->rny, RT, RTx, s0, s1, m0, m1);
            if (angle) {
                if (P->use_input_grad) {
                    interp_volume_linear(rgx, rgx_v, P->rny, nzx, rposf, rpos, P->ry0, P->rdy, s0, s1);
                    interp_volume_linear(rgz, rgz_v, P->rny, nzx, rposf, rpos, P->ry0, P->rdy, s0, s1);
                }
                leg_gradient(P, RT, rgx, rgz, grx, grz, t1, t2);
            }
#pragma omp parallel for
            for (long i = 0; i < nzx; i++) {
                const int iz = (int)(i % nz);
                const int ix = (int)((i - iz) / nz);
                const R zdist = MAXV(R_FABS((R)iz * dz), MAXV(RF(1.0e-12), RF(1.0e-6) * R_FABS(dz)));
                const R ximg = x0 + (R)ix * dxg;
                const R dsx = R_FABS(s - ximg);
                const R drx = R_FABS(rpos - ximg);
                const R as_deg = R_ATAN(dsx / zdist) * RF(180.0) / R_PI;
                const R ar_deg = R_ATAN(drx / zdist) * RF(180.0) / R_PI;
                const R ws = MAXV(aperture_leg_weight(as_deg, RF(P->aper), RF(P->aperture_taper)),
                                  aperture_floor_weight(dsx, RF(P->aperture_rmin), RF(P->aperture_rtaper)));
                const R wr = MAXV(aperture_leg_weight(ar_deg, RF(P->aper), RF(P->aperture_taper)),
                                  aperture_floor_weight(drx, RF(P->aperture_rmin), RF(P->aperture_rtaper)));
                const R apw = ws * wr;
                if (apw <= RF(0)) continue;
                const R ti = ST[i] + RT[i] + tau;
                const R tx = MAXV(R_FABS(STx[i] * ds), R_FABS(RTx[i] * dh));
                if (angle) {
                    const R ang = angle_from_grad(gsx[i], gsz[i], grx[i], grz[i], P->half_angle);
                    const R aw = angle_taper_weight(ang, RF(P->angle_taper_start), RF(P->angle_taper_end)) *
                                 depth_mute_weight(ang, iz, nz, RF(P->oazmin), RF(P->oazmax), RF(P->oaztaper)) *
                                 trace_w * apw;
                    if (aw <= RF(0)) continue;
                    if (P->angle_interp) {
                        int ig0 = -1, ig1 = -1;
                        R w0 = RF(0), w1 = RF(0);
                        if (!linear_bins(ang, g0, dg, ng, &ig0, &ig1, &w0, &w1)) continue;
                        R picked = kirmig_pick(ti, tx * aal, trace, nt, dt, t0);
                        picked *= aw;
                        out[(long)ig0 * nzx + i] += w0 * picked;
                        if (ig1 != ig0 && w1 > RF(0)) out[(long)ig1 * nzx + i] += w1 * picked;
                    } else {
                        const int ig = nearest_bin(ang, g0, dg, ng);
                        if (ig < 0) continue;
                        const R picked = kirmig_pick(ti, tx * aal, trace, nt, dt, t0);
                        out[(long)ig * nzx + i] += aw * picked;
                    }
                } else {
                    const int ig = P->cig ? ig_offset : 0;
                    const R picked = kirmig_pick(ti, tx * aal, trace, nt, dt, t0);
                    out[(long)ig * nzx + i] += trace_w * apw * picked;
                }
            }
        }
    }
    for (long i = 0; i < nzx * ng; i++) image[i] = (double)out[i];
    free(buf);
    free(trace);
    free(out);
    return 0;
}

/* kirchmig2d_cig.cpp adj=0 (:1110-1147, :1300-1312, :1340-1351): forward
 * modelling of data [ns][nh][nt] from an image [ng][nx][nz] with the weights
 * of the adjoint path; each trace is the sum of the sprayed picks, then
 * doubint (its own adjoint).  No direct mute and no diff2 are applied, as in
 * the reference's forward branch.  Serial (the trace is the scatter target). */
/* ------------------------------------------------------------ kirchmig2d --
 * src/kirchmig2d.cpp:366-540 (adj=1), the plain Kirchhoff tool: the table
 * index is the truncated float quotient, and a position in the first
 * interval takes slice 0 unchanged (:372-395, :413-440); a trace is dropped
 * when |iht - ist| >= aperture_trace (:423); a pair is dropped outside the
 * cone test of :455-488, evaluated in the reference's float arithmetic in
 * both builds; ti = t1 + t2 + tau; the pick goes to image ih (cig=1) or 0.
 * P->ng must be nh (cig=1) or 1. */
static int table_at_k2d(const oracle_params *P, const float *tab, const float *der, float posf, R pos, float of,
                        float df, int n, R *T, R *Tx, R *s0, R *s1, R *m0, R *m1)
{
    const long nzx = (long)P->nz * P->nx;
    const int it = (df != 0.0f) ? (int)((posf - of) / df) : 0;
    if (it <= 0) {
        load_slice(T, tab, 0, nzx);
        load_slice(Tx, der, 0, nzx);
    } else if (it >= n - 1) {
        load_slice(T, tab, n - 1, nzx);
        load_slice(Tx, der, n - 1, nzx);
    } else {
        const R coord = pos - ((R)of + (R)it * (R)df);
        load_slice(s0, tab, it, nzx);
        load_slice(s1, tab, it + 1, nzx);
        load_slice(m0, der, it, nzx);
        load_slice(m1, der, it + 1, nzx);
        interp_slices(P->interp_type, T, Tx, coord, (R)df, s0, s1, m0, m1, P->nz, (int)nzx, RF(P->dx));
    }
    return it;
}

static int cone_cut(float num, float zi, float aper)
{
    return atanf(num / zi) * 180. / 3.14159265358979323846 > aper;
}

int oracle_kirchmig2d_adj(const oracle_params *P, const float *data, const float *stab, const float *sder,
                          const float *rtab, const float *rder, double *image)
{
    const int nz = P->nz, nx = P->nx, nt = P->nt, ng = P->ng;
    const long nzx = (long)nz * nx;
    const float dsf = P->ns == 1 ? 0.0f : P->ds, dhf = P->nh == 1 ? 0.0f : P->dh;
    const R ds = RF(dsf), dh = RF(dhf);
    R *buf = (R *)malloc(sizeof(R) * (size_t)nzx * 8);
    R *trace = (R *)malloc(sizeof(R) * (size_t)nt * 2);
    R *out = (R *)calloc((size_t)nzx * ng, sizeof(R));
    if (!buf || !trace || !out) { free(buf); free(trace); free(out); return -1; }
    R *ST = buf, *STx = buf + nzx, *RT = buf + 2 * nzx, *RTx = buf + 3 * nzx;
    R *s0 = buf + 4 * nzx, *s1 = buf + 5 * nzx, *m0 = buf + 6 * nzx, *m1 = buf + 7 * nzx;
    const R t0 = RF(P->t0), dt = RF(P->dt), tau = RF(P->tau), aal = RF(P->aal);
    for (int is = 0; is < P->ns; is++) {
        const float sf = P->s0 + (float)is * dsf;
        const R s = RF(P->s0) + (R)is * ds;
        const int ist = table_at_k2d(P, stab, sder, sf, s, P->sy0, P->sdy, P->sny, ST, STx, s0, s1, m0, m1);
        for (int ih = 0; ih < P->nh; ih++) {
            const float hf = P->h0 + (float)ih * dhf;
            const R h = RF(P->h0) + (R)ih * dh;
            const float rposf = P->cmp ? sf + hf : hf;
            const R rpos = P->cmp ? s + h : h;
            const int iht = (P->rdy != 0.0f) ? (int)((rposf - P->ry0) / P->rdy) : 0;
            if (P->aperture_trace != -1 && fabs((double)(iht - ist)) >= (double)P->aperture_trace) continue;
            const float *src = data + ((long)is * P->nh + ih) * nt;
            for (int it = 0; it < nt; it++) trace[it] = (R)src[it];
            doubint(nt, trace);
            if (P->isdiff == 1) diff2(trace, nt, dt, trace + nt);
            (void)table_at_k2d(P, rtab, rder, rposf, rpos, P->ry0, P->rdy, P->rny, RT, RTx, s0, s1, m0, m1);
            R *img = out + (long)(P->cig ? ih : 0) * nzx;
#pragma omp parallel for
            for (long i = 0; i < nzx; i++) {
                const int iz = (int)(i % nz), ix = (int)(i / nz);
                const float zi = (float)iz * P->dz, xd = (float)ix * P->dx;
                int cut;
                if (P->cmp) {
                    if (hf >= 0.0f)
                        cut = cone_cut(sf - P->x0 - xd, zi, P->aper) || cone_cut(P->x0 + xd - sf - hf, zi, P->aper);
                    else
                        cut = cone_cut(sf + hf - P->x0 - xd, zi, P->aper) || cone_cut(P->x0 + xd - sf, zi, P->aper);
                } else {
                    if (hf - sf >= 0.0f)
                        cut = cone_cut(sf - P->x0 - xd, zi, P->aper) || cone_cut(P->x0 + xd - hf, zi, P->aper);
                    else
                        cut = cone_cut(hf - P->x0 - xd, zi, P->aper) || cone_cut(P->x0 + xd - sf, zi, P->aper);
                }
                if (cut) continue;
                const R ti = ST[i] + RT[i] + tau;
                const R tx = MAXV(R_FABS(STx[i] * ds), R_FABS(RTx[i] * dh));
                img[i] += kirmig_pick(ti, tx * aal, trace, nt, dt, t0);
            }
        }
    }
    for (long i = 0; i < nzx * ng; i++) image[i] = (double)out[i];
    free(buf);
    free(trace);
    free(out);
    return 0;
}

int oracle_model_fwd(const oracle_params *P, const float *image, const float *stab, const float *sder,
                     const float *rtab, const float *rder, const float *sgx_v, const float *sgz_v,
                     const float *rgx_v, const float *rgz_v, double *data)
{
    const int nz = P->nz, nx = P->nx, nt = P->nt, ng = P->ng;
    const long nzx = (long)nz * nx;
    const int angle = P->cig && P->cig_is_angle;
    const R ds = RF(P->ns == 1 ? 0.0f : P->ds);
    const R dh = RF(P->nh == 1 ? 0.0f : P->dh);
    R *buf = (R *)malloc(sizeof(R) * (size_t)nzx * 18);
    R *trace = (R *)malloc(sizeof(R) * (size_t)nt);
    if (!buf || !trace) { free(buf); free(trace); return -1; }
    R *ST = buf, *STx = buf + nzx, *RT = buf + 2 * nzx, *RTx = buf + 3 * nzx;
    R *s0 = buf + 4 * nzx, *s1 = buf + 5 * nzx, *m0 = buf + 6 * nzx, *m1 = buf + 7 * nzx;
    R *gsx = buf + 8 * nzx, *gsz = buf + 9 * nzx, *grx = buf + 10 * nzx, *grz = buf + 11 * nzx;
    R *t1 = buf + 12 * nzx, *t2 = buf + 13 * nzx, *sgx = buf + 14 * nzx, *sgz = buf + 15 * nzx;
    R *rgx = buf + 16 * nzx, *rgz = buf + 17 * nzx;
    const R t0 = RF(P->t0), dt = RF(P->dt), tau = RF(P->tau), aal = RF(P->aal);
    const R dz = RF(P->dz), dxg = RF(P->dx), x0 = RF(P->x0);
    const R g0 = RF(P->g0), dg = RF(P->dg);

    for (int is = 0; is < P->ns; is++) {
        const R s = RF(P->s0) + (R)is * ds;
        const float sf = P->s0 + (float)is * (P->ns == 1 ? 0.0f : P->ds);
        const int ist = table_at(1, P, stab, sder, sf, s, P->sy0, P->sdy, P->sny, ST, STx,
                                 s0, s1, m0, m1);
        if (angle) {
            if (P->use_input_grad) {
                interp_volume_linear(sgx, sgx_v, P->sny, nzx, sf, s, P->sy0, P->sdy, s0, s1);
                interp_volume_linear(sgz, sgz_v, P->sny, nzx, sf, s, P->sy0, P->sdy, s0, s1);
            }
            leg_gradient(P, ST, sgx, sgz, gsx, gsz, t1, t2);
        }
        for (int ih = 0; ih < P->nh; ih++) {
            const R h = RF(P->h0) + (R)ih * dh;
            const R rpos = P->cmp ? (s + h) : h;
            const float hf = P->h0 + (float)ih * (P->nh == 1 ? 0.0f : P->dh);
            const float rposf = P->cmp ? (sf + hf) : hf;
            float rf = 0.0f;
            if (P->rny > 1 && P->rdy != 0.0f) rf = (rposf - P->ry0) / P->rdy;
            const int iht = (P->rny > 1 && P->rdy != 0.0f) ? (int)floorf(rf) : 0;
            double *dst = data + ((long)is * P->nh + ih) * nt;
            for (int it = 0; it < nt; it++) { trace[it] = RF(0); dst[it] = 0.0; }
            R trace_w = RF(1);
            if (P->aperture_trace != -1) {
                const R ad = R_FABS((R)(iht - ist));
                if (ad >= (R)P->aperture_trace) continue;
                if (P->aperture_trace_taper > 0) {
                    const R tb = MAXV(RF(0), (R)(P->aperture_trace - P->aperture_trace_taper));
                    if (ad > tb) {
                        const R den = (R)P->aperture_trace - tb;
                        if (den > RF(0)) trace_w = RF(0.5) * (RF(1) + R_COS(R_PI * ((ad - tb) / den)));
                    }
                }
            }
            int ig_offset = 0;
            if (P->cig && !P->cig_is_angle) {
                const float u = (hf - P->g0) / P->dg + 0.5f;
                ig_offset = (ng <= 0 || P->dg <= 0.0f || !isfinite(hf)) ? -1 : (int)floorf(u);
                if (ig_offset >= ng) ig_offset = -1;
                if (ig_offset < 0) continue;
            }
            table_at(0, P, rtab, rder, rposf, rpos, P->ry0, P->rdy, P->rny, RT, RTx, s0, s1, m0, m1);
            if (angle) {
                if (P->use_input_grad) {
                    interp_volume_linear(rgx, rgx_v, P->rny, nzx, rposf, rpos, P->ry0, P->rdy, s0, s1);
                    interp_volume_linear(rgz, rgz_v, P->rny, nzx, rposf, rpos, P->ry0, P->rdy, s0, s1);
                }
                leg_gradient(P, RT, rgx, rgz, grx, grz, t1, t2);
            }
            for (long i = 0; i < nzx; i++) {
                const int iz = (int)(i % nz);
                const int ix = (int)((i - iz) / nz);
                const R zdist = MAXV(R_FABS((R)iz * dz), MAXV(RF(1.0e-12), RF(1.0e-6) * R_FABS(dz)));
                const R ximg = x0 + (R)ix * dxg;
                const R dsx = R_FABS(s - ximg);
                const R drx = R_FABS(rpos - ximg);
                const R as_deg = R_ATAN(dsx / zdist) * RF(180.0) / R_PI;
                const R ar_deg = R_ATAN(drx / zdist) * RF(180.0) / R_PI;
                const R ws = MAXV(aperture_leg_weight(as_deg, RF(P->aper), RF(P->aperture_taper)),
                                  aperture_floor_weight(dsx, RF(P->aperture_rmin), RF(P->aperture_rtaper)));
                const R wr = MAXV(aperture_leg_weight(ar_deg, RF(P->aper), RF(P->aperture_taper)),
                                  aperture_floor_weight(drx, RF(P->aperture_rmin), RF(P->aperture_rtaper)));
                const R apw = ws * wr;
                if (apw <= RF(0)) continue;
                const R ti = ST[i] + RT[i] + tau;
                const R tx = MAXV(R_FABS(STx[i] * ds), R_FABS(RTx[i] * dh));
                if (angle) {
                    const R ang = angle_from_grad(gsx[i], gsz[i], grx[i], grz[i], P->half_angle);
                    const R aw = angle_taper_weight(ang, RF(P->angle_taper_start), RF(P->angle_taper_end)) *
                                 depth_mute_weight(ang, iz, nz, RF(P->oazmin), RF(P->oazmax), RF(P->oaztaper)) *
                                 trace_w * apw;
                    if (aw <= RF(0)) continue;
                    if (P->angle_interp) {
                        int ig0 = -1, ig1 = -1;
                        R w0 = RF(0), w1 = RF(0);
                        if (!linear_bins(ang, g0, dg, ng, &ig0, &ig1, &w0, &w1)) continue;
                        kirmig_spray(ti, tx * aal, aw * w0 * (R)image[(long)ig0 * nzx + i], trace, nt, dt, t0);
                        if (ig1 != ig0 && w1 > RF(0))
                            kirmig_spray(ti, tx * aal, aw * w1 * (R)image[(long)ig1 * nzx + i], trace, nt, dt, t0);
                    } else {
                        const int ig = nearest_bin(ang, g0, dg, ng);
                        if (ig < 0) continue;
                        kirmig_spray(ti, tx * aal, aw * (R)image[(long)ig * nzx + i], trace, nt, dt, t0);
                    }
                } else {
                    const int ig = P->cig ? ig_offset : 0;
                    kirmig_spray(ti, tx * aal, trace_w * apw * (R)image[(long)ig * nzx + i], trace, nt, dt, t0);
                }
            }
            doubint(nt, trace);
            for (int it = 0; it < nt; it++) dst[it] = (double)trace[it];
        }
    }
    free(buf);
    free(trace);
    return 0;
}
