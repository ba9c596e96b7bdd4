// sm_100a kernels of the adjoint angle-domain Kirchhoff summation.
//
//   K1 k_prelude_cta  per-trace direct mute + doubint (FP64 running sums) +
//                     optional diff2, written as {D[i], D[i+1]-D[i]} pairs so
//                     a linear-interpolated pick is one 16-byte load and one
//                     fused multiply-add.
//   K2 k_leg_*        per source/receiver position: table interpolation along
//                     the position axis, traveltime gradient, triangle
//                     smoothing and the aperture leg weight ("leg fields").
//   K3 k_sum          the summation: one CTA owns an image tile, keeps its
//                     angle bins in shared memory, and loops over every trace.
//
// Reference: src/kirchmig2d_cig.cpp (the adj=1 loop :979-1339),
// SERECKIRCH/src/kirmig.cpp (doubint :8-24, kirmig_pick :34-58) and
// SERECKIRCH/src/tinterpsr.cpp (:37-188).
#include <math.h>
#include <stdio.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include "kcig_aperture.h"
#include "kcig_common.h"
#include "kcig_tc.h"

namespace kcig {


// =============================================================== K1 prelude ==
// doubint of one trace per warp (the building block kcig_doubint_device and
// the forward modelling's final integration): the trace is staged in shared
// memory as double and integrated causally and anticausally (kirmig.cpp:8-24)
// with every running sum in FP64: each lane scans a contiguous chunk and a
// warp scan of the chunk totals links the chunks.  FP64 sums keep the later
// second differences (the pick) accurate, which an FP32 running sum of a long
// trace does not.  The migration's prelude is k_prelude_cta further down.
__device__ __forceinline__ double warp_excl_scan(double v, double *total)
{
    const int lane = threadIdx.x & 31;
    double x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        double y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    *total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
}

__device__ __forceinline__ double warp_excl_suffix_scan(double v, double *total)
{
    const int lane = threadIdx.x & 31;
    double x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        double y = __shfl_down_sync(0xffffffffu, x, o);
        if (lane + o < 32) x += y;
    }
    *total = __shfl_sync(0xffffffffu, x, 0);
    return x - v;
}

__device__ void doubint_warp(double *s, int nt)
{
    const int lane = threadIdx.x & 31;
    const int chunk = (nt + 31) / 32;
    const int a = min(nt, lane * chunk), b = min(nt, a + chunk);
    double tot, loc = 0.0;
    for (int i = a; i < b; i++) loc += s[i];
    double off = warp_excl_scan(loc, &tot);
    for (int i = a; i < b; i++) { off += s[i]; s[i] = off; }
    __syncwarp();
    loc = 0.0;
    for (int i = a; i < b; i++) loc += s[i];
    off = warp_excl_suffix_scan(loc, &tot);
    for (int i = b - 1; i >= a; i--) { off += s[i]; s[i] = off; }
    __syncwarp();
}

__device__ void diff2_warp(double *s, int nt, double dt)
{
    // kirchmig2d_cig.cpp:381-394: central difference, one-sided at the ends.
    // Each lane rewrites its chunk in place, carrying the original values of
    // the neighbours it still needs; chunk-boundary neighbours are read first.
    const int lane = threadIdx.x & 31;
    if (nt < 2) return;
    const int chunk = (nt + 31) / 32;
    const int a = min(nt, lane * chunk), b = min(nt, a + chunk);
    double prev = (a > 0 && a < nt) ? s[a - 1] : 0.0;
    const double nextv = (b < nt && a < b) ? s[b] : 0.0;
    double cur = (a < b) ? s[a] : 0.0;
    __syncwarp();
    for (int i = a; i < b; i++) {
        const double nx = (i + 1 < b) ? s[i + 1] : nextv;
        double v;
        if (i == 0) v = (nx - cur) / dt;
        else if (i == nt - 1) v = (cur - prev) / dt;
        else v = (nx - prev) / (2.0 * dt);
        s[i] = v;
        prev = cur;
        cur = nx;
    }
    __syncwarp();
}

template <typename IN, typename OUT>
__global__ void __launch_bounds__(64) k_doubint_plain(const IN *in, OUT *out, int ntr, int nt,
                                                      int isdiff, double dt)
{
    extern __shared__ double smem_d[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tr = blockIdx.x * (blockDim.x >> 5) + warp;
    if (tr >= ntr) return;
    double *s = smem_d + (size_t)warp * nt;
    for (int i = lane; i < nt; i += 32) s[i] = (double)in[(size_t)tr * nt + i];
    __syncwarp();
    doubint_warp(s, nt);
    if (isdiff == 1) diff2_warp(s, nt, dt);
    for (int i = lane; i < nt; i += 32) out[(size_t)tr * nt + i] = (OUT)s[i];
}

int set_dyn_smem(const void *fn, int bytes, int carveout)
{
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, int> done;
    int dev = 0;
    KCIG_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    int &have = done[std::make_pair(dev, fn)];
    if (bytes <= have) return KCIG_OK;
    KCIG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    if (carveout >= 0) KCIG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, carveout));
    have = bytes;
    return KCIG_OK;
}

static int prelude_block(int nt, int *warps)
{
    const size_t per = (size_t)nt * sizeof(double);
    if (per * 2 <= 96 * 1024) { *warps = 2; return 0; }
    if (per <= 200 * 1024) { *warps = 1; return 0; }
    return -1;
}

// K1 with one CTA of PW warps per trace.  The trace is staged in shared
// memory as FP64 with coalesced loads (the mute applied on the way).  Each
// warp owns a contiguous segment of 32-sample rows and scans it row by row
// with a 32-wide shuffle scan, carrying the running total from row to row;
// the segments' totals are scanned across the warps first (in a fixed order),
// so every running sum is FP64 and every shared-memory access is one
// consecutive row (no bank conflicts).  Causal sum, then anticausal sum
// (kirmig.cpp:8-24), then the optional centred difference (:381-394); the
// {D[i], D[i+1]-D[i]} pairs leave with coalesced 16-byte stores.
__device__ __forceinline__ double warp_incl_scan(double v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
    }
    return v;
}

__device__ __forceinline__ double warp_incl_suffix_scan(double v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_down_sync(0xffffffffu, v, o);
        if (lane + o < 32) v += y;
    }
    return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

constexpr int kPreludeWarps = 4;

__global__ void __launch_bounds__(32 * kPreludeWarps) k_prelude_cta(PreludeArgs a)
{
    constexpr int PW = kPreludeWarps, PT = 32 * PW;
    extern __shared__ double pd[];  // [nt] (+ [nt] of the differenced trace with diff=1)
    __shared__ double wtot[PW], woff[PW];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
    const int tr = blockIdx.x;
    const int k = tr / a.nhc, rr = tr % a.nhc;
    const float *x = a.data + ((size_t)(a.shot0 + k) * a.nh + (a.rcv0 + rr)) * a.nt;
    int nt = a.nt;
    if (a.toff) {  // ragged shots: own samples, own length (padding traces are never read)
        const long long off = a.toff[tr];
        if (off < 0) return;
        x = a.data + off;
        nt = a.tnt[tr];
    }
    double boundary = 0.0;
    const bool mute = a.mute_sx != nullptr;
    if (mute) {
        const double off = a.slope * fabs(a.mute_rx[tr] - a.mute_sx[tr]);
        boundary = a.invert ? a.intercept - off : a.intercept + off;
    }
    for (int i = tid; i < nt; i += PT) {
        double v = (double)__ldg(x + i);
        if (mute) {
            const double t = a.t0 + (double)i * a.dt;
            double w = 0.0;
            if (t >= boundary + a.taper) w = 1.0;
            else if (t > boundary) w = 0.5 * (1.0 - cospi((t - boundary) / a.taper));
            v *= w;
        }
        pd[i] = v;
    }
    __syncthreads();
    const int rows = (nt + 31) >> 5, R = (rows + PW - 1) / PW;
    const int i0 = min(nt, warp * R * 32), i1 = min(nt, (warp + 1) * R * 32);

    // causal running sum
    double sv = 0.0;
    for (int i = i0 + lane; i < i1; i += 32) sv += pd[i];
    sv = warp_sum(sv);
    if (lane == 0) wtot[warp] = sv;
    __syncthreads();
    if (tid == 0) {
        double acc = 0.0;
        for (int w = 0; w < PW; w++) {
            woff[w] = acc;
            acc += wtot[w];
        }
    }
    __syncthreads();
    double carry = woff[warp];
    for (int b = i0; b < i1; b += 32) {
        const int i = b + lane;
        const double v = warp_incl_scan(i < i1 ? pd[i] : 0.0) + carry;
        if (i < i1) pd[i] = v;
        carry = __shfl_sync(0xffffffffu, v, 31);
    }
    __syncthreads();

    // anticausal running sum of that: D[i] = sum over j >= i
    sv = 0.0;
    for (int i = i0 + lane; i < i1; i += 32) sv += pd[i];
    sv = warp_sum(sv);
    if (lane == 0) wtot[warp] = sv;
    __syncthreads();
    if (tid == 0) {
        double acc = 0.0;
        for (int w = PW - 1; w >= 0; w--) {
            woff[w] = acc;
            acc += wtot[w];
        }
    }
    __syncthreads();
    carry = woff[warp];
    if (i1 > i0) {
        for (int b = i0 + ((i1 - 1 - i0) & ~31); b >= i0; b -= 32) {
            const int i = b + lane;
            const double v = warp_incl_suffix_scan(i < i1 ? pd[i] : 0.0) + carry;
            if (i < i1) pd[i] = v;
            carry = __shfl_sync(0xffffffffu, v, 0);
        }
    }
    __syncthreads();

    const double *D = pd;
    if (a.isdiff == 1 && nt >= 2) {
        // central first derivative, one-sided at the ends, into the second half
        double *q = pd + nt;
        for (int i = tid; i < nt; i += PT) {
            double v;
            if (i == 0) v = (pd[1] - pd[0]) / a.dt;
            else if (i == nt - 1) v = (pd[nt - 1] - pd[nt - 2]) / a.dt;
            else v = (pd[i + 1] - pd[i - 1]) / (2.0 * a.dt);
            q[i] = v;
        }
        __syncthreads();
        D = q;
    }
    double2 *out = a.D + (size_t)tr * a.nt;
    for (int i = tid; i < nt; i += PT) {
        double2 e;
        e.x = D[i];
        e.y = (i + 1 < nt) ? D[i + 1] - D[i] : 0.0;
        out[i] = e;
    }
}

int launch_prelude(const PreludeArgs &a, cudaStream_t st)
{
    if (a.ntr <= 0) return KCIG_OK;
    const size_t sm = (size_t)(a.isdiff == 1 ? 2 : 1) * a.nt * sizeof(double);
    if (sm > 200 * 1024)
        return set_error(KCIG_ERR_UNSUPPORTED, "nt=%d exceeds the on-chip trace limit (%d, %d with diff=1)", a.nt,
                         25600, 12800);
    KCIG_TRY(set_dyn_smem((const void *)k_prelude_cta, (int)sm));
    k_prelude_cta<<<a.ntr, 32 * kPreludeWarps, sm, st>>>(a);
    KCIG_CUDA(cudaGetLastError());
    return KCIG_OK;
}

int launch_doubint_f32(const double *in, float *out, int ntr, int nt, cudaStream_t st)
{
    if (ntr <= 0) return KCIG_OK;
    int warps;
    if (prelude_block(nt, &warps))
        return set_error(KCIG_ERR_UNSUPPORTED, "nt=%d exceeds the on-chip trace limit (25600)", nt);
    const size_t sm = (size_t)warps * nt * sizeof(double);
    KCIG_TRY(set_dyn_smem((const void *)k_doubint_plain<double, float>, (int)sm));
    k_doubint_plain<double, float><<<(ntr + warps - 1) / warps, 32 * warps, sm, st>>>(in, out, ntr, nt, 0, 1.0);
    KCIG_CUDA(cudaGetLastError());
    return KCIG_OK;
}

int launch_doubint_plain(const float *in, double *out, int ntr, int nt, int isdiff, double dt,
                         cudaStream_t st)
{
    if (ntr <= 0) return KCIG_OK;
    int warps;
    if (prelude_block(nt, &warps))
        return set_error(KCIG_ERR_UNSUPPORTED, "nt=%d exceeds the on-chip trace limit (25600)", nt);
    const size_t sm = (size_t)warps * nt * sizeof(double);
    KCIG_TRY(set_dyn_smem((const void *)k_doubint_plain<float, double>, (int)sm));
    k_doubint_plain<float, double><<<(ntr + warps - 1) / warps, 32 * warps, sm, st>>>(in, out, ntr, nt, isdiff, dt);
    KCIG_CUDA(cudaGetLastError());
    return KCIG_OK;
}

// ============================================================ K2 leg fields ==
// Table interpolation (tinterpsr.cpp:37-188) in double, aperture weight, and
// the input-gradient interpolation (kirchmig2d_cig.cpp:294-322).
__global__ void k_leg_interp(FieldArgs a, LegFields out, double *work)
{
    const int nzx = a.nz * a.nx;
    const int j = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nzx) return;
    const LegInterp L = a.legs[j];
    const size_t base = (size_t)j * nzx;
    double T, Tx;
    if (L.i1 < 0) {
        T = a.tab[(size_t)L.i0 * nzx + i];
        Tx = a.der[(size_t)L.i0 * nzx + i];
    } else if (L.type == 'p') {
        // tinterp_partial / dinterp_partial (tinterpsr.cpp:72-140).  The
        // reference's right-slice derivative terms index below the slice for
        // the first k2 lateral columns (tinterpsr.cpp:119-124), and with one
        // lateral column a one-sided term indexes past it; such an index is
        // clamped to the first/last column at the same depth, so every read
        // stays inside the table.
        const float *p0 = a.tab + (size_t)L.i0 * nzx, *p1 = a.tab + (size_t)L.i1 * nzx;
        const int n1 = a.nz, k1 = L.k1, k2 = L.k2, nn = nzx;
        const double t = L.t, dd = a.dx, dxp = L.dxp;
        auto cl = [&](int j) -> int { return j < 0 ? i % n1 : (j >= nn ? nn - n1 + i % n1 : j); };
        auto P1 = [&](int j) -> double { return (double)p1[cl(j)]; };
        auto P0 = [&](int j) -> double { return (double)p0[cl(j)]; };
        if (i - k1 * n1 >= 0 && i + k2 * n1 < nn) {
            T = (1.0 - t) * p0[i - k1 * n1] + t * p1[i + k2 * n1];
            double dv = (-(double)p0[i - k1 * n1] + p1[i + k2 * n1]) / dxp;
            if (i - (k1 + 1) * n1 >= 0 && i - (k1 - 1) * n1 < nn)
                dv -= (1.0 - t) * (-(double)p0[i - (k1 + 1) * n1] + p0[i - (k1 - 1) * n1]) / (2.0 * dd);
            else if (i - (k1 + 1) * n1 < 0)
                dv -= (1.0 - t) * (-(double)p0[i - k1 * n1] + P0(i - (k1 - 1) * n1)) / dd;
            else
                dv -= (1.0 - t) * (-(double)p0[i - (k1 + 1) * n1] + p0[i - k1 * n1]) / dd;
            if (i - (k2 + 1) * n1 >= 0 && i - (k2 - 1) * n1 < nn)
                dv -= t * (-(double)p1[i - (k2 + 1) * n1] + p1[i - (k2 - 1) * n1]) / (2.0 * dd);
            else if (i - (k2 + 1) * n1 < 0)
                dv -= t * (-P1(i - k2 * n1) + P1(i - (k2 - 1) * n1)) / dd;
            else
                dv -= t * (-(double)p1[i - (k2 + 1) * n1] + p1[i - k2 * n1]) / dd;
            Tx = dv;
        } else {
            T = (1.0 - t) * p0[i] + t * p1[i];
            Tx = (-(double)p0[i] + p1[i]) / dxp;
        }
    } else {
        const double p0 = a.tab[(size_t)L.i0 * nzx + i], p1 = a.tab[(size_t)L.i1 * nzx + i];
        const double m0 = a.der[(size_t)L.i0 * nzx + i], m1 = a.der[(size_t)L.i1 * nzx + i];
        T = L.c[0] * p0 + L.c[1] * m0 + L.c[2] * p1 + L.c[3] * m1;
        Tx = L.e[0] * p0 + L.e[1] * m0 + L.e[2] * p1 + L.e[3] * m1;
    }
    const int iz = i % a.nz, ix = i / a.nz;
    double w;
    if (a.cone) {
        // kirchmig2d.cpp:455-488 in its float arithmetic: the pair is dropped
        // when the image point lies beyond the cone of the left leg on its
        // left or of the right leg on its right.  w = 1 (left-side test
        // passes) + 2 (right-side test passes); the pair's kernel picks the
        // left leg's bit 1 and the right leg's bit 2.
        const float zi = __fmul_rn((float)iz, a.dz), xd = __fmul_rn((float)ix, a.dx);
        const float lnum = __fsub_rn(__fsub_rn(L.posf, a.x0), xd);   // p - x0 - ix*dx
        const float rnum = L.cexact ? __fsub_rn(__fsub_rn(__fadd_rn(a.x0, xd), L.cs), L.ch)  // x0 + ix*dx - s - h
                                    : __fsub_rn(__fadd_rn(a.x0, xd), L.posf);              // x0 + ix*dx - p
        const bool lcut = (double)atanf(__fdiv_rn(lnum, zi)) * 180. / M_PI > (double)a.aper;
        const bool rcut = (double)atanf(__fdiv_rn(rnum, zi)) * 180. / M_PI > (double)a.aper;
        w = (lcut ? 0.0 : 1.0) + (rcut ? 0.0 : 2.0);
    } else {
        w = leg_aperture_weight(L.pos, iz, ix, a.dz, a.x0, a.dx, a.aper, a.aper_taper, a.rmin, a.rtaper);
    }
    out.TP[base + i] = make_double2(T, 0.0);
    // reference: stablex[i]*ds, an FP32 product of the FP32 table derivative
    out.XW[base + i] = make_float2((float)Tx * L.scale, (float)w);
    if (a.angle && a.use_grad) {
        double gx, gz;
        const size_t s0 = (size_t)L.gi0 * nzx + i;
        if (L.gw == 0.0) {
            gx = a.gxv[s0];
            gz = a.gzv[s0];
        } else {
            const size_t s1 = (size_t)L.gi1 * nzx + i;
            gx = (1.0 - L.gw) * a.gxv[s0] + L.gw * a.gxv[s1];
            gz = (1.0 - L.gw) * a.gzv[s0] + L.gw * a.gzv[s1];
        }
        work[(size_t)j * 4 * nzx + i] = gx;
        work[(size_t)j * 4 * nzx + nzx + i] = gz;
    }
}

// compute_grad_plane (kirchmig2d_cig.cpp:130-152, :424-435) in double.
__global__ void k_leg_fd(FieldArgs a, LegFields out, double *work)
{
    const int nzx = a.nz * a.nx;
    const int j = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nzx) return;
    const double2 *T = out.TP + (size_t)j * nzx;
    const int iz = i % a.nz, ix = i / a.nz;
    const int r = a.radius < 1 ? 1 : a.radius;
    double gx = 0.0, gz = 0.0;
    if (a.nx > 1 && a.dx != 0.0f) {
        const int il = max(0, ix - r), ir = min(a.nx - 1, ix + r);
        if (ir != il) gx = (T[(size_t)ir * a.nz + iz].x - T[(size_t)il * a.nz + iz].x) / ((double)(ir - il) * a.dx);
    }
    if (a.nz > 1 && a.dz != 0.0f) {
        const int it = max(0, iz - r), ib = min(a.nz - 1, iz + r);
        if (ib != it) gz = (T[(size_t)ix * a.nz + ib].x - T[(size_t)ix * a.nz + it].x) / ((double)(ib - it) * a.dz);
    }
    work[(size_t)j * 4 * nzx + i] = gx;
    work[(size_t)j * 4 * nzx + nzx + i] = gz;
}

// One box average (kirchmig2d_cig.cpp:438-466) along z (axis=0) or x (axis=1)
// of planes pin -> pout of every position (component c: planes c and c+2).
__global__ void k_box(int nz, int nx, int r, int axis, int pin, int pout, double *work)
{
    const int nzx = nz * nx;
    const int j = blockIdx.y;
    const int c = blockIdx.z;  // component
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nzx) return;
    const double *in = work + ((size_t)j * 4 + pin + c) * nzx;
    double *o = work + ((size_t)j * 4 + pout + c) * nzx;
    const int iz = i % nz, ix = i / nz;
    double s = 0.0;
    int a0, b0;
    if (axis == 0) {
        a0 = max(0, iz - r); b0 = min(nz - 1, iz + r);
        for (int k = a0; k <= b0; k++) s += in[(size_t)ix * nz + k];
    } else {
        a0 = max(0, ix - r); b0 = min(nx - 1, ix + r);
        for (int k = a0; k <= b0; k++) s += in[(size_t)k * nz + iz];
    }
    o[i] = s / (double)(b0 - a0 + 1);
}

// Direction of the stabilised gradient.  scattering_angle_deg_from_grad
// (:171-187) returns NaN when either gradient vanishes; phi = NaN carries that.
__global__ void k_leg_pack(FieldArgs a, LegFields out, const double *work)
{
    const int nzx = a.nz * a.nx;
    const int j = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nzx) return;
    const double gx = work[(size_t)j * 4 * nzx + i];
    const double gz = work[(size_t)j * 4 * nzx + nzx + i];
    double2 *tp = out.TP + (size_t)j * nzx + i;
    const double phi = (sqrt(gx * gx + gz * gz) <= 1.0e-12) ? __longlong_as_double(0x7ff8000000000000ll)
                                                             : atan2(gz, gx);
    tp->y = phi;
}

// compute_grad_plane + smooth_grad_component x2 + the direction, fused for
// one kGradTile x kGradTile block of image points of one position.  The
// interpolated traveltime is staged in shared memory with a halo of r + 2s
// samples; the centred differences (radius r), the four box averages (radius
// s; z, x, z, x as :438-492, both components per pass) and the arc tangent
// all run there in FP64, and only the direction goes back to HBM.  Every
// window is clamped to the GRID, as the reference's full-plane passes are,
// so a tile reproduces them; divisions by a window's length are
// multiplications by its reciprocal (one rounding apart).
constexpr int kGradTile = 32;

// One box average along z (AXIS 0) or x (AXIS 1) of the local cells
// [z0,z1) x [x0,x1), already clipped to the grid; the window is clamped to
// the grid's local range [glo, ghi) of that axis.  rcp[k] = 1 / (k + 1).
// Every cell of [z0,z1) x [x0,x1), walked by all threads of the block as one
// flat range: consecutive threads take consecutive depths (rows stay
// coalesced in shared memory) and no lane idles at the end of a row, as it
// would with a row per 32 lanes on a halo tile 44 wide.  The column of flat
// index q is q / nzr, taken exactly as a float product with the reciprocal:
// (q + 0.5) / nzr lies at least 0.5 / nzr from an integer, far above the
// float error for the tile sizes here (q < 2^20, nzr <= 1024).
template <class F>
__device__ __forceinline__ void for_cells(int z0, int z1, int x0, int x1, F f)
{
    const int nzr = z1 - z0, nxr = x1 - x0;
    if (nzr <= 0 || nxr <= 0) return;
    const int n = nzr * nxr;
    const float inv = 1.0f / (float)nzr;
    const int nthr = blockDim.x * blockDim.y;
    for (int q = threadIdx.y * blockDim.x + threadIdx.x; q < n; q += nthr) {
        const int cx = (int)(((float)q + 0.5f) * inv);
        f(z0 + (q - cx * nzr), x0 + cx);
    }
}

template <int AXIS>
__device__ __forceinline__ void box_tile(const double *in0, double *out0, const double *in1, double *out1, int W,
                                         int s, int z0, int z1, int x0, int x1, int glo, int ghi, const double *rcp)
{
    for_cells(z0, z1, x0, x1, [&](int lz, int lx) {
        const int c = AXIS == 0 ? lz : lx;
        const int a0 = max(c - s, glo), b0 = min(c + s, ghi - 1);
        const int step = AXIS == 0 ? 1 : W;
        const int base = AXIS == 0 ? lx * W + a0 : a0 * W + lz;
        double s0 = 0.0, s1 = 0.0;
        for (int k = 0; k <= b0 - a0; k++) {
            s0 += in0[base + k * step];
            s1 += in1[base + k * step];
        }
        out0[lx * W + lz] = s0 * rcp[b0 - a0];
        out1[lx * W + lz] = s1 * rcp[b0 - a0];
    });
}

// The same box pass for radius 2 (the default angle_smooth) on pairs of
// cells along z: a thread takes cells c, c+1 (c even, so that with W even a
// pair is one aligned 16-byte word) and loads each value of the two windows
// once, as 16-byte words -- three per component along z, five along x --
// instead of ten 8-byte loads.  The sums run in the generic pass's order
// (0.0, then the window from its first cell), so the results are the same
// bit for bit.  Pairs with a cell outside [z0, z1) or a window clamped to the
// grid take the generic per-cell code.
template <int AXIS>
__device__ __forceinline__ void box_tile_s2(const double *in0, double *out0, const double *in1, double *out1, int W,
                                            int z0, int z1, int x0, int x1, int glo, int ghi, const double *rcp)
{
    constexpr int S = 2;
    const int pz0 = z0 & ~1;
    const double rc = rcp[2 * S];
    auto cell = [&](int lz, int lx) {
        const int c = AXIS == 0 ? lz : lx;
        const int a0 = max(c - S, glo), b0 = min(c + S, ghi - 1);
        const int step = AXIS == 0 ? 1 : W;
        const int base = AXIS == 0 ? lx * W + a0 : a0 * W + lz;
        double s0 = 0.0, s1 = 0.0;
        for (int k = 0; k <= b0 - a0; k++) {
            s0 += in0[base + k * step];
            s1 += in1[base + k * step];
        }
        out0[lx * W + lz] = s0 * rcp[b0 - a0];
        out1[lx * W + lz] = s1 * rcp[b0 - a0];
    };
    for_cells(0, (z1 - pz0 + 1) >> 1, x0, x1, [&](int q, int lx) {
        const int c = pz0 + 2 * q;
        const bool both = c >= z0 && c + 1 < z1;
        const bool inner = AXIS == 0 ? (c - S >= glo && c + 1 + S <= ghi - 1) : (lx - S >= glo && lx + S <= ghi - 1);
        if (!(both && inner)) {
            if (c >= z0 && c < z1) cell(c, lx);
            if (c + 1 >= z0 && c + 1 < z1) cell(c + 1, lx);
            return;
        }
        double2 r0, r1;
        if (AXIS == 0) {
            // values c-2 .. c+3 of the column as three aligned words
            const double2 *p0 = reinterpret_cast<const double2 *>(in0 + lx * W + c - S);
            const double2 *p1 = reinterpret_cast<const double2 *>(in1 + lx * W + c - S);
            const double2 u0 = p0[0], u1 = p0[1], u2 = p0[2], v0 = p1[0], v1 = p1[1], v2 = p1[2];
            r0.x = ((((0.0 + u0.x) + u0.y) + u1.x) + u1.y) + u2.x;
            r0.y = ((((0.0 + u0.y) + u1.x) + u1.y) + u2.x) + u2.y;
            r1.x = ((((0.0 + v0.x) + v0.y) + v1.x) + v1.y) + v2.x;
            r1.y = ((((0.0 + v0.y) + v1.x) + v1.y) + v2.x) + v2.y;
        } else {
            // the pair's word in columns lx-2 .. lx+2
            double2 s0 = make_double2(0.0, 0.0), s1 = make_double2(0.0, 0.0);
#pragma unroll
            for (int k = -S; k <= S; k++) {
                const double2 u = *reinterpret_cast<const double2 *>(in0 + (lx + k) * W + c);
                const double2 v = *reinterpret_cast<const double2 *>(in1 + (lx + k) * W + c);
                s0.x += u.x;
                s0.y += u.y;
                s1.x += v.x;
                s1.y += v.y;
            }
            r0 = s0;
            r1 = s1;
        }
        *reinterpret_cast<double2 *>(out0 + lx * W + c) = make_double2(r0.x * rc, r0.y * rc);
        *reinterpret_cast<double2 *>(out1 + lx * W + c) = make_double2(r1.x * rc, r1.y * rc);
    });
}

template <int AXIS>
__device__ __forceinline__ void box_pass(const double *in0, double *out0, const double *in1, double *out1, int W,
                                         int s, int z0, int z1, int x0, int x1, int glo, int ghi, const double *rcp)
{
    if (s == 2)
        box_tile_s2<AXIS>(in0, out0, in1, out1, W, z0, z1, x0, x1, glo, ghi, rcp);
    else
        box_tile<AXIS>(in0, out0, in1, out1, W, s, z0, z1, x0, x1, glo, ghi, rcp);
}

// Centred differences of the staged traveltimes P0 on the cells
// [max(r, zlo), min(W - r, zhi)) x [max(r, xlo), min(W - r, xhi)): gx -> P1,
// gz -> P2, each window clamped to the grid's local range (compute_grad_plane,
// :130-152).  For r = 2 (the default angle_grad_radius) cells go in pairs
// along z as in box_tile_s2 (the same arithmetic, 16-byte words).
__device__ __forceinline__ void centred_diffs(const double *P0, double *P1, double *P2, int W, int r, int zlo,
                                              int zhi, int xlo, int xhi, bool dox, bool doz, const double *rcpx,
                                              const double *rcpz)
{
    auto cell = [&](int lz, int lx) {
        double vx = 0.0, vz = 0.0;
        if (dox) {
            const int il = max(xlo, lx - r), ir = min(xhi - 1, lx + r);
            if (ir != il) vx = (P0[ir * W + lz] - P0[il * W + lz]) * rcpx[ir - il];
        }
        if (doz) {
            const int it = max(zlo, lz - r), ib = min(zhi - 1, lz + r);
            if (ib != it) vz = (P0[lx * W + ib] - P0[lx * W + it]) * rcpz[ib - it];
        }
        P1[lx * W + lz] = vx;
        P2[lx * W + lz] = vz;
    };
    const int z0 = max(r, zlo), z1 = min(W - r, zhi), x0 = max(r, xlo), x1 = min(W - r, xhi);
    if (r != 2) {
        for_cells(z0, z1, x0, x1, cell);
        return;
    }
    const int pz0 = z0 & ~1;
    const double cx = rcpx[4], cz = rcpz[4];
    for_cells(0, (z1 - pz0 + 1) >> 1, x0, x1, [&](int q, int lx) {
        const int c = pz0 + 2 * q;
        const bool both = c >= z0 && c + 1 < z1;
        const bool inner = lx - 2 >= xlo && lx + 2 <= xhi - 1 && c - 2 >= zlo && c + 3 <= zhi - 1;
        if (!(both && inner)) {
            if (c >= z0 && c < z1) cell(c, lx);
            if (c + 1 >= z0 && c + 1 < z1) cell(c + 1, lx);
            return;
        }
        double2 gx = make_double2(0.0, 0.0), gz = make_double2(0.0, 0.0);
        if (dox) {
            const double2 l = *reinterpret_cast<const double2 *>(P0 + (lx - 2) * W + c);
            const double2 h = *reinterpret_cast<const double2 *>(P0 + (lx + 2) * W + c);
            gx = make_double2((h.x - l.x) * cx, (h.y - l.y) * cx);
        }
        if (doz) {
            const double2 t = *reinterpret_cast<const double2 *>(P0 + lx * W + c - 2);
            const double2 b = *reinterpret_cast<const double2 *>(P0 + lx * W + c + 2);
            gz = make_double2((b.x - t.x) * cz, (b.y - t.y) * cz);
        }
        *reinterpret_cast<double2 *>(P1 + lx * W + c) = gx;
        *reinterpret_cast<double2 *>(P2 + lx * W + c) = gz;
    });
}

__global__ void __launch_bounds__(256) k_leg_grad_fused(FieldArgs a, LegFields out)
{
    extern __shared__ double gsm[];
    const int nz = a.nz, nx = a.nx;
    const size_t nzx = (size_t)nz * nx;
    const int r = a.radius < 1 ? 1 : a.radius, s = a.smooth;
    const int H = r + 2 * s, W = kGradTile + 2 * H;
    const int tiles_z = (nz + kGradTile - 1) / kGradTile;
    const int gz0 = (int)(blockIdx.x % tiles_z) * kGradTile - H, gx0 = (int)(blockIdx.x / tiles_z) * kGradTile - H;
    // the grid in local coordinates
    const int zlo = max(0, -gz0), zhi = min(W, nz - gz0), xlo = max(0, -gx0), xhi = min(W, nx - gx0);
    double *P0 = gsm, *P1 = P0 + W * W, *P2 = P1 + W * W, *P3 = P2 + W * W;
    double *rcpb = P3 + W * W, *rcpx = rcpb + 2 * s + 1, *rcpz = rcpx + 2 * r + 1;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * blockDim.y;
    const double2 *TP = out.TP + (size_t)blockIdx.y * nzx;
    double2 *TPo = out.TP + (size_t)blockIdx.y * nzx;

    // the traveltimes of the tile and its halo, all loads in flight at once
    for_cells(zlo, zhi, xlo, xhi, [&](int lz, int lx) {
        const unsigned dst = (unsigned)__cvta_generic_to_shared(P0 + lx * W + lz);
        const double2 *src = TP + (size_t)(gx0 + lx) * nz + (gz0 + lz);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
    });
    for (int k = tid; k <= 2 * s; k += nthr) rcpb[k] = 1.0 / (double)(k + 1);
    for (int k = tid; k <= 2 * r; k += nthr) {
        rcpx[k] = k ? 1.0 / ((double)k * a.dx) : 0.0;
        rcpz[k] = k ? 1.0 / ((double)k * a.dz) : 0.0;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();

    // centred differences on [r, W-r)^2: gx -> P1, gz -> P2
    const bool dox = nx > 1 && a.dx != 0.0f, doz = nz > 1 && a.dz != 0.0f;
    centred_diffs(P0, P1, P2, W, r, zlo, zhi, xlo, xhi, dox, doz, rcpx, rcpz);
    __syncthreads();

    if (s > 0) {
        // each pass narrows the cells it must produce by s along its own
        // axis; the cells the next pass reads are always inside
        const int i1 = r + s, i2 = H;
        box_pass<0>(P1, P0, P2, P3, W, s, max(i1, zlo), min(W - i1, zhi), max(r, xlo), min(W - r, xhi), zlo, zhi,
                    rcpb);
        __syncthreads();
        box_pass<1>(P0, P1, P3, P2, W, s, max(i1, zlo), min(W - i1, zhi), max(i1, xlo), min(W - i1, xhi), xlo, xhi,
                    rcpb);
        __syncthreads();
        box_pass<0>(P1, P0, P2, P3, W, s, max(i2, zlo), min(W - i2, zhi), max(i1, xlo), min(W - i1, xhi), zlo, zhi,
                    rcpb);
        __syncthreads();
        box_pass<1>(P0, P1, P3, P2, W, s, max(i2, zlo), min(W - i2, zhi), max(i2, xlo), min(W - i2, xhi), xlo, xhi,
                    rcpb);
        __syncthreads();
    }
    // scattering_angle_deg_from_grad (:171-187) returns NaN for a vanishing gradient
    for (int lx = max(H, xlo) + (int)threadIdx.y; lx < min(W - H, xhi); lx += blockDim.y)
        for (int lz = max(H, zlo) + (int)threadIdx.x; lz < min(W - H, zhi); lz += blockDim.x) {
            const double vx = P1[lx * W + lz], vz = P2[lx * W + lz];
            const double phi = (sqrt(vx * vx + vz * vz) <= 1.0e-12) ? __longlong_as_double(0x7ff8000000000000ll)
                                                                     : atan2(vz, vx);
            TPo[(size_t)(gx0 + lx) * nz + (gz0 + lz)].y = phi;
        }
}

size_t leg_grad_fused_smem(int radius, int smooth)
{
    const int r = radius < 1 ? 1 : radius, W = kGradTile + 2 * (r + 2 * smooth);
    return (4 * (size_t)W * W + 2 * smooth + 1 + 2 * (2 * r + 1)) * sizeof(double);
}

// K2 in one pass from the tables: interpolation along the position axis
// (tinterpsr.cpp:37-70, :142-188), the gradient with its smoothing and
// direction (as k_leg_grad_fused), and the aperture weight, for one
// kGradTile x kGradTile block of image points of one leg.  The table slices
// the block and its halo need (p0, m0 and, between two positions, p1, m1)
// are staged in shared memory by the TMA engine: one bulk copy per column
// and slice, completing on an mbarrier's transaction count.  A table column
// starts at ix*nz floats, which is 16-byte aligned only when nz is a multiple
// of 4, so a tiled tensor map cannot describe the tables in general: each
// column segment is placed in shared memory at the same 16-byte phase as in
// global memory, its aligned interior goes by bulk copy and its ragged ends
// (at most three floats each) by plain loads.  The staging buffer is then
// reused for the gradient planes.  Every interpolated traveltime stays on
// chip; only the block's own {T, phi} and {Tx*scale, w} are written.
constexpr int kLegTileMaxW = 96;  // widest halo tile the host launches (one byte of phase per column)

__host__ __device__ inline int leg_tile_pitch(int W) { return (W + 6) & ~3; }  // >= W + 3 floats, 16-byte rows

size_t leg_tile_smem(int radius, int smooth)
{
    const int r = radius < 1 ? 1 : radius, W = kGradTile + 2 * (r + 2 * smooth);
    const size_t stage = (size_t)4 * W * leg_tile_pitch(W) * sizeof(float);
    const size_t planes = (size_t)3 * W * W * sizeof(double);
    return (size_t)W * W * sizeof(double) + std::max(stage, planes) +
           (size_t)(2 * smooth + 1 + 2 * (2 * r + 1)) * sizeof(double);
}

__global__ void __launch_bounds__(256, 3) k_leg_tile(FieldArgs a, LegFields out)
{
    extern __shared__ __align__(16) unsigned char lsm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ unsigned char phs[4][kLegTileMaxW];  // 16-byte phase (in floats) of each staged column
    const int nz = a.nz, nx = a.nx;
    const size_t nzx = (size_t)nz * nx;
    const int r = a.radius < 1 ? 1 : a.radius, s = a.smooth;
    const int H = r + 2 * s, W = kGradTile + 2 * H, SW = leg_tile_pitch(W);
    const int tiles_z = (nz + kGradTile - 1) / kGradTile;
    const int gz0 = (int)(blockIdx.x % tiles_z) * kGradTile - H, gx0 = (int)(blockIdx.x / tiles_z) * kGradTile - H;
    const int zlo = max(0, -gz0), zhi = min(W, nz - gz0), xlo = max(0, -gx0), xhi = min(W, nx - gx0);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * blockDim.y;
    const LegInterp &L = a.legs[blockIdx.y];
    const int i0 = L.i0, i1 = L.i1;
    const bool two = i1 >= 0;  // between two positions: p0, m0, p1, m1; else p0, m0
    const int nsl = two ? 4 : 2;
    double *P0 = reinterpret_cast<double *>(lsm);
    unsigned char *regB = lsm + (size_t)W * W * sizeof(double);
    float *stage = reinterpret_cast<float *>(regB);
    double *P1 = reinterpret_cast<double *>(regB), *P2 = P1 + W * W, *P3 = P2 + W * W;
    const size_t stage_bytes = (size_t)4 * W * SW * sizeof(float), plane_bytes = (size_t)3 * W * W * sizeof(double);
    const size_t regB_bytes = stage_bytes > plane_bytes ? stage_bytes : plane_bytes;
    double *rcpb = reinterpret_cast<double *>(regB + regB_bytes), *rcpx = rcpb + 2 * s + 1, *rcpz = rcpx + 2 * r + 1;

    // ---- stage the slices' columns of the block and its halo
    if (tid == 0) tc::mbar_init(&bar, 1);
    __syncthreads();
    const int ncol = xhi - xlo, nseg = zhi - zlo;
    for (int j = tid; j < nsl * ncol; j += nthr) {
        const int q = j / ncol, lx = xlo + j % ncol;
        const float *base = (q & 1) ? a.der : a.tab;
        const float *gp = base + (size_t)(q < 2 ? i0 : i1) * nzx + (size_t)(gx0 + lx) * nz + (gz0 + zlo);
        const uintptr_t ad = reinterpret_cast<uintptr_t>(gp);
        const bool aligned4 = (ad & 3) == 0;
        const int ph = aligned4 ? (int)((ad >> 2) & 3) : 0;
        const int head = aligned4 ? min(nseg, (4 - ph) & 3) : nseg;
        const int nb = ((nseg - head) >> 2) << 2;
        float *dp = stage + (size_t)(q * W + lx) * SW + ph;  // segment element k at dp[k]
        phs[q][lx] = (unsigned char)ph;
        for (int k = 0; k < head; k++) dp[k] = __ldg(gp + k);
        for (int k = head + nb; k < nseg; k++) dp[k] = __ldg(gp + k);
        if (nb > 0) {
            tc::mbar_expect_tx(&bar, (uint32_t)nb * 4u);
            tc::bulk_g2s(dp + head, gp + head, (uint32_t)nb * 4u, &bar);
        }
    }
    for (int k = tid; k <= 2 * s; k += nthr) rcpb[k] = 1.0 / (double)(k + 1);
    for (int k = tid; k <= 2 * r; k += nthr) {
        rcpx[k] = k ? 1.0 / ((double)k * a.dx) : 0.0;
        rcpz[k] = k ? 1.0 / ((double)k * a.dz) : 0.0;
    }
    __syncthreads();  // every transfer announced before the arrival
    if (tid == 0) tc::mbar_arrive(&bar);
    // bounded wait; a block whose copies did not land raises the flag, waits
    // once more (bounded) for them and leaves
    if (!__syncthreads_and(tc::mbar_wait(&bar, 0))) {
        if (tid == 0 && a.status) atomicExch(a.status, 1);
        tc::mbar_wait(&bar, 0);
        return;
    }

    // ---- interpolated traveltime (FP64) on the block and its halo
    double2 *TPo = out.TP + (size_t)blockIdx.y * nzx;
    const double hc0 = L.c[0], hc1 = L.c[1], hc2 = L.c[2], hc3 = L.c[3];
    for_cells(zlo, zhi, xlo, xhi, [&](int lz, int lx) {
        const int o = lz - zlo;
        double T;
        if (!two) {
            T = stage[(size_t)(0 * W + lx) * SW + phs[0][lx] + o];
        } else {
            const double p0 = stage[(size_t)(0 * W + lx) * SW + phs[0][lx] + o];
            const double m0 = stage[(size_t)(1 * W + lx) * SW + phs[1][lx] + o];
            const double p1 = stage[(size_t)(2 * W + lx) * SW + phs[2][lx] + o];
            const double m1 = stage[(size_t)(3 * W + lx) * SW + phs[3][lx] + o];
            T = hc0 * p0 + hc1 * m0 + hc2 * p1 + hc3 * m1;
        }
        P0[lx * W + lz] = T;
    });
    // ---- the block's own points, lanes aligned with its kGradTile rows (one
    // full warp pass per row): T, Tx and the aperture weight written
    {
        const int lz = H + (int)threadIdx.x;  // blockDim.x == kGradTile
        const bool zin = lz >= zlo && lz < zhi;
        for (int lx = max(H, xlo) + (int)threadIdx.y; lx < min(H + kGradTile, xhi); lx += blockDim.y) {
            if (!zin) continue;
            const double p0 = stage[(size_t)(0 * W + lx) * SW + phs[0][lx] + (lz - zlo)];
            const double m0 = stage[(size_t)(1 * W + lx) * SW + phs[1][lx] + (lz - zlo)];
            double T, Tx;
            if (!two) {
                T = p0;
                Tx = m0;
            } else {
                const double p1 = stage[(size_t)(2 * W + lx) * SW + phs[2][lx] + (lz - zlo)];
                const double m1 = stage[(size_t)(3 * W + lx) * SW + phs[3][lx] + (lz - zlo)];
                T = hc0 * p0 + hc1 * m0 + hc2 * p1 + hc3 * m1;
                Tx = L.e[0] * p0 + L.e[1] * m0 + L.e[2] * p1 + L.e[3] * m1;
            }
            const int iz = gz0 + lz, ix = gx0 + lx;
            const double w = leg_aperture_weight(L.pos, iz, ix, a.dz, a.x0, a.dx, a.aper, a.aper_taper, a.rmin,
                                                 a.rtaper);
            TPo[(size_t)ix * nz + iz].x = T;
            out.XW[(size_t)blockIdx.y * nzx + (size_t)ix * nz + iz] = make_float2((float)Tx * L.scale, (float)w);
        }
    }
    __syncthreads();  // the staging buffer is free: it becomes P1..P3

    // ---- centred differences on [r, W-r)^2: gx -> P1, gz -> P2
    const bool dox = nx > 1 && a.dx != 0.0f, doz = nz > 1 && a.dz != 0.0f;
    centred_diffs(P0, P1, P2, W, r, zlo, zhi, xlo, xhi, dox, doz, rcpx, rcpz);
    __syncthreads();
    // ---- the four box passes (z, x, z, x; both components per pass), P0 and
    // P3 as scratch (the block's traveltimes are already written)
    if (s > 0) {
        const int i1 = r + s, i2 = H;
        box_pass<0>(P1, P0, P2, P3, W, s, max(i1, zlo), min(W - i1, zhi), max(r, xlo), min(W - r, xhi), zlo, zhi,
                    rcpb);
        __syncthreads();
        box_pass<1>(P0, P1, P3, P2, W, s, max(i1, zlo), min(W - i1, zhi), max(i1, xlo), min(W - i1, xhi), xlo, xhi,
                    rcpb);
        __syncthreads();
        box_pass<0>(P1, P0, P2, P3, W, s, max(i2, zlo), min(W - i2, zhi), max(i1, xlo), min(W - i1, xhi), zlo, zhi,
                    rcpb);
        __syncthreads();
        box_pass<1>(P0, P1, P3, P2, W, s, max(i2, zlo), min(W - i2, zhi), max(i2, xlo), min(W - i2, xhi), xlo, xhi,
                    rcpb);
        __syncthreads();
    }
    // scattering_angle_deg_from_grad (:171-187) returns NaN for a vanishing gradient
    for (int lx = max(H, xlo) + (int)threadIdx.y; lx < min(W - H, xhi); lx += blockDim.y)
        for (int lz = max(H, zlo) + (int)threadIdx.x; lz < min(W - H, zhi); lz += blockDim.x) {
            const double vx = P1[lx * W + lz], vz = P2[lx * W + lz];
            const double phi = (sqrt(vx * vx + vz * vz) <= 1.0e-12) ? __longlong_as_double(0x7ff8000000000000ll)
                                                                     : atan2(vz, vx);
            TPo[(size_t)(gx0 + lx) * nz + (gz0 + lz)].y = phi;
        }
}

int launch_leg_interp(const FieldArgs &a, LegFields out, double *work, cudaStream_t st, int *launches)
{
    if (a.n <= 0) return KCIG_OK;
    const int nzx = a.nz * a.nx;
    k_leg_interp<<<dim3((nzx + 255) / 256, a.n), dim3(256), 0, st>>>(a, out, work);
    KCIG_CUDA(cudaGetLastError());
    if (launches) (*launches)++;
    return KCIG_OK;
}

int launch_leg_grad(const FieldArgs &a, LegFields out, double *work, cudaStream_t st, int *launches)
{
    if (a.n <= 0 || !a.angle) return KCIG_OK;
    int nl = 0;
    struct Count {
        int *dst;
        int &n;
        ~Count() { if (dst) *dst += n; }
    } count{launches, nl};
    const int nzx = a.nz * a.nx;
    const dim3 blk(256), grd((nzx + 255) / 256, a.n);
    const size_t fsm = leg_grad_fused_smem(a.radius, a.smooth);
    if (!a.use_grad && fsm <= 200 * 1024) {
        KCIG_TRY(set_dyn_smem((const void *)k_leg_grad_fused, (int)fsm));
        const int tiles = ((a.nz + kGradTile - 1) / kGradTile) * ((a.nx + kGradTile - 1) / kGradTile);
        k_leg_grad_fused<<<dim3(tiles, a.n), dim3(32, 8), fsm, st>>>(a, out);
        nl++;
        KCIG_CUDA(cudaGetLastError());
        return KCIG_OK;
    }
    if (!a.use_grad) {
        k_leg_fd<<<grd, blk, 0, st>>>(a, out, work);
        nl++;
        KCIG_CUDA(cudaGetLastError());
    }
    if (a.smooth > 0) {
        // smooth_grad_component (:486-492): two separable passes z then x;
        // planes {0,1} hold (gx,gz), {2,3} are the scratch pair.
        const dim3 g3((nzx + 255) / 256, a.n, 2);
        for (int pass = 0; pass < 2; pass++) {
            k_box<<<g3, blk, 0, st>>>(a.nz, a.nx, a.smooth, 0, 0, 2, work);
            k_box<<<g3, blk, 0, st>>>(a.nz, a.nx, a.smooth, 1, 2, 0, work);
            nl += 2;
        }
        KCIG_CUDA(cudaGetLastError());
    }
    k_leg_pack<<<grd, blk, 0, st>>>(a, out, work);
    nl++;
    KCIG_CUDA(cudaGetLastError());
    return KCIG_OK;
}

bool leg_grad_needs_work(const FieldArgs &a)
{
    return a.angle && (a.use_grad || leg_grad_fused_smem(a.radius, a.smooth) > 200 * 1024);
}

// The one-pass kernel covers the default interpolations (Hermite and linear
// between two positions, or a clamped end) with the angle on and no gradient
// volumes; the partial-shift interpolation, gradient volumes, the kirchmig2d
// cone flags and halos wider than its shared memory take the two-stage path.
static bool leg_tile_applies(const FieldArgs &a)
{
    if (!a.angle || a.use_grad || a.cone || a.type_p) return false;
    const int r = a.radius < 1 ? 1 : a.radius, W = kGradTile + 2 * (r + 2 * a.smooth);
    return W <= kLegTileMaxW && leg_tile_smem(a.radius, a.smooth) <= 200 * 1024;
}

int launch_leg_fields(const FieldArgs &a, LegFields out, double *work, cudaStream_t st, int *launches)
{
    int nl = 0;
    if (a.n > 0 && leg_tile_applies(a)) {
        const size_t sm = leg_tile_smem(a.radius, a.smooth);
        KCIG_TRY(set_dyn_smem((const void *)k_leg_tile, (int)sm));
        const int tiles = ((a.nz + kGradTile - 1) / kGradTile) * ((a.nx + kGradTile - 1) / kGradTile);
        k_leg_tile<<<dim3(tiles, a.n), dim3(32, 8), sm, st>>>(a, out);
        KCIG_CUDA(cudaGetLastError());
        if (launches) *launches = 1;
        return KCIG_OK;
    }
    const int rc = launch_leg_interp(a, out, work, st, &nl);
    if (rc == KCIG_OK && a.angle) {
        const int rc2 = launch_leg_grad(a, out, work, st, &nl);
        if (launches) *launches = nl;
        return rc2;
    }
    if (launches) *launches = nl;
    return rc;
}

// ============================================================ K3 summation ==
// kirchmig2d_cig.cpp:226-238 (cosine ramp helpers) in the FP32 of the
// reference: weights only scale a pick, so FP32 rounding is harmless here.
__device__ __forceinline__ float taper_weight(float ang, float start, float end)
{
    if (start < 0.0f || end <= start) return 1.0f;
    if (ang <= start) return 1.0f;
    if (ang >= end) return 0.0f;
    const float x = (ang - start) / (end - start);
    return 0.5f * (1.0f + cospif(x));  // cos(pi x) for x in [0, 1]: no large-argument path
}

__device__ __forceinline__ float depth_weight(float ang, float cutoff, float band)
{
    if (band <= 0.0f) return (ang <= cutoff) ? 1.0f : 0.0f;
    if (ang <= cutoff) return 1.0f;
    if (ang >= cutoff + band) return 0.0f;
    const float u = (ang - cutoff) / band;
    return 0.5f * (1.0f + cospif(u));
}

// floor(x) + 1.5 * 2^52 for 0 <= x < 2^31 (also -1 <= x < 0), exact: the sum
// is rounded down onto the integer grid of [2^52, 2^53), so its low mantissa
// word is floor(x) as a two's-complement int (__double2loint) and subtracting
// the shift again gives floor(x) as a double.  Two FP64 adds instead of a
// round-to-integer and a conversion.
static constexpr double kFloorShift = 6755399441055744.0;
__device__ __forceinline__ double floor_shift(double x) { return __dadd_rd(x, kFloorShift); }

// One CTA owns a TZ x TX image tile (one thread per image point) and keeps
// its [bins][points] FP32 accumulators in shared memory: each thread only
// touches its own column, so there are no atomics and no block barriers.
// Shots are taken KB at a time with their leg fields in registers; each
// receiver's leg fields are loaded once per shot block when receivers are
// shared by all shots (cmp=0), one receiver ahead of use.  Per pair
// (kirchmig2d_cig.cpp:1206-1339), cheapest rejections first: trace weight,
// aperture gate, opening angle as the folded difference of the two legs'
// gradient directions (exact in FP64, no per-pair arc tangent) and its bin
// range, the angle tapers, then the antialiased pick from {D[i], D[i+1]-D[i]}
// with its time-to-sample mapping and six-term sum in FP64.  Rejections are
// mostly uniform across a warp (32 neighbouring image points), so skipping
// them costs little.
// Resident CTAs of 128 threads per SM the register allocation must allow
// (scaled for other tile sizes, so every tile gets 28 warps and at most 72
// registers): 7 CTAs of 128 threads is the most the 61-bin accumulators'
// shared memory admits (7 x 31 KB); occupancy is what this latency- and
// issue-bound loop needs (measured on the benchmark: 6 CTAs/SM at 80
// registers 500 ms per launch, 7 CTAs/SM 482 ms; earlier 16x16 tiles at 2
// CTAs/SM were slower still; 8x8 tiles of ragged shots at 82 registers held
// 10 CTAs, 20 warps, and waited on their gathers).
#ifndef KCIG_SUM_MINB
#define KCIG_SUM_MINB 7
#endif

// The unshared-receiver variant (its own receiver stream per shot) can trade
// resident CTAs for streams in flight: its own count.
#ifndef KCIG_SUM_MINB_UNSHARED
#define KCIG_SUM_MINB_UNSHARED KCIG_SUM_MINB
#endif

template <int TZ, int TX, int KB, bool SHARED_R, int MODE>
__global__ void __launch_bounds__(TZ *TX, (SHARED_R ? KCIG_SUM_MINB : KCIG_SUM_MINB_UNSHARED) * 128 / (TZ * TX))
    k_sum(const __grid_constant__ SumArgs a)
{
    constexpr int P = TZ * TX;
    constexpr double kPiD = 3.141592653589793238463, kTwoPi = 6.283185307179586476925;
    extern __shared__ float acc[];  // [nbins][P]
    const int tid = threadIdx.x;
    const int tiles_z = (a.nz + TZ - 1) / TZ;
    const int tz = blockIdx.x % tiles_z, tx = blockIdx.x / tiles_z;
    const int iz = tz * TZ + (tid % TZ), ix = tx * TX + (tid / TZ);
    const bool valid = (iz < a.nz) && (ix < a.nx);
    const int nzx = a.nz * a.nx;
    const int i = valid ? ix * a.nz + iz : 0;
    const int gc0 = a.gchunk0, nb = a.gchunk1 - a.gchunk0;
    // this CTA row's share of the shots (whole blocks of KB)
    int s_lo = 0, s_hi = a.nsb;
    float *out = a.image;
    if (a.nsplit > 1) {
        const int nblk = (a.nsb + KB - 1) / KB;
        s_lo = (int)((long long)nblk * blockIdx.y / a.nsplit) * KB;
        s_hi = min(a.nsb, (int)((long long)nblk * (blockIdx.y + 1) / a.nsplit) * KB);
        out = a.partial + (size_t)blockIdx.y * a.ng * nzx;
    }
    const bool fresh = a.zero_init || a.nsplit > 1;

    for (int b = 0; b < nb; b++)
        acc[b * P + tid] = (fresh || !valid) ? 0.0f : a.image[(size_t)(gc0 + b) * nzx + i];
    if (!valid) return;  // no block-wide synchronisation follows

    // cutoff of angle_depth_mute_weight (:200-211) depends only on depth
    const float zf = (a.nz > 1) ? (float)iz / (float)(a.nz - 1) : 0.0f;
    const float cutoff = a.oazmin + zf * (a.oazmax - a.oazmin);
    // angles (radians) at or below this carry both weights 1 when the angle
    // taper is off: no FP32 angle is formed for them (the depth weight is
    // continuous at the cutoff, so the comparison's rounding is immaterial)
    const bool no_taper = a.ats < 0.0f || a.ate <= a.ats;
    const double th_one = no_taper ? (double)cutoff / a.deg : -1.0;
    const double ulo = -1.0e-5, uhi = (double)(a.ng - 1) + 1.0e-5;
    const double uk = a.deg * a.uinv, ub = a.ug0 * a.uinv;  // u = th*uk - ub
    const double top = (double)(a.nt - 1);
    const float inv_dt_f = (float)a.inv_dt;
    const bool aal_pos = a.aal >= 0.0f;
    const float aal_abs = fabsf(a.aal), aal_sgn = aal_pos ? 1.0f : -1.0f;

    // receiver streams: one shared by a block's KB shots (cmp=0), or one per
    // shot (receivers not shared), so that KB independent (shot, receiver)
    // gather chains are in flight per thread either way
    constexpr int KR = SHARED_R ? 1 : KB;
    for (int sb = s_lo; sb < s_hi; sb += KB) {
        double2 sTP[KB];
        float2 sXW[KB];
#pragma unroll
        for (int k = 0; k < KB; k++) {
            if (sb + k < s_hi) {
                sTP[k] = __ldg(a.STP + (size_t)(sb + k) * nzx + i);
                sXW[k] = __ldg(a.SXW + (size_t)(sb + k) * nzx + i);
                // the shot's share of the pick position and of the
                // antialias width, once per shot block instead of per pair
                sTP[k].x = (sTP[k].x + a.tau - a.t0) * a.inv_dt;
                sXW[k].x = fabsf(sXW[k].x) * aal_abs * inv_dt_f;
            } else {
                sTP[k] = make_double2(0.0, 0.0);
                sXW[k] = make_float2(0.f, 0.f);
            }
        }
        // per stream: the last usable sample of its traces and its receiver
        // count (ragged shots carry their own), and its fields loaded one
        // receiver ahead of use (through the trace's field index when not
        // shared, with the index of the receiver after next loaded too, so
        // the index load does not stand in front of the field load)
        double topk[KR];
        int nrk[KR], fnext[KR];
        double2 nTP[KR];
        float2 nXW[KR];
        int nr = 0;
#pragma unroll
        for (int j = 0; j < KR; j++) {
            const bool live = SHARED_R || sb + j < s_hi;
            topk[j] = (!SHARED_R && a.stop && live) ? (double)__ldg(a.stop + sb + j) : top;
            nrk[j] = !live ? 0 : ((!SHARED_R && a.snh) ? __ldg(a.snh + sb + j) : a.nh);
            nr = max(nr, nrk[j]);
            fnext[j] = 0;
            nTP[j] = make_double2(0.0, 0.0);
            nXW[j] = make_float2(0.f, 0.f);
            if (nrk[j] > 0) {
                const int *rfi_j = a.rfi + (size_t)(sb + j) * a.nh;
                const size_t f0 = SHARED_R ? 0 : (size_t)__ldg(rfi_j);
                nTP[j] = __ldg(a.RTP + f0 * nzx + i);
                nXW[j] = __ldg(a.RXW + f0 * nzx + i);
                if (!SHARED_R && nrk[j] > 1) fnext[j] = __ldg(rfi_j + 1);
            }
        }
        for (int r = 0; r < nr; r++) {
            double2 rTP[KR];
            float2 rXW[KR];
#pragma unroll
            for (int j = 0; j < KR; j++) {
                rTP[j] = nTP[j];
                rXW[j] = nXW[j];
                // the receiver's share, once per receiver for the stream's shots
                rTP[j].x *= a.inv_dt;
                rXW[j].x = fabsf(rXW[j].x) * aal_abs * inv_dt_f;
                if (r + 1 < nrk[j]) {  // next receiver, one ahead of use
                    const size_t f1 = SHARED_R ? (size_t)(r + 1) : (size_t)fnext[j];
                    nTP[j] = __ldg(a.RTP + f1 * nzx + i);
                    nXW[j] = __ldg(a.RXW + f1 * nzx + i);
                    if (!SHARED_R && r + 2 < nrk[j]) fnext[j] = __ldg(a.rfi + (size_t)(sb + j) * a.nh + r + 2);
                }
            }
#pragma unroll
            for (int k = 0; k < KB; k++) {
                if (sb + k >= s_hi) break;
                const int j = SHARED_R ? 0 : k;  // this shot's receiver stream
                if (!SHARED_R && r >= nrk[j]) continue;
                const double2 rTPk = rTP[j];
                const float2 rXWk = rXW[j];
                const double topj = topk[j];
                const int trc = (sb + k) * a.nh + r;
                const float tw = a.unit_tw ? 1.0f : __ldg(a.trw + trc);
                if (tw == 0.0f) continue;  // trace removed by aperture_trace / offset bin
                const float apw = sXW[k].y * rXWk.y;
                if (!(apw > 0.0f)) continue;
                int b0 = 0;
                float w0 = 1.0f, w1 = 0.0f, aw;
                if (MODE == 3) {
                    // kirchmig2d (:455-488): the trace weight's sign says
                    // whether the source is the left leg; each leg's w holds
                    // its cone flags (1: left side inside, 2: right side inside)
                    const int sw = (int)sXW[k].y, rw = (int)rXWk.y;
                    const bool keep = tw > 0.0f ? ((sw & 1) && (rw & 2)) : ((rw & 1) && (sw & 2));
                    if (!keep) continue;
                    b0 = __ldg(a.igo + trc) - gc0;
                    if (b0 < 0 || b0 >= nb) continue;
                    aw = 1.0f;
                } else if (MODE == 2) {
                    b0 = __ldg(a.igo + trc) - gc0;
                    if (b0 < 0 || b0 >= nb) continue;
                    aw = tw * apw;
                } else {
                    // opening angle (:171-187): atan2(|s x r|, s.r) is the
                    // difference of the gradient directions folded to [0, pi]
                    double th = fabs(sTP[k].y - rTPk.y);
                    th = (th > kPiD) ? kTwoPi - th : th;
                    const double u = fma(th, uk, -ub);  // bin coordinate; NaN: vanishing gradient
                    double fl = 0.0;
                    if (MODE == 0) {
                        // value_to_linear_bins (:54-79)
                        if (!(u >= ulo && u <= uhi)) continue;
                    } else {
                        // value_to_nearest_bin (:35-41)
                        fl = floor(u + 0.5);
                        if (!(fl >= 0.0 && fl < (double)a.ng)) continue;
                    }
                    if (th <= th_one) {
                        aw = tw * apw;
                    } else {
                        const float ang = (float)(th * a.deg);
                        aw = taper_weight(ang, a.ats, a.ate) * depth_weight(ang, cutoff, a.oaztaper) * tw * apw;
                        if (!(aw > 0.0f)) continue;
                    }
                    if (MODE == 0) {
                        if (u <= 0.0) { b0 = 0; w0 = 1.0f; w1 = 0.0f; }
                        else if (u >= (double)(a.ng - 1)) { b0 = a.ng - 1; w0 = 1.0f; w1 = 0.0f; }
                        else {
                            const double fu = floor_shift(u);  // u in (0, ng - 1)
                            b0 = __double2loint(fu);
                            w1 = (float)(u - (fu - kFloorShift));
                            w0 = 1.0f - w1;
                        }
                    } else {
                        b0 = (int)fl;
                    }
                    b0 -= gc0;
                }
                // kirmig_pick (kirmig.cpp:34-58): sample positions of t,
                // t-deltat-dt and t+deltat+dt in FP64; every test fails on NaN
                // ft0 = (Ts + Tr + tau - t0) / dt from the two shares; the
                // half window in samples, 1 + max(|dTs ds|, |dTr dh|) * aal / dt,
                // as 1 + sign(aal) * (max of the shares scaled by |aal| / dt):
                // the scale is >= 0 and rounding is monotone, and negation is
                // exact; in FP32: it only sets the window
                const double ft0 = sTP[k].x + rTPk.x;
                const float shf = fmaf(aal_sgn, fmaxf(sXW[k].x, rXWk.x), 1.0f);
                const double sh = (double)shf;
                const double ftm0 = ft0 - sh, ftp0 = ft0 + sh;
                // the reference's six tests on the three floors (0 <= flm <=
                // fl0 <= flp < top); with aal >= 0 the half window is >= 1 or
                // NaN, so fl0 lies between the other two and the tests reduce
                // to ftm0 >= 0 and ftp0 < top (top is an integer; NaN fails)
                if (aal_pos) {
                    if (!(ftm0 >= 0.0 && ftp0 < topj)) continue;
                } else {
                    const double fl0 = floor(ft0), flm = floor(ftm0), flp = floor(ftp0);
                    if (!(fl0 >= 0.0 && fl0 < topj && flm >= 0.0 && flm <= fl0 && flp >= fl0 && flp < topj)) continue;
                }
                // all three positions are now in [0, nt - 1): floors by the
                // shifted add, the sample indices from its low word
                const double f0s = floor_shift(ft0), fms = floor_shift(ftm0), fps = floor_shift(ftp0);
                const double2 *Dk = a.D + (size_t)trc * a.nt;
                const double2 q0 = __ldg(Dk + __double2loint(f0s));
                const double2 qm = __ldg(Dk + __double2loint(fms));
                const double2 qp = __ldg(Dk + __double2loint(fps));
                const float r1 = __fdividef(1.0f, fmaf(2.0f, shf, 1.0f));  // dt / (dt + tp - tm), 2 ulp
                const double sum = 2.0 * fma(ft0 - (f0s - kFloorShift), q0.y, q0.x) -
                                   fma(ftm0 - (fms - kFloorShift), qm.y, qm.x) -
                                   fma(ftp0 - (fps - kFloorShift), qp.y, qp.x);
                const float picked = (float)sum * (r1 * r1 * aw);
                // 0 <= b < nb as one unsigned test each
                if ((unsigned)b0 < (unsigned)nb) acc[b0 * P + tid] += w0 * picked;
                if (MODE == 0 && w1 > 0.0f && (unsigned)(b0 + 1) < (unsigned)nb) acc[(b0 + 1) * P + tid] += w1 * picked;
            }
        }
    }
    for (int b = 0; b < nb; b++) out[(size_t)(gc0 + b) * nzx + i] = acc[b * P + tid];
}

// ------------------------------------------------------- forward modelling --
// kirchmig2d_cig adj=0 (:1300-1312, kirmig.cpp:59-68): one CTA per shot and
// block of RB receivers, the RB traces accumulated in shared memory in FP64
// (the trace is integrated twice afterwards, which would amplify FP32
// accumulation error; threads sweep the image points, and neighbouring points
// land on different samples), the same gates, weights and pick positions as
// k_sum.
template <int MODE, int RB>
__global__ void __launch_bounds__(256) k_spray(const __grid_constant__ SprayArgs a)
{
    constexpr double kPiD = 3.141592653589793238463, kTwoPi = 6.283185307179586476925;
    extern __shared__ double tr[];  // [RB][nt]
    const int nrb = (a.nh + RB - 1) / RB;
    const int k = blockIdx.x / nrb, r0 = (blockIdx.x % nrb) * RB;
    const int nr = min(RB, a.nh - r0);
    for (int q = threadIdx.x; q < RB * a.nt; q += blockDim.x) tr[q] = 0.0;
    float tw[RB];
    int ri[RB], ig[RB];
#pragma unroll
    for (int j = 0; j < RB; j++) {
        const int trc = k * a.nh + r0 + j;
        tw[j] = j < nr ? __ldg(a.trw + trc) : 0.0f;
        ri[j] = j < nr ? __ldg(a.rfi + trc) : 0;
        ig[j] = j < nr ? __ldg(a.igo + trc) : 0;
    }
    __syncthreads();
    const int nzx = a.nz * a.nx;
    const double top = (double)(a.nt - 1);
    const double ulo = -1.0e-5, uhi = (double)(a.ng - 1) + 1.0e-5;
    const double uk = a.deg * a.uinv, ub = a.ug0 * a.uinv;
    for (int i = threadIdx.x; i < nzx; i += blockDim.x) {
        const double2 sTP = __ldg(a.STP + (size_t)k * nzx + i);
        const float2 sXW = __ldg(a.SXW + (size_t)k * nzx + i);
        if (!(sXW.y > 0.0f)) continue;
        const int iz = i % a.nz;
        const float zf = (a.nz > 1) ? (float)iz / (float)(a.nz - 1) : 0.0f;
        const float cutoff = a.oazmin + zf * (a.oazmax - a.oazmin);
#pragma unroll
        for (int j = 0; j < RB; j++) {
            if (tw[j] == 0.0f) continue;
            const double2 rTP = __ldg(a.RTP + (size_t)ri[j] * nzx + i);
            const float2 rXW = __ldg(a.RXW + (size_t)ri[j] * nzx + i);
            const float apw = sXW.y * rXW.y;
            if (!(apw > 0.0f)) continue;
            int b0 = 0;
            float w0 = 1.0f, w1 = 0.0f, aw;
            if (MODE == 2) {
                b0 = ig[j];
                aw = tw[j] * apw;
            } else {
                double th = fabs(sTP.y - rTP.y);
                th = (th > kPiD) ? kTwoPi - th : th;
                const double u = fma(th, uk, -ub);
                double fl;
                if (MODE == 0) {
                    if (!(u >= ulo && u <= uhi)) continue;
                    fl = floor(u);
                } else {
                    fl = floor(u + 0.5);
                    if (!(fl >= 0.0 && fl < (double)a.ng)) continue;
                }
                const float ang = (float)(th * a.deg);
                aw = taper_weight(ang, a.ats, a.ate) * depth_weight(ang, cutoff, a.oaztaper) * tw[j] * apw;
                if (!(aw > 0.0f)) continue;
                if (MODE == 0) {
                    if (u <= 0.0) { b0 = 0; w0 = 1.0f; w1 = 0.0f; }
                    else if (u >= (double)(a.ng - 1)) { b0 = a.ng - 1; w0 = 1.0f; w1 = 0.0f; }
                    else {
                        b0 = (int)fl;
                        const double f1 = u - fl;
                        w1 = (float)f1;
                        w0 = (float)(1.0 - f1);
                    }
                } else {
                    b0 = (int)fl;
                }
            }
            const double ft0 = (sTP.x + rTP.x + a.tau - a.t0) * a.inv_dt;
            const double sh = fma((double)(fmaxf(fabsf(sXW.x), fabsf(rXW.x)) * a.aal), a.inv_dt, 1.0);
            const double ftm0 = ft0 - sh, ftp0 = ft0 + sh;
            const double fl0 = floor(ft0), flm = floor(ftm0), flp = floor(ftp0);
            if (!(fl0 >= 0.0 && fl0 < top && flm >= 0.0 && flm <= fl0 && flp >= fl0 && flp < top)) continue;
            float val = w0 * __ldg(a.image + (size_t)b0 * nzx + i);
            if (MODE == 0 && w1 > 0.0f) val += w1 * __ldg(a.image + (size_t)(b0 + 1) * nzx + i);
            const float r1 = 1.0f / (1.0f + 2.0f * (float)sh);  // dt / (dt + tp - tm)
            const double sv = (double)(r1 * r1 * (aw * val));
            double *t = tr + j * a.nt;
            const double f0 = ft0 - fl0, fm = ftm0 - flm, fp = ftp0 - flp;
            atomicAdd(t + (int)fl0, 2.0 * (1.0 - f0) * sv);
            atomicAdd(t + (int)fl0 + 1, 2.0 * f0 * sv);
            atomicAdd(t + (int)flm, -(1.0 - fm) * sv);
            atomicAdd(t + (int)flm + 1, -fm * sv);
            atomicAdd(t + (int)flp, -(1.0 - fp) * sv);
            atomicAdd(t + (int)flp + 1, -fp * sv);
        }
    }
    __syncthreads();
    for (int j = 0; j < nr; j++)
        for (int q = threadIdx.x; q < a.nt; q += blockDim.x)
            a.raw[((size_t)k * a.nh + r0 + j) * a.nt + q] = tr[j * a.nt + q];
}

int launch_spray(const SprayArgs &a, cudaStream_t st)
{
    if (a.nsb <= 0 || a.nh <= 0) return KCIG_OK;
    constexpr int RB = 4;
    const size_t sm = (size_t)RB * a.nt * sizeof(double);
    if (sm > 200 * 1024) return set_error(KCIG_ERR_UNSUPPORTED, "nt=%d too long for forward modelling", a.nt);
    const int grid = a.nsb * ((a.nh + RB - 1) / RB);
    if (a.mode == 0) {
        KCIG_TRY(set_dyn_smem((const void *)k_spray<0, RB>, (int)sm));
        k_spray<0, RB><<<grid, 256, sm, st>>>(a);
    } else if (a.mode == 1) {
        KCIG_TRY(set_dyn_smem((const void *)k_spray<1, RB>, (int)sm));
        k_spray<1, RB><<<grid, 256, sm, st>>>(a);
    } else {
        KCIG_TRY(set_dyn_smem((const void *)k_spray<2, RB>, (int)sm));
        k_spray<2, RB><<<grid, 256, sm, st>>>(a);
    }
    KCIG_CUDA(cudaGetLastError());
    return KCIG_OK;
}

// image (+)= the split rows' partial images, rows in order (deterministic)
__global__ void k_sum_reduce(float *image, const float *partial, int nsplit, size_t n, int zero_init)
{
    const size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    float v = zero_init ? 0.0f : image[j];
    for (int y = 0; y < nsplit; y++) v += partial[(size_t)y * n + j];
    image[j] = v;
}

template <int TZ, int TX, int KB, bool SR, int MODE>
static int launch_sum_t(const SumArgs &a, int nb, cudaStream_t st)
{
    constexpr int P = TZ * TX;
    const size_t sm = (size_t)nb * P * sizeof(float);
    auto kern = k_sum<TZ, TX, KB, SR, MODE>;
    // all of the unified L1/shared memory as shared: the accumulators of as
    // many CTAs as the registers allow (the driver's own choice held 8x8
    // tiles to 10 CTAs per SM)
    KCIG_TRY(set_dyn_smem((const void *)kern, (int)sm, cudaSharedmemCarveoutMaxShared));
    const int tiles = ((a.nz + TZ - 1) / TZ) * ((a.nx + TX - 1) / TX);
    kern<<<dim3(tiles, a.nsplit > 1 ? a.nsplit : 1), P, sm, st>>>(a);
    KCIG_CUDA(cudaGetLastError());
    return KCIG_OK;
}

// Shots per block when receivers are not shared (each shot its own receiver
// stream): the independent gather chains a thread keeps in flight.
#ifndef KCIG_KB_UNSHARED
#define KCIG_KB_UNSHARED 2
#endif

template <int TZ, int TX, int KB>
static int launch_sum_mode(const SumArgs &a, int nb, cudaStream_t st)
{
    if (a.shared_r) {
        if (a.mode == 0) return launch_sum_t<TZ, TX, KB, true, 0>(a, nb, st);
        if (a.mode == 1) return launch_sum_t<TZ, TX, KB, true, 1>(a, nb, st);
        if (a.mode == 3) return launch_sum_t<TZ, TX, KB, true, 3>(a, nb, st);
        return launch_sum_t<TZ, TX, KB, true, 2>(a, nb, st);
    }
    if (a.mode == 0) return launch_sum_t<TZ, TX, KCIG_KB_UNSHARED, false, 0>(a, nb, st);
    if (a.mode == 1) return launch_sum_t<TZ, TX, KCIG_KB_UNSHARED, false, 1>(a, nb, st);
    if (a.mode == 3) return launch_sum_t<TZ, TX, KCIG_KB_UNSHARED, false, 3>(a, nb, st);
    return launch_sum_t<TZ, TX, KCIG_KB_UNSHARED, false, 2>(a, nb, st);
}

// Shots per block of the receiver-shared path (register-resident source
// legs) and the tile of one CTA while the bins fit in 100 KB.
#ifndef KCIG_KB
#define KCIG_KB 4
#endif
#ifndef KCIG_TZ
#define KCIG_TZ 16
#endif
#ifndef KCIG_TX
#define KCIG_TX 8
#endif

// Shared memory holds [bins][points] FP32 accumulators: TZ x TX-point tiles
// while a launch's bins fit in 200 KB, 8x8 tiles beyond, and launches of at
// most 384 bins.
const int kSumTileShape[kSumTiles][3] = {{0, 0, 0}, {16, 8, 4}, {8, 8, 4}, {8, 16, 4}, {16, 8, 2}};

int launch_sum(const SumArgs &a0, cudaStream_t st, int *launches)
{
    const int maxb = 384;
    for (int g = 0; g < a0.ng; g += maxb) {
        SumArgs a = a0;
        a.gchunk0 = g;
        a.gchunk1 = min(a0.ng, g + maxb);
        const int nb = a.gchunk1 - a.gchunk0;
        int rc;
        const bool fits128 = (size_t)nb * 128 * 4 <= 200 * 1024;  // every variant but 8x8 holds 128 points
        if (a.tile == 1 && fits128) rc = launch_sum_mode<16, 8, 4>(a, nb, st);
        else if (a.tile == 2) rc = launch_sum_mode<8, 8, 4>(a, nb, st);
        else if (a.tile == 3 && fits128) rc = launch_sum_mode<8, 16, 4>(a, nb, st);
        else if (a.tile == 4 && fits128) rc = launch_sum_mode<16, 8, 2>(a, nb, st);
        else if ((size_t)nb * KCIG_TZ * KCIG_TX * 4 <= 200 * 1024) rc = launch_sum_mode<KCIG_TZ, KCIG_TX, KCIG_KB>(a, nb, st);
        else rc = launch_sum_mode<8, 8, KCIG_KB>(a, nb, st);
        if (rc) return rc;
        if (launches) (*launches)++;
    }
    if (a0.nsplit > 1) {
        const size_t n = (size_t)a0.ng * a0.nz * a0.nx;
        k_sum_reduce<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a0.image, a0.partial, a0.nsplit, n, a0.zero_init);
        KCIG_CUDA(cudaGetLastError());  // (counted by the caller: `launches` counts k_sum launches)
    }
    return KCIG_OK;
}

// A summation is split over shots into partial images when its tiles fill
// fewer than KCIG_SPLIT_BELOW waves of resident CTAs: with shared receivers
// to the split of least waves x shot blocks per row (below), with ragged shots
// aiming for KCIG_SPLIT_WAVES waves (a partial last wave costs less the more
// waves there are; each split adds a partial image).  A grid of more waves is split into
// up to 4 parts only when that fills its last wave clearly better: the
// 601 x 1601 grid's 7638 tiles are 7.37 waves of 1036 slots (the last one 37%
// full), as two parts 14.75 waves (75% full), measured 1.7% faster.
#ifndef KCIG_SPLIT_BELOW
#define KCIG_SPLIT_BELOW 2
#endif
#ifndef KCIG_SPLIT_WAVES
#define KCIG_SPLIT_WAVES 8
#endif

int sum_nsplit(int nz, int nx, int nsb, bool shared_r)
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            sms = 148;
    }
    const long long tiles = (long long)((nz + 15) / 16) * ((nx + 7) / 8);
    const long long slots = (long long)sms * KCIG_SUM_MINB;  // resident CTAs of one wave
    const int blocks = shared_r ? (nsb + KCIG_KB - 1) / KCIG_KB : (nsb + KCIG_KB_UNSHARED - 1) / KCIG_KB_UNSHARED;
    if (tiles >= (long long)KCIG_SPLIT_BELOW * slots) {
        // fill(n): the waves of n parts over whole waves
        auto fill = [&](int n) {
            const double w = (double)(n * tiles) / (double)slots;
            return w / ceil(w);
        };
        int best = 1;
        for (int n = 2; n <= std::min(4, blocks); n++)
            if (fill(n) > fill(best) + 0.02) best = n;
        return best;
    }
    if (shared_r) {
        // shots shared by every tile: a CTA row's duration is its number of
        // shot blocks, so take the split with the fewest waves x blocks per
        // row (whole waves, the longest row); more parts only for 5% less.  The
        // v(z) 201 x 401 survey (663 tiles, 16 blocks): 16 parts of one block
        // each, 11 units, against 13 parts (the 8-wave aim) at 9 x 2 = 18 --
        // measured 4.80 -> 4.42 ms
        long long best = 1, cost = -1;
        for (long long n = 1; n <= std::min(blocks, 64); n++) {
            const long long c = ((n * tiles + slots - 1) / slots) * ((blocks + n - 1) / n);
            if (cost < 0 || 20 * c < 19 * cost) {
                cost = c;
                best = n;
            }
        }
        return (int)best;
    }
    const long long want = (long long)KCIG_SPLIT_WAVES * slots;
    long long ns = (want + tiles - 1) / tiles;
    ns = std::min<long long>(ns, std::min(blocks, 64));
    return (int)std::max<long long>(1, ns);
}

}  // namespace kcig
