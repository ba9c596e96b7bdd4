// Learned traveltime surrogate on the fifth-generation tensor cores
// (tcgen05 MMAs, TMEM accumulators), in place of the traveltime tables.
//
// The network (no counterpart in the reference, which reads tables):
//   u_i = (v_i - lo_i) * 2 / (hi_i - lo_i) - 1   for v = (xs, z, x) in km
//   f   = interleaved [sin th_ik, cos th_ik], th_ik = (k+1) * fstep * u_i,
//         k < 64, fstep = pi * fmax / 64                 -> 384 features
//   h_1 = SiLU(W_1 f + b_1), h_l = SiLU(W_l h_{l-1} + b_l), l = 2..4 (128 wide)
//   out = w_o . h_4 + b_o
//   T   = Tb + rscale * out   (additive residual, rscale > 0), or
//   T   = Tb * (1 + out)      (factored form, rscale = 0)
// with Tb the first-arrival time of a background medium vref + vgrad (z -
// zsrc) (closed form; straight rays at vgrad = 0): the network learns what
// the background misses.  BF16 operands (weights, features, activations,
// backpropagated gradients) with FP32 accumulation in TMEM; biases, output
// layer and the traveltime algebra in FP32 (FP64 for the traveltime a leg
// field stores).  Input gradients come from the backward pass of the same
// network: dT/dxs for the antialias width, and -- on request -- dT/dz, dT/dx
// for the scattering angle; by default a plan takes the angle from the
// traveltime's finite-difference gradient, as with tables.  A 128-point tile
// is one M=128 MMA row block; each TMEM lane (row) is shared by the threads
// of the warps that read it, each taking a share of its 128 columns.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "kcig_aperture.h"
#include "kcig_common.h"
#include "kcig_tc.h"

namespace kcig {

// The three operand views the surrogate's kernels use, on one 128x128 tile
// pair X, W (row-major in global memory, staged in the canonical layout):
//   D0 = X W^T   (A K-major,  B K-major)   -- forward layer
//   D1 = X W     (A K-major,  B MN-major)  -- backward through a layer
//   D2 = X^T W   (A MN-major, B MN-major)  -- weight gradient
__global__ void __launch_bounds__(128, 1) k_tc_selftest(const __nv_bfloat16 *X, const __nv_bfloat16 *W, float *D,
                                                        int *status)
{
    extern __shared__ __align__(1024) unsigned char dsm[];
    unsigned char *sx = dsm, *sw = dsm + 128 * 128 * 2;
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5;

    if (warp == 0) tc::tmem_alloc(&tslot, 512);
    if (tid == 0) tc::mbar_init(&bar, 1);
    // stage: thread = row, 16 groups of 8 columns
    for (int g = 0; g < 16; g++) {
        const uint4 vx = *reinterpret_cast<const uint4 *>(X + tid * 128 + g * 8);
        const uint4 vw = *reinterpret_cast<const uint4 *>(W + tid * 128 + g * 8);
        *reinterpret_cast<uint4 *>(sx + tc::canon_off(tid, g * 8, 128)) = vx;
        *reinterpret_cast<uint4 *>(sw + tc::canon_off(tid, g * 8, 128)) = vw;
    }
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tbase = tslot;
    if (warp == 0 && tc::elect_one()) {
        const uint32_t ax = tc::smem_u32(sx), aw = tc::smem_u32(sw);
        tc::gemm(tbase + 0, ax, 2048, 128, aw, 2048, 128, 128, tc::idesc_bf16(128, 128, 0, 0), false);
        tc::gemm(tbase + 128, ax, 2048, 128, aw, 128, 2048, 128, tc::idesc_bf16(128, 128, 0, 1), false);
        tc::gemm(tbase + 256, ax, 128, 2048, aw, 128, 2048, 128, tc::idesc_bf16(128, 128, 1, 1), false);
        tc::commit(&bar);
    }
    const bool ok = __syncthreads_and(tc::mbar_wait(&bar, 0));  // uniform: the loads below are warp-collective
    tc::fence_after();
    if (ok) {
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
        for (int m = 0; m < 3; m++)
            for (int c = 0; c < 4; c++) {
                float v[32];
                tc::tmem_ld32(tbase + lane_base + m * 128 + c * 32, v);
                float *o = D + (size_t)m * 128 * 128 + (size_t)tid * 128 + c * 32;
#pragma unroll
                for (int i = 0; i < 32; i++) o[i] = v[i];
            }
    } else if (tid == 0) {
        atomicExch(status, 1);
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tbase, 512);
}


// ================================================================ network ==
namespace sg {
constexpr int NF = 64, H = 128, FEAT = 384;
constexpr int OFF_W1 = 0, OFF_W2 = H * FEAT, OFF_W3 = OFF_W2 + H * H, OFF_W4 = OFF_W3 + H * H;
constexpr int OFF_B1 = OFF_W4 + H * H, OFF_B2 = OFF_B1 + H, OFF_B3 = OFF_B2 + H, OFF_B4 = OFF_B3 + H;
constexpr int OFF_WO = OFF_B4 + H, OFF_BO = OFF_WO + H, NPARAM = OFF_BO + 1;
constexpr int NWB = OFF_B1;                 // matrix weights, kept as BF16 for the MMAs
constexpr int PSTRIDE = NPARAM + 3;         // one tile's partial gradient + loss, padded to 16 B
constexpr int TB = 128 * 128 * 2;           // bytes of one 128x128 BF16 operand tile
constexpr uint32_t ID_KK = tc::idesc_bf16(128, 128, 0, 0);  // A K-major,  B K-major
constexpr uint32_t ID_KM = tc::idesc_bf16(128, 128, 0, 1);  // A K-major,  B MN-major
constexpr uint32_t ID_MM = tc::idesc_bf16(128, 128, 1, 1);  // A MN-major, B MN-major
constexpr uint32_t LBO_K = 2048, SBO_K = 128;  // K-major view of a 128-row canonical tile
constexpr uint32_t LBO_M = 128, SBO_M = 2048;  // MN-major view of the same bytes
}  // namespace sg

struct SgNet {
    const __nv_bfloat16 *W;  // [NWB] BF16 copy of W_1..W_4 (row = output)
    const float *P;          // [NPARAM] FP32 parameters
    float lo[3], sc[3];      // u = (v - lo) * sc - 1
    float fstep, vref, zsrc;
    float vgrad;             // background velocity vref + vgrad * (z - zsrc)
    float rscale;            // > 0: T = Tb + rscale * out (s); 0: T = Tb * (1 + out)
};

__device__ __forceinline__ float sg_sig(float z) { return __fdividef(1.0f, 1.0f + __expf(-z)); }
__device__ __forceinline__ float sg_silu(float z) { return z * sg_sig(z); }
__device__ __forceinline__ float sg_dsilu(float z)
{
    const float s = sg_sig(z);
    return s * (1.0f + z * (1.0f - s));
}

// Background traveltime Tb(xs, z, x) and its derivatives: the first arrival
// in the medium v(z) = vref + vgrad (z - zsrc) from a source at (xs, zsrc),
// the closed form for a constant velocity gradient g,
//     Tb = acosh(1 + eps) / g,   eps = g^2 r^2 / (2 vs vp),
// vs = vref at the source, vp = v at the point, r the distance; written as
//     Tb = r / sqrt(vs vp) * log1p(eps + sqrt(eps (2 + eps))) / sqrt(2 eps)
// so that it tends to the straight-ray time r / vref as g -> 0 without
// cancellation.  Its gradient, from dTb/dA = 1 / (g sqrt(A^2 - 1)) with
// A = 1 + eps:  dTb/dx = (x - xs) k,  dTb/dz = (z - zsrc - r^2 g / (2 vp)) k,
// k = sqrt(2 / (vs vp (2 + eps))) / r,  dTb/dxs = -dTb/dx (0 at r = 0).
template <typename F>
__device__ __forceinline__ void sg_background(const SgNet &n, F xs, F z, F x, F &Tb, F &dxs, F &dz, F &dx)
{
    const F ex = x - xs, ez = z - (F)n.zsrc, g = (F)n.vgrad, vs = (F)n.vref;
    const F r2 = ex * ex + ez * ez, r = sqrt(r2);
    F vp = vs + g * ez;
    vp = vp > (F)1e-3 * vs ? vp : (F)1e-3 * vs;
    const F q = vs * vp, eps = g * g * r2 / ((F)2 * q);
    const F fac = eps < (F)1e-6 ? (F)1 - eps / (F)12 : log1p(eps + sqrt(eps * ((F)2 + eps))) / sqrt((F)2 * eps);
    Tb = r * fac / sqrt(q);
    if (r > (F)0) {
        const F k = sqrt((F)2 / (q * ((F)2 + eps))) / r;
        dx = ex * k;
        dxs = -dx;
        dz = (ez - r2 * g / ((F)2 * vp)) * k;
    } else {
        dx = dxs = dz = (F)0;
    }
}

// The network's output `out` (w_o . h_4 + b_o) and the background combine as
// T = Tb + osc * out: osc = rscale for an additive residual, osc = Tb for the
// factored form T = Tb (1 + out).  dT/dv = dTb/dv (1 + m out) + osc dout/dv
// with m = 0 (additive) or 1 (factored).
template <typename F>
__device__ __forceinline__ F sg_out_scale(const SgNet &n, F Tb, F &m)
{
    m = n.rscale > 0.0f ? (F)0 : (F)1;
    return n.rscale > 0.0f ? (F)n.rscale : Tb;
}

// 128x128 block of a row-major BF16 matrix (rows = outputs, row stride ld,
// columns c0..c0+127) into a canonical shared tile
__device__ __forceinline__ void sg_stage_w(unsigned char *dst, const __nv_bfloat16 *src, int ld, int c0)
{
    for (int q = threadIdx.x; q < 2048; q += blockDim.x) {
        const int row = q >> 4, g = q & 15;
        const uint4 v = *reinterpret_cast<const uint4 *>(src + (size_t)row * ld + c0 + g * 8);
        *reinterpret_cast<uint4 *>(dst + tc::canon_off(row, g * 8, 128)) = v;
    }
}

// Fourier features of one input for row r, pairs [p0, p0 + np) (np a
// multiple of 4): column 2k = sin th_k, 2k+1 = cos th_k, by rotation from
// th_{p0} in steps of fstep*u
__device__ __forceinline__ void sg_features(unsigned char *act, int r, int p0, int np, float u, float fstep)
{
    const float d = fstep * u;
    float s, c, sd, cd;
    // angles as multiples of pi (sincospif: no large-argument reduction)
    const float dp = d * 0.318309886f;
    sincospif(dp * (float)(p0 + 1), &s, &c);
    sincospif(dp, &sd, &cd);
    for (int g = 0; g < np / 4; g++) {
        uint32_t pk[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            __nv_bfloat162 b = __floats2bfloat162_rn(s, c);
            pk[j] = *reinterpret_cast<uint32_t *>(&b);
            const float s2 = s * cd + c * sd, c2 = c * cd - s * sd;
            s = s2;
            c = c2;
        }
        *reinterpret_cast<uint4 *>(act + tc::canon_off(r, 2 * p0 + 8 * g, 128)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
}

// d tau / d u of one input from 32*nq columns of d tau / d f starting at
// column c0 (G, FP32 from TMEM): sum over its pairs of G_sin (k+1) fstep cos th - G_cos (k+1) fstep sin th
__device__ __forceinline__ float sg_feature_grad(uint32_t tG, int c0, int nq, float u, float fstep)
{
    const float d = fstep * u;
    float s, c, sd, cd;
    const float dp = d * 0.318309886f;
    sincospif(dp * (float)(c0 / 2 + 1), &s, &c);
    sincospif(dp, &sd, &cd);
    float acc = 0.0f;
    for (int q = 0; q < nq; q++) {
        float v[32];
        tc::tmem_ld32(tG + c0 + 32 * q, v);
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const float kf = (float)(c0 / 2 + 16 * q + j + 1) * fstep;
            acc += kf * (v[2 * j] * c - v[2 * j + 1] * s);
            const float s2 = s * cd + c * sd, c2 = c * cd - s * sd;
            s = s2;
            c = c2;
        }
    }
    return acc;
}

__device__ __forceinline__ void sg_store8(unsigned char *dst, int r, int col, const float *x)
{
    __nv_bfloat162 b0 = __floats2bfloat162_rn(x[0], x[1]), b1 = __floats2bfloat162_rn(x[2], x[3]);
    __nv_bfloat162 b2 = __floats2bfloat162_rn(x[4], x[5]), b3 = __floats2bfloat162_rn(x[6], x[7]);
    *reinterpret_cast<uint4 *>(dst + tc::canon_off(r, col, 128)) =
        make_uint4(*reinterpret_cast<uint32_t *>(&b0), *reinterpret_cast<uint32_t *>(&b1),
                   *reinterpret_cast<uint32_t *>(&b2), *reinterpret_cast<uint32_t *>(&b3));
}

// forward epilogue: h = SiLU(acc + bias) as BF16 into dst (row r, the
// thread's columns cb .. cb + 32*nq)
__device__ __forceinline__ void sg_epi_silu(uint32_t tacc, const float *bias, unsigned char *dst, int r, int cb,
                                            int nq)
{
    for (int q = 0; q < nq; q++) {
        float v[32];
        const int c0 = cb + 32 * q;
        tc::tmem_ld32(tacc + c0, v);
#pragma unroll
        for (int j = 0; j < 32; j++) v[j] = sg_silu(v[j] + bias[c0 + j]);
#pragma unroll
        for (int g = 0; g < 4; g++) sg_store8(dst, r, c0 + 8 * g, v + 8 * g);
    }
}

// backward epilogue: g = G * SiLU'(z + bias) as BF16 into dst; returns the
// sum over the thread's columns of bf16(g) * vdot (vdot may be null).
// colsum (may be null): this warp's column sums over its 32 rows, stored
// (not added) at colsum[c] -- one slot array per row group, so every slot
// has one writer and the caller adds the groups in a fixed order
__device__ __forceinline__ float sg_epi_back(uint32_t tG, uint32_t tZ, const float *bias, unsigned char *dst, int r,
                                             int cb, int nq, const float *vdot, float *colsum)
{
    float dot = 0.0f;
    for (int q = 0; q < nq; q++) {
        float G[32], Z[32];
        const int c0 = cb + 32 * q;
        tc::tmem_ld32(tG + c0, G);
        tc::tmem_ld32(tZ + c0, Z);
#pragma unroll
        for (int j = 0; j < 32; j++) {
            const float g = G[j] * sg_dsilu(Z[j] + bias[c0 + j]);
            G[j] = __bfloat162float(__float2bfloat16_rn(g));
        }
        if (vdot) {
#pragma unroll
            for (int j = 0; j < 32; j++) dot += G[j] * vdot[c0 + j];
        }
        if (colsum) {
#pragma unroll
            for (int j = 0; j < 32; j++) {
                float x = G[j];
                x += __shfl_xor_sync(0xffffffffu, x, 16);
                x += __shfl_xor_sync(0xffffffffu, x, 8);
                x += __shfl_xor_sync(0xffffffffu, x, 4);
                x += __shfl_xor_sync(0xffffffffu, x, 2);
                x += __shfl_xor_sync(0xffffffffu, x, 1);
                if ((threadIdx.x & 31) == 0) colsum[c0 + j] = x;
            }
        }
#pragma unroll
        for (int g = 0; g < 4; g++) sg_store8(dst, r, c0 + 8 * g, G + 8 * g);
    }
    return dot;
}

// all threads' shared-memory operand writes and TMEM reads are done; the
// tensor core may start
__device__ __forceinline__ void sg_sync_for_mma()
{
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
}

// all wait (bounded) for the step thread 0 issued and committed with
// sg_issue_end.  false: the tensor core did not answer
__device__ __forceinline__ bool sg_wait(uint64_t *bar, uint32_t &phase)
{
    const bool ok = __syncthreads_and(tc::mbar_wait(bar, phase));
    phase ^= 1u;
    tc::fence_after();
    return ok;
}

// ------------------------------------------------------------ leg fields --
// Persistent kernel: the work items (leg, 128-point tile) are split into one
// contiguous range per CTA, so a CTA changes leg rarely.  Per leg, the xs
// features are constant: their part of layer 1 folds into a per-leg bias and
// their input gradient into a per-leg vector (d tau/d u_xs = g_1 . v_leg),
// so only the z and x features go through the tensor core.  All matrix
// weights stay in shared memory (160 KB) next to two activation tiles.
struct SgFieldArgs {
    SgNet net;
    const LegInterp *legs;  // .pos and .scale of each leg
    int nlegs, nz, nx;
    float z0, dz, x0, dx;
    float aper, aper_taper, rmin, rtaper;
    LegFields out;
    int *status;
};
constexpr int kSgFieldSmem = 7 * sg::TB;
// what a launch computes: the traveltime only (its position derivative and
// the aperture weight come from the tables, its direction from the
// finite-difference pass), the traveltime and its source-position
// derivative from the network's backward pass (direction from the
// finite-difference pass), or also the direction from the network's input
// gradient in depth and lateral position
enum { SGF_T = 0, SGF_TX = 1, SGF_ALL = 2 };

template <int MODE>
__global__ void __launch_bounds__(512, 1) k_sg_fields(SgFieldArgs a)
{
    using namespace sg;
    extern __shared__ __align__(1024) unsigned char dsm[];
    unsigned char *sW1z = dsm, *sW1x = dsm + TB, *sW2 = dsm + 2 * TB, *sW3 = dsm + 3 * TB, *sW4 = dsm + 4 * TB;
    unsigned char *actA = dsm + 5 * TB, *actB = dsm + 6 * TB;
    // the dynamic tiles take 224 of the 227 KB a CTA may hold; the small
    // per-leg arrays fit in the rest
    __shared__ float b1p[H], vleg[H];
    __shared__ float fx[H], dfx[H];  // per-leg xs features and their derivatives
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tslot;
    const SgNet &n = a.net;
    const int tid = threadIdx.x, warp = tid >> 5, h = warp >> 2, r = (warp & 3) * 32 + (tid & 31);
    const int nzx = a.nz * a.nx;

    if (warp == 0) tc::tmem_alloc(&tslot, 512);
    if (tid == 0) tc::mbar_init(&bar, 1);
    sg_stage_w(sW1z, n.W + OFF_W1, FEAT, 128);
    sg_stage_w(sW1x, n.W + OFF_W1, FEAT, 256);
    sg_stage_w(sW2, n.W + OFF_W2, H, 0);
    sg_stage_w(sW3, n.W + OFF_W3, H, 0);
    sg_stage_w(sW4, n.W + OFF_W4, H, 0);
    const float *bias2 = n.P + OFF_B2, *bias3 = n.P + OFF_B3, *bias4 = n.P + OFF_B4, *wo = n.P + OFF_WO;
    sg_sync_for_mma();
    const uint32_t lane = (uint32_t)((warp & 3) * 32) << 16;
    const uint32_t D1 = tslot + lane, D2 = D1 + 128, D3 = D1 + 256, D4 = D1 + 384;
    const uint32_t aW1z = tc::smem_u32(sW1z), aW1x = tc::smem_u32(sW1x), aW2 = tc::smem_u32(sW2);
    const uint32_t aW3 = tc::smem_u32(sW3), aW4 = tc::smem_u32(sW4), aA = tc::smem_u32(actA), aB = tc::smem_u32(actB);
    const uint32_t T1 = tslot, T2 = tslot + 128, T3 = tslot + 256, T4 = tslot + 384;  // MMA targets
    const float bo = n.P[OFF_BO];

    const int ntiles = (nzx + 127) / 128;
    const long long total = (long long)a.nlegs * ntiles;
    const long long per = (total + gridDim.x - 1) / gridDim.x;
    const long long it0 = (long long)blockIdx.x * per, it1 = (it0 + per < total) ? it0 + per : total;
    int cur = -1;
    uint32_t phase = 0;
    bool ok = true;
    for (long long item = it0; item < it1 && ok; item++) {
        const int j = (int)(item / ntiles), t = (int)(item % ntiles);
        const LegInterp &L = a.legs[j];
        const float xs = (float)L.pos;
        if (j != cur) {
            // per-leg bias and input-gradient vector of the xs features
            cur = j;
            const float u0 = (xs - n.lo[0]) * n.sc[0] - 1.0f;
            if (tid < NF) {
                float sn, cs;
                const float th = (float)(tid + 1) * n.fstep * u0;
                sincospif(th * 0.318309886f, &sn, &cs);
                fx[2 * tid] = __bfloat162float(__float2bfloat16_rn(sn));
                fx[2 * tid + 1] = __bfloat162float(__float2bfloat16_rn(cs));
                dfx[2 * tid] = (float)(tid + 1) * n.fstep * cs;
                dfx[2 * tid + 1] = -(float)(tid + 1) * n.fstep * sn;
            }
            __syncthreads();
            {   // four threads per output row, 32 columns each
                const int o = tid >> 2, c0 = 32 * (tid & 3);
                float acc = 0.0f, accv = 0.0f;
                const __nv_bfloat16 *w = n.W + OFF_W1 + (size_t)o * FEAT;
                for (int c = c0; c < c0 + 32; c++) {
                    const float wc = __bfloat162float(w[c]);
                    acc += wc * fx[c];
                    accv += wc * dfx[c];
                }
                acc += __shfl_xor_sync(0xffffffffu, acc, 1);
                accv += __shfl_xor_sync(0xffffffffu, accv, 1);
                acc += __shfl_xor_sync(0xffffffffu, acc, 2);
                accv += __shfl_xor_sync(0xffffffffu, accv, 2);
                if ((tid & 3) == 0) {
                    b1p[o] = n.P[OFF_B1 + o] + acc;
                    vleg[o] = accv;
                }
            }
            __syncthreads();
        }
        const int i = t * 128 + r;
        const bool valid = i < nzx;
        const int ic = valid ? i : nzx - 1, iz = ic % a.nz, ix = ic / a.nz;
        const float zf = a.z0 + (float)iz * a.dz, xf = a.x0 + (float)ix * a.dx;
        const float uz = (zf - n.lo[1]) * n.sc[1] - 1.0f, ux = (xf - n.lo[2]) * n.sc[2] - 1.0f;

        sg_features(actA, r, 16 * h, 16, uz, n.fstep);
        sg_features(actB, r, 16 * h, 16, ux, n.fstep);
        sg_sync_for_mma();
        if (warp == 0 && tc::elect_one()) {
            tc::gemm(T1, aA, LBO_K, SBO_K, aW1z, LBO_K, SBO_K, 128, ID_KK, false);
            tc::gemm(T1, aB, LBO_K, SBO_K, aW1x, LBO_K, SBO_K, 128, ID_KK, true);
            tc::commit(&bar);
        }
        if (!(ok = sg_wait(&bar, phase))) break;
        sg_epi_silu(D1, b1p, actA, r, 32 * h, 1);
        sg_sync_for_mma();
        if (warp == 0 && tc::elect_one()) {
            tc::gemm(T2, aA, LBO_K, SBO_K, aW2, LBO_K, SBO_K, 128, ID_KK, false);
            tc::commit(&bar);
        }
        if (!(ok = sg_wait(&bar, phase))) break;
        sg_epi_silu(D2, bias2, actB, r, 32 * h, 1);
        sg_sync_for_mma();
        if (warp == 0 && tc::elect_one()) {
            tc::gemm(T3, aB, LBO_K, SBO_K, aW3, LBO_K, SBO_K, 128, ID_KK, false);
            tc::commit(&bar);
        }
        if (!(ok = sg_wait(&bar, phase))) break;
        sg_epi_silu(D3, bias3, actA, r, 32 * h, 1);
        sg_sync_for_mma();
        if (warp == 0 && tc::elect_one()) {
            tc::gemm(T4, aA, LBO_K, SBO_K, aW4, LBO_K, SBO_K, 128, ID_KK, false);
            tc::commit(&bar);
        }
        if (!(ok = sg_wait(&bar, phase))) break;
        float out_part, xs_part = 0.0f, gz_part = 0.0f, gx_part = 0.0f;
        {   // output layer and the start of the backward pass (d out / d out = 1)
            float part = 0.0f, v[32];
            const int c0 = 32 * h;
            tc::tmem_ld32(D4 + c0, v);
#pragma unroll
            for (int jj = 0; jj < 32; jj++) {
                const float z = v[jj] + bias4[c0 + jj];
                part += sg_silu(z) * wo[c0 + jj];
                v[jj] = wo[c0 + jj] * sg_dsilu(z);
            }
            if (MODE != SGF_T) {
#pragma unroll
                for (int g = 0; g < 4; g++) sg_store8(actB, r, c0 + 8 * g, v + 8 * g);
            }
            out_part = part;
        }
        if (MODE != SGF_T) {
            sg_sync_for_mma();
            if (warp == 0 && tc::elect_one()) {
                tc::gemm(T4, aB, LBO_K, SBO_K, aW4, LBO_M, SBO_M, 128, ID_KM, false);
                tc::commit(&bar);
            }
            if (!(ok = sg_wait(&bar, phase))) break;
            sg_epi_back(D4, D3, bias3, actA, r, 32 * h, 1, nullptr, nullptr);
            sg_sync_for_mma();
            if (warp == 0 && tc::elect_one()) {
                tc::gemm(T3, aA, LBO_K, SBO_K, aW3, LBO_M, SBO_M, 128, ID_KM, false);
                tc::commit(&bar);
            }
            if (!(ok = sg_wait(&bar, phase))) break;
            sg_epi_back(D3, D2, bias2, actB, r, 32 * h, 1, nullptr, nullptr);
            sg_sync_for_mma();
            if (warp == 0 && tc::elect_one()) {
                tc::gemm(T2, aB, LBO_K, SBO_K, aW2, LBO_M, SBO_M, 128, ID_KM, false);
                tc::commit(&bar);
            }
            if (!(ok = sg_wait(&bar, phase))) break;
            xs_part = sg_epi_back(D2, D1, b1p, actA, r, 32 * h, 1, vleg, nullptr);
        }
        if (MODE == SGF_ALL) {
            sg_sync_for_mma();
            if (warp == 0 && tc::elect_one()) {
                tc::gemm(T3, aA, LBO_K, SBO_K, aW1z, LBO_M, SBO_M, 128, ID_KM, false);
                tc::gemm(T4, aA, LBO_K, SBO_K, aW1x, LBO_M, SBO_M, 128, ID_KM, false);
                tc::commit(&bar);
            }
            if (!(ok = sg_wait(&bar, phase))) break;
            // each column quarter: its part of d out/d u_z (G0z) and d out/d u_x (G0x)
            gz_part = sg_feature_grad(D3, 32 * h, 1, uz, n.fstep);
            gx_part = sg_feature_grad(D4, 32 * h, 1, ux, n.fstep);
        }
        // the four column quarters' partials of each quantity meet in actB,
        // which no MMA reads any more in this item
        {
            float *xq = reinterpret_cast<float *>(actB);  // [quantity][quarter][row]
            xq[(0 * 4 + h) * 128 + r] = out_part;
            xq[(1 * 4 + h) * 128 + r] = xs_part;
            xq[(2 * 4 + h) * 128 + r] = gz_part;
            xq[(3 * 4 + h) * 128 + r] = gx_part;
        }
        tc::fence_before();
        __syncthreads();
        if (h == 0 && valid) {
            const float *xq = reinterpret_cast<const float *>(actB);
            float sum[4];
#pragma unroll
            for (int k = 0; k < 4; k++)
                sum[k] = (xq[(k * 4) * 128 + r] + xq[(k * 4 + 1) * 128 + r]) +
                         (xq[(k * 4 + 2) * 128 + r] + xq[(k * 4 + 3) * 128 + r]);
            const float out = sum[0] + bo;
            // the traveltime in FP64: background plus the network's term
            double Tb, bxs, bz, bx, m;
            sg_background<double>(n, (double)L.pos, (double)zf, (double)xf, Tb, bxs, bz, bx);
            const double osc = sg_out_scale<double>(n, Tb, m);
            const double T = Tb + osc * (double)out;
            const size_t o = (size_t)j * nzx + i;
            if (MODE == SGF_T) {
                a.out.TP[o].x = T;  // Tx and w come from the tables, phi from the traveltime's gradient
            } else {
                const double gxs = (double)(sum[1] * n.sc[0]);
                const double Txs = bxs * (1.0 + m * out) + osc * gxs;
                double phi = 0.0;  // MODE SGF_TX: written by the finite-difference pass
                if (MODE == SGF_ALL) {
                    const double Tz = bz * (1.0 + m * out) + osc * (double)(sum[2] * n.sc[1]);
                    const double Tx = bx * (1.0 + m * out) + osc * (double)(sum[3] * n.sc[2]);
                    phi = (sqrt(Tx * Tx + Tz * Tz) <= 1.0e-12) ? __longlong_as_double(0x7ff8000000000000ll)
                                                               : atan2(Tz, Tx);
                }
                const double w = leg_aperture_weight(L.pos, iz, ix, a.dz, a.x0, a.dx, a.aper, a.aper_taper, a.rmin,
                                                     a.rtaper);
                a.out.TP[o] = make_double2(T, phi);
                a.out.XW[o] = make_float2((float)Txs * L.scale, (float)w);
            }
        }
        __syncthreads();
    }
    if (!ok && tid == 0) atomicExch(a.status, 1);
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tslot, 512);
}

// --------------------------------------------------- training / evaluation --
// One CTA per 128-sample tile, weights staged per use (the xs features vary
// per sample).  TRAIN: forward, loss mean((1000 (T - Ttrue))^2) over ntotal
// samples, and this tile's gradient of every parameter into part[tile][*]
// (loss at index NPARAM); summed later in a fixed order.  EVAL: T and
// dT/d(xs, z, x).
enum { SG_TRAIN = 0, SG_EVAL = 1 };
struct SgTileArgs {
    SgNet net;
    const float *xs, *z, *x, *Ttrue;  // [n]
    int n, ntotal;
    float *part;                      // TRAIN: [tiles][PSTRIDE]
    float *T, *Txs, *Tz, *Tx;         // EVAL: [n]
    float *stages;                    // EVAL, optional: accumulators of tile 0, [5][128][128]
    int *status;
};

// a canonical BF16 operand tile decoded to FP32 [128][128] (tile 0 only)
__device__ __forceinline__ void sg_dump_tile(float *dst, const unsigned char *tile)
{
    if (!dst || blockIdx.x != 0) return;
    for (int q = threadIdx.x; q < 128 * 128; q += blockDim.x) {
        const int row = q >> 7, col = q & 127;
        dst[q] = __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(tile + tc::canon_off(row, col, 128)));
    }
}

// stage dump of the first tile (kcig_surrogate_eval_stages): row = TMEM lane
__device__ __forceinline__ void sg_dump(float *dst, uint32_t tD, int r, int h)
{
    if (!dst || blockIdx.x != 0) return;
    for (int q = 0; q < 2; q++) {
        float v[32];
        tc::tmem_ld32(tD + 64 * h + 32 * q, v);
        for (int j = 0; j < 32; j++) dst[r * 128 + 64 * h + 32 * q + j] = v[j];
    }
}
constexpr int kSgTileSmem = 6 * sg::TB;

template <int MODE>
__global__ void __launch_bounds__(256, 1) k_sg_tile(SgTileArgs a)
{
    using namespace sg;
    extern __shared__ __align__(1024) unsigned char dsm[];
    unsigned char *wbuf = dsm, *fbuf = dsm + TB, *H1 = dsm + 2 * TB, *H2 = dsm + 3 * TB, *H3 = dsm + 4 * TB;
    unsigned char *gbuf = dsm + 5 * TB;
    __shared__ float bias[4][H], wo[H], red[4][2][H];
    // per row group (32 samples each) partial sums, added in a fixed order
    // at the end so that a tile's gradient is the same on every run
    __shared__ float colpart[4][4][H], cwopart[4][H], lpart[4], dpart[4];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tslot;
    const SgNet &n = a.net;
    const int tid = threadIdx.x, warp = tid >> 5, h = warp >> 2, r = (warp & 3) * 32 + (tid & 31);
    const int s_idx = blockIdx.x * 128 + r;
    const bool valid = s_idx < a.n;
    const int sc = valid ? s_idx : a.n - 1;

    if (warp == 0) tc::tmem_alloc(&tslot, 512);
    if (tid == 0) tc::mbar_init(&bar, 1);
    const int rg = warp & 3;  // row group of this warp
    for (int q = tid; q < H; q += blockDim.x) {
        for (int l = 0; l < 4; l++) bias[l][q] = n.P[OFF_B1 + l * H + q];
        wo[q] = n.P[OFF_WO + q];
    }
    const float vxs = a.xs[sc], vz = a.z[sc], vx = a.x[sc];
    const float u0 = (vxs - n.lo[0]) * n.sc[0] - 1.0f, u1 = (vz - n.lo[1]) * n.sc[1] - 1.0f;
    const float u2 = (vx - n.lo[2]) * n.sc[2] - 1.0f;
    __syncthreads();
    const uint32_t lane = (uint32_t)((warp & 3) * 32) << 16;
    const uint32_t D1 = tslot + lane, D2 = D1 + 128, D3 = D1 + 256, D4 = D1 + 384;
    const uint32_t T1 = tslot, T2 = tslot + 128, T3 = tslot + 256, T4 = tslot + 384;
    const uint32_t aW = tc::smem_u32(wbuf), aF = tc::smem_u32(fbuf), aH1 = tc::smem_u32(H1);
    const uint32_t aH2 = tc::smem_u32(H2), aH3 = tc::smem_u32(H3), aG = tc::smem_u32(gbuf);
    uint32_t phase = 0;
    bool ok = true;
    float *part = MODE == SG_TRAIN ? a.part + (size_t)blockIdx.x * PSTRIDE : nullptr;

    do {
        // layer 1, three feature chunks
        for (int c = 0; c < 3 && ok; c++) {
            sg_stage_w(wbuf, n.W + OFF_W1, FEAT, 128 * c);
            sg_features(fbuf, r, 32 * h, 32, c == 0 ? u0 : (c == 1 ? u1 : u2), n.fstep);
            sg_sync_for_mma();
            if (warp == 0 && tc::elect_one()) {
                tc::gemm(T1, aF, LBO_K, SBO_K, aW, LBO_K, SBO_K, 128, ID_KK, c > 0);
                tc::commit(&bar);
            }
            ok = sg_wait(&bar, phase);
        }
        if (!ok) break;
        sg_epi_silu(D1, bias[0], H1, r, 64 * h, 2);
        sg_stage_w(wbuf, n.W + OFF_W2, H, 0);
        sg_sync_for_mma();
        if (warp == 0 && tc::elect_one()) {
            tc::gemm(T2, aH1, LBO_K, SBO_K, aW, LBO_K, SBO_K, 128, ID_KK, false);
            tc::commit(&bar);
        }
        if (!(ok = sg_wait(&bar, phase))) break;
        sg_epi_silu(D2, bias[1], H2, r, 64 * h, 2);
        sg_stage_w(wbuf, n.W + OFF_W3, H, 0);
        sg_sync_for_mma();
        if (warp == 0 && tc::elect_one()) {
            tc::gemm(T3, aH2, LBO_K, SBO_K, aW, LBO_K, SBO_K, 128, ID_KK, false);
            tc::commit(&bar);
        }
        if (!(ok = sg_wait(&bar, phase))) break;
        sg_epi_silu(D3, bias[2], H3, r, 64 * h, 2);
        sg_stage_w(wbuf, n.W + OFF_W4, H, 0);
        sg_sync_for_mma();
        if (warp == 0 && tc::elect_one()) {
            tc::gemm(T4, aH3, LBO_K, SBO_K, aW, LBO_K, SBO_K, 128, ID_KK, false);
            tc::commit(&bar);
        }
        if (!(ok = sg_wait(&bar, phase))) break;

        if (MODE == SG_EVAL) sg_dump(a.stages, D4, r, h);
        // output layer
        float z4[64];
        {
            float part_out = 0.0f;
#pragma unroll
            for (int q = 0; q < 2; q++) {
                float v[32];
                tc::tmem_ld32(D4 + 64 * h + 32 * q, v);
#pragma unroll
                for (int jj = 0; jj < 32; jj++) {
                    const int c = 64 * h + 32 * q + jj;
                    z4[32 * q + jj] = v[jj] + bias[3][c];
                    part_out += sg_silu(z4[32 * q + jj]) * wo[c];
                }
            }
            red[0][h][r] = part_out;
        }
        __syncthreads();
        const float out = red[0][0][r] + red[0][1][r] + n.P[OFF_BO];
        float Tb, bxs, bz, bx, mfac;
        sg_background<float>(n, vxs, vz, vx, Tb, bxs, bz, bx);
        const float osc = sg_out_scale<float>(n, Tb, mfac);
        float gout = 1.0f;  // EVAL: d out / d out
        if (MODE == SG_TRAIN) {
            const float res = valid ? 1000.0f * (Tb + osc * out - a.Ttrue[sc]) : 0.0f;
            gout = 2.0f * res * 1000.0f * osc / (float)a.ntotal;
            if (h == 0) {
                float l = res * res / (float)a.ntotal, d = gout;
#pragma unroll
                for (int m = 16; m >= 1; m >>= 1) {
                    l += __shfl_xor_sync(0xffffffffu, l, m);
                    d += __shfl_xor_sync(0xffffffffu, d, m);
                }
                if ((tid & 31) == 0) {
                    lpart[rg] = l;
                    dpart[rg] = d;
                }
            }
        }
        // g4 = gout * wo * SiLU'(z4) -> gbuf; TRAIN: d wo, d b4 column sums
#pragma unroll
        for (int q = 0; q < 2; q++) {
            float g[32];
#pragma unroll
            for (int jj = 0; jj < 32; jj++) {
                const int c = 64 * h + 32 * q + jj;
                const float z = z4[32 * q + jj];
                g[jj] = __bfloat162float(__float2bfloat16_rn(gout * wo[c] * sg_dsilu(z)));
                if (MODE == SG_TRAIN) {
                    float hw = gout * sg_silu(z), gb = g[jj];
#pragma unroll
                    for (int m = 16; m >= 1; m >>= 1) {
                        hw += __shfl_xor_sync(0xffffffffu, hw, m);
                        gb += __shfl_xor_sync(0xffffffffu, gb, m);
                    }
                    if ((tid & 31) == 0) {
                        cwopart[rg][c] = hw;
                        colpart[3][rg][c] = gb;
                    }
                }
            }
#pragma unroll
            for (int g8 = 0; g8 < 4; g8++) sg_store8(gbuf, r, 64 * h + 32 * q + 8 * g8, g + 8 * g8);
        }
        // backward through layers 4..2: weight gradient (TRAIN), then data gradient
        // step k works on layer 4 - k: its accumulator columns, the previous
        // layer's, and that layer's input activations (H3, H2, H1 are
        // consecutive tiles).  Plain arithmetic, no per-thread index arrays.
        for (int k = 0; k < 3 && ok; k++) {
            const uint32_t Tk = T4 - 128u * k, Dk = D4 - 128u * k, Dpk = D3 - 128u * k;
            const uint32_t aHp = aH3 - (uint32_t)(TB * k);
            const int offW = OFF_W4 - k * H * H;
            if (MODE == SG_TRAIN) {
                sg_sync_for_mma();
                if (warp == 0 && tc::elect_one()) {
                    tc::gemm(Tk, aG, LBO_M, SBO_M, aHp, LBO_M, SBO_M, 128, ID_MM, false);
                    tc::commit(&bar);
                }
                if (!(ok = sg_wait(&bar, phase))) break;
                for (int q = 0; q < 2; q++) {
                    float v[32];
                    tc::tmem_ld32(Dk + 64 * h + 32 * q, v);
                    float4 *dst = reinterpret_cast<float4 *>(part + offW + (size_t)r * H + 64 * h + 32 * q);
#pragma unroll
                    for (int g4 = 0; g4 < 8; g4++)
                        dst[g4] = make_float4(v[4 * g4], v[4 * g4 + 1], v[4 * g4 + 2], v[4 * g4 + 3]);
                }
            }
            if (k > 0) sg_stage_w(wbuf, n.W + offW, H, 0);  // W4 is still staged for k = 0
            sg_sync_for_mma();
            if (warp == 0 && tc::elect_one()) {
                tc::gemm(Tk, aG, LBO_K, SBO_K, aW, LBO_M, SBO_M, 128, ID_KM, false);
                tc::commit(&bar);
            }
            if (!(ok = sg_wait(&bar, phase))) break;
            if (MODE == SG_EVAL) sg_dump(a.stages ? a.stages + (1 + k) * 16384 : nullptr, Dk, r, h);
            if (MODE == SG_EVAL && k == 0 && a.stages) {
                sg_dump_tile(a.stages + 5 * 16384, gbuf);
                sg_dump_tile(a.stages + 6 * 16384, wbuf);
            }
            sg_epi_back(Dk, Dpk, bias[2 - k], gbuf, r, 64 * h, 2, nullptr,
                        MODE == SG_TRAIN ? colpart[2 - k][rg] : nullptr);
        }
        if (!ok) break;
        // layer 1: weight gradient per feature chunk (TRAIN) or input gradient (EVAL)
        for (int c = 0; c < 3 && ok; c++) {
            if (MODE == SG_TRAIN) {
                sg_features(fbuf, r, 32 * h, 32, c == 0 ? u0 : (c == 1 ? u1 : u2), n.fstep);
                sg_sync_for_mma();
                if (warp == 0 && tc::elect_one()) {
                    tc::gemm(T1, aG, LBO_M, SBO_M, aF, LBO_M, SBO_M, 128, ID_MM, false);
                    tc::commit(&bar);
                }
                if (!(ok = sg_wait(&bar, phase))) break;
                for (int q = 0; q < 2; q++) {
                    float v[32];
                    tc::tmem_ld32(D1 + 64 * h + 32 * q, v);
                    float4 *dst =
                        reinterpret_cast<float4 *>(part + OFF_W1 + (size_t)r * FEAT + 128 * c + 64 * h + 32 * q);
#pragma unroll
                    for (int g4 = 0; g4 < 8; g4++)
                        dst[g4] = make_float4(v[4 * g4], v[4 * g4 + 1], v[4 * g4 + 2], v[4 * g4 + 3]);
                }
            } else {
                sg_stage_w(wbuf, n.W + OFF_W1, FEAT, 128 * c);
                sg_sync_for_mma();
                if (warp == 0 && tc::elect_one()) {
                    tc::gemm(T1, aG, LBO_K, SBO_K, aW, LBO_M, SBO_M, 128, ID_KM, false);
                    tc::commit(&bar);
                }
                if (!(ok = sg_wait(&bar, phase))) break;
                if (c == 0) sg_dump(a.stages ? a.stages + 4 * 16384 : nullptr, D1, r, h);
                red[1 + c][h][r] = sg_feature_grad(D1, 64 * h, 2, c == 0 ? u0 : (c == 1 ? u1 : u2), n.fstep);
            }
        }
        if (!ok) break;
        tc::fence_before();
        __syncthreads();
        if (MODE == SG_TRAIN) {
            for (int q = tid; q < H; q += blockDim.x) {
                for (int l = 0; l < 4; l++)
                    part[OFF_B1 + l * H + q] = ((colpart[l][0][q] + colpart[l][1][q]) + colpart[l][2][q]) + colpart[l][3][q];
                part[OFF_WO + q] = ((cwopart[0][q] + cwopart[1][q]) + cwopart[2][q]) + cwopart[3][q];
            }
            if (tid == 0) {
                part[OFF_BO] = ((dpart[0] + dpart[1]) + dpart[2]) + dpart[3];
                part[NPARAM] = ((lpart[0] + lpart[1]) + lpart[2]) + lpart[3];
            }
        } else if (h == 0 && valid) {
            const float gxs = (red[1][0][r] + red[1][1][r]) * n.sc[0];
            const float gz = (red[2][0][r] + red[2][1][r]) * n.sc[1];
            const float gx = (red[3][0][r] + red[3][1][r]) * n.sc[2];
            a.T[s_idx] = Tb + osc * out;
            a.Txs[s_idx] = bxs * (1.0f + mfac * out) + osc * gxs;
            a.Tz[s_idx] = bz * (1.0f + mfac * out) + osc * gz;
            a.Tx[s_idx] = bx * (1.0f + mfac * out) + osc * gx;
        }
    } while (false);
    if (!ok && tid == 0) atomicExch(a.status, 1);
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tslot, 512);
}

// Sum of the tiles' partial gradients in tile order (deterministic), then
// one Adam step on the FP32 parameters and their BF16 matrix copy; with
// lr = 0 only the summed gradient is written (grad_out, may be null).
__global__ void k_sg_adam(float *P, float *m, float *v, __nv_bfloat16 *Wb, const float *part, int ntiles, float lr,
                          float beta1, float beta2, float eps, float bc1, float bc2, float *grad_out, float *loss_out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > sg::NPARAM) return;
    float g = 0.0f;
    for (int t = 0; t < ntiles; t++) g += part[(size_t)t * sg::PSTRIDE + p];
    if (p == sg::NPARAM) {
        if (loss_out) *loss_out = g;
        return;
    }
    if (grad_out) grad_out[p] = g;
    if (lr == 0.0f) return;
    const float mm = beta1 * m[p] + (1.0f - beta1) * g;
    const float vv = beta2 * v[p] + (1.0f - beta2) * g * g;
    m[p] = mm;
    v[p] = vv;
    const float np = P[p] - lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
    P[p] = np;
    if (p < sg::NWB) Wb[p] = __float2bfloat16_rn(np);
}

__global__ void k_sg_pack(const float *P, __nv_bfloat16 *Wb)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < sg::NWB) Wb[p] = __float2bfloat16_rn(P[p]);
}

// uniform samples (position, depth, lateral) of a table volume [npos][nx][nz]
__device__ __forceinline__ uint64_t sg_mix(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__global__ void k_sg_sample(const float *table, int npos, float p0, float dp, int nz, int nx, float z0, float dz,
                            float x0, float dx, uint64_t seed, int B, float *xs, float *z, float *x, float *Tt)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const uint64_t hsh = sg_mix(seed ^ sg_mix((uint64_t)b));
    const int ip = (int)((hsh & 0xFFFFFull) % (uint64_t)npos);
    const int iz = (int)(((hsh >> 20) & 0xFFFFFull) % (uint64_t)nz);
    const int ix = (int)(((hsh >> 40) & 0xFFFFFFull) % (uint64_t)nx);
    xs[b] = p0 + (float)ip * dp;
    z[b] = z0 + (float)iz * dz;
    x[b] = x0 + (float)ix * dx;
    Tt[b] = table[((size_t)ip * nx + ix) * nz + iz];
}

static int launch_sg_fields(const SgNet &net, const LegInterp *legs, int nlegs, const kcig_geometry &g,
                            const kcig_params &p, LegFields out, int *status, int mode, cudaStream_t st)
{
    if (nlegs <= 0) return KCIG_OK;
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        KCIG_CUDA(cudaGetDevice(&dev));
        KCIG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    SgFieldArgs a;
    a.net = net;
    a.legs = legs;
    a.nlegs = nlegs;
    a.nz = g.nz;
    a.nx = g.nx;
    a.z0 = g.z0;
    a.dz = g.dz;
    a.x0 = g.x0;
    a.dx = g.dx;
    a.aper = p.aperture;
    a.aper_taper = p.aperture_taper;
    a.rmin = p.aperture_rmin;
    a.rtaper = p.aperture_rtaper;
    a.out = out;
    a.status = status;
    const long long items = (long long)nlegs * ((g.nz * g.nx + 127) / 128);
    const int grid = (int)std::min<long long>(sms, items);
    if (mode == SGF_T) {
        KCIG_TRY(set_dyn_smem((const void *)k_sg_fields<SGF_T>, kSgFieldSmem));
        k_sg_fields<SGF_T><<<grid, 512, kSgFieldSmem, st>>>(a);
    } else if (mode == SGF_TX) {
        KCIG_TRY(set_dyn_smem((const void *)k_sg_fields<SGF_TX>, kSgFieldSmem));
        k_sg_fields<SGF_TX><<<grid, 512, kSgFieldSmem, st>>>(a);
    } else {
        KCIG_TRY(set_dyn_smem((const void *)k_sg_fields<SGF_ALL>, kSgFieldSmem));
        k_sg_fields<SGF_ALL><<<grid, 512, kSgFieldSmem, st>>>(a);
    }
    KCIG_CUDA(cudaGetLastError());
    return KCIG_OK;
}

}  // namespace kcig

using namespace kcig;

extern "C" int kcig_tc_selftest(const void *X, const void *W, float *D, int *status, void *stream)
{
    if (!X || !W || !D || !status) return set_error(KCIG_ERR_ARG, "kcig_tc_selftest: null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    KCIG_CUDA(cudaMemsetAsync(status, 0, sizeof(int), st));
    const int smem = 2 * 128 * 128 * 2;
    KCIG_CUDA(cudaFuncSetAttribute(k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_tc_selftest<<<1, 128, smem, st>>>((const __nv_bfloat16 *)X, (const __nv_bfloat16 *)W, D, status);
    KCIG_CUDA(cudaGetLastError());
    KCIG_CUDA(cudaStreamSynchronize(st));
    return KCIG_OK;
}

// ================================================================ C ABI ==
struct kcig_surrogate {
    kcig_surrogate_config cfg;
    int device = 0;
    float *P = nullptr, *m = nullptr, *v = nullptr;  // [NPARAM]
    __nv_bfloat16 *Wb = nullptr;                     // [NWB]
    float *part = nullptr;                           // [tiles][PSTRIDE]
    size_t part_tiles = 0;
    float *batch = nullptr;                          // xs, z, x, Ttrue of one training batch
    size_t batch_cap = 0;
    float *scal = nullptr;                           // device scalars: loss
    int *status = nullptr;
    long long step = 0;                              // Adam steps taken
};

namespace kcig {

static SgNet sg_net(const kcig_surrogate *s);

int launch_surrogate_fields(kcig_surrogate *s, const LegInterp *legs, int nlegs, const kcig_geometry &g,
                            const kcig_params &p, LegFields out, int mode, cudaStream_t st)
{
    return launch_sg_fields(sg_net(s), legs, nlegs, g, p, out, s->status, mode, st);
}

int sg_reset_status(kcig_surrogate *s, cudaStream_t st)
{
    KCIG_CUDA(cudaMemsetAsync(s->status, 0, sizeof(int), st));
    return KCIG_OK;
}

static SgNet sg_net(const kcig_surrogate *s)
{
    SgNet n;
    n.W = s->Wb;
    n.P = s->P;
    for (int i = 0; i < 3; i++) {
        n.lo[i] = s->cfg.lo[i];
        n.sc[i] = 2.0f / (s->cfg.hi[i] - s->cfg.lo[i]);
    }
    n.fstep = 3.14159265358979f * s->cfg.fmax / (float)sg::NF;
    n.vref = s->cfg.vref;
    n.zsrc = s->cfg.zsrc;
    n.vgrad = s->cfg.vgrad;
    n.rscale = s->cfg.residual_ms * 1e-3f;
    return n;
}

int sg_device_check(const kcig_surrogate *s)
{
    int dev = -1;
    KCIG_CUDA(cudaGetDevice(&dev));
    if (dev != s->device) return set_error(KCIG_ERR_ARG, "surrogate: created on device %d, current device %d", s->device, dev);
    return KCIG_OK;
}

int sg_ensure_part(kcig_surrogate *s, size_t tiles)
{
    if (tiles <= s->part_tiles) return KCIG_OK;
    if (s->part) cudaFree(s->part);
    s->part = nullptr;
    s->part_tiles = 0;
    KCIG_CUDA(cudaMalloc(&s->part, tiles * sg::PSTRIDE * sizeof(float)));
    s->part_tiles = tiles;
    return KCIG_OK;
}

int sg_launch_tile(kcig_surrogate *s, int mode, const float *xs, const float *z, const float *x, const float *Tt, int n,
                   float *T, float *Txs, float *Tz, float *Tx, cudaStream_t st, float *stages = nullptr)
{
    SgTileArgs a;
    a.net = sg_net(s);
    a.xs = xs;
    a.z = z;
    a.x = x;
    a.Ttrue = Tt;
    a.n = n;
    a.ntotal = n;
    a.part = s->part;
    a.T = T;
    a.Txs = Txs;
    a.Tz = Tz;
    a.Tx = Tx;
    a.stages = stages;
    a.status = s->status;
    const int tiles = (n + 127) / 128;
    if (mode == SG_TRAIN) {
        KCIG_TRY(set_dyn_smem((const void *)k_sg_tile<SG_TRAIN>, kSgTileSmem));
        k_sg_tile<SG_TRAIN><<<tiles, 256, kSgTileSmem, st>>>(a);
    } else {
        KCIG_TRY(set_dyn_smem((const void *)k_sg_tile<SG_EVAL>, kSgTileSmem));
        k_sg_tile<SG_EVAL><<<tiles, 256, kSgTileSmem, st>>>(a);
    }
    KCIG_CUDA(cudaGetLastError());
    return KCIG_OK;
}

int sg_check_status(kcig_surrogate *s, cudaStream_t st)
{
    int h = 0;
    KCIG_CUDA(cudaMemcpyAsync(&h, s->status, sizeof(int), cudaMemcpyDeviceToHost, st));
    KCIG_CUDA(cudaStreamSynchronize(st));
    if (h) return set_error(KCIG_ERR_DEVICE, "surrogate: a tensor-core step did not complete");
    return KCIG_OK;
}

}  // namespace kcig

extern "C" int kcig_surrogate_nparams(void) { return sg::NPARAM; }

extern "C" int kcig_surrogate_create(const kcig_surrogate_config *cfg, unsigned long long seed, kcig_surrogate **out)
{
    if (!cfg || !out) return set_error(KCIG_ERR_ARG, "kcig_surrogate_create: null argument");
    *out = nullptr;
    for (int i = 0; i < 3; i++)
        if (!(cfg->hi[i] > cfg->lo[i])) return set_error(KCIG_ERR_ARG, "kcig_surrogate_create: need hi > lo on every input");
    if (!(cfg->vref > 0.0f) || !(cfg->fmax > 0.0f)) return set_error(KCIG_ERR_ARG, "kcig_surrogate_create: need vref > 0 and fmax > 0");
    if (!std::isfinite(cfg->vgrad) || !(cfg->residual_ms >= 0.0f))
        return set_error(KCIG_ERR_ARG, "kcig_surrogate_create: need a finite vgrad and residual_ms >= 0");
    kcig_surrogate *s = new kcig_surrogate();
    s->cfg = *cfg;
    int rc = KCIG_OK;
    cudaError_t e = cudaGetDevice(&s->device);
    if (e == cudaSuccess) e = cudaMalloc(&s->P, sg::NPARAM * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&s->m, sg::NPARAM * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&s->v, sg::NPARAM * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&s->Wb, sg::NWB * sizeof(__nv_bfloat16));
    if (e == cudaSuccess) e = cudaMalloc(&s->scal, 4 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&s->status, sizeof(int));
    if (e != cudaSuccess) rc = cuda_error(e, "kcig_surrogate_create");
    if (!rc) {
        // seeded initial parameters: uniform with the fan-in bound sqrt(6/fan_in)
        // for W_1..W_4, +-0.01 for the output weights, zero biases
        std::vector<float> p(sg::NPARAM, 0.0f);
        uint64_t st = seed * 0x9E3779B97F4A7C15ull + 0x1234567ull;
        auto next = [&]() {
            st ^= st >> 12;
            st ^= st << 25;
            st ^= st >> 27;
            return (double)((st * 2685821657736338717ull) >> 11) * (1.0 / 9007199254740992.0);
        };
        const int offs[4] = {sg::OFF_W1, sg::OFF_W2, sg::OFF_W3, sg::OFF_W4};
        const int fans[4] = {sg::FEAT, sg::H, sg::H, sg::H};
        for (int l = 0; l < 4; l++) {
            const double lim = std::sqrt(6.0 / fans[l]);
            for (int k = 0; k < sg::H * fans[l]; k++) p[offs[l] + k] = (float)((2.0 * next() - 1.0) * lim);
        }
        for (int k = 0; k < sg::H; k++) p[sg::OFF_WO + k] = (float)((2.0 * next() - 1.0) * 0.01);
        rc = kcig_surrogate_set_params(s, p.data());
    }
    if (rc) {
        kcig_surrogate_destroy(s);
        return rc;
    }
    *out = s;
    return KCIG_OK;
}

extern "C" void kcig_surrogate_destroy(kcig_surrogate *s)
{
    if (!s) return;
    cudaFree(s->P);
    cudaFree(s->m);
    cudaFree(s->v);
    cudaFree(s->Wb);
    cudaFree(s->part);
    cudaFree(s->batch);
    cudaFree(s->scal);
    cudaFree(s->status);
    delete s;
}

extern "C" int kcig_surrogate_set_params(kcig_surrogate *s, const float *params)
{
    if (!s || !params) return set_error(KCIG_ERR_ARG, "kcig_surrogate_set_params: null argument");
    KCIG_TRY(sg_device_check(s));
    KCIG_CUDA(cudaMemcpy(s->P, params, sg::NPARAM * sizeof(float), cudaMemcpyHostToDevice));
    KCIG_CUDA(cudaMemset(s->m, 0, sg::NPARAM * sizeof(float)));
    KCIG_CUDA(cudaMemset(s->v, 0, sg::NPARAM * sizeof(float)));
    k_sg_pack<<<(sg::NWB + 255) / 256, 256>>>(s->P, s->Wb);
    KCIG_CUDA(cudaGetLastError());
    KCIG_CUDA(cudaDeviceSynchronize());
    s->step = 0;
    return KCIG_OK;
}

extern "C" int kcig_surrogate_get_params(const kcig_surrogate *s, float *params)
{
    if (!s || !params) return set_error(KCIG_ERR_ARG, "kcig_surrogate_get_params: null argument");
    KCIG_TRY(sg_device_check(s));
    KCIG_CUDA(cudaMemcpy(params, s->P, sg::NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    return KCIG_OK;
}

extern "C" int kcig_surrogate_eval(kcig_surrogate *s, int n, const float *xs, const float *z, const float *x, float *T,
                                   float *dTdxs, float *dTdz, float *dTdx, void *stream)
{
    if (!s || n < 0 || (n > 0 && (!xs || !z || !x || !T || !dTdxs || !dTdz || !dTdx)))
        return set_error(KCIG_ERR_ARG, "kcig_surrogate_eval: bad arguments");
    if (n == 0) return KCIG_OK;
    KCIG_TRY(sg_device_check(s));
    cudaStream_t st = (cudaStream_t)stream;
    KCIG_CUDA(cudaMemsetAsync(s->status, 0, sizeof(int), st));
    KCIG_TRY(sg_launch_tile(s, SG_EVAL, xs, z, x, nullptr, n, T, dTdxs, dTdz, dTdx, st));
    return sg_check_status(s, st);
}

extern "C" int kcig_surrogate_eval_stages(kcig_surrogate *s, int n, const float *xs, const float *z, const float *x,
                                          float *stages, void *stream)
{
    if (!s || n < 1 || !xs || !z || !x || !stages) return set_error(KCIG_ERR_ARG, "kcig_surrogate_eval_stages: bad arguments");
    KCIG_TRY(sg_device_check(s));
    cudaStream_t st = (cudaStream_t)stream;
    float *tmp = nullptr;
    KCIG_CUDA(cudaMallocAsync(&tmp, 4 * (size_t)n * sizeof(float), st));
    KCIG_CUDA(cudaMemsetAsync(s->status, 0, sizeof(int), st));
    int rc = sg_launch_tile(s, SG_EVAL, xs, z, x, nullptr, n, tmp, tmp + n, tmp + 2 * n, tmp + 3 * n, st, stages);
    cudaFreeAsync(tmp, st);
    if (rc) return rc;
    return sg_check_status(s, st);
}

extern "C" int kcig_surrogate_loss_grad(kcig_surrogate *s, int n, const float *xs, const float *z, const float *x,
                                        const float *Ttrue, float *loss, float *grad, void *stream)
{
    if (!s || n < 1 || !xs || !z || !x || !Ttrue) return set_error(KCIG_ERR_ARG, "kcig_surrogate_loss_grad: bad arguments");
    KCIG_TRY(sg_device_check(s));
    cudaStream_t st = (cudaStream_t)stream;
    const int tiles = (n + 127) / 128;
    KCIG_TRY(sg_ensure_part(s, tiles));
    KCIG_CUDA(cudaMemsetAsync(s->status, 0, sizeof(int), st));
    KCIG_TRY(sg_launch_tile(s, SG_TRAIN, xs, z, x, Ttrue, n, nullptr, nullptr, nullptr, nullptr, st));
    k_sg_adam<<<(sg::NPARAM + 256) / 256, 256, 0, st>>>(s->P, s->m, s->v, s->Wb, s->part, tiles, 0.0f, 0.f, 0.f, 0.f,
                                                       1.f, 1.f, grad, s->scal);
    KCIG_CUDA(cudaGetLastError());
    if (loss) KCIG_CUDA(cudaMemcpyAsync(loss, s->scal, sizeof(float), cudaMemcpyDeviceToDevice, st));
    return sg_check_status(s, st);
}

extern "C" int kcig_surrogate_train(kcig_surrogate *s, const float *table, int npos, float p0, float dp, int nz, int nx,
                                    float z0, float dz, float x0, float dx, int steps, int batch, float lr,
                                    float lr_final, unsigned long long seed, float *losses, void *stream)
{
    if (!s || !table || npos < 1 || nz < 1 || nx < 1 || steps < 0 || batch < 128 || batch % 128 != 0 || !(lr > 0.0f))
        return set_error(KCIG_ERR_ARG, "kcig_surrogate_train: bad arguments (batch must be a positive multiple of 128)");
    KCIG_TRY(sg_device_check(s));
    cudaStream_t st = (cudaStream_t)stream;
    const int tiles = batch / 128;
    KCIG_TRY(sg_ensure_part(s, tiles));
    if ((size_t)batch > s->batch_cap) {
        if (s->batch) cudaFree(s->batch);
        s->batch = nullptr;
        s->batch_cap = 0;
        KCIG_CUDA(cudaMalloc(&s->batch, 4 * (size_t)batch * sizeof(float)));
        s->batch_cap = batch;
    }
    float *dloss = nullptr;
    if (losses && steps > 0) KCIG_CUDA(cudaMallocAsync(&dloss, steps * sizeof(float), st));
    KCIG_CUDA(cudaMemsetAsync(s->status, 0, sizeof(int), st));
    float *bx = s->batch, *bz = bx + batch, *bxx = bz + batch, *bt = bxx + batch;
    const float b1 = 0.9f, b2 = 0.999f;
    int rc = KCIG_OK;
    for (int k = 0; k < steps && rc == KCIG_OK; k++) {
        // cosine decay from lr to lr_final
        const double f = steps > 1 ? (double)k / (steps - 1) : 0.0;
        const float lrk = (float)(lr_final + 0.5 * (lr - lr_final) * (1.0 + std::cos(3.14159265358979 * f)));
        k_sg_sample<<<(batch + 255) / 256, 256, 0, st>>>(table, npos, p0, dp, nz, nx, z0, dz, x0, dx,
                                                         seed * 0x100000001B3ull + (uint64_t)s->step, batch, bx, bz,
                                                         bxx, bt);
        rc = sg_launch_tile(s, SG_TRAIN, bx, bz, bxx, bt, batch, nullptr, nullptr, nullptr, nullptr, st);
        if (rc) break;
        s->step++;
        const float bc1 = 1.0f - (float)std::pow(b1, (double)s->step), bc2 = 1.0f - (float)std::pow(b2, (double)s->step);
        k_sg_adam<<<(sg::NPARAM + 256) / 256, 256, 0, st>>>(s->P, s->m, s->v, s->Wb, s->part, tiles, lrk, b1, b2, 1e-8f,
                                                           bc1, bc2, nullptr, dloss ? dloss + k : nullptr);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_error(e, "k_sg_adam");
    }
    if (!rc && dloss) {
        cudaError_t e = cudaMemcpyAsync(losses, dloss, steps * sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) rc = cuda_error(e, "kcig_surrogate_train(losses)");
    }
    if (dloss) cudaFreeAsync(dloss, st);
    if (!rc) rc = sg_check_status(s, st);
    return rc;
}
