// Datuming between depth levels on the device: the frequency-domain
// Kirchhoff extrapolation of the reference's kirchdat2d_freq
// (src/kirchdat2d_frequency_cs.cpp) and the datum-depth slice of greensol_auto
// (src/greensol_auto.cpp).
//
// Layout in HBM.  After the forward transforms the spectra are kept
// frequency-major, U[iw][is][ih] (complex FP32): one ns x nh matrix per
// frequency.  For cmp = 0 the receiver operator is the same for every shot
// and the source operator the same for every receiver, so each side is one
// complex matrix product per frequency:
//     receiver side  Utmp[iw] = U[iw] . Kr[iw],   Kr[ic][ih]  (nh x nh)
//     source side    Uout[iw] = Ks[iw] . Utmp[iw], Ks[is][ic]  (ns x ns)
// (k_cgemm, batched over a chunk of frequencies, skipping the K tiles outside
// the aperture band).  The operators of a chunk are built on the device
// (k_dat_op): per term the weight of :508-523 (aperture taper, distance,
// tau) precomputed on the host in the reference's arithmetic, times the
// anti-aliasing weight (:197-226) and the filter H(tau, w) (:98-182), which is
// evaluated in FP64 with exact phase reduction (the reference's FP32 phase
// omega * m loses ~1e-3 rad at high frequencies).  For cmp = 1 the receiver
// operator moves with the shot and the source side walks common-receiver
// gathers (:556-619), so the sums run term by term (k_dat_rcv_cmp1,
// k_dat_src_cmp1) over per-chunk tables of aH for the table pairs they use.
// Transforms: cuFFT R2C / C2R of length nfft on batches of traces
// (k_dat_prep reverses, tapers and pads; k_dat_finish scales, reverses and
// trims), with tiled transposes between trace-major and frequency-major.
#include <cuda_runtime.h>
#include <cufft.h>
#include <math.h>

#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "kcig_common.h"
#include "kcig_tc.h"

namespace kcig {
namespace {

constexpr int kFilterMax = 64;  // filter samples kept in shared memory (longer filters recompute them)

struct DatEntry {
    float w;     // term weight before the anti-alias weight (0: no term)
    float tau;   // table traveltime of the term
    float dtau;  // |slope| x coordinate step, the anti-alias phase increment
};

struct DatOpArgs {
    const DatEntry *ent;
    int ne;
    float2 *out;  // [nf][ne]
    int f0, nf, nfft, K;
    float dt, antialias;
};

// antialias_weight_iw (:197-226), in the reference's float arithmetic, its
// per-term part (fnyq, fmax, fpass) taken once per term and the frequency
// iw / (nfft dt) once per chunk: the same float operations, the same weights.
// mode 1: the weight is 1 at every frequency; 0: 0 at iw > 0; 2: the taper
// between fpass and fmax
struct DatAa {
    int mode;
    float fpass, fmax, den;
};

__device__ __forceinline__ DatAa dat_aa_term(float antialias, float dtau, float dt)
{
    DatAa t{1, 0.0f, 0.0f, 0.0f};
    if (antialias <= 0.0f) return t;
    dtau = __fmul_rn(fabsf(dtau), antialias);
    if (dtau <= 1e-12f || !isfinite(dtau)) return t;
    const float fnyq = __fdiv_rn(0.5f, dt);
    const float fmax = __fdiv_rn(0.5f, dtau);
    if (fmax >= fnyq) return t;
    if (fmax <= 0.0f) {
        t.mode = 0;
        return t;
    }
    t.mode = 2;
    t.fmax = fmax;
    t.fpass = __fmul_rn(0.8f, fmax);
    t.den = __fsub_rn(fmax, t.fpass);
    return t;
}

// freq = iw / (nfft dt) as dat_aa forms it
__device__ __forceinline__ float dat_aa_at(const DatAa &t, int iw, float freq)
{
    if (t.mode == 1 || iw <= 0) return 1.0f;
    if (t.mode == 0) return 0.0f;
    if (freq <= t.fpass) return 1.0f;
    if (freq >= t.fmax) return 0.0f;
    const float x = __fdiv_rn(__fsub_rn(freq, t.fpass), t.den);
    return __fmul_rn(0.5f, __fadd_rn(1.0f, cospif(x)));
}

// sqrt(t^2 - 1) for t = 1 + u, written without the cancellation of t^2 - 1
__device__ __forceinline__ double dat_root(int j, double dt_over_tau)
{
    if (j < 0) return 0.0;
    const double u = (double)(j + 1) * dt_over_tau;
    return sqrt(u * (2.0 + u));
}

// One thread per operator term, looping over the chunk's frequencies:
// out[c][e] = w aa(iw) H(tau, iw), H = lin . sum_k F[k]/dt exp(-i w k) with
// F the second differences of sqrt(t^2 - 1) (build_filter_F, :98-116), lin =
// (1-delta) exp(-i w m) + delta exp(-i w (m-1)), m = ceil(tau/dt) (:128-181).
__global__ void __launch_bounds__(128) k_dat_op(const DatOpArgs a)
{
    extern __shared__ double zs[];  // [nf][2]: cos w, sin w of the chunk's frequencies; [nf] frequencies; filters
    float *fq = reinterpret_cast<float *>(zs + 2 * a.nf);
    const float fden = __fmul_rn((float)a.nfft, a.dt);
    for (int c = threadIdx.x; c < a.nf; c += blockDim.x) {
        double s, co;
        sincospi(2.0 * (double)(a.f0 + c) / (double)a.nfft, &s, &co);
        zs[2 * c] = co;
        zs[2 * c + 1] = s;
        fq[c] = __fdiv_rn((float)(a.f0 + c), fden);
    }
    __syncthreads();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.ne) return;
    const DatEntry d = a.ent[e];
    float2 *o = a.out + e;
    if (d.w == 0.0f || !(d.tau > 0.0f) || !isfinite(d.tau) || a.K <= 0) {
        for (int c = 0; c < a.nf; c++) o[(size_t)c * a.ne] = make_float2(0.0f, 0.0f);
        return;
    }
    const double r = (double)a.dt / (double)d.tau, inv_dt = 1.0 / (double)a.dt;
    const int K = a.K;
    // the filter samples in shared memory, F[128 k] of this thread (in a
    // local array they spilled past L1; 21 -> 17 ms at the benchmark size)
    const bool cached = K <= kFilterMax;
    double *F = reinterpret_cast<double *>(zs + 2 * a.nf + (a.nf + 1) / 2) + threadIdx.x;
    if (cached) {
        double p2 = 0.0, p1 = 0.0;
        for (int k = 0; k < K; k++) {
            const double ck = dat_root(k, r);
            F[128 * k] = (ck - 2.0 * p1 + p2) * inv_dt;
            p2 = p1;
            p1 = ck;
        }
    }
    const double q = (double)d.tau * inv_dt, mceil = ceil(q), delta = mceil - q;
    const long long m = (long long)mceil;
    const DatAa aa = dat_aa_term(a.antialias, d.dtau, a.dt);
    for (int c = 0; c < a.nf; c++) {
        const int iw = a.f0 + c;
        const float wa = __fmul_rn(d.w, dat_aa_at(aa, iw, fq[c]));
        if (fabsf(wa) < 1e-20f) {  // the reference skips these terms (:525)
            o[(size_t)c * a.ne] = make_float2(0.0f, 0.0f);
            continue;
        }
        const double zr = zs[2 * c], zi = zs[2 * c + 1];  // exp(-i w) = zr - i zi
        // Horner from the last filter sample down: S = ((F[K-1] z + F[K-2]) z + ...) z + F[0]
        double sr, si = 0.0;
        if (cached) {
            sr = F[128 * (K - 1)];
            for (int k = K - 2; k >= 0; k--) {
                const double tr = sr * zr + si * zi, ti = si * zr - sr * zi;
                sr = tr + F[128 * k];
                si = ti;
            }
        } else {  // long filters: the samples from three running roots
            double c0 = dat_root(K - 1, r), c1 = dat_root(K - 2, r), c2 = dat_root(K - 3, r);
            sr = (c0 - 2.0 * c1 + c2) * inv_dt;
            for (int k = K - 2; k >= 0; k--) {
                c0 = c1;
                c1 = c2;
                c2 = dat_root(k - 2, r);
                const double tr = sr * zr + si * zi, ti = si * zr - sr * zi;
                sr = tr + (c0 - 2.0 * c1 + c2) * inv_dt;
                si = ti;
            }
        }
        // exp(-i w m) with the phase reduced exactly: (iw m) mod nfft, nfft a
        // power of two and iw m >= 0
        const long long red = ((long long)iw * m) & (long long)(a.nfft - 1);
        float es, ec;
        sincospif(__fdiv_rn(2.0f * (float)red, (float)a.nfft), &es, &ec);
        const double lr = (1.0 - delta) + delta * zr, li = delta * zi;  // (1-delta) + delta exp(+i w)
        const double mr = (double)ec * lr + (double)es * li, mi = (double)ec * li - (double)es * lr;
        const double hr = mr * sr - mi * si, hi = mr * si + mi * sr;
        o[(size_t)c * a.ne] = make_float2((float)(wa * hr), (float)(wa * hi));
    }
}

// Batched complex GEMM, FP32: C[z] = A[z] . B[z] (row-major, complex
// interleaved), 64x64 tiles of C per CTA, 4x4 per thread, K in steps of 8.
// band >= 0: the nonzero terms satisfy |k - m| <= band (band_rows) or
// |k - n| <= band, so a tile reads only the K range that can touch it.
struct CGemmArgs {
    const float2 *A;
    const float2 *B;
    float2 *C;
    long long sA, sB, sC;  // batch strides (elements)
    int lda, ldb, ldc;
    int M, N, K;
    int band, band_rows;
    int a_trans;           // tensor-core kernel only: A(m, k) at A[k * lda + m]
    int a_vec;             // tensor-core kernel only: row-major A rows start on 16 bytes (lda, sA even)
};

__global__ void __launch_bounds__(256) k_cgemm(const CGemmArgs a)
{
    constexpr int BM = 64, BN = 64, BK = 8;
    __shared__ __align__(16) float2 As[BK][BM + 2];
    __shared__ __align__(16) float2 Bs[BK][BN + 2];
    const int z = blockIdx.z;
    const float2 *A = a.A + (size_t)z * a.sA;
    const float2 *B = a.B + (size_t)z * a.sB;
    float2 *C = a.C + (size_t)z * a.sC;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    int k_lo = 0, k_hi = a.K;
    if (a.band >= 0) {
        const int c0 = a.band_rows ? m0 : n0, c1 = (a.band_rows ? min(a.M, m0 + BM) : min(a.N, n0 + BN)) - 1;
        k_lo = max(0, c0 - a.band);
        k_hi = min(a.K, c1 + a.band + 1);
    }
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    float ar[4][4], ai[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) ar[i][j] = ai[i][j] = 0.0f;
    for (int k0 = k_lo; k0 < k_hi; k0 += BK) {
#pragma unroll
        for (int rr = 0; rr < 2; rr++) {
            const int e = tid + 256 * rr;
            const int mm = e >> 3, kk = e & 7, gm = m0 + mm, gk = k0 + kk;
            As[kk][mm] = (gm < a.M && gk < k_hi) ? A[(size_t)gm * a.lda + gk] : make_float2(0.0f, 0.0f);
            const int kb = e >> 6, nn = e & 63, gkb = k0 + kb, gn = n0 + nn;
            Bs[kb][nn] = (gkb < k_hi && gn < a.N) ? B[(size_t)gkb * a.ldb + gn] : make_float2(0.0f, 0.0f);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            const float4 a01 = *reinterpret_cast<const float4 *>(&As[kk][ty * 4]);
            const float4 a23 = *reinterpret_cast<const float4 *>(&As[kk][ty * 4 + 2]);
            const float4 b01 = *reinterpret_cast<const float4 *>(&Bs[kk][tx * 4]);
            const float4 b23 = *reinterpret_cast<const float4 *>(&Bs[kk][tx * 4 + 2]);
            const float xr[4] = {a01.x, a01.z, a23.x, a23.z}, xi[4] = {a01.y, a01.w, a23.y, a23.w};
            const float yr[4] = {b01.x, b01.z, b23.x, b23.z}, yi[4] = {b01.y, b01.w, b23.y, b23.w};
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    ar[i][j] = fmaf(xr[i], yr[j], ar[i][j]);
                    ar[i][j] = fmaf(-xi[i], yi[j], ar[i][j]);
                    ai[i][j] = fmaf(xr[i], yi[j], ai[i][j]);
                    ai[i][j] = fmaf(xi[i], yr[j], ai[i][j]);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int gm = m0 + ty * 4 + i;
        if (gm >= a.M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int gn = n0 + tx * 4 + j;
            if (gn < a.N) C[(size_t)gm * a.ldc + gn] = make_float2(ar[i][j], ai[i][j]);
        }
    }
}

// The same batched complex GEMM on the tensor cores (tcgen05, kind::tf32,
// accumulators in TMEM) with FP32 accuracy from three TF32 products:
// x = hi + lo (hi = TF32(x), lo = TF32(x - hi), both rounded to nearest),
// a.b ~ ah.bh + ah.bl + al.bh,
// the dropped al.bl and the TF32 rounding of lo being ~2^-22 relative.
// The complex product runs as four real products on separate real and
// imaginary planes of both operands: Cr = Ar.Br - Ai.Bi and Ci = Ar.Bi +
// Ai.Br, the minus by the instruction's negate-A bit, so no operand value is
// stored twice.  CTA tile: 128 rows x TNC complex columns (Cr and Ci each a
// 128 x TNC FP32 accumulator in TMEM); K in chunks of 8 complex through S
// pipeline stages, each holding the hi and lo of Ar, Ai (128 x 8) and Br, Bi
// (TNC x 8) in the canonical K-major layout.  Two groups of 8 producer warps
// take alternate chunks: each loads its next chunk while it splits and
// stores the current one; after the main loop all 16 warps read the
// accumulators out.  Warp 16 allocates TMEM and one of its lanes issues the
// MMAs (12 per chunk).  One CTA per SM.  Every mbarrier wait is bounded; a
// wait that gives up sets *status, and the CTA stops issuing work, waits
// (bounded) for its own MMAs and frees its TMEM.
#ifndef KCIG_CGEMM_TNC
#define KCIG_CGEMM_TNC 208  // complex columns of a CTA tile: 400 columns in two tiles (4% padding)
#endif
#ifndef KCIG_CGEMM_STAGES
#define KCIG_CGEMM_STAGES 4
#endif
namespace tcg {
constexpr int TM = 128, TNC = KCIG_CGEMM_TNC, KC = 8, S = KCIG_CGEMM_STAGES;
static_assert(TNC % 16 == 0 && TNC >= 16 && TNC <= 256, "an M = 128 MMA takes N = 16 .. 256 in steps of 16");
constexpr int TMEM_COLS = TNC <= 64 ? 128 : TNC <= 128 ? 256 : 512;  // Cr at column 0, Ci at TMEM_COLS / 2
constexpr int AK = TM * 16 + 32;                    // byte stride of an A plane's two k-groups (padded)
constexpr int BK = TNC * 16;                        // byte stride of a B plane's two k-groups
constexpr int A_PLANE = 2 * AK, B_PLANE = 2 * BK;   // one plane: 8 real k = two 16-byte k-groups
constexpr int STAGE = 4 * A_PLANE + 4 * B_PLANE;    // Ar, Ai, Br, Bi, each hi and lo
constexpr int SMEM = S * STAGE + 128;               // + barriers and slots
constexpr int PRODUCERS = 16;                       // warps
constexpr int THREADS = 32 * (PRODUCERS + 1);
constexpr int RB = (2 * TNC + 255) / 256;           // B items (column, k-group) per producer thread
static_assert(SMEM <= 227 * 1024, "shared memory of one CTA");
}  // namespace tcg

// a bounded mbarrier wait: at most 2^22 polls, each suspending the thread for
// up to 1 us (a few seconds in all; a tile's whole main loop takes ~20 us)
__device__ __forceinline__ bool dat_wait(uint64_t *bar, uint32_t parity)
{
    const uint32_t addr = tc::smem_u32(bar);
    for (uint32_t i = 0; i < (1u << 22); i++) {
        uint32_t ready;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ready)
            : "r"(addr), "r"(parity), "r"(1000u)
            : "memory");
        if (ready) return true;
    }
    return false;
}

// x rounded to 10 mantissa bits (half an ulp added to the magnitude's bits,
// the low 13 bits cleared): the TF32 value nearest x, on the integer pipes
__device__ __forceinline__ float tf32_round(float x)
{
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

__device__ __forceinline__ void tc_store_split(uint8_t *hi, uint8_t *lo, uint32_t off, float4 v)
{
    float4 h, l;
    h.x = tf32_round(v.x);
    h.y = tf32_round(v.y);
    h.z = tf32_round(v.z);
    h.w = tf32_round(v.w);
    l.x = tf32_round(v.x - h.x);
    l.y = tf32_round(v.y - h.y);
    l.z = tf32_round(v.z - h.z);
    l.w = tf32_round(v.w - h.w);
    *reinterpret_cast<float4 *>(hi + off) = h;
    *reinterpret_cast<float4 *>(lo + off) = l;
}

// the real parts and the imaginary parts of four complex values, split into
// TF32 hi / lo, into one 16-byte row segment of the four planes re_hi, re_lo,
// im_hi, im_lo (`plane` bytes apart, in that order)
__device__ __forceinline__ void tc_store_planes(uint8_t *base, int plane, uint32_t off, const float2 *v)
{
    tc_store_split(base, base + plane, off, make_float4(v[0].x, v[1].x, v[2].x, v[3].x));
    tc_store_split(base + 2 * plane, base + 3 * plane, off, make_float4(v[0].y, v[1].y, v[2].y, v[3].y));
}

__global__ void __launch_bounds__(tcg::THREADS, 1) k_cgemm_tc(const CGemmArgs a, int *status)
{
    using namespace tcg;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + S * STAGE);
    uint64_t *empty = full + S;
    uint64_t *done = empty + S;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(done + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tslot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int z = blockIdx.z;
    const float2 *A = a.A + (size_t)z * a.sA;
    const float2 *B = a.B + (size_t)z * a.sB;
    float2 *C = a.C + (size_t)z * a.sC;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TNC;
    int k_lo = 0, k_hi = a.K;
    if (a.band >= 0) {
        const int c0 = a.band_rows ? m0 : n0, c1 = (a.band_rows ? min(a.M, m0 + TM) : min(a.N, n0 + TNC)) - 1;
        // even start (16-byte loads of A cover k, k+1); the terms added below
        // the band have zero operator entries
        k_lo = max(0, c0 - a.band) & ~1;
        k_hi = min(a.K, c1 + a.band + 1);
    }
    const int nchunks = k_hi > k_lo ? (k_hi - k_lo + KC - 1) / KC : 0;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            tc::mbar_init(&full[s], 8);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(done, 1);
        *abort_flag = 0;
    }
    if (warp == PRODUCERS) tc::tmem_alloc(tslot, TMEM_COLS);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tslot;

    if (warp < PRODUCERS) {
        // ---- producers: group g (warps 8g .. 8g+7) stores chunks g, g+2, ...
        // into stage i % S.  A item: (row t % 128, k-group t / 128), four
        // complex k; B item e: (column e % TNC, k-group e / TNC), four complex k
        const int g = warp >> 3, t = threadIdx.x & 255;
        struct Chunk {
            float2 a[4], b[RB][4];
        };
        const int arow = t & 127, aj = t >> 7;
        auto load = [&](int i, Chunk &c) {
            const int k0 = k_lo + i * KC + 4 * aj;  // even
            const int gm = m0 + arow;
#pragma unroll
            for (int q = 0; q < 4; q++) c.a[q] = make_float2(0.0f, 0.0f);
            if (gm < a.M) {
                if (a.a_trans) {
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        if (k0 + q < k_hi) c.a[q] = A[(size_t)(k0 + q) * a.lda + gm];
                } else {
                    const float2 *src = A + (size_t)gm * a.lda + k0;
                    if (a.a_vec && k0 + 3 < k_hi) {  // two 16-byte loads
                        const float4 p = *reinterpret_cast<const float4 *>(src);
                        const float4 r = *reinterpret_cast<const float4 *>(src + 2);
                        c.a[0] = make_float2(p.x, p.y);
                        c.a[1] = make_float2(p.z, p.w);
                        c.a[2] = make_float2(r.x, r.y);
                        c.a[3] = make_float2(r.z, r.w);
                    } else {
#pragma unroll
                        for (int q = 0; q < 4; q++)
                            if (k0 + q < k_hi) c.a[q] = src[q];
                    }
                }
            }
#pragma unroll
            for (int rr = 0; rr < RB; rr++) {
                const int e = t + 256 * rr, j = e / TNC, n = e - j * TNC, gn = n0 + n;
                const int kb = k_lo + i * KC + 4 * j;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    c.b[rr][q] = make_float2(0.0f, 0.0f);
                    if (e < 2 * TNC && gn < a.N && kb + q < k_hi) c.b[rr][q] = B[(size_t)(kb + q) * a.ldb + gn];
                }
            }
        };
        // group g takes chunks g, g+2, g+4, ...: the loads of its next chunk
        // are issued before the current one is split and stored
        Chunk nxt;
        if (g < nchunks) load(g, nxt);
        for (int i = g; i < nchunks; i += 2) {
            const int slot = i % S;
            const Chunk c = nxt;
            if (i + 2 < nchunks) load(i + 2, nxt);
            if (i >= S && !dat_wait(&empty[slot], ((i / S) - 1) & 1)) {
                atomicExch(status, 1);
                *abort_flag = 1;
            }
            if (__any_sync(0xffffffffu, *abort_flag)) break;  // warp-uniform, as the arrival below is per warp
            uint8_t *st = smem + slot * STAGE;
            // row r of a plane, k-group j: j * stride + (r / 8) * 128 + (r % 8) * 16
            tc_store_planes(st, A_PLANE, (uint32_t)(aj * AK + (arow >> 3) * 128 + (arow & 7) * 16), c.a);
#pragma unroll
            for (int rr = 0; rr < RB; rr++) {
                const int e = t + 256 * rr, j = e / TNC, n = e - j * TNC;
                if (e < 2 * TNC)
                    tc_store_planes(st + 4 * A_PLANE, B_PLANE, (uint32_t)(j * BK + (n >> 3) * 128 + (n & 7) * 16),
                                    c.b[rr]);
            }
            tc::fence_async_smem();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&full[slot]);
        }
    } else if (lane == 0) {
        // ---- MMA issuer: Cr += Ar.Br - Ai.Bi, Ci += Ar.Bi + Ai.Br, three
        // TF32 products each
        const uint32_t id = tc::idesc_tf32(TM, TNC), id_neg = id | (1u << 13);  // bit 13: negate A
        const uint32_t Dr = tmem, Di = tmem + TMEM_COLS / 2;
        for (int i = 0; i < nchunks; i++) {
            const int slot = i % S;
            if (!dat_wait(&full[slot], (i / S) & 1)) {
                atomicExch(status, 2);
                *abort_flag = 1;
            }
            if (*abort_flag) break;
            tc::fence_after();
            const uint32_t st = tc::smem_u32(smem + slot * STAGE), sb = st + 4 * A_PLANE;
            const uint64_t arh = tc::sdesc(st, AK, 128), arl = tc::sdesc(st + A_PLANE, AK, 128);
            const uint64_t aih = tc::sdesc(st + 2 * A_PLANE, AK, 128), ail = tc::sdesc(st + 3 * A_PLANE, AK, 128);
            const uint64_t brh = tc::sdesc(sb, BK, 128), brl = tc::sdesc(sb + B_PLANE, BK, 128);
            const uint64_t bih = tc::sdesc(sb + 2 * B_PLANE, BK, 128), bil = tc::sdesc(sb + 3 * B_PLANE, BK, 128);
            const uint32_t acc = i > 0 ? 1u : 0u;
            tc::mma_tf32(Dr, arh, brh, id, acc);
            tc::mma_tf32(Dr, arh, brl, id, 1u);
            tc::mma_tf32(Dr, arl, brh, id, 1u);
            tc::mma_tf32(Dr, aih, bih, id_neg, 1u);
            tc::mma_tf32(Dr, aih, bil, id_neg, 1u);
            tc::mma_tf32(Dr, ail, bih, id_neg, 1u);
            tc::mma_tf32(Di, arh, bih, id, acc);
            tc::mma_tf32(Di, arh, bil, id, 1u);
            tc::mma_tf32(Di, arl, bih, id, 1u);
            tc::mma_tf32(Di, aih, brh, id, 1u);
            tc::mma_tf32(Di, aih, brl, id, 1u);
            tc::mma_tf32(Di, ail, brh, id, 1u);
            tc::commit(&empty[slot]);
        }
        tc::commit(done);  // tracks every MMA issued, also after an abort
    }
    __syncwarp();
    // ---- epilogue: warps 0-15 read the accumulators; warp w owns TMEM lanes
    // 32 (w % 4) .. +31 and a quarter of the columns, 32 at a time
    bool ok = true;
    if (warp < PRODUCERS || lane == 0) ok = dat_wait(done, 0);
    if (!ok) atomicExch(status, 3);
    if (warp < PRODUCERS) {
        tc::fence_after();
        constexpr int QC = (TNC / 4 + 31) / 32 * 32;  // columns per quarter, whole 32-column loads
        const int q = warp & 3, quarter = warp >> 2;
        const int gm = m0 + 32 * q + lane;
        const uint32_t lanes = (uint32_t)(32 * q) << 16;
        const bool live = __all_sync(0xffffffffu, ok && !*abort_flag);  // warp-uniform: TMEM loads are collective
        for (int cb = 0; cb < QC; cb += 32) {
            const int c0 = quarter * QC + cb;
            if (c0 >= TNC) break;  // the accumulators' unused columns
            float vr[32], vi[32];
            if (nchunks > 0 && live) {
                tc::tmem_ld32(tmem + lanes + c0, vr);
                tc::tmem_ld32(tmem + lanes + TMEM_COLS / 2 + c0, vi);
            } else {
#pragma unroll
                for (int c = 0; c < 32; c++) vr[c] = vi[c] = 0.0f;
            }
            if (gm < a.M && live) {
                float2 *dst = C + (size_t)gm * a.ldc + n0 + c0;
#pragma unroll
                for (int c = 0; c < 32; c++)
                    if (c0 + c < TNC && n0 + c0 + c < a.N) dst[c] = make_float2(vr[c], vi[c]);
            }
        }
    }
    tc::fence_before();
    __syncthreads();
    if (warp == PRODUCERS) tc::tmem_free(tmem, TMEM_COLS);
}

// cmp = 1 receiver side (:493-546 with s_abs = s0 + is ds): one thread per
// (frequency, shot, trace), the sum over the aperture of
// geom[ih][ic] tau (aH)[pair], pair = (table row cc = cabs[is][ic], column
// c = cabs[is][ih]) looked up in the chunk's band table P[c][row][j],
// j = c - cc + band.
struct RcvCmp1Args {
    const float2 *U;   // [nf][ns][nh] (the chunk's input spectra)
    float2 *Utmp;      // [nf][ns][nh]
    const float2 *P;   // [nf][nrow * (2 band + 1)]
    const float *Ptau; // [nrow * (2 band + 1)]
    const int *cabs;   // [ns][nh]
    const float *geom; // [nh][nh]
    int ns, nh, aper, band, row0, nrow;
    long long sU;      // U batch stride
};

__global__ void __launch_bounds__(128) k_dat_rcv_cmp1(const RcvCmp1Args a)
{
    const int tr = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
    const int ntr = a.ns * a.nh;
    if (tr >= ntr) return;
    const int is = tr / a.nh, ih = tr - is * a.nh;
    const float2 *U = a.U + (size_t)c * a.sU + (size_t)is * a.nh;
    const int wid = 2 * a.band + 1;
    const float2 *P = a.P + (size_t)c * a.nrow * wid;
    const int cih = a.cabs[tr];
    float sr = 0.0f, si = 0.0f;
    const int left = max(0, ih - a.aper), right = min(a.nh - 1, ih + a.aper);
    for (int ic = left; ic <= right; ic++) {
        const float g = a.geom[(size_t)ih * a.nh + ic];
        if (g == 0.0f) continue;
        const int cc = a.cabs[(size_t)is * a.nh + ic];
        const size_t pi = (size_t)(cc - a.row0) * wid + (cih - cc + a.band);
        const float w = __fmul_rn(g, a.Ptau[pi]);
        const float2 h = P[pi], u = U[ic];
        sr = fmaf(w, u.x * h.x - u.y * h.y, sr);
        si = fmaf(w, u.x * h.y + u.y * h.x, si);
    }
    a.Utmp[(size_t)c * ntr + tr] = make_float2(sr, si);
}

// cmp = 1 source side (:556-619): one thread per (frequency, shot); it walks
// the common-receiver gathers r that hold the shot (ir in [ir_lo, ir_hi]),
// and adds the sum over the gather's neighbouring shots to its own trace
// ih(r) of the output, so every output row has one writer and a fixed order.
struct SrcCmp1Args {
    const float2 *Utmp;  // [nf][ns][nh]
    float2 *Uout;        // [nf][ns][nh] (zeroed)
    const float2 *P;     // [nf][ns][ns]: aH of pair (c_s[ic], c_s[is]) at [is][ic]
    const float *Ptau;   // [ns][ns]
    const int *sleft, *sright;  // [nr] the gather's shot range
    const int *ihmap;    // [nr][ns]: trace of shot is in gather r, -1 outside
    const int *ir_lo, *ir_hi;   // [ns]
    int ns, nh, nr, aper, jump, tap;
    float ds, sdatum;
    long long sUout;
};

__device__ __forceinline__ float dat_taper(int left, int center, int right, int tap, int stride)
{
    if (center < left || center > right) return 0.0f;
    if (tap <= 0) return 1.0f;
    if (stride < 1) stride = 1;
    const float width = __fmul_rn((float)tap, (float)stride);
    const float ul = fminf(1.0f, fmaxf(0.0f, __fdiv_rn((float)(center - left), width)));
    const float ur = fminf(1.0f, fmaxf(0.0f, __fdiv_rn((float)(right - center), width)));
    return __fmul_rn(__fmul_rn(__fmul_rn(0.5f, __fsub_rn(1.0f, cospif(ul))), 0.5f), __fsub_rn(1.0f, cospif(ur)));
}

__global__ void __launch_bounds__(128) k_dat_src_cmp1(const SrcCmp1Args a)
{
    const int is = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
    if (is >= a.ns) return;
    const int ntr = a.ns * a.nh;
    const float2 *Ut = a.Utmp + (size_t)c * ntr;
    float2 *Uo = a.Uout + (size_t)c * a.sUout + (size_t)is * a.nh;
    const float2 *P = a.P + (size_t)c * a.ns * a.ns + (size_t)is * a.ns;
    const float *Pt = a.Ptau + (size_t)is * a.ns;
    const double kw = (double)a.ds * (double)a.sdatum / 3.14159265358979323846;
    for (int ir = a.ir_lo[is]; ir <= a.ir_hi[is]; ir++) {
        const int sl = a.sleft[ir], sr = a.sright[ir];
        if (is < sl || is > sr || (is - sl) % a.jump) continue;
        const int ih = a.ihmap[(size_t)ir * a.ns + is];
        if (ih < 0) continue;
        const int il = max(sl, is - a.jump * a.aper), iu = min(sr, is + a.jump * a.aper);
        float accr = 0.0f, acci = 0.0f;
        for (int ic = il; ic <= iu; ic += a.jump) {
            const int hh = a.ihmap[(size_t)ir * a.ns + ic];
            if (hh < 0) continue;
            const float coef = dat_taper(il, ic, iu, a.tap, a.jump);
            const float dist = __fadd_rn(__fmul_rn(a.sdatum, a.sdatum),
                                         __fmul_rn(__fmul_rn((float)((ic - is) * (ic - is)), a.ds), a.ds));
            const float w = (float)((double)coef * kw * (double)Pt[ic] / (double)dist);
            const float2 h = P[ic], u = Ut[(size_t)ic * a.nh + hh];
            accr = fmaf(w, u.x * h.x - u.y * h.y, accr);
            acci = fmaf(w, u.x * h.y + u.y * h.x, acci);
        }
        float2 o = Uo[ih];
        o.x += accr;
        o.y += acci;
        Uo[ih] = o;
    }
}

// reverse in time, edge taper and zero-pad one batch of traces (:287-306):
// a thread writes four consecutive samples of a padded trace (one 16-byte
// store; nfft is a power of two >= 4), up to 1024 block rows walk the
// batch's traces (several traces per block: ~10 waves at full size)
__global__ void k_dat_prep(const float *in, const float *wtr, float *pad, int tr0, int nb, int nt, int nfft)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (nfft >> 2)) return;
    for (int b = blockIdx.y; b < nb; b += gridDim.y) {
        const float w = wtr[tr0 + b];
        const float *src = in + (size_t)(tr0 + b) * nt + (nt - 1);  // src[-t]: sample nt - 1 - t
        float v[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int t = 4 * q + j;
            float x = 0.0f;
            if (t < nt) {
                const float y = src[-t];
                x = w == 1.0f ? y : __fmul_rn(w, y);
            }
            v[j] = x;
        }
        reinterpret_cast<float4 *>(pad + (size_t)b * nfft)[q] = make_float4(v[0], v[1], v[2], v[3]);
    }
}

// scale by 1/nfft, optionally reverse, trim to nt (:476-487): threads along
// the output samples, up to 1024 block rows walk the batch's traces
__global__ void k_dat_finish(const float *pad, float *out, int tr0, int nb, int nt, int nfft, float scale, int reverse)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const int ts = reverse ? nt - 1 - t : t;
    for (int b = blockIdx.y; b < nb; b += gridDim.y)
        out[(size_t)(tr0 + b) * nt + t] = __fmul_rn(pad[(size_t)b * nfft + ts], scale);
}

// tiled transposes between spec[b][nw] (a batch of traces) and U[iw][ntr]
__global__ void k_dat_to_fmajor(const float2 *spec, float2 *U, int tr0, int nb, int nw, int ntr)
{
    __shared__ float2 tile[32][33];
    const int w0 = blockIdx.x * 32, b0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int b = b0 + r, w = w0 + threadIdx.x;
        if (b < nb && w < nw) tile[r][threadIdx.x] = spec[(size_t)b * nw + w];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int w = w0 + r, b = b0 + threadIdx.x;
        if (b < nb && w < nw) U[(size_t)w * ntr + tr0 + b] = tile[threadIdx.x][r];
    }
}

__global__ void k_dat_to_tmajor(const float2 *U, float2 *spec, int tr0, int nb, int nw, int ntr)
{
    __shared__ float2 tile[32][33];
    const int w0 = blockIdx.y * 32, b0 = blockIdx.x * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int w = w0 + r, b = b0 + threadIdx.x;
        if (b < nb && w < nw) tile[r][threadIdx.x] = U[(size_t)w * ntr + tr0 + b];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int b = b0 + r, w = w0 + threadIdx.x;
        if (b < nb && w < nw) spec[(size_t)b * nw + w] = tile[threadIdx.x][r];
    }
}

__global__ void k_green_gather(const float *table, const int *ix, float *out, int ngx, int nx, int nz, int idatum)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ngx * ngx) return;
    const int i1 = i / ngx, i2 = i - i1 * ngx;
    out[i] = table[((size_t)i1 * nx + ix[i2]) * nz + idatum];
}

// ------------------------------------------------------------ host side --

// the reference's float arithmetic for indices and weights (x86-64 SSE, no
// contraction): every operation below rounds to float as it does there
inline int f2i(float x) { return (int)x; }

float taper_host(int left, int center, int right, int tap, int stride)  // taper_weight (:229-240)
{
    if (center < left || center > right) return 0.0f;
    if (tap <= 0) return 1.0f;
    if (stride < 1) stride = 1;
    const float width = (float)tap * (float)stride;
    const float ul = fminf(1.0f, fmaxf(0.0f, (float)(center - left) / width));
    const float ur = fminf(1.0f, fmaxf(0.0f, (float)(right - center) / width));
    return 0.5f * (1.0f - cosf((float)M_PI * ul)) * 0.5f * (1.0f - cosf((float)M_PI * ur));
}

float edge_host(int i, int n, int tap)  // data_edge_taper_weight (:255-279)
{
    if (tap <= 0 || n <= 1) return 1.0f;
    int ntap = tap;
    const int max_tap = (n - 1) / 2;
    if (ntap > max_tap) ntap = max_tap;
    if (ntap <= 0) return 1.0f;
    if (i < ntap) return 0.5f * (1.0f - cosf((float)M_PI * ((float)i / (float)ntap)));
    if (i > n - 1 - ntap) return 0.5f * (1.0f - cosf((float)M_PI * ((float)(n - 1 - i) / (float)ntap)));
    return 1.0f;
}

float slope_host(const float *t, int n, int row, int col, float dcoord)  // :184-194, t[row][col] row-major n x n
{
    if (n <= 1 || dcoord == 0.0f) return 0.0f;
    if (row <= 0) return (t[(size_t)1 * n + col] - t[col]) / dcoord;
    if (row >= n - 1) return (t[(size_t)(n - 1) * n + col] - t[(size_t)(n - 2) * n + col]) / dcoord;
    return 0.5f * (t[(size_t)(row + 1) * n + col] - t[(size_t)(row - 1) * n + col]) / dcoord;
}

int rcv_index(const kcig_datum_params &p, int is, int ih)  // :502, :507
{
    const float s = p.cmp ? p.s0 + (float)is * p.ds : 0.0f;
    return f2i((s + p.h0 + (float)ih * p.dh - p.rg0) / p.drg + 0.5f);
}

int src_index(const kcig_datum_params &p, int is)  // :583, :638
{
    return f2i((p.s0 + (float)is * p.ds - p.sg0) / p.dsg + 0.5f);
}

// w = coef / M_PI * d * datum * tau / dist, in double as written, then float
float term_weight(float coef, float d, float datum, float tau, float dist)
{
    return (float)(coef / M_PI * d * datum * tau / dist);
}

struct Stage {
    cudaEvent_t ev[6] = {};
};

thread_local float g_last_ms[5] = {0, 0, 0, 0, 0};
thread_local int g_last_launches = 0;

struct DBuf {
    void *p = nullptr;
    ~DBuf()
    {
        if (p) cudaFree(p);
    }
    template <class T>
    T *as() const
    {
        return (T *)p;
    }
};

int dalloc(DBuf &b, size_t bytes, const char *what)
{
    if (bytes == 0) bytes = 16;
    const cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return set_error(KCIG_ERR_NOMEM, "kcig_green_slice: cannot allocate %.3f GB for %s on the device",
                         bytes / 1e9, what);
    }
    return KCIG_OK;
}

template <class T>
int upload(DBuf &b, const std::vector<T> &v, cudaStream_t st, const char *what)
{
    KCIG_TRY(dalloc(b, v.size() * sizeof(T), what));
    if (!v.empty()) KCIG_CUDA(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return KCIG_OK;
}

int cufft_error(cufftResult r, const char *what)
{
    return set_error(KCIG_ERR_CUDA, "%s failed: cufftResult %d", what, (int)r);
}

// ---- device buffers and transform plans kept between calls
// The spectra alone take nw x traces x 8 bytes (10.5 GB for 400 x 400
// traces and 8193 frequencies); allocating them, planning the transforms and
// freeing it all again cost a fifth of a call.  One cache per device, held
// by a call for its whole run (kcig_datum_freq is synchronous on its
// stream), so calls on one device from several threads run one after the
// other.  Buffers only grow.  A call that cannot allocate frees every cached
// buffer and tries once more; kcig_datum_release frees a device's cache.
enum CacheSlot {
    CB_U,       // spectra, frequency-major [nw][ntr]
    CB_UFULL,   // receiver-side spectra kept for interm
    CB_UT,      // receiver-side spectra of one chunk of frequencies
    CB_KR,      // receiver operator of one chunk
    CB_KS,      // source operator of one chunk
    CB_PAD,     // one batch of padded traces
    CB_SPEC,    // one batch of trace-major spectra
    CB_WORK,    // cuFFT work area, shared by the four plans
    CB_IN,      // host-memory calls: the input, output and interm cubes
    CB_OUT,
    CB_INTERM,
    CB_STATUS,  // tensor-core GEMM status word
    CB_WTR,     // uploads: trace weights, operator entries, cmp = 1 walk tables
    CB_RCV,
    CB_SRC,
    CB_CABS,
    CB_GEOM,
    CB_RTAU,
    CB_STAU,
    CB_SL,
    CB_SR,
    CB_IHM,
    CB_IRL,
    CB_IRH,
    CB_COUNT
};

const char *const kSlotName[CB_COUNT] = {
    "the spectra", "the receiver-side spectra", "the receiver-side chunk", "the receiver operator",
    "the source operator", "the transform buffer", "the transform buffer", "the transform work area",
    "the input traces", "the output traces", "the intermediate traces", "a status word", "trace weights",
    "receiver terms", "source terms", "receiver indices", "receiver weights", "receiver pair times",
    "source pair times", "gather ranges", "gather ranges", "gather traces", "gather ranges", "gather ranges"};

struct CBuf {
    void *p = nullptr;
    size_t n = 0;
    template <class T>
    T *as() const
    {
        return (T *)p;
    }
};

// an R2C / C2R plan pair of one transform length and batch
struct FftPair {
    cufftHandle f = 0, b = 0;
    bool ok = false;
    int nfft = 0, batch = 0;
    size_t work = 0;
};

struct DatumCache {
    std::mutex mu;
    CBuf buf[CB_COUNT];
    FftPair full, tail;
    std::vector<cudaEvent_t> ev;
    cudaStream_t copy = nullptr;  // host-memory calls: the cubes' copies, batch by batch
};

std::mutex g_caches_mu;
std::map<int, DatumCache *> g_caches;  // never destroyed: the process exit or kcig_datum_release frees them

DatumCache &cache_of(int dev)
{
    std::lock_guard<std::mutex> g(g_caches_mu);
    DatumCache *&c = g_caches[dev];
    if (!c) c = new DatumCache;
    return *c;
}

void free_buffers(DatumCache &c)
{
    for (CBuf &b : c.buf) {
        if (b.p) cudaFree(b.p);
        b = CBuf{};
    }
}

void free_pair(FftPair &q)
{
    if (q.ok) {
        cufftDestroy(q.f);
        cufftDestroy(q.b);
    }
    q = FftPair{};
}

// the plan pair for (nfft, batch), work area left to the caller
int make_pair(FftPair &q, int nfft, int nw, int batch)
{
    if (q.ok && q.nfft == nfft && q.batch == batch) return KCIG_OK;
    free_pair(q);
    cufftResult cr;
    if ((cr = cufftCreate(&q.f)) != CUFFT_SUCCESS) return cufft_error(cr, "cufftCreate");
    if ((cr = cufftCreate(&q.b)) != CUFFT_SUCCESS) {
        cufftDestroy(q.f);
        q = FftPair{};
        return cufft_error(cr, "cufftCreate");
    }
    q.ok = true;
    int n = nfft;
    size_t wf = 0, wb = 0;
    if ((cr = cufftSetAutoAllocation(q.f, 0)) != CUFFT_SUCCESS || (cr = cufftSetAutoAllocation(q.b, 0)) != CUFFT_SUCCESS) {
        free_pair(q);
        return cufft_error(cr, "cufftSetAutoAllocation");
    }
    if ((cr = cufftMakePlanMany(q.f, 1, &n, nullptr, 1, nfft, nullptr, 1, nw, CUFFT_R2C, batch, &wf)) != CUFFT_SUCCESS) {
        free_pair(q);
        return cufft_error(cr, "cufftPlanMany (R2C)");
    }
    if ((cr = cufftMakePlanMany(q.b, 1, &n, nullptr, 1, nw, nullptr, 1, nfft, CUFFT_C2R, batch, &wb)) != CUFFT_SUCCESS) {
        free_pair(q);
        return cufft_error(cr, "cufftPlanMany (C2R)");
    }
    q.nfft = nfft;
    q.batch = batch;
    q.work = std::max(wf, wb);
    return KCIG_OK;
}

// every slot at least need[slot] bytes (0: not used by this call)
int ensure_buffers(DatumCache &c, const size_t *need)
{
    for (int attempt = 0; attempt < 2; attempt++) {
        int bad = -1;
        for (int i = 0; i < CB_COUNT && bad < 0; i++) {
            CBuf &b = c.buf[i];
            if (need[i] == 0 || b.n >= need[i]) continue;
            if (b.p) cudaFree(b.p);
            b = CBuf{};
            if (cudaMalloc(&b.p, need[i]) != cudaSuccess) {
                cudaGetLastError();
                b.p = nullptr;
                bad = i;
            } else {
                b.n = need[i];
            }
        }
        if (bad < 0) return KCIG_OK;
        free_buffers(c);
        if (attempt == 1)
            return set_error(KCIG_ERR_NOMEM, "kcig_datum_freq: cannot allocate %.3f GB for %s on the device",
                             need[bad] / 1e9, kSlotName[bad]);
    }
    return KCIG_OK;
}

template <class T>
size_t upload_bytes(const std::vector<T> &v)
{
    return std::max<size_t>(16, v.size() * sizeof(T));
}

template <class T>
int upload_to(const CBuf &b, const std::vector<T> &v, cudaStream_t st)
{
    if (!v.empty()) KCIG_CUDA(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return KCIG_OK;
}

int validate(const kcig_datum_params &p)
{
    if (p.cmp != 0 && p.cmp != 1) return set_error(KCIG_ERR_ARG, "cmp must be 0 or 1.");
    if (p.bf_p <= 0 || p.bf_n_leaf <= 1) return set_error(KCIG_ERR_ARG, "Need bf_p > 0 and bf_n_leaf > 1.");
    if (p.bf_p >= p.bf_n_leaf)
        return set_error(KCIG_ERR_ARG,
                         "Need bf_p < bf_n_leaf for meaningful butterfly interpolation / exact leaf-stage settings.");
    if (p.data_taper < 0) return set_error(KCIG_ERR_ARG, "data_taper must be >= 0.");
    if (!(p.antialias >= 0.0f)) return set_error(KCIG_ERR_ARG, "antialias must be >= 0.");
    if (p.nt <= 0 || p.nh <= 0 || p.ns <= 0 || p.nsg <= 0 || p.nrg <= 0)
        return set_error(KCIG_ERR_ARG, "kcig_datum_freq: sizes must be positive");
    if (!(p.dt > 0.0f)) return set_error(KCIG_ERR_ARG, "kcig_datum_freq: dt must be positive");
    if ((long long)p.ns * p.nh > 0x7fffffffLL) return set_error(KCIG_ERR_ARG, "kcig_datum_freq: too many traces");
    return KCIG_OK;
}

int sizes(const kcig_datum_params &p, const float *st, const float *rt, int *nsam_out, int *nfft_out)
{
    const float ratio = p.length / p.dt;
    if (!(fabsf(ratio) < 1e8f)) return set_error(KCIG_ERR_ARG, "kcig_datum_freq: length / dt out of range");
    const int nsam = f2i(ratio) + 2;
    float max_tau = 0.0f;  // choose_nfft (:82-96)
    for (size_t i = 0; i < (size_t)p.nrg * p.nrg; i++)
        if (rt[i] > max_tau) max_tau = rt[i];
    for (size_t i = 0; i < (size_t)p.nsg * p.nsg; i++)
        if (st[i] > max_tau) max_tau = st[i];
    const float steps = ceilf(max_tau / p.dt);
    if (!(steps < 5e8f)) return set_error(KCIG_ERR_ARG, "kcig_datum_freq: table traveltimes too long for an FFT");
    const long long need = (long long)p.nt + (long long)steps + (nsam - 2) + 2;
    long long n = 1;
    while (n < need) n <<= 1;
    if (n > (1LL << 30)) return set_error(KCIG_ERR_ARG, "kcig_datum_freq: nfft %lld too large", n);
    *nsam_out = nsam;
    *nfft_out = (int)n;
    return KCIG_OK;
}

// Operator terms of one side in the reference's arithmetic.  Dense matrices
// of DatEntry: receiver (cmp 0) at [ic][ih] (the K x N operand), source
// (cmp 0) at [is][ic]; for cmp = 1, the band table of receiver pairs and the
// source pair matrix, whose entries carry w = 1 (the geometric factor is
// applied by the sums).
struct Host {
    std::vector<DatEntry> rcv, src;
    // cmp = 1 receiver side
    std::vector<int> cabs;        // [ns][nh]
    std::vector<float> geom, rtau;  // [nh][nh], [nrow][2 band + 1]
    int band = 0, row0 = 0, nrow = 0;
    // cmp = 1 source side
    std::vector<float> stau;  // [ns][ns]
    std::vector<int> sleft, sright, ihmap, ir_lo, ir_hi;
    int nr = 0, jump = 1;
};

int build_receiver(const kcig_datum_params &p, const float *rt, Host &h)
{
    const int nh = p.nh, ns = p.ns, aper = p.aperture, nrg = p.nrg;
    if (p.cmp == 0) {
        h.rcv.assign((size_t)nh * nh, DatEntry{0.0f, 0.0f, 0.0f});
        for (int ih = 0; ih < nh; ih++) {
            const int c = rcv_index(p, 0, ih);
            const int left = std::max(0, ih - aper), right = std::min(nh - 1, ih + aper);
            for (int ic = left; ic <= right; ic++) {
                const int cc = rcv_index(p, 0, ic);
                if (c < 0 || c >= nrg || cc < 0 || cc >= nrg) return set_error(KCIG_ERR_ARG, "Receiver table too small.");
                const float coef = taper_host(left, ic, right, p.taper, 1);
                const float tau = rt[(size_t)cc * nrg + c];
                const float dist = p.rdatum * p.rdatum + (float)((ic - ih) * (ic - ih)) * p.dh * p.dh;
                DatEntry &e = h.rcv[(size_t)ic * nh + ih];
                e.w = term_weight(coef, p.dh, p.rdatum, tau, dist);
                e.tau = tau;
                e.dtau = slope_host(rt, nrg, cc, c, p.drg) * fabsf(p.dh);
            }
        }
        return KCIG_OK;
    }
    h.cabs.resize((size_t)ns * nh);
    int lo = 0x7fffffff, hi = -0x7fffffff - 1;
    for (int is = 0; is < ns; is++)
        for (int ih = 0; ih < nh; ih++) {
            const int c = rcv_index(p, is, ih);
            h.cabs[(size_t)is * nh + ih] = c;
            if (aper >= 0 && (c < 0 || c >= nrg)) return set_error(KCIG_ERR_ARG, "Receiver table too small.");
            lo = std::min(lo, c);
            hi = std::max(hi, c);
        }
    h.geom.assign((size_t)nh * nh, 0.0f);
    int band = 0;
    for (int ih = 0; ih < nh; ih++) {
        const int left = std::max(0, ih - aper), right = std::min(nh - 1, ih + aper);
        for (int ic = left; ic <= right; ic++) {
            const float coef = taper_host(left, ic, right, p.taper, 1);
            const float dist = p.rdatum * p.rdatum + (float)((ic - ih) * (ic - ih)) * p.dh * p.dh;
            h.geom[(size_t)ih * nh + ic] = (float)(coef / M_PI * p.dh * p.rdatum / dist);
        }
        for (int is = 0; is < ns && left <= right; is++) {
            const int c = h.cabs[(size_t)is * nh + ih];
            band = std::max(band, std::abs(c - h.cabs[(size_t)is * nh + left]));
            band = std::max(band, std::abs(c - h.cabs[(size_t)is * nh + right]));
        }
    }
    if (aper < 0 || lo > hi) {
        lo = hi = 0;
    }
    h.band = band;
    h.row0 = lo;
    h.nrow = hi - lo + 1;
    const int wid = 2 * band + 1;
    h.rcv.assign((size_t)h.nrow * wid, DatEntry{0.0f, 0.0f, 0.0f});
    h.rtau.assign((size_t)h.nrow * wid, 0.0f);
    for (int r = 0; r < h.nrow; r++)
        for (int j = 0; j < wid; j++) {
            const int cc = h.row0 + r, c = cc + j - band;
            if (cc < 0 || cc >= nrg || c < 0 || c >= nrg) continue;
            DatEntry &e = h.rcv[(size_t)r * wid + j];
            e.w = 1.0f;
            e.tau = rt[(size_t)cc * nrg + c];
            e.dtau = slope_host(rt, nrg, cc, c, p.drg) * fabsf(p.dh);
            h.rtau[(size_t)r * wid + j] = e.tau;
        }
    return KCIG_OK;
}

int build_source(const kcig_datum_params &p, const float *st, Host &h)
{
    const int ns = p.ns, nh = p.nh, aper = p.aperture, nsg = p.nsg;
    std::vector<int> cs(ns);
    for (int is = 0; is < ns; is++) cs[is] = src_index(p, is);
    if (p.cmp == 0) {
        h.src.assign((size_t)ns * ns, DatEntry{0.0f, 0.0f, 0.0f});
        for (int is = 0; is < ns; is++) {
            const int c = cs[is];
            if (c < 0 || c >= nsg) return set_error(KCIG_ERR_ARG, "Source table too small.");
            const int left = std::max(0, is - aper), right = std::min(ns - 1, is + aper);
            for (int ic = left; ic <= right; ic++) {
                const int cc = cs[ic];
                if (cc < 0 || cc >= nsg) return set_error(KCIG_ERR_ARG, "Source table too small.");
                const float coef = taper_host(left, ic, right, p.taper, 1);
                const float tau = st[(size_t)cc * nsg + c];
                const float dist = p.sdatum * p.sdatum + (float)((ic - is) * (ic - is)) * p.ds * p.ds;
                DatEntry &e = h.src[(size_t)is * ns + ic];
                e.w = term_weight(coef, p.ds, p.sdatum, tau, dist);
                e.tau = tau;
                e.dtau = slope_host(st, nsg, cc, c, p.dsg) * fabsf(p.ds);
            }
        }
        return KCIG_OK;
    }
    // the common-receiver walk (:556-579), in float as the reference
    const float ds = p.ds, dh = p.dh;
    const float s = fabsf((float)(ns - 1) * ds), hl = fabsf((float)(nh - 1) * dh);
    const bool wide = fabsf(ds) >= fabsf(dh);
    const int jump = wide ? 1 : f2i(dh / ds + 0.5f);
    const float dr = wide ? fabsf(dh) : fabsf(ds);
    const int nr = f2i((s + hl) / dr + 1.5f);
    if (jump < 1) return set_error(KCIG_ERR_ARG, "kcig_datum_freq: cmp=1 needs dh / ds >= 1 when |ds| < |dh|");
    if (nr < 0 || (long long)nr * ns > 0x7fffffffLL) return set_error(KCIG_ERR_ARG, "kcig_datum_freq: cmp=1 gather count");
    h.nr = nr;
    h.jump = jump;
    h.sleft.resize(nr);
    h.sright.resize(nr);
    h.ihmap.assign((size_t)nr * ns, -1);
    h.ir_lo.assign(ns, 0);
    h.ir_hi.assign(ns, -1);
    const float as = ds <= 0.f ? -1.f : 0.f, ah = dh <= 0.f ? -1.f : 0.f, bl = ds <= 0.f ? 0.f : -1.f;
    for (int ir = 0; ir < nr; ir++) {
        const float r = (float)ir * dr + as * s + ah * hl;
        int sl = f2i(((float)ir * dr + as * s + bl * hl) / ds + 0.5f);
        int sr = f2i(((float)ir * dr + as * s + as * hl) / ds + 0.5f);
        if (sl < 0) sl = 0;
        if (sr > ns - 1) sr = ns - 1;
        const int left = f2i((r - (float)sl * ds) / dh + 0.5f);
        if (left < 0 || left > nh - 1) sl++;
        const int right = f2i((r - (float)sr * ds) / dh + 0.5f);
        if (right < 0 || right > nh - 1) sr--;
        h.sleft[ir] = sl;
        h.sright[ir] = sr;
        for (int is = sl; is <= sr; is += jump) {
            if (is < 0 || is >= ns) continue;
            const int c = cs[is];
            if (c < 0 || c >= nsg) return set_error(KCIG_ERR_ARG, "Source table too small.");
            const int ih = f2i((r - (float)is * ds) / dh + 0.5f);
            h.ihmap[(size_t)ir * ns + is] = (ih >= 0 && ih < nh) ? ih : -1;
            if (h.ir_hi[is] < h.ir_lo[is]) h.ir_lo[is] = ir;
            h.ir_hi[is] = ir;
        }
    }
    h.src.assign((size_t)ns * ns, DatEntry{0.0f, 0.0f, 0.0f});
    h.stau.assign((size_t)ns * ns, 0.0f);
    const float jds = fabsf((float)jump * ds);
    for (int is = 0; is < ns; is++)
        for (int ic = std::max(0, is - jump * aper); ic <= std::min(ns - 1, is + jump * aper); ic++) {
            const int c = cs[is], cc = cs[ic];
            if (c < 0 || c >= nsg || cc < 0 || cc >= nsg) continue;
            DatEntry &e = h.src[(size_t)is * ns + ic];
            e.w = 1.0f;
            e.tau = st[(size_t)cc * nsg + c];
            e.dtau = slope_host(st, nsg, cc, c, p.dsg) * jds;
            h.stau[(size_t)is * ns + ic] = e.tau;
        }
    return KCIG_OK;
}

int launch_op(const DatEntry *ent, int ne, float2 *out, int f0, int nf, int nfft, int K, const kcig_datum_params &p,
              cudaStream_t st, int &launches)
{
    if (ne <= 0) return KCIG_OK;
    DatOpArgs a;
    a.ent = ent;
    a.ne = ne;
    a.out = out;
    a.f0 = f0;
    a.nf = nf;
    a.nfft = nfft;
    a.K = K;
    a.dt = p.dt;
    a.antialias = p.antialias;
    // shared memory: cos, sin and frequency of the chunk's frequencies, then
    // each thread's filter samples (128 threads)
    const size_t sm = (size_t)nf * 2 * sizeof(double) + (size_t)(nf + 1) / 2 * sizeof(double) +
                      (size_t)std::min(K, kFilterMax) * 128 * sizeof(double);
    KCIG_TRY(set_dyn_smem((const void *)k_dat_op, (int)sm));
    k_dat_op<<<(ne + 127) / 128, 128, sm, st>>>(a);
    launches++;
    KCIG_CUDA(cudaGetLastError());
    return KCIG_OK;
}

int launch_gemm(const float2 *A, long long sA, int lda, const float2 *B, long long sB, int ldb, float2 *C,
                long long sC, int ldc, int M, int N, int K, int band, int band_rows, int batch, cudaStream_t st,
                int &launches)
{
    CGemmArgs g;
    g.a_trans = 0;
    g.a_vec = 0;
    g.A = A;
    g.B = B;
    g.C = C;
    g.sA = sA;
    g.sB = sB;
    g.sC = sC;
    g.lda = lda;
    g.ldb = ldb;
    g.ldc = ldc;
    g.M = M;
    g.N = N;
    g.K = K;
    g.band = band;
    g.band_rows = band_rows;
    for (int z0 = 0; z0 < batch; z0 += 65535) {
        const int nz = std::min(65535, batch - z0);
        CGemmArgs gz = g;
        gz.A += (size_t)z0 * sA;
        gz.B += (size_t)z0 * sB;
        gz.C += (size_t)z0 * sC;
        k_cgemm<<<dim3((N + 63) / 64, (M + 63) / 64, nz), 256, 0, st>>>(gz);
        launches++;
        KCIG_CUDA(cudaGetLastError());
    }
    return KCIG_OK;
}

int launch_gemm_tc(const float2 *A, long long sA, int lda, const float2 *B, long long sB, int ldb, float2 *C,
                   long long sC, int ldc, int M, int N, int K, int band, int band_rows, int batch, int *status,
                   cudaStream_t st, int &launches, int a_trans = 0)
{
    CGemmArgs g;
    g.a_trans = a_trans;
    g.a_vec = !a_trans && lda % 2 == 0 && sA % 2 == 0 && ((uintptr_t)A & 15) == 0;
    g.A = A;
    g.B = B;
    g.C = C;
    g.sA = sA;
    g.sB = sB;
    g.sC = sC;
    g.lda = lda;
    g.ldb = ldb;
    g.ldc = ldc;
    g.M = M;
    g.N = N;
    g.K = K;
    g.band = band;
    g.band_rows = band_rows;
    KCIG_TRY(set_dyn_smem((const void *)k_cgemm_tc, tcg::SMEM));
    for (int z0 = 0; z0 < batch; z0 += 65535) {
        const int nz = std::min(65535, batch - z0);
        CGemmArgs gz = g;
        gz.A += (size_t)z0 * sA;
        gz.B += (size_t)z0 * sB;
        gz.C += (size_t)z0 * sC;
        k_cgemm_tc<<<dim3((N + tcg::TNC - 1) / tcg::TNC, (M + tcg::TM - 1) / tcg::TM, nz), tcg::THREADS, tcg::SMEM, st>>>(
            gz, status);
        launches++;
        KCIG_CUDA(cudaGetLastError());
    }
    return KCIG_OK;
}

// the GEMMs of cmp = 0 run on the tensor cores; KCIG_DATUM_GEMM=simt selects
// the FP32 CUDA-core kernel instead (a diagnostic comparison)
bool gemm_on_tensor_cores()
{
    const char *e = getenv("KCIG_DATUM_GEMM");
    return !(e && strcmp(e, "simt") == 0);
}

// traces per transform batch: as many as keep a batch's padded traces at
// 1 GB, or KCIG_DATUM_BATCH (smaller batches and a tail batch on small cases)
long long transform_batch(long long ntr, int nfft)
{
    long long b = ((long long)1 << 28) / nfft;
    const char *e = getenv("KCIG_DATUM_BATCH");
    if (e && atoll(e) > 0) b = std::min(b, atoll(e));
    return std::max<long long>(1, std::min<long long>(ntr, b));
}

}  // namespace
}  // namespace kcig

using namespace kcig;

extern "C" int kcig_datum_params_init(kcig_datum_params *p)
{
    if (!p) return set_error(KCIG_ERR_ARG, "kcig_datum_params_init: null");
    *p = kcig_datum_params{};
    p->aperture = 50;
    p->taper = 10;
    p->data_taper = 0;
    p->cmp = 1;
    p->antialias = 1.0f;
    p->length = 0.025f;
    p->use_bf = 1;
    p->bf_p = 12;
    p->bf_n_leaf = 16;
    p->bf_panel_levels = 1;
    p->bf_amp_eps = 1e-20f;
    p->bf_phase_tol = 2.0f;
    return KCIG_OK;
}

extern "C" int kcig_datum_sizes(const kcig_datum_params *p, const float *stable, const float *rtable, int *nsam,
                                int *nfft)
{
    if (!p || !stable || !rtable || !nsam || !nfft) return set_error(KCIG_ERR_ARG, "kcig_datum_sizes: null argument");
    KCIG_TRY(validate(*p));
    return sizes(*p, stable, rtable, nsam, nfft);
}

extern "C" int kcig_datum_release(void)
{
    int dev = 0;
    KCIG_CUDA(cudaGetDevice(&dev));
    DatumCache &c = cache_of(dev);
    std::lock_guard<std::mutex> hold(c.mu);
    free_buffers(c);
    free_pair(c.full);
    free_pair(c.tail);
    for (cudaEvent_t e : c.ev) cudaEventDestroy(e);
    c.ev.clear();
    if (c.copy) cudaStreamDestroy(c.copy);
    c.copy = nullptr;
    return KCIG_OK;
}

extern "C" int kcig_datum_last_timing(float *ms5, int *launches)
{
    if (ms5)
        for (int i = 0; i < 5; i++) ms5[i] = g_last_ms[i];
    if (launches) *launches = g_last_launches;
    return KCIG_OK;
}

extern "C" int kcig_green_slice(const float *table, int nz, int nx, int ngx, float oz, float ox, float dz, float dx,
                                float ogx, float dgx, float datum, float *tgreen, int memory, void *stream)
{
    if (!table || !tgreen || nz <= 0 || nx <= 0 || ngx <= 0) return set_error(KCIG_ERR_ARG, "kcig_green_slice: bad arguments");
    if (memory != KCIG_MEM_HOST && memory != KCIG_MEM_DEVICE) return set_error(KCIG_ERR_ARG, "kcig_green_slice: bad memory kind");
    // src/greensol_auto.cpp:68-69 and :75-82: float operands, double 0.5
    const int idatum = (int)((datum - oz) / dz + 0.5);
    if (idatum < 0 || idatum >= nz) return set_error(KCIG_ERR_ARG, "Datum out of range.");
    std::vector<int> ix(ngx);
    for (int i = 0; i < ngx; i++) {
        const float gx = ogx + (float)i * dgx;
        ix[i] = (int)((gx - ox) / dx + 0.5);
        if (ix[i] < 0 || ix[i] >= nx) return set_error(KCIG_ERR_ARG, "Receiver table too small.");
    }
    if (memory == KCIG_MEM_HOST) {
        for (int i1 = 0; i1 < ngx; i1++)
            for (int i2 = 0; i2 < ngx; i2++)
                tgreen[(size_t)i1 * ngx + i2] = table[((size_t)i1 * nx + ix[i2]) * nz + idatum];
        return KCIG_OK;
    }
    cudaStream_t st = (cudaStream_t)stream;
    DBuf dix;
    KCIG_TRY(upload(dix, ix, st, "table indices"));
    const int n = ngx * ngx;
    k_green_gather<<<(n + 255) / 256, 256, 0, st>>>(table, dix.as<int>(), tgreen, ngx, nx, nz, idatum);
    KCIG_CUDA(cudaGetLastError());
    KCIG_CUDA(cudaStreamSynchronize(st));
    return KCIG_OK;
}

extern "C" int kcig_datum_freq(const kcig_datum_params *pp, const float *stable, const float *rtable, const float *in,
                               float *out, float *interm, int memory, void *stream)
{
    if (!pp || !stable || !rtable || !in || !out) return set_error(KCIG_ERR_ARG, "kcig_datum_freq: null argument");
    if (memory != KCIG_MEM_HOST && memory != KCIG_MEM_DEVICE) return set_error(KCIG_ERR_ARG, "kcig_datum_freq: bad memory kind");
    const kcig_datum_params p = *pp;
    KCIG_TRY(validate(p));
    cudaStream_t st = (cudaStream_t)stream;
    // host copies of the tables (indices, weights and nfft are decided there)
    std::vector<float> sth, rth;
    const float *stp = stable, *rtp = rtable;
    if (memory == KCIG_MEM_DEVICE) {
        sth.resize((size_t)p.nsg * p.nsg);
        rth.resize((size_t)p.nrg * p.nrg);
        KCIG_CUDA(cudaMemcpyAsync(sth.data(), stable, sth.size() * 4, cudaMemcpyDeviceToHost, st));
        KCIG_CUDA(cudaMemcpyAsync(rth.data(), rtable, rth.size() * 4, cudaMemcpyDeviceToHost, st));
        KCIG_CUDA(cudaStreamSynchronize(st));
        stp = sth.data();
        rtp = rth.data();
    }
    int nsam = 0, nfft = 0;
    KCIG_TRY(sizes(p, stp, rtp, &nsam, &nfft));
    if (nfft < 4) return set_error(KCIG_ERR_ARG, "kcig_datum_freq: transform length %d below 4", nfft);
    const int nw = nfft / 2 + 1, K = nsam - 1;
    const int ns = p.ns, nh = p.nh, nt = p.nt;
    const long long ntr = (long long)ns * nh;
    Host h;
    KCIG_TRY(build_receiver(p, rtp, h));  // the receiver side's checks come first, as in the reference
    KCIG_TRY(build_source(p, stp, h));
    // cmp = 0 with shots and receivers on the same positions, tables and
    // datums: Ks[a][b] == Kr[b][a] term for term, so one operator serves both
    // sides (the source side reads it transposed) and is built once
    bool shared_op = p.cmp == 0 && ns == nh && gemm_on_tensor_cores();
    for (size_t a0 = 0; shared_op && a0 < (size_t)ns; a0++)
        for (size_t b0 = 0; b0 < (size_t)ns; b0++) {
            const DatEntry &x = h.src[a0 * ns + b0], &y = h.rcv[b0 * nh + a0];
            if (memcmp(&x, &y, sizeof(DatEntry)) != 0) {
                shared_op = false;
                break;
            }
        }
    std::vector<float> wtr((size_t)ntr);
    for (int is = 0; is < ns; is++) {
        const float ws = edge_host(is, ns, p.data_taper);
        for (int ih = 0; ih < nh; ih++) wtr[(size_t)is * nh + ih] = ws * edge_host(ih, nh, p.data_taper);
    }

    // ---- device buffers and transform plans, kept between calls on this device
    int dev = 0;
    KCIG_CUDA(cudaGetDevice(&dev));
    DatumCache &c = cache_of(dev);
    std::lock_guard<std::mutex> hold(c.mu);
    // declared after the lock: on every return the stream is idle before
    // the next call may reuse the buffers
    struct StreamIdle {
        cudaStream_t s, s2;
        ~StreamIdle()
        {
            cudaStreamSynchronize(s);
            if (s2) cudaStreamSynchronize(s2);
        }
    } idle{st, nullptr};
    int launches = 0;
    const size_t spec_bytes = (size_t)nw * ntr * sizeof(float2);
    const bool tcore = gemm_on_tensor_cores();
    // per-frequency bytes of a chunk: Utmp + both operators
    const size_t op_r = h.rcv.size(), op_s = shared_op ? 0 : h.src.size();
    const size_t per_f = (interm ? 0 : (size_t)ntr * sizeof(float2)) + (op_r + op_s) * sizeof(float2);
    int chunk = (int)std::max<size_t>(1, std::min<size_t>(256, ((size_t)1536 << 20) / std::max<size_t>(per_f, 1)));
    chunk = std::min(chunk, nw);
    // transform batches
    const int B = (int)transform_batch(ntr, nfft);
    const int tail = (int)(ntr % B);
    // plans first (their work area is sized with the buffers); a plan that
    // does not fit beside the cached buffers gets a second try without them
    for (int attempt = 0;; attempt++) {
        int rc = make_pair(c.full, nfft, nw, B);
        if (rc == KCIG_OK && tail) rc = make_pair(c.tail, nfft, nw, tail);
        if (rc == KCIG_OK) break;
        if (attempt == 1) return rc;
        free_buffers(c);
    }
    size_t need[CB_COUNT] = {};
    need[CB_U] = spec_bytes;
    if (interm)
        need[CB_UFULL] = spec_bytes;
    else
        need[CB_UT] = (size_t)chunk * ntr * sizeof(float2);
    need[CB_KR] = (size_t)chunk * std::max<size_t>(op_r, 1) * sizeof(float2);
    need[CB_KS] = (size_t)chunk * std::max<size_t>(op_s, 1) * sizeof(float2);
    need[CB_PAD] = (size_t)B * nfft * 4;
    need[CB_SPEC] = (size_t)B * nw * sizeof(float2);
    need[CB_WORK] = std::max<size_t>(16, std::max(c.full.work, tail ? c.tail.work : 0));
    if (memory == KCIG_MEM_HOST) {
        need[CB_IN] = need[CB_OUT] = (size_t)ntr * nt * 4;
        if (interm) need[CB_INTERM] = (size_t)ntr * nt * 4;
    }
    need[CB_STATUS] = sizeof(int);
    need[CB_WTR] = upload_bytes(wtr);
    need[CB_RCV] = upload_bytes(h.rcv);
    need[CB_SRC] = upload_bytes(h.src);
    if (p.cmp == 1) {
        need[CB_CABS] = upload_bytes(h.cabs);
        need[CB_GEOM] = upload_bytes(h.geom);
        need[CB_RTAU] = upload_bytes(h.rtau);
        need[CB_STAU] = upload_bytes(h.stau);
        need[CB_SL] = upload_bytes(h.sleft);
        need[CB_SR] = upload_bytes(h.sright);
        need[CB_IHM] = upload_bytes(h.ihmap);
        need[CB_IRL] = upload_bytes(h.ir_lo);
        need[CB_IRH] = upload_bytes(h.ir_hi);
    }
    KCIG_TRY(ensure_buffers(c, need));
    const CBuf *bf = c.buf;
    cufftResult cr;
    for (FftPair *q : {&c.full, &c.tail}) {
        if (q == &c.tail && !tail) continue;
        for (cufftHandle hq : {q->f, q->b}) {
            if ((cr = cufftSetWorkArea(hq, bf[CB_WORK].p)) != CUFFT_SUCCESS) return cufft_error(cr, "cufftSetWorkArea");
            if ((cr = cufftSetStream(hq, st)) != CUFFT_SUCCESS) return cufft_error(cr, "cufftSetStream");
        }
    }
    const float *d_in = in;
    float *d_out = out, *d_interm = interm;
    cudaStream_t cs = nullptr;
    if (memory == KCIG_MEM_HOST) {
        if (!c.copy) KCIG_CUDA(cudaStreamCreateWithFlags(&c.copy, cudaStreamNonBlocking));
        cs = idle.s2 = c.copy;
        d_in = bf[CB_IN].as<float>();
        d_out = bf[CB_OUT].as<float>();
        if (interm) d_interm = bf[CB_INTERM].as<float>();
    }
    KCIG_CUDA(cudaMemsetAsync(bf[CB_STATUS].p, 0, sizeof(int), st));
    KCIG_TRY(upload_to(bf[CB_WTR], wtr, st));
    KCIG_TRY(upload_to(bf[CB_RCV], h.rcv, st));
    KCIG_TRY(upload_to(bf[CB_SRC], h.src, st));
    if (p.cmp == 1) {
        KCIG_TRY(upload_to(bf[CB_CABS], h.cabs, st));
        KCIG_TRY(upload_to(bf[CB_GEOM], h.geom, st));
        KCIG_TRY(upload_to(bf[CB_RTAU], h.rtau, st));
        KCIG_TRY(upload_to(bf[CB_STAU], h.stau, st));
        KCIG_TRY(upload_to(bf[CB_SL], h.sleft, st));
        KCIG_TRY(upload_to(bf[CB_SR], h.sright, st));
        KCIG_TRY(upload_to(bf[CB_IHM], h.ihmap, st));
        KCIG_TRY(upload_to(bf[CB_IRL], h.ir_lo, st));
        KCIG_TRY(upload_to(bf[CB_IRH], h.ir_hi, st));
    }
    float2 *const U = bf[CB_U].as<float2>();
    float2 *const Kr = bf[CB_KR].as<float2>(), *const Ks = bf[CB_KS].as<float2>();
    float *const pad = bf[CB_PAD].as<float>();
    float2 *const spec = bf[CB_SPEC].as<float2>();
    int *const dstatus = bf[CB_STATUS].as<int>();
    // events: four stage bounds, four per chunk of frequencies (read once
    // the call has finished, so the chunks are queued back to back), and for
    // host-memory calls per batch of traces: its input copied, its interm
    // and output traces finished
    const int nchunk = (nw + chunk - 1) / chunk;
    const int nbatch = (int)((ntr + B - 1) / B);
    while (c.ev.size() < 4 + 4 * (size_t)nchunk + 3 * (size_t)nbatch) {
        cudaEvent_t e;
        KCIG_CUDA(cudaEventCreate(&e));
        c.ev.push_back(e);
    }
    cudaEvent_t *const ev = c.ev.data();
    cudaEvent_t *const bev = ev + 4 + 4 * nchunk;
    // host-memory calls: a batch's input goes over on the copy stream while
    // the batch before it is transformed; its output comes back once its
    // inverse transform is done, while later batches are transformed
    auto copy_in = [&](int ib) -> int {
        const long long t0 = (long long)ib * B;
        const size_t n = (size_t)std::min<long long>(B, ntr - t0) * nt;
        KCIG_CUDA(cudaMemcpyAsync(bf[CB_IN].as<float>() + t0 * nt, in + t0 * nt, n * 4, cudaMemcpyHostToDevice, cs));
        KCIG_CUDA(cudaEventRecord(bev[ib], cs));
        return KCIG_OK;
    };
    if (cs) KCIG_TRY(copy_in(0));
    KCIG_CUDA(cudaEventRecord(ev[0], st));
    // ---- forward: reverse, taper, pad, R2C, to frequency-major
    for (long long t0 = 0, ib = 0; t0 < ntr; t0 += B, ib++) {
        const int nb = (int)std::min<long long>(B, ntr - t0);
        if (cs) KCIG_CUDA(cudaStreamWaitEvent(st, bev[ib], 0));
        k_dat_prep<<<dim3((nfft / 4 + 255) / 256, std::min(nb, 1024)), 256, 0, st>>>(d_in, bf[CB_WTR].as<float>(), pad,
                                                                                    (int)t0, nb, nt, nfft);
        launches++;
        KCIG_CUDA(cudaGetLastError());
        if ((cr = cufftExecR2C(nb == B ? c.full.f : c.tail.f, (cufftReal *)pad, (cufftComplex *)spec)) != CUFFT_SUCCESS)
            return cufft_error(cr, "cufftExecR2C");
        launches++;
        k_dat_to_fmajor<<<dim3((nw + 31) / 32, (nb + 31) / 32), dim3(32, 8), 0, st>>>(spec, U, (int)t0, nb, nw,
                                                                                     (int)ntr);
        launches++;
        KCIG_CUDA(cudaGetLastError());
        if (cs && ib + 1 < nbatch) KCIG_TRY(copy_in((int)ib + 1));
    }
    KCIG_CUDA(cudaEventRecord(ev[1], st));
    // ---- per chunk of frequencies: operators, receiver side, source side
    for (int f0 = 0, ic = 0; f0 < nw; f0 += chunk, ic++) {
        const int nf = std::min(chunk, nw - f0);
        cudaEvent_t *const ce = ev + 4 + 4 * ic;
        float2 *Uc = U + (size_t)f0 * ntr;
        float2 *Utc = interm ? bf[CB_UFULL].as<float2>() + (size_t)f0 * ntr : bf[CB_UT].as<float2>();
        KCIG_CUDA(cudaEventRecord(ce[0], st));
        KCIG_TRY(launch_op(bf[CB_RCV].as<DatEntry>(), (int)op_r, Kr, f0, nf, nfft, K, p, st, launches));
        if (op_s) KCIG_TRY(launch_op(bf[CB_SRC].as<DatEntry>(), (int)op_s, Ks, f0, nf, nfft, K, p, st, launches));
        KCIG_CUDA(cudaEventRecord(ce[1], st));
        if (p.cmp == 0) {
            if (tcore)
                KCIG_TRY(launch_gemm_tc(Uc, ntr, nh, Kr, (long long)nh * nh, nh, Utc, ntr, nh, ns, nh, nh,
                                        p.aperture >= 0 ? p.aperture : 0, 0, nf, dstatus, st, launches));
            else
                KCIG_TRY(launch_gemm(Uc, ntr, nh, Kr, (long long)nh * nh, nh, Utc, ntr, nh, ns, nh, nh,
                                     p.aperture >= 0 ? p.aperture : 0, 0, nf, st, launches));
        } else {
            RcvCmp1Args a;
            a.U = Uc;
            a.Utmp = Utc;
            a.P = Kr;
            a.Ptau = bf[CB_RTAU].as<float>();
            a.cabs = bf[CB_CABS].as<int>();
            a.geom = bf[CB_GEOM].as<float>();
            a.ns = ns;
            a.nh = nh;
            a.aper = p.aperture;
            a.band = h.band;
            a.row0 = h.row0;
            a.nrow = h.nrow;
            a.sU = ntr;
            k_dat_rcv_cmp1<<<dim3((unsigned)((ntr + 127) / 128), nf), 128, 0, st>>>(a);
            launches++;
            KCIG_CUDA(cudaGetLastError());
        }
        KCIG_CUDA(cudaEventRecord(ce[2], st));
        if (p.cmp == 0) {
            if (tcore && shared_op)
                KCIG_TRY(launch_gemm_tc(Kr, (long long)nh * nh, nh, Utc, ntr, nh, Uc, ntr, nh, ns, nh, ns,
                                        p.aperture >= 0 ? p.aperture : 0, 1, nf, dstatus, st, launches, 1));
            else if (tcore)
                KCIG_TRY(launch_gemm_tc(Ks, (long long)ns * ns, ns, Utc, ntr, nh, Uc, ntr, nh, ns, nh, ns,
                                        p.aperture >= 0 ? p.aperture : 0, 1, nf, dstatus, st, launches));
            else
                KCIG_TRY(launch_gemm(Ks, (long long)ns * ns, ns, Utc, ntr, nh, Uc, ntr, nh, ns, nh, ns,
                                     p.aperture >= 0 ? p.aperture : 0, 1, nf, st, launches));
        } else {
            KCIG_CUDA(cudaMemsetAsync(Uc, 0, (size_t)nf * ntr * sizeof(float2), st));
            SrcCmp1Args a;
            a.Utmp = Utc;
            a.Uout = Uc;
            a.P = Ks;
            a.Ptau = bf[CB_STAU].as<float>();
            a.sleft = bf[CB_SL].as<int>();
            a.sright = bf[CB_SR].as<int>();
            a.ihmap = bf[CB_IHM].as<int>();
            a.ir_lo = bf[CB_IRL].as<int>();
            a.ir_hi = bf[CB_IRH].as<int>();
            a.ns = ns;
            a.nh = nh;
            a.nr = h.nr;
            a.aper = p.aperture;
            a.jump = h.jump;
            a.tap = p.taper;
            a.ds = p.ds;
            a.sdatum = p.sdatum;
            a.sUout = ntr;
            k_dat_src_cmp1<<<dim3((ns + 127) / 128, nf), 128, 0, st>>>(a);
            launches++;
            KCIG_CUDA(cudaGetLastError());
        }
        KCIG_CUDA(cudaEventRecord(ce[3], st));
    }
    KCIG_CUDA(cudaEventRecord(ev[2], st));
    // ---- inverse: to trace-major, C2R, scale, reverse, trim
    auto inverse = [&](const float2 *Usrc, float *dst, int reverse, cudaEvent_t *done) -> int {
        for (long long t0 = 0, ib = 0; t0 < ntr; t0 += B, ib++) {
            const int nb = (int)std::min<long long>(B, ntr - t0);
            k_dat_to_tmajor<<<dim3((nb + 31) / 32, (nw + 31) / 32), dim3(32, 8), 0, st>>>(Usrc, spec, (int)t0, nb, nw,
                                                                                         (int)ntr);
            launches++;
            KCIG_CUDA(cudaGetLastError());
            if ((cr = cufftExecC2R(nb == B ? c.full.b : c.tail.b, (cufftComplex *)spec, (cufftReal *)pad)) != CUFFT_SUCCESS)
                return cufft_error(cr, "cufftExecC2R");
            launches++;
            k_dat_finish<<<dim3((nt + 255) / 256, std::min(nb, 1024)), 256, 0, st>>>(pad, dst, (int)t0, nb, nt, nfft,
                                                                                  1.0f / (float)nfft, reverse);
            launches++;
            KCIG_CUDA(cudaGetLastError());
            if (cs) KCIG_CUDA(cudaEventRecord(done[ib], st));
        }
        return KCIG_OK;
    };
    cudaEvent_t *const done_im = bev + nbatch, *const done_out = bev + 2 * nbatch;
    if (interm) KCIG_TRY(inverse(bf[CB_UFULL].as<float2>(), d_interm, 0, done_im));
    KCIG_TRY(inverse(U, d_out, 1, done_out));
    KCIG_CUDA(cudaEventRecord(ev[3], st));
    if (cs) {
        // queued after every inverse launch, so a copy to pageable memory
        // (which holds the host until it is done) leaves the device busy
        auto copy_out = [&](float *host, const float *dev_src, const cudaEvent_t *done) -> int {
            for (long long t0 = 0, ib = 0; t0 < ntr; t0 += B, ib++) {
                const size_t n = (size_t)std::min<long long>(B, ntr - t0) * nt;
                KCIG_CUDA(cudaStreamWaitEvent(cs, done[ib], 0));
                KCIG_CUDA(cudaMemcpyAsync(host + t0 * nt, dev_src + t0 * nt, n * 4, cudaMemcpyDeviceToHost, cs));
            }
            return KCIG_OK;
        };
        if (interm) KCIG_TRY(copy_out(interm, d_interm, done_im));
        KCIG_TRY(copy_out(out, d_out, done_out));
        KCIG_CUDA(cudaStreamSynchronize(cs));
    }
    int dev_status = 0;
    KCIG_CUDA(cudaMemcpyAsync(&dev_status, dstatus, sizeof(int), cudaMemcpyDeviceToHost, st));
    KCIG_CUDA(cudaStreamSynchronize(st));
    if (dev_status)
        return set_error(KCIG_ERR_DEVICE, "kcig_datum_freq: a tensor-core GEMM gave up waiting (stage %d)", dev_status);
    float t, ms_op = 0.0f, ms_r = 0.0f, ms_s = 0.0f;
    for (int ic = 0; ic < nchunk; ic++) {
        const cudaEvent_t *ce = ev + 4 + 4 * ic;
        cudaEventElapsedTime(&t, ce[0], ce[1]);
        ms_op += t;
        cudaEventElapsedTime(&t, ce[1], ce[2]);
        ms_r += t;
        cudaEventElapsedTime(&t, ce[2], ce[3]);
        ms_s += t;
    }
    cudaEventElapsedTime(&t, ev[0], ev[1]);
    g_last_ms[0] = t;
    g_last_ms[1] = ms_op;
    g_last_ms[2] = ms_r;
    g_last_ms[3] = ms_s;
    cudaEventElapsedTime(&t, ev[2], ev[3]);
    g_last_ms[4] = t;
    g_last_launches = launches;
    return KCIG_OK;
}
