// ADCIG stitching of depth windows (src/layercom_cig.cpp:412-556): each
// window's image volume [n3][n2][n1w] is scaled and written into the
// full-depth volume [n3][n2][n1] at its depth range; rows it shares with the
// window above keep the upper values for the first rows of the overlap and are
// blended with complementary raised-cosine weights over the rest.
//
// One pass over the window's samples: 4 B read from the window and 4 B
// written in the output per sample, 4 B more read in the blended rows
// (HBM-bound).  The blend weights and the
// lateral taper are formed on the host in double exactly as the reference
// forms them (:455-466, :522-528) and rounded once to float; the kernel keeps
// the reference's float operations separate (no fused multiply-add), so the
// output is the reference's, bit for bit.
#include <math.h>
#include <string.h>

#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "kcig_common.h"

namespace kcig {

struct StitchArgs {
    float *out;             // [n3][n2][n1] full-depth volume
    const float *layer;     // [n3][n2][n1w] this window
    const float *blend_w;   // [blend_count] weights of the window's rows past keep_upper
    const float *lateral;   // [n2] lateral taper, or null (1)
    unsigned long long *nonfinite;
    int n1, n2, n3, n1w, start, previous_end, keep_upper, blend_count, overlap;
    float layer_scale;
};

// One warp per depth column (i3, i2) of the window, its lanes along the
// contiguous depth rows: the column's scale is formed once, every access is
// coalesced, and no index is divided per sample.
__global__ void __launch_bounds__(256) k_stitch_layer(const StitchArgs a)
{
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    const int ncol = a.n2 * a.n3;  // < 2^31 (checked on the host)
    unsigned long long bad = 0;
    for (int col = blockIdx.x * warps + (threadIdx.x >> 5); col < ncol; col += gridDim.x * warps) {
        const int i2 = col % a.n2;
        const float sx = a.lateral ? a.lateral[i2] : 1.0f;
        const float scale = __fmul_rn(a.layer_scale, sx);
        const float *src = a.layer + (size_t)col * a.n1w;
        float *dst = a.out + (size_t)col * a.n1 + a.start;
        for (int i1 = lane; i1 < a.n1w; i1 += 32) {
            float v = __fmul_rn(src[i1], scale);
            if (!isfinite(v)) {
                ++bad;
                v = 0.0f;
            }
            if (a.overlap > 0 && a.start + i1 <= a.previous_end) {
                if (i1 < a.keep_upper || a.blend_count == 0) continue;
                const float w = a.blend_w[i1 - a.keep_upper];
                dst[i1] = __fadd_rn(__fmul_rn(dst[i1], __fsub_rn(1.0f, w)), __fmul_rn(v, w));
            } else {
                dst[i1] = v;
            }
        }
    }
    // one atomic per warp at most
    for (int off = 16; off > 0; off >>= 1) bad += __shfl_down_sync(0xffffffffu, bad, off);
    if (lane == 0 && bad) atomicAdd(a.nonfinite, bad);
}

// Device scratch of the calls (counter + weights), one per device, grown on
// demand and kept for the life of the process: a call allocates nothing once
// warm.  Calls hold the lock until they have synchronised.
static std::mutex g_scratch_mu;
static std::map<int, std::pair<void *, size_t>> g_scratch;

}  // namespace kcig

using namespace kcig;

extern "C" int kcig_stitch_window(float *out, int n1, int n2, int n3, const float *layer, int start, int end,
                                  int previous_end, int stitch_blend, float layer_scale, int use_lateral,
                                  int scalex_aper, double scalex_scale, long long *nonfinite, void *stream)
{
    if (!out || !layer || !nonfinite || n1 <= 0 || n2 <= 0 || n3 <= 0)
        return set_error(KCIG_ERR_ARG, "kcig_stitch_window: bad arguments");
    if ((long long)n2 * n3 > 0x7fffffffLL) return set_error(KCIG_ERR_ARG, "kcig_stitch_window: n2*n3 too large");
    if (start < 0 || end < start || end >= n1)
        return set_error(KCIG_ERR_ARG, "Invalid layer range [%d,%d]", start, end);
    if (stitch_blend < -1) return set_error(KCIG_ERR_ARG, "stitch_blend must be -1 or nonnegative");
    if (scalex_aper < 0) return set_error(KCIG_ERR_ARG, "scalex_aper must be nonnegative");
    // overlap with the window above (:490-499): every window but the first
    // must share rows with it
    int overlap = 0;
    if (previous_end >= 0) {
        overlap = previous_end - start + 1;
        if (overlap <= 0) return set_error(KCIG_ERR_ARG, "no overlap with the window above");
    }
    int blend_count = overlap;
    if (overlap > 0 && stitch_blend >= 0) blend_count = std::min(stitch_blend, overlap);
    const int keep_upper = overlap - blend_count;
    const int n1w = end - start + 1;

    // complementary cosine weights (:522-528), in double, rounded once
    std::vector<float> host((size_t)blend_count + (use_lateral ? n2 : 0));
    for (int bi = 0; bi < blend_count; bi++) {
        const double u = blend_count > 1 ? (double)bi / (double)(blend_count - 1) : 1.0;
        host[bi] = (float)(0.5 * (1.0 - cos(3.14159265358979323846 * u)));
    }
    // lateral taper towards both edges (:455-466)
    if (use_lateral) {
        float *lat = host.data() + blend_count;
        for (int i2 = 0; i2 < n2; i2++) {
            lat[i2] = 1.0f;
            const int edge = std::min(i2, n2 - 1 - i2);
            if (scalex_aper > 0 && edge < scalex_aper) {
                const double taper = scalex_aper == 1 ? 1.0 : 1.0 - (double)edge / (double)(scalex_aper - 1);
                lat[i2] = (float)(1.0 + (scalex_scale - 1.0) * taper);
            }
        }
    }
    cudaStream_t st = (cudaStream_t)stream;
    // device scratch: the counter first (8-byte aligned), then the weights
    const size_t bytes = sizeof(unsigned long long) + host.size() * sizeof(float);
    int dev = 0;
    KCIG_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    std::pair<void *, size_t> &buf = g_scratch[dev];
    if (buf.second < bytes) {
        if (buf.first) cudaFree(buf.first);
        buf = {nullptr, 0};
        KCIG_CUDA(cudaMalloc(&buf.first, std::max<size_t>(bytes, 64 << 10)));
        buf.second = std::max<size_t>(bytes, 64 << 10);
    }
    void *scratch = buf.first;
    unsigned long long *d_bad = (unsigned long long *)scratch;
    float *d_w = (float *)(d_bad + 1);
    int rc = KCIG_OK;
    cudaError_t e = cudaMemsetAsync(d_bad, 0, sizeof *d_bad, st);
    if (e == cudaSuccess && !host.empty())
        e = cudaMemcpyAsync(d_w, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        StitchArgs a;
        a.out = out;
        a.layer = layer;
        a.blend_w = d_w;
        a.lateral = use_lateral ? d_w + blend_count : nullptr;
        a.nonfinite = d_bad;
        a.n1 = n1;
        a.n2 = n2;
        a.n3 = n3;
        a.n1w = n1w;
        a.start = start;
        a.previous_end = previous_end;
        a.keep_upper = keep_upper;
        a.blend_count = blend_count;
        a.overlap = overlap;
        a.layer_scale = layer_scale;
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const size_t want = ((size_t)n2 * n3 + 7) / 8;  // 8 columns (warps) per block
        const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>(want, (size_t)sms * 16));
        k_stitch_layer<<<grid, 256, 0, st>>>(a);
        e = cudaGetLastError();
    }
    unsigned long long bad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = cuda_error(e, "kcig_stitch_window");
    *nonfinite = (long long)bad;
    return rc;
}

// ------------------------------------------------- all windows, one pass --
// The windows of one stitch in a single kernel.  Each warp owns an output
// column (i3, i2) and keeps it in shared memory: zeroed, then every window
// applied in order with exactly the per-window rule above (write; keep the
// upper value; or blend), its lanes along the window's rows (each row of a
// window has one lane, so a window's updates never collide), then written
// out once.  The result equals the window-by-window calls on a zeroed volume
// bit for bit (rows no window covers stay 0).  Each window sample is read
// once and each output sample written once; the window records are
// warp-uniform loads, once per column; one launch, one upload of the weights
// and one read-back of the counters.
namespace kcig {

struct StitchWin {
    const float *layer;  // [n3][n2][n1w]
    int start, n1w, keep_upper, blend_count, overlap, previous_end, lateral, woff;
    float scale;
};

struct StitchAllArgs {
    float *out;
    const StitchWin *win;     // [nwin]
    const float *weights;     // blend weights of every window (at win.woff)
    const float *lateral;     // lateral taper [n2], or null
    unsigned long long *nonfinite;  // [nwin]
    int n1, n2, n3, nwin;
};

__global__ void __launch_bounds__(256) k_stitch_all(const StitchAllArgs a)
{
    extern __shared__ float colbuf[];  // [warps][n1]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    float *buf = colbuf + (size_t)warp * a.n1;
    const int ncol = a.n2 * a.n3;
    for (int col = blockIdx.x * warps + warp; col < ncol; col += gridDim.x * warps) {
        const int i2 = col % a.n2;
        const float sx = a.lateral ? a.lateral[i2] : 1.0f;
        for (int r = lane; r < a.n1; r += 32) buf[r] = 0.0f;
        __syncwarp();
        for (int k = 0; k < a.nwin; k++) {
            const StitchWin w = a.win[k];
            const float scale = __fmul_rn(w.scale, w.lateral ? sx : 1.0f);
            const float *src = w.layer + (size_t)col * w.n1w;
            unsigned long long bad = 0;
            // eight loads per lane in flight before the first is used: a
            // window column is 256 samples or fewer in the common case, one
            // round of independent loads instead of a dependent chain
            for (int base = 0; base < w.n1w; base += 256) {
                float ld[8];
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int i1 = base + lane + 32 * u;
                    ld[u] = i1 < w.n1w ? __ldcs(src + i1) : 0.0f;
                }
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int i1 = base + lane + 32 * u;
                    if (i1 >= w.n1w) continue;
                    float v = __fmul_rn(ld[u], scale);
                    if (!isfinite(v)) {
                        ++bad;
                        v = 0.0f;
                    }
                    const int r = w.start + i1;
                    if (w.overlap > 0 && r <= w.previous_end) {
                        if (i1 < w.keep_upper || w.blend_count == 0) continue;
                        const float bw = a.weights[w.woff + i1 - w.keep_upper];
                        buf[r] = __fadd_rn(__fmul_rn(buf[r], __fsub_rn(1.0f, bw)), __fmul_rn(v, bw));
                    } else {
                        buf[r] = v;
                    }
                }
            }
            for (int off = 16; off > 0; off >>= 1) bad += __shfl_down_sync(0xffffffffu, bad, off);
            if (lane == 0 && bad) atomicAdd(a.nonfinite + k, bad);
            __syncwarp();
        }
        float *dst = a.out + (size_t)col * a.n1;
        for (int r = lane; r < a.n1; r += 32) dst[r] = buf[r];
        __syncwarp();
    }
}

}  // namespace kcig

extern "C" int kcig_stitch_windows(float *out, int n1, int n2, int n3, int nwin, const float *const *layers,
                                   const int *starts, const int *ends, int stitch_blend, const float *scales,
                                   int use_lateral, int scalex_aper, double scalex_scale, long long *nonfinite,
                                   void *stream)
{
    if (!out || !layers || !starts || !ends || !scales || !nonfinite || n1 <= 0 || n2 <= 0 || n3 <= 0 || nwin < 1)
        return set_error(KCIG_ERR_ARG, "kcig_stitch_windows: bad arguments");
    if ((long long)n2 * n3 > 0x7fffffffLL) return set_error(KCIG_ERR_ARG, "kcig_stitch_windows: n2*n3 too large");
    if (stitch_blend < -1) return set_error(KCIG_ERR_ARG, "stitch_blend must be -1 or nonnegative");
    if (scalex_aper < 0) return set_error(KCIG_ERR_ARG, "scalex_aper must be nonnegative");
    std::vector<StitchWin> win(nwin);
    std::vector<float> wts;
    for (int k = 0; k < nwin; k++) {
        const int start = starts[k], end = ends[k];
        if (!layers[k] || start < 0 || end < start || end >= n1)
            return set_error(KCIG_ERR_ARG, "Invalid layer range [%d,%d]", start, end);
        const int previous_end = k > 0 ? ends[k - 1] : -1;
        int overlap = 0;
        if (previous_end >= 0) {
            overlap = previous_end - start + 1;
            if (overlap <= 0) return set_error(KCIG_ERR_ARG, "no overlap with the window above");
        }
        int blend_count = overlap;
        if (overlap > 0 && stitch_blend >= 0) blend_count = std::min(stitch_blend, overlap);
        StitchWin &w = win[k];
        w.layer = layers[k];
        w.start = start;
        w.n1w = end - start + 1;
        w.keep_upper = overlap - blend_count;
        w.blend_count = blend_count;
        w.overlap = overlap;
        w.previous_end = previous_end;
        w.lateral = use_lateral && k > 0;
        w.scale = scales[k];
        w.woff = (int)wts.size();
        // complementary cosine weights (:522-528), in double, rounded once
        for (int bi = 0; bi < blend_count; bi++) {
            const double u = blend_count > 1 ? (double)bi / (double)(blend_count - 1) : 1.0;
            wts.push_back((float)(0.5 * (1.0 - cos(3.14159265358979323846 * u))));
        }
    }
    const int lat_off = (int)wts.size();
    if (use_lateral) {  // lateral taper towards both edges (:455-466)
        for (int i2 = 0; i2 < n2; i2++) {
            float v = 1.0f;
            const int edge = std::min(i2, n2 - 1 - i2);
            if (scalex_aper > 0 && edge < scalex_aper) {
                const double taper = scalex_aper == 1 ? 1.0 : 1.0 - (double)edge / (double)(scalex_aper - 1);
                v = (float)(1.0 + (scalex_scale - 1.0) * taper);
            }
            wts.push_back(v);
        }
    }
    // a column of the output per warp in shared memory
    const size_t col_bytes = (size_t)n1 * sizeof(float);
    if (col_bytes > 200 * 1024) return set_error(KCIG_ERR_ARG, "kcig_stitch_windows: n1=%d rows exceed one column buffer", n1);
    const int warps = (int)std::max<size_t>(1, std::min<size_t>(8, (96 * 1024) / col_bytes));
    // one staging upload: counters, window records, weights
    const size_t o_bad = 0, o_win = o_bad + (((size_t)nwin * 8 + 15) & ~(size_t)15);
    const size_t o_w = o_win + (((size_t)nwin * sizeof(StitchWin) + 15) & ~(size_t)15);
    const size_t bytes = o_w + std::max<size_t>(1, wts.size()) * 4;
    std::vector<unsigned char> host(bytes, 0);
    memcpy(host.data() + o_win, win.data(), nwin * sizeof(StitchWin));
    if (!wts.empty()) memcpy(host.data() + o_w, wts.data(), wts.size() * 4);
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    KCIG_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    std::pair<void *, size_t> &buf = g_scratch[dev];
    if (buf.second < bytes) {
        if (buf.first) cudaFree(buf.first);
        buf = {nullptr, 0};
        KCIG_CUDA(cudaMalloc(&buf.first, std::max<size_t>(bytes, 64 << 10)));
        buf.second = std::max<size_t>(bytes, 64 << 10);
    }
    unsigned char *d = (unsigned char *)buf.first;
    cudaError_t e = cudaMemcpyAsync(d, host.data(), bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        StitchAllArgs a;
        a.out = out;
        a.win = (const StitchWin *)(d + o_win);
        a.weights = (const float *)(d + o_w);
        a.lateral = use_lateral ? a.weights + lat_off : nullptr;
        a.nonfinite = (unsigned long long *)(d + o_bad);
        a.n1 = n1;
        a.n2 = n2;
        a.n3 = n3;
        a.nwin = nwin;
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int smem = (int)(warps * col_bytes);
        int rc = set_dyn_smem((const void *)k_stitch_all, smem);
        if (rc) return rc;
        const size_t want = ((size_t)n2 * n3 + warps - 1) / warps;
        const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>(want, (size_t)sms * 32));
        k_stitch_all<<<grid, 32 * warps, smem, st>>>(a);
        e = cudaGetLastError();
    }
    std::vector<unsigned long long> bad(nwin, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(bad.data(), d + o_bad, nwin * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_error(e, "kcig_stitch_windows");
    for (int k = 0; k < nwin; k++) nonfinite[k] = (long long)bad[k];
    return KCIG_OK;
}
