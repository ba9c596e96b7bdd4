// ADCIG stitching of depth windows (src/layercom_cig.cpp:412-556): each
// window's image volume [n3][n2][n1w] is scaled and written into the
// full-depth volume [n3][n2][n1] at its depth range; rows it shares with the
// window above keep the upper values for the first rows of the overlap and are
// blended with complementary raised-cosine weights over the rest.
//
// One pass over the window's samples, one thread per sample in a grid-stride
// loop along the contiguous depth axis: 4 B read from the window, 4 B read
// and 4 B written in the output (HBM-bound).  The blend weights and the
// lateral taper are formed on the host in double exactly as the reference
// forms them (:455-466, :522-528) and rounded once to float; the kernel keeps
// the reference's float operations separate (no fused multiply-add), so the
// output is the reference's, bit for bit.
#include <math.h>

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

__global__ void __launch_bounds__(256) k_stitch_layer(const StitchArgs a)
{
    const size_t total = (size_t)a.n1w * a.n2 * a.n3;
    unsigned long long bad = 0;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int i1 = (int)(idx % a.n1w);
        const size_t col = idx / a.n1w;  // i3 * n2 + i2
        const int i2 = (int)(col % a.n2);
        const float sx = a.lateral ? a.lateral[i2] : 1.0f;
        const float scale = __fmul_rn(a.layer_scale, sx);
        float v = __fmul_rn(a.layer[idx], scale);
        if (!isfinite(v)) {
            ++bad;
            v = 0.0f;
        }
        const int g1 = a.start + i1;
        float *o = a.out + col * a.n1 + g1;
        if (a.overlap > 0 && g1 <= a.previous_end) {
            if (i1 < a.keep_upper || a.blend_count == 0) continue;
            const float w = a.blend_w[i1 - a.keep_upper];
            *o = __fadd_rn(__fmul_rn(*o, __fsub_rn(1.0f, w)), __fmul_rn(v, w));
        } else {
            *o = v;
        }
    }
    // one atomic per warp at most
    for (int off = 16; off > 0; off >>= 1) bad += __shfl_down_sync(0xffffffffu, bad, off);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(a.nonfinite, bad);
}

}  // namespace kcig

using namespace kcig;

extern "C" int kcig_stitch_window(float *out, int n1, int n2, int n3, const float *layer, int start, int end,
                                  int previous_end, int stitch_blend, float layer_scale, int use_lateral,
                                  int scalex_aper, double scalex_scale, long long *nonfinite, void *stream)
{
    if (!out || !layer || !nonfinite || n1 <= 0 || n2 <= 0 || n3 <= 0)
        return set_error(KCIG_ERR_ARG, "kcig_stitch_window: bad arguments");
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
    void *scratch = nullptr;
    const size_t bytes = sizeof(unsigned long long) + host.size() * sizeof(float);
    KCIG_CUDA(cudaMalloc(&scratch, bytes));
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
        const size_t total = (size_t)n1w * n2 * n3;
        int sms = 148, dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const size_t want = (total + 255) / 256;
        const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>(want, (size_t)sms * 8));
        k_stitch_layer<<<grid, 256, 0, st>>>(a);
        e = cudaGetLastError();
    }
    unsigned long long bad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = cuda_error(e, "kcig_stitch_window");
    cudaFree(scratch);
    *nonfinite = (long long)bad;
    return rc;
}
