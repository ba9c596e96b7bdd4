// First-arrival traveltime tables on the GPU: the role eikods2d plays for
// the migration (src/eikods2d.cpp:149-765, SERECKIRCH/src/eikods.cpp:66-211):
// for each source position a [nx][nz] table of first-arrival times and the
// derivative of the time with respect to the source position.
//
// Method: fast sweeping with a first-order Godunov upwind update, run as
// Gauss-Seidel sweeps in the four diagonal orderings.  Points on one
// anti-diagonal of a sweep depend only on the previous anti-diagonal, so a
// CTA (one per source) updates a whole anti-diagonal in parallel and
// synchronises between anti-diagonals.  Near the source, inside the same
// (b1, b2) box eikods2d uses (eikods.cpp:66-111, neighbors.cpp), times are the
// straight-ray distance times the source slowness.  The iteration count is
// fixed by the caller: there is no data-dependent loop and no wait.
//
// The position derivative is the centred difference of adjacent positions'
// tables (one-sided at the ends) -- a stand-in for eikods2d's tds1 transport.
#include <math.h>

#include <vector>

#include "kcig_common.h"

namespace kcig {

static constexpr float kBig = 1.0e30f;

__global__ void __launch_bounds__(1024) k_fsm(const float *__restrict__ slow, float *__restrict__ T, int nz, int nx,
                                              float dz, float dx, float z0, float x0, const float *__restrict__ px,
                                              float zs, int b1, int b2, int iters)
{
    const int j = blockIdx.x;
    const size_t nzx = (size_t)nz * nx;
    float *t = T + (size_t)j * nzx;
    const float xs = px[j];
    const int isz = (int)lrintf((zs - z0) / dz), isx = (int)lrintf((xs - x0) / dx);
    const int csz = min(max(isz, 0), nz - 1), csx = min(max(isx, 0), nx - 1);
    const float s0 = slow[(size_t)csx * nz + csz];
    for (size_t i = threadIdx.x; i < nzx; i += blockDim.x) {
        const int iz = (int)(i % nz), ix = (int)(i / nz);
        float v = kBig;
        if (abs(iz - isz) <= b1 && abs(ix - isx) <= b2) {
            const float ddz = z0 + iz * dz - zs, ddx = x0 + ix * dx - xs;
            v = s0 * sqrtf(ddz * ddz + ddx * ddx);
        }
        t[i] = v;
    }
    __syncthreads();
    const double idx2 = 1.0 / ((double)dx * dx), idz2 = 1.0 / ((double)dz * dz);
    for (int it = 0; it < iters; it++) {
        for (int dir = 0; dir < 4; dir++) {
            const bool fz = (dir & 1) == 0, fx = (dir & 2) == 0;
            for (int k = 0; k <= nz + nx - 2; k++) {
                const int ulo = max(0, k - (nx - 1)), uhi = min(nz - 1, k);
                for (int u = ulo + (int)threadIdx.x; u <= uhi; u += blockDim.x) {
                    const int v = k - u;
                    const int iz = fz ? u : nz - 1 - u, ix = fx ? v : nx - 1 - v;
                    const size_t i = (size_t)ix * nz + iz;
                    const float cur = t[i];
                    const float a = fminf(ix > 0 ? t[i - nz] : kBig, ix < nx - 1 ? t[i + nz] : kBig);
                    const float b = fminf(iz > 0 ? t[i - 1] : kBig, iz < nz - 1 ? t[i + 1] : kBig);
                    if (a >= kBig && b >= kBig) continue;
                    const double f = slow[i];
                    double tn;
                    const double ta = (double)a + f * dx, tb = (double)b + f * dz;
                    if (a >= kBig) tn = tb;
                    else if (b >= kBig) tn = ta;
                    else {
                        // ((t-a)/dx)^2 + ((t-b)/dz)^2 = f^2, accepted when t >= max(a, b)
                        const double A = idx2 + idz2;
                        const double B = -2.0 * ((double)a * idx2 + (double)b * idz2);
                        const double C = (double)a * a * idx2 + (double)b * b * idz2 - f * f;
                        const double disc = B * B - 4.0 * A * C;
                        tn = fmin(ta, tb);
                        if (disc >= 0.0) {
                            const double q = (-B + sqrt(disc)) / (2.0 * A);
                            if (q >= fmax((double)a, (double)b)) tn = fmin(tn, q);
                        }
                    }
                    if ((float)tn < cur) t[i] = (float)tn;
                }
                __syncthreads();
            }
        }
    }
}

__global__ void k_pos_deriv(const float *__restrict__ T, float *__restrict__ D, int npos, size_t nzx, float dp)
{
    const int j = blockIdx.y;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nzx) return;
    float v = 0.0f;
    if (npos > 1) {
        const int a = max(0, j - 1), b = min(npos - 1, j + 1);
        v = (T[(size_t)b * nzx + i] - T[(size_t)a * nzx + i]) / ((float)(b - a) * dp);
    }
    D[(size_t)j * nzx + i] = v;
}

__global__ void k_slowness(const float *__restrict__ vel, float *__restrict__ s, size_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) s[i] = 1.0f / vel[i];
}

}  // namespace kcig

using namespace kcig;

extern "C" int kcig_eikonal_tables(const float *vel, int nz, int nx, float dz, float dx, float z0, float x0, int npos,
                                   float p0, float dp, float zsrc, int b1, int b2, int iterations, float *time,
                                   float *deriv, void *stream)
{
    if (!vel || !time || nz < 2 || nx < 2 || npos < 1 || !(dz > 0.0f) || !(dx > 0.0f) || iterations < 1)
        return set_error(KCIG_ERR_ARG, "kcig_eikonal_tables: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nzx = (size_t)nz * nx;
    float *slow = nullptr, *px = nullptr;
    KCIG_CUDA(cudaMallocAsync(&slow, nzx * sizeof(float), st));
    cudaError_t e = cudaMallocAsync(&px, (size_t)npos * sizeof(float), st);
    if (e != cudaSuccess) {
        cudaFreeAsync(slow, st);
        return cuda_error(e, "cudaMallocAsync");
    }
    std::vector<float> hp(npos);
    for (int j = 0; j < npos; j++) hp[j] = p0 + (float)j * dp;
    int rc = KCIG_OK;
    e = cudaMemcpyAsync(px, hp.data(), npos * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) rc = cuda_error(e, "cudaMemcpyAsync(positions)");
    if (!rc) {
        k_slowness<<<(unsigned)((nzx + 255) / 256), 256, 0, st>>>(vel, slow, nzx);
        const int diag = nz < nx ? nz : nx;
        const int threads = diag >= 1024 ? 1024 : ((diag + 31) / 32) * 32;
        k_fsm<<<npos, threads, 0, st>>>(slow, time, nz, nx, dz, dx, z0, x0, px, zsrc, b1, b2, iterations);
        if (deriv) k_pos_deriv<<<dim3((unsigned)((nzx + 255) / 256), npos), 256, 0, st>>>(time, deriv, npos, nzx, dp);
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_error(e, "kcig_eikonal_tables launch");
    }
    cudaFreeAsync(slow, st);
    cudaFreeAsync(px, st);
    e = cudaStreamSynchronize(st);
    if (!rc && e != cudaSuccess) rc = cuda_error(e, "kcig_eikonal_tables");
    return rc;
}
