// Traveltime surrogate on the fifth-generation tensor cores (tcgen05, TMEM).
//
// This file holds the tensor-core GEMM self-test; the surrogate's training and
// field kernels follow it.
#include <cuda_bf16.h>

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
    if (tid == 0) {
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
