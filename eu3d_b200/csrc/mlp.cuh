// Learned chemistry surrogate: BF16 tensor-core (tcgen05) kernels with FP32
// accumulation for the MLP 12 -> 128 -> 128 -> 128 -> 10 (GELU) that maps a
// cell's (T, log p, Y_k, log dt) to (dY_k, dT) over one chemistry step.
//
// k_gemm_tc is the generic building block of training: C (+)= A B^T with A
// (M x K) and B (N x K) bf16 row-major (K contiguous), C (M x N) f32.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "tc.cuh"

namespace eu3d {

constexpr int GEMM_KC = 64;  // K columns staged per pass

__device__ __forceinline__ uint32_t tmem_cols_for(int n)
{
    uint32_t c = 32;
    while (c < (uint32_t)n) c <<= 1;
    return c;
}

// One CTA of 128 threads computes rows [128 b, 128 b + 128) x all N columns.
__global__ void __launch_bounds__(128) k_gemm_tc(const __nv_bfloat16 *__restrict__ A, const __nv_bfloat16 *__restrict__ B,
                                                float *__restrict__ C, int M, int N, int K, int accumulate,
                                                int *__restrict__ err)
{
    extern __shared__ __align__(128) unsigned char gsm[];
    unsigned char *As = gsm;                             // 128 x GEMM_KC
    unsigned char *Bs = gsm + 128 * GEMM_KC * 2;         // N x GEMM_KC
    uint64_t *mbar = reinterpret_cast<uint64_t *>(Bs + 256 * GEMM_KC * 2);
    uint32_t *slot = reinterpret_cast<uint32_t *>(mbar + 1);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int m0 = blockIdx.x * 128;
    const uint32_t ncols = tmem_cols_for(N);
    if (warp == 0) tc::tmem_alloc(slot, ncols);
    if (tid == 0) {
        tc::mbar_init(tc::smem_u32(mbar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *slot;
    const uint32_t idesc = tc::idesc_bf16(128, N);
    uint32_t phase = 0;
    bool ok = true;
    for (int k0 = 0; k0 < K; k0 += GEMM_KC) {
        const int kc = min(GEMM_KC, K - k0);
        const int vec = kc >> 3;  // 16-byte vectors per row
        for (int v = tid; v < 128 * vec; v += 128) {
            const int r = v / vec, kk = (v % vec) * 8;
            const uint4 x = *reinterpret_cast<const uint4 *>(A + (size_t)(m0 + r) * K + k0 + kk);
            *reinterpret_cast<uint4 *>(As + tc::op_off(128, r, kk)) = x;
        }
        for (int v = tid; v < N * vec; v += 128) {
            const int r = v / vec, kk = (v % vec) * 8;
            const uint4 x = *reinterpret_cast<const uint4 *>(B + (size_t)r * K + k0 + kk);
            *reinterpret_cast<uint4 *>(Bs + tc::op_off(N, r, kk)) = x;
        }
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after();
            for (int s = 0; s < (kc >> 4); s++)
                tc::mma(tmem, tc::sdesc(tc::smem_u32(As + s * 128 * 32)), tc::sdesc(tc::smem_u32(Bs + s * N * 32)),
                        idesc, (k0 > 0 || s > 0) ? 1u : 0u);
            tc::commit(tc::smem_u32(mbar));
        }
        ok = tc::mbar_wait(tc::smem_u32(mbar), phase) && ok;
        phase ^= 1;
        tc::fence_after();
        __syncthreads();  // the MMAs have read this pass's tiles; the next pass may overwrite them
    }
    if (!ok && err) atomicExch(err, 1);
    // epilogue: thread tid owns row m0 + tid (TMEM lane tid)
    const int row = m0 + tid;
    const uint32_t lane = (uint32_t)(warp * 32) << 16;
    for (int c0 = 0; c0 < N; c0 += 32) {
        float v[32];
        if (N - c0 >= 32) {
            tc::tmem_ld32(tmem + lane + c0, v);
        } else {
            tc::tmem_ld16(tmem + lane + c0, v);
        }
        const int nn = min(32, N - c0);
        float *dst = C + (size_t)row * N + c0;
        for (int i = 0; i < nn; i++) dst[i] = accumulate ? dst[i] + v[i] : v[i];
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tmem, ncols);
}

inline size_t gemm_smem_bytes() { return (size_t)(128 + 256) * GEMM_KC * 2 + 16; }

}  // namespace eu3d
