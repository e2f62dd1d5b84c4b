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
// With gridDim.y > 1 the K range is split into chunks of kchunk columns, one
// per blockIdx.y, and the partial products are added into C atomically (C
// must hold zeros, or the values to accumulate onto).
__global__ void __launch_bounds__(128) k_gemm_tc(const __nv_bfloat16 *__restrict__ A, const __nv_bfloat16 *__restrict__ B,
                                                float *__restrict__ C, int M, int N, int K, int accumulate,
                                                int *__restrict__ err, int kchunk = 0)
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
    const bool split = gridDim.y > 1;
    const int kbeg = split ? blockIdx.y * kchunk : 0;
    const int kend = split ? min(K, kbeg + kchunk) : K;
    for (int k0 = kbeg; k0 < kend; k0 += GEMM_KC) {
        const int kc = min(GEMM_KC, kend - k0);
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
                        idesc, (k0 > kbeg || s > 0) ? 1u : 0u);
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
        if (split) {
            if (kbeg < kend)
                for (int i = 0; i < nn; i++) atomicAdd(dst + i, v[i]);
        } else {
            for (int i = 0; i < nn; i++) dst[i] = accumulate ? dst[i] + v[i] : v[i];
        }
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tmem, ncols);
}

inline size_t gemm_smem_bytes() { return (size_t)(128 + 256) * GEMM_KC * 2 + 16; }

}  // namespace eu3d

namespace eu3d {

// ---------------------------------------------------------------- model
constexpr int SUR_NIN = 12;   // T, log p, Y_0..Y_8, log dt
constexpr int SUR_NOUT = 10;  // Y_s rates (9) and T rate
constexpr int SUR_IN = 16, SUR_H = 128, SUR_OUT = 16;  // padded widths
// flat FP32 parameter vector: W1[16][128] b1[128] W2[128][128] b2 W3[128][128] b3 W4[128][16] b4[16]
constexpr int SUR_OFF_W1 = 0;
constexpr int SUR_OFF_B1 = SUR_OFF_W1 + SUR_IN * SUR_H;
constexpr int SUR_OFF_W2 = SUR_OFF_B1 + SUR_H;
constexpr int SUR_OFF_B2 = SUR_OFF_W2 + SUR_H * SUR_H;
constexpr int SUR_OFF_W3 = SUR_OFF_B2 + SUR_H;
constexpr int SUR_OFF_B3 = SUR_OFF_W3 + SUR_H * SUR_H;
constexpr int SUR_OFF_W4 = SUR_OFF_B3 + SUR_H;
constexpr int SUR_OFF_B4 = SUR_OFF_W4 + SUR_H * SUR_OUT;
constexpr int SUR_NPARAM = SUR_OFF_B4 + SUR_OUT;

// hardware tanh (PTX tanh.approx.f32, about 2^-11 relative error)
__device__ __forceinline__ float tanh_hw(float x)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// GELU in the tanh form of Hendrycks & Gimpel (2016):
// 0.5 z (1 + tanh(c (z + 0.044715 z^3))), c = sqrt(2 / pi).  Training and
// inference evaluate the same expression.
__device__ __forceinline__ float gelu_f(float z)
{
    const float c = 0.7978845608028654f, c3 = 0.7978845608028654f * 0.044715f;
    const float u = z * fmaf(c3, z * z, c);
    const float hz = 0.5f * z;
    return fmaf(hz, tanh_hw(u), hz);
}

// GELU of two values in packed BF16 arithmetic (the network's activation in
// training and inference): z = bf16(z0, z1); u = z (c + c3 z^2); h = z/2 +
// z/2 tanh(u), each packed operation rounded to BF16.  Returns the packed
// BF16 pair (z0 in the low half).
__device__ __forceinline__ uint32_t gelu_bf16x2(float z0, float z1)
{
    uint32_t z, z2, a, u, t, hz, h;
    // packed constants: c = sqrt(2/pi), c3 = c * 0.044715, 0.5
    const uint32_t C1 = 0x3F4C3F4Cu, C3 = 0x3D123D12u, HALF = 0x3F003F00u, NZ = 0x80008000u;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(z) : "f"(z1), "f"(z0));
    asm("fma.rn.bf16x2 %0, %1, %1, %2;" : "=r"(z2) : "r"(z), "r"(NZ));
    asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(a) : "r"(z2), "r"(C3), "r"(C1));
    asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(u) : "r"(z), "r"(a), "r"(NZ));
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(u));
    asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(hz) : "r"(z), "r"(HALF), "r"(NZ));
    asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(h) : "r"(hz), "r"(t), "r"(hz));
    return h;
}

// Twice gelu_bf16x2, in one packed operation fewer: h2 = z + z tanh(u).
// Because halving and doubling are exact in BF16, h2 = 2 gelu_bf16x2(z0, z1)
// bit for bit; the inference kernel feeds h2 to weights staged at half
// their value, so every tensor-core product equals the unscaled one.
__device__ __forceinline__ uint32_t gelu2_bf16x2(float z0, float z1)
{
    uint32_t z, z2, a, u, t, h;
    const uint32_t C1 = 0x3F4C3F4Cu, C3 = 0x3D123D12u, NZ = 0x80008000u;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(z) : "f"(z1), "f"(z0));
    asm("fma.rn.bf16x2 %0, %1, %1, %2;" : "=r"(z2) : "r"(z), "r"(NZ));
    asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(a) : "r"(z2), "r"(C3), "r"(C1));
    asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(u) : "r"(z), "r"(a), "r"(NZ));
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(u));
    asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(h) : "r"(z), "r"(t), "r"(z));
    return h;
}

__device__ __forceinline__ float gelu_grad_f(float z)
{
    const float c = 0.7978845608028654f, c3 = 0.7978845608028654f * 0.044715f;
    const float t = tanh_hw(z * fmaf(c3, z * z, c));
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * fmaf(3.0f * c3, z * z, c);
}

// ------------------------------------------------------- training kernels
// Z = acc + b; H = gelu(Z) (bf16 pairs, row-major and transposed); N even
__global__ void k_sur_fwd_act(const float *__restrict__ acc, const float *__restrict__ b, float *__restrict__ Z,
                              __nv_bfloat16 *__restrict__ H, __nv_bfloat16 *__restrict__ Ht, int B, int N)
{
    const long long n = (long long)B * N / 2;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long e = 2 * t;
        const int r = (int)(e / N), c = (int)(e % N);
        const float z0 = acc[e] + b[c], z1 = acc[e + 1] + b[c + 1];
        Z[e] = z0;
        Z[e + 1] = z1;
        const uint32_t h = gelu_bf16x2(z0, z1);
        *reinterpret_cast<uint32_t *>(H + e) = h;
        Ht[(long long)c * B + r] = __ushort_as_bfloat16((unsigned short)(h & 0xFFFFu));
        Ht[(long long)(c + 1) * B + r] = __ushort_as_bfloat16((unsigned short)(h >> 16));
    }
}

// output layer: out = acc + b; loss = sum over rows r and output columns of
// w_r (out - y)^2 / (B SUR_NOUT), w_r = y[r][15] (0 drops a sample);
// dZ = 2 w_r (out - y) / (B SUR_NOUT) as bf16 (row-major and transposed)
__global__ void k_sur_loss(const float *__restrict__ acc, const float *__restrict__ b, const float *__restrict__ y,
                           float *__restrict__ out, __nv_bfloat16 *__restrict__ dZ, __nv_bfloat16 *__restrict__ dZt,
                           float *__restrict__ loss, int B)
{
    const long long n = (long long)B * SUR_OUT;
    const float scale = 1.0f / ((float)B * SUR_NOUT);
    float local = 0.f;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t / SUR_OUT), c = (int)(t % SUR_OUT);
        const float o = acc[t] + b[c];
        out[t] = o;
        float g = 0.f;
        if (c < SUR_NOUT) {
            const float w = y[(long long)r * SUR_OUT + 15];
            const float d = o - y[t];
            local += w * d * d * scale;
            g = 2.f * w * d * scale;
        }
        const __nv_bfloat16 gb = __float2bfloat16_rn(g);
        dZ[t] = gb;
        dZt[(long long)c * B + r] = gb;
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, local);
}

// dZ = dH * gelu'(Z) (bf16, row-major and transposed)
__global__ void k_sur_bwd_act(const float *__restrict__ dH, const float *__restrict__ Z, __nv_bfloat16 *__restrict__ dZ,
                              __nv_bfloat16 *__restrict__ dZt, int B, int N)
{
    const long long n = (long long)B * N;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t / N), c = (int)(t % N);
        const __nv_bfloat16 g = __float2bfloat16_rn(dH[t] * gelu_grad_f(Z[t]));
        dZ[t] = g;
        dZt[(long long)c * B + r] = g;
    }
}

// db[c] = sum_r dZ[r][c]  (bf16 input, FP32 sum); one block per column
__global__ void k_sur_colsum(const __nv_bfloat16 *__restrict__ dZt, float *__restrict__ db, int B)
{
    const int c = blockIdx.x;
    float s = 0.f;
    for (int r = threadIdx.x; r < B; r += blockDim.x) s += __bfloat162float(dZt[(long long)c * B + r]);
    __shared__ float sm[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.f;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) db[c] = s;
    }
}

// gather the weight gradients of the padded GEMM outputs into the flat layout
// (dW1 is rows 0..15 of a 128-row product; the others are full)
__global__ void k_sur_gather_grads(const float *__restrict__ dW1, const float *__restrict__ dW2,
                                   const float *__restrict__ dW3, const float *__restrict__ dW4,
                                   const float *__restrict__ db1, const float *__restrict__ db2,
                                   const float *__restrict__ db3, const float *__restrict__ db4, float *__restrict__ g)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < SUR_NPARAM; t += gridDim.x * blockDim.x) {
        float v;
        if (t < SUR_OFF_B1) v = dW1[t];
        else if (t < SUR_OFF_W2) v = db1[t - SUR_OFF_B1];
        else if (t < SUR_OFF_B2) v = dW2[t - SUR_OFF_W2];
        else if (t < SUR_OFF_W3) v = db2[t - SUR_OFF_B2];
        else if (t < SUR_OFF_B3) v = dW3[t - SUR_OFF_W3];
        else if (t < SUR_OFF_W4) v = db3[t - SUR_OFF_B3];
        else if (t < SUR_OFF_B4) v = dW4[t - SUR_OFF_W4];
        else v = db4[t - SUR_OFF_B4];
        g[t] = v;
    }
}

// bf16 copies of the weights: W (in x out, row-major) and W^T (out x in)
__device__ __forceinline__ void sur_weight_dims(int l, int &off, int &in, int &out)
{
    const int offs[4] = {SUR_OFF_W1, SUR_OFF_W2, SUR_OFF_W3, SUR_OFF_W4};
    const int ins[4] = {SUR_IN, SUR_H, SUR_H, SUR_H};
    const int outs[4] = {SUR_H, SUR_H, SUR_H, SUR_OUT};
    off = offs[l];
    in = ins[l];
    out = outs[l];
}

struct SurBf16 {
    __nv_bfloat16 *W[4], *Wt[4];
};

__global__ void k_sur_refresh_bf16(const float *__restrict__ p, SurBf16 w)
{
    for (int l = 0; l < 4; l++) {
        int off, in, out;
        sur_weight_dims(l, off, in, out);
        for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < in * out; t += gridDim.x * blockDim.x) {
            const int i = t / out, o = t % out;
            const __nv_bfloat16 v = __float2bfloat16_rn(p[off + t]);
            w.W[l][t] = v;
            w.Wt[l][o * in + i] = v;
        }
    }
}

// Adam with bias correction (t = step count, from 1)
__global__ void k_sur_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                           float *__restrict__ v, float lr, float b1, float b2, float eps, int t)
{
    const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < SUR_NPARAM; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// inputs: X (B x 16 f32) -> bf16 row-major and transposed (padded to 128 rows)
__global__ void k_sur_input(const float *__restrict__ X, __nv_bfloat16 *__restrict__ H0,
                            __nv_bfloat16 *__restrict__ H0t, int B)
{
    const long long n = (long long)B * SUR_IN;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t / SUR_IN), c = (int)(t % SUR_IN);
        const __nv_bfloat16 v = __float2bfloat16_rn(X[t]);
        H0[t] = v;
        H0t[(long long)c * B + r] = v;
    }
}

}  // namespace eu3d
