// Fifth-generation tensor core (tcgen05) building blocks for sm_100a, in
// inline PTX: TMEM allocation, shared-memory matrix descriptors, BF16 MMA with
// FP32 accumulation in TMEM, commit to an mbarrier, TMEM -> register loads.
//
// Operand layout in shared memory (K-major, no swizzle).  A tile of R rows
// (R a multiple of 8) by K bf16 columns (K a multiple of 16) is stored as K/16
// slabs of R*32 bytes; inside a slab, rows come in groups of 8 (256 bytes per
// group), each group holding two 8 x 16-byte core matrices: columns k%16 < 8
// first, then k%16 >= 8 (128 bytes apart).  One MMA reads one slab with
// leading byte offset 128 (between the two K halves) and stride byte offset
// 256 (between 8-row groups).
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

namespace eu3d {
namespace tc {

constexpr uint32_t LBO = 128, SBO = 256;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (r, k) of an R-row operand tile
__host__ __device__ __forceinline__ uint32_t op_off(int R, int r, int k)
{
    return (uint32_t)((k >> 4) * (R * 32) + (r >> 3) * 256 + ((k >> 3) & 1) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor (no swizzle, Blackwell version bit)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((LBO >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((SBO >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor: A, B bf16 K-major, D f32; M in {64, 128}, N % 16 == 0
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// arrive on mbar when all previously issued MMAs of this thread complete
__device__ __forceinline__ void commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// non-blocking test of an mbarrier phase
__device__ __forceinline__ bool mbar_test(uint32_t mbar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}

// potentially blocking test without a suspend-time hint: the hardware
// resumes the thread when the phase completes (or after its own time limit,
// then false)
__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// bounded wait on an mbarrier phase: false when the bound ran out, so that
// no caller can spin forever.  The bound is max_tries attempts and at most
// one second of the global timer, whichever ends first.  Waiting threads
// block in try_wait, which the hardware ends as soon as the phase completes;
// a suspend-time hint is not given (with one, a wait that found the copy
// still in flight slept out the hint, which set the pace of the flux ring).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint32_t max_tries = (1u << 19))
{
    uint64_t t0 = 0;
    for (uint32_t t = 0; t < max_tries; t++) {
        if (mbar_try(mbar, parity)) return true;
        const uint64_t now = global_ns();
        if (t == 0)
            t0 = now;
        else if (now - t0 > 1000000000ull)
            return false;
    }
    return false;
}

// arm an mbarrier for one arrival plus `bytes` of asynchronous copy
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// make mbarrier initialisation visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// TMA tiled load of one 4-D box (coordinates innermost first) into shared
// memory, completing on mbar.  No multicast.  The innermost coordinate x
// times the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const void *tmap, int x, int y, int z, int w, uint32_t mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(dst),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(w), "r"(mbar)
        : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// make generic-proxy shared-memory writes visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMEM allocation by one full warp; the base address lands in *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes 32w..32w+31)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float v[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive FP32 columns
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace eu3d
