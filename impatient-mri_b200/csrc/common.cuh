// Shared device helpers for the IMPATIENT B200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

namespace imp {

// Error bits a kernel can raise in the context's device error word.
enum : unsigned {
    DEV_ERR_TIMEOUT = 1u,   // a bounded mbarrier wait ran out
    DEV_ERR_RANGE = 2u,     // an input coordinate is outside the fixed-point phase range
};

constexpr double kTwoPi = 6.283185307179586476925286766559;

// ---------------------------------------------------------------------------
// mbarrier + bulk-copy (TMA, non-tensor) primitives.  Every wait is bounded:
// on expiry the kernel records DEV_ERR_TIMEOUT and carries on, so all threads
// still reach the same barriers and the launch ends.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: about 2^22 polls (each try_wait may itself suspend briefly).
__device__ __forceinline__ void mbar_wait_bounded(uint64_t *bar, unsigned parity,
                                                  unsigned *err) {
    for (unsigned it = 0; it < (1u << 22); ++it)
        if (mbar_try_wait(bar, parity)) return;
    if (err) atomicOr(err, DEV_ERR_TIMEOUT);
}

// Global -> shared bulk copy completing on an mbarrier.  Both addresses
// 16-byte aligned, bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_g2s(void *smem_dst, const void *gmem_src, unsigned bytes,
                                         uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// ---------------------------------------------------------------------------
// Block reductions (FP64) used by the CG scalars.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the block; the result is valid in thread 0.  `sh` holds >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double *sh) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        r = lane < nw ? sh[lane] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

// Deterministic sum of `n` per-block partials, computed redundantly by every
// block that needs it (n is small: a few hundred).  Valid in all threads.
__device__ __forceinline__ double sum_partials(const double *p, int n, double *sh) {
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v += p[i];
    v = block_sum(v, sh);
    __syncthreads();
    if (threadIdx.x == 0) sh[32] = v;
    __syncthreads();
    return sh[32];
}

__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

}  // namespace imp
