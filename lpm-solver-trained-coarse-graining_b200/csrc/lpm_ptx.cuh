// Inline-PTX helpers shared by the TMA-fed operators: mbarriers with bounded waits, 4D tiled TMA loads (no
// multicast), proxy fences, and the packed FP32x2 arithmetic of sm_100a.
#pragma once
#include <cuda.h>

#include <cstdint>

namespace lpm {
namespace ptx {

constexpr unsigned kWaitLimit = 1u << 22;  // try_wait polls before a wait is declared expired

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_arrive(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase of `bar` with the given parity (at most `limit` polls); false on expiry.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned limit = kWaitLimit)
{
    for (unsigned n = 0; n < limit; ++n)
        if (mbar_test(bar, parity)) return true;
    return false;
}

// 4D tiled bulk tensor load global -> shared of this CTA, completion counted on `bar` (no multicast).
__device__ __forceinline__ void tma_load4(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                          int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(saddr(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// ---------------------------------------------------------------------------------------- packed FP32 pairs
// A pair holds the same quantity of two systems (low half: first system).  Round-to-nearest, no flush-to-zero.
using pair_t = unsigned long long;

__device__ __forceinline__ pair_t pk(float a, float b)
{
    pair_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ pair_t dup(float a) { return pk(a, a); }
__device__ __forceinline__ void unpk(pair_t v, float& a, float& b)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ pair_t add2(pair_t a, pair_t b)
{
    pair_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ pair_t sub2(pair_t a, pair_t b)
{
    pair_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ pair_t mul2(pair_t a, pair_t b)
{
    pair_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ pair_t fma2(pair_t a, pair_t b, pair_t c)
{
    pair_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// One FP64 system in place of a pair (the FP64 instantiation of the pair operator): the same names, scalar
// round-to-nearest arithmetic without contraction, as the packed instructions.
__device__ __forceinline__ double dup(double a) { return a; }
__device__ __forceinline__ double add2(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub2(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul2(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fma2(double a, double b, double c) { return __fma_rn(a, b, c); }

}  // namespace ptx
}  // namespace lpm
