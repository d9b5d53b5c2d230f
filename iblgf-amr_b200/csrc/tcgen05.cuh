// Fifth-generation tensor-core primitives of sm_100a (tcgen05) used by the
// tensor-core spectral MAC: tensor-memory allocation, register <-> tensor
// memory copies, the TF32 MMA with its A operand in tensor memory and B in
// shared memory, and the commit that signals an mbarrier when the issued
// MMAs have completed.
//
// Layouts (M = 128, one CTA):
//   tensor memory address = lane << 16 | column, 32-bit cells;
//   A (M x K, K-major): row m in lane m, element k in column a + k;
//   D (M x N, FP32):    row m in lane m, element n in column d + n;
//   B (N x K, K-major) in shared memory without swizzle: 8 x 4 core
//   matrices of 8 rows x 16 bytes (rows 16 bytes apart); the core matrix
//   holding k + 4 is kLbo bytes after the one holding k, the one holding
//   n + 8 is kSbo bytes after the one holding n.
// A warp reaches the 32 lanes 32 (warp % 4) .. + 31 of tensor memory.
#pragma once
#include <cuda_runtime.h>

#include "tma.cuh"

namespace iblgf_b200
{
namespace tc
{
constexpr unsigned kLbo = 128, kSbo = 256;

// TF32 of x, rounded to nearest (ties away), as the 32-bit pattern the MMA reads
__device__ __forceinline__ unsigned tf32_round(float x)
{
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// x = hi + lo with hi a TF32 value: the 3-product split (hi*hi + lo*hi +
// hi*lo) of two such pairs keeps FP32 accuracy in the TF32 MMA
__device__ __forceinline__ void split(float x, unsigned& hi, unsigned& lo)
{
    hi = tf32_round(x);
    lo = __float_as_uint(x - __uint_as_float(hi));
}

// shared-memory matrix descriptor of a K-major B tile without swizzle
__device__ __forceinline__ unsigned long long smem_desc(const void* p)
{
    const unsigned a = smem_addr(p);
    unsigned long long d = (unsigned long long)((a >> 4) & 0x3FFF);
    d |= (unsigned long long)((kLbo >> 4) & 0x3FFF) << 16;
    d |= (unsigned long long)((kSbo >> 4) & 0x3FFF) << 32;
    d |= 1ull << 46;  // descriptor version of sm_100
    return d;
}

// instruction descriptor: D FP32, A and B TF32, both K-major, M x N
__host__ __device__ constexpr unsigned idesc_tf32(int M, int N)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(M >> 4) << 24);
}

// executed by one whole warp
__device__ __forceinline__ void alloc(unsigned* slot, unsigned cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// executed by the warp that allocated
__device__ __forceinline__ void dealloc(unsigned base, unsigned cols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 16 consecutive columns of this thread's lane
__device__ __forceinline__ void st16(unsigned addr, const unsigned (&v)[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(addr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
        "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
}

// 8 consecutive columns of this thread's lane
__device__ __forceinline__ void st8(unsigned addr, const unsigned (&v)[8])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(addr), "r"(v[0]),
                 "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
                 : "memory");
}

__device__ __forceinline__ void ld8(unsigned addr, unsigned (&v)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(addr)
                 : "memory");
}

__device__ __forceinline__ void ld16(unsigned addr, unsigned (&v)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(addr)
        : "memory");
}

// D (+)= A B, A in tensor memory, B described by bdesc; accumulate = false
// overwrites D. Issued by one thread.
__device__ __forceinline__ void mma_tf32(unsigned d, unsigned a, unsigned long long bdesc, unsigned idesc,
                                         bool accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
        "r"(a), "l"(bdesc), "r"(idesc), "r"(accumulate ? 1u : 0u)
        : "memory");
}

// the mbarrier receives one arrival when every MMA this thread issued before
// has completed
__device__ __forceinline__ void commit(unsigned long long* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}
}  // namespace tc
}  // namespace iblgf_b200
