// Minimal complex helpers on CUDA vector types, FP64 and FP32.
#pragma once
#include <cuda_runtime.h>

namespace iblgf_b200
{
template<class R>
struct Cx;
template<>
struct Cx<double>
{
    using t = double2;
};
template<>
struct Cx<float>
{
    using t = float2;
};
template<class R>
using cx = typename Cx<R>::t;

template<class R>
__device__ __forceinline__ cx<R> mk(R a, R b)
{
    cx<R> r;
    r.x = a;
    r.y = b;
    return r;
}
// a += b * c
template<class R>
__device__ __forceinline__ void cmac(cx<R>& a, const cx<R>& b, const cx<R>& c)
{
    a.x = fma(b.x, c.x, fma(-b.y, c.y, a.x));
    a.y = fma(b.x, c.y, fma(b.y, c.x, a.y));
}
// a += b * conj(c)
template<class R>
__device__ __forceinline__ void cmac_conj(cx<R>& a, const cx<R>& b, const cx<R>& c)
{
    a.x = fma(b.x, c.x, fma(b.y, c.y, a.x));
    a.y = fma(b.y, c.x, fma(-b.x, c.y, a.y));
}
// a += r * c (real times complex)
template<class R>
__device__ __forceinline__ void rmac(cx<R>& a, R r, const cx<R>& c)
{
    a.x = fma(r, c.x, a.x);
    a.y = fma(r, c.y, a.y);
}
}  // namespace iblgf_b200
