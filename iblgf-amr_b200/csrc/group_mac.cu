// Sibling-group spectral MAC with the fast block-Toeplitz product.
//
// Contract (include/iblgf/utilities/convolution.hpp:204-221, per pair
// acc += G_hat(u) * S_hat, summed over a target's neighbour and influence
// lists, fmm.hpp:907-1027): for a sibling group (the 8 children c of one
// parent) and a frequency f,
//     acc[c] = sum_n sum_c' G(c - c' - 2n) * s_n[c'],
// n over the parent's 27 neighbour parents, c' over their children. For a
// fixed n the 8 x 8 matrix M_n[c][c'] = G(c - c' - 2n) depends on c - c' in
// {-1,0,1}^3 only: a 3-level block-Toeplitz matrix (2 x 2 Toeplitz along each
// axis). Along one axis [[a0, a-1], [a1, a0]] (x0, x1) equals
//     y0 = m + p, y1 = m + q,  m = a0 (x0 + x1), p = (a-1 - a0) x1,
//                              q = (a1 - a0) x0,
// three products instead of four; the tensor product of the three axes
// multiplies M_n by a vector with 27 products instead of 64. The output
// combination (y0, y1 from m, p, q) does not depend on n, so each thread
// accumulates the 27 products over all neighbour parents and combines them
// into the 8 children once at the end: per (group, frequency, parent) 8
// source loads, 19 complex additions and 27 complex multiply-adds (the direct
// product takes 64). The 27 coefficients of a parent are finite-difference
// combinations of the 27 offsets around -2n; the CTA forms them once per
// frequency chunk for all its groups.
//
// CTA = (tile of sibling groups, chunk of F frequencies, half of the tile:
// NG groups), one group per thread row, F consecutive frequencies per row.
// The neighbour parents are taken in three z-slabs (nz = -1, 0, 1). Per slab
// the three z-planes of LGF spectrum rows the slab reads (3 x 49 rows of F
// frequencies) are brought into shared memory with bulk asynchronous copies
// (cp.async.bulk + transaction mbarrier; the next slab's rows are in flight
// while the current slab computes), the 9 x 27 coefficient rows are formed
// from them, and every thread walks the slab's 9 parents of its group.
// Excluded offsets (coarse targets take only non-adjacent sources) are zero
// rows, exactly as in the direct kernel. Tiles of the integrating factor
// (adjacent pairs only, 27 of 216) keep the direct kernel, which skips the
// others.
#include <type_traits>

#include "cplx.cuh"
#include "ctx.hpp"
#include "tma.cuh"

namespace iblgf_b200
{
namespace
{
template<class R>
__device__ __forceinline__ cx<R> cadd(const cx<R>& a, const cx<R>& b)
{
    return mk<R>(a.x + b.x, a.y + b.y);
}

// the 27 products of one neighbour parent: gt = coefficient rows of the
// parent (27 rows of F, this thread's frequency), s = the parent's 8
// children's source values (c' = x + 2y + 4z)
template<class R, int F>
__device__ __forceinline__ void toeplitz_parent(const cx<R>* gt, const cx<R> (&s)[8], cx<R> (&A)[27])
{
#pragma unroll
    for (int tz = 0; tz < 3; ++tz)
    {
        // along z: m = x0 + x1, p = x1, q = x0 (x0 / x1: c'z = 0 / 1)
        cx<R> v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] = tz == 0 ? cadd<R>(s[q], s[q + 4]) : (tz == 1 ? s[q + 4] : s[q]);
#pragma unroll
        for (int ty = 0; ty < 3; ++ty)
        {
            cx<R> w0, w1;  // c'x = 0, 1
            if (ty == 0)
            {
                w0 = cadd<R>(v[0], v[2]);
                w1 = cadd<R>(v[1], v[3]);
            }
            else if (ty == 1)
            {
                w0 = v[2];
                w1 = v[3];
            }
            else
            {
                w0 = v[0];
                w1 = v[1];
            }
            const int t0 = 3 * ty + 9 * tz;
            cmac<R>(A[t0], gt[t0 * F], cadd<R>(w0, w1));
            cmac<R>(A[t0 + 1], gt[(t0 + 1) * F], w1);
            cmac<R>(A[t0 + 2], gt[(t0 + 2) * F], w0);
        }
    }
}

// the 8 children from the 27 accumulated products: along each axis
// y0 = m + p, y1 = m + q
template<class R>
__device__ __forceinline__ void toeplitz_combine(const cx<R> (&A)[27], cx<R> (&y)[8])
{
    cx<R> b[2][3][3];  // [cx][ty][tz]
#pragma unroll
    for (int tz = 0; tz < 3; ++tz)
#pragma unroll
        for (int ty = 0; ty < 3; ++ty)
        {
            const int t0 = 3 * ty + 9 * tz;
            b[0][ty][tz] = cadd<R>(A[t0], A[t0 + 1]);
            b[1][ty][tz] = cadd<R>(A[t0], A[t0 + 2]);
        }
#pragma unroll
    for (int cxx = 0; cxx < 2; ++cxx)
#pragma unroll
        for (int cy = 0; cy < 2; ++cy)
        {
            cx<R> cz3[3];
#pragma unroll
            for (int tz = 0; tz < 3; ++tz) cz3[tz] = cadd<R>(b[cxx][0][tz], b[cxx][cy ? 2 : 1][tz]);
            y[cxx + 2 * cy] = cadd<R>(cz3[0], cz3[1]);
            y[cxx + 2 * cy + 4] = cadd<R>(cz3[0], cz3[2]);
        }
}

// shared memory: raw [3][49][F] | coefficients [9][27][F] | candidate rows
// [NG][216] | slot per offset [344] | mbarrier
template<class R, int F, int NG>
struct ToeplitzSmem
{
    static constexpr size_t raw = (size_t)147 * F * sizeof(cx<R>);
    static constexpr size_t coef = (size_t)243 * F * sizeof(cx<R>);
    static constexpr size_t jr = (size_t)NG * 216 * sizeof(int);
    static constexpr size_t sl = (size_t)344 * sizeof(int);
    static constexpr size_t total = raw + coef + jr + sl + 16;
};

template<class R, int F, int NG, int NB>
__global__ void __launch_bounds__(NG* F, 1)
    toeplitz_mac_kernel(const cx<R>* __restrict__ G, const cx<R>* __restrict__ S,
                        const int* __restrict__ tile_gptr, const int* __restrict__ tile_jr,
                        const int* __restrict__ tile_tab, const int* __restrict__ tile_coarse,
                        const int* __restrict__ spec_u, const unsigned* __restrict__ grp_pm,
                        const int* __restrict__ grp_tgt, cx<R>* __restrict__ ACC, int* __restrict__ status)
{
    constexpr int P = 2 * NB - 1;
    constexpr long long NC = (long long)(P / 2 + 1) * P * P;
    constexpr int NT = NG * F;
    using SM = ToeplitzSmem<R, F, NG>;
    static_assert(F % 16 == 0 && NG % 2 == 0, "rows of 16-byte pieces");
    extern __shared__ __align__(128) unsigned char smraw[];
    cx<R>* rawS = reinterpret_cast<cx<R>*>(smraw);
    cx<R>* Gt = reinterpret_cast<cx<R>*>(smraw + SM::raw);
    int* Jr = reinterpret_cast<int*>(smraw + SM::raw + SM::coef);
    int* Sl = reinterpret_cast<int*>(smraw + SM::raw + SM::coef + SM::jr);
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smraw + SM::raw + SM::coef + SM::jr + SM::sl);

    const int tile = blockIdx.x;
    const int g0 = tile_gptr[tile] + (int)blockIdx.z * NG;
    const int g1 = min(tile_gptr[tile + 1], g0 + NG);
    if (g0 >= g1) return;  // uniform over the CTA
    const long long f0 = (long long)blockIdx.y * F;
    const int valid = (int)(NC - f0 < F ? NC - f0 : F);  // frequencies of this chunk inside the row
    const unsigned row_bytes = (unsigned)(valid * sizeof(cx<R>));
    const int lane = threadIdx.x % F, row = threadIdx.x / F;
    const int mode = tile_coarse[tile];  // 0 all pairs, 1 non-adjacent only
    const int* su = spec_u + 343 * tile_tab[tile];
    const cx<R> zero = mk<R>(0, 0);

    if (threadIdx.x == 0) mbar_init(bar, 1);
    for (int r = threadIdx.x; r < 343; r += NT)
    {
        const int ux = r % 7 - 3, uy = (r / 7) % 7 - 3, uz = r / 49 - 3;
        const bool adj = ux >= -1 && ux <= 1 && uy >= -1 && uy <= 1 && uz >= -1 && uz <= 1;
        Sl[r] = (mode == 1 && adj) ? -1 : su[r];
    }
    __syncthreads();

    // rows of slab s (nz = s - 1): plane pz = dz + 1 holds uz = dz - 2 nz
    auto stage = [&](int s) {
        const int nz = s - 1;
        if (threadIdx.x < 32)
        {
            if (threadIdx.x == 0)
            {
                unsigned bytes = s == 0 ? (unsigned)(NG * 216 * sizeof(int)) : 0u;
                for (int q = 0; q < 147; ++q)
                {
                    const int uz = q / 49 - 1 - 2 * nz;
                    if (Sl[q % 49 + 49 * (uz + 3)] >= 0) bytes += row_bytes;
                }
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(bar, bytes);
            }
            __syncwarp();
            if (s == 0 && threadIdx.x == 0)
                bulk_g2s(Jr, tile_jr + ((size_t)tile * kGroupTileCap + blockIdx.z * NG) * 216,
                         (unsigned)(NG * 216 * sizeof(int)), bar);
            for (int q = threadIdx.x; q < 147; q += 32)
            {
                const int uz = q / 49 - 1 - 2 * nz;
                const int slot = Sl[q % 49 + 49 * (uz + 3)];
                if (slot >= 0) bulk_g2s(rawS + (size_t)q * F, G + (size_t)slot * NC + f0, row_bytes, bar);
            }
        }
        // excluded rows and the part of a row past the spectrum's end: zeros
        for (int i = threadIdx.x; i < 147 * F; i += NT)
        {
            const int q = i / F, f = i % F;
            const int uz = q / 49 - 1 - 2 * nz;
            if (Sl[q % 49 + 49 * (uz + 3)] < 0 || f >= valid) rawS[i] = zero;
        }
    };

    // the 9 x 27 coefficient rows of slab s from its raw rows:
    // C[t] = sum over the axes' stencils of +-G(d - 2n), per axis
    // m: {d = 0: +1}, p: {d = -1: +1, d = 0: -1}, q: {d = +1: +1, d = 0: -1}
    auto build = [&]() {
        for (int i = threadIdx.x; i < 243 * F; i += NT)
        {
            const int f = i % F, e = i / F;
            const int nxy = e / 27, t = e % 27;
            const int nx = nxy % 3 - 1, ny = nxy / 3 - 1;
            const int tt[3] = {t % 3, (t / 3) % 3, t / 9};
            cx<R> sum = zero;
#pragma unroll
            for (int az = 0; az < 2; ++az)
            {
                if (az == 1 && tt[2] == 0) continue;
                const int dz = az ? 0 : (tt[2] == 0 ? 0 : (tt[2] == 1 ? -1 : 1));
                const R sz = az ? R(-1) : R(1);
#pragma unroll
                for (int ay = 0; ay < 2; ++ay)
                {
                    if (ay == 1 && tt[1] == 0) continue;
                    const int dy = ay ? 0 : (tt[1] == 0 ? 0 : (tt[1] == 1 ? -1 : 1));
                    const R syz = ay ? -sz : sz;
#pragma unroll
                    for (int ax = 0; ax < 2; ++ax)
                    {
                        if (ax == 1 && tt[0] == 0) continue;
                        const int dx = ax ? 0 : (tt[0] == 0 ? 0 : (tt[0] == 1 ? -1 : 1));
                        const R sg = ax ? -syz : syz;
                        const cx<R> g = rawS[((dz + 1) * 49 + (dy - 2 * ny + 3) * 7 + (dx - 2 * nx + 3)) * F + f];
                        sum.x = fma(sg, g.x, sum.x);
                        sum.y = fma(sg, g.y, sum.y);
                    }
                }
            }
            Gt[(size_t)e * F + f] = sum;
        }
    };

    const int g = g0 + row;
    const bool active = g < g1;
    const unsigned pm = active ? grp_pm[g] : 0u;
    const long long f = f0 + lane;
    const cx<R>* Sf = S + (f < NC ? f : NC - 1);  // clamped column for the tail chunk
    cx<R> A[27];
#pragma unroll
    for (int t = 0; t < 27; ++t) A[t] = zero;

    bool timed_out = false;
    stage(0);
    for (int s = 0; s < 3; ++s)
    {
        __syncthreads();  // zero-filled rows visible
        timed_out = !mbar_wait(bar, (unsigned)(s & 1));
        if (__syncthreads_or(timed_out))
        {
            // the wait ran out: report it, give the copies in flight one more
            // bounded wait, and leave without touching the outputs
            if (threadIdx.x == 0)
            {
                atomicOr(status, kStatusTimeout);
                mbar_wait(bar, (unsigned)(s & 1));
            }
            __syncthreads();
            return;
        }
        build();
        __syncthreads();  // raw rows consumed, coefficients ready
        if (s < 2) stage(s + 1);  // the next slab's rows arrive while this one computes
        if (active)
        {
            const int* jr = Jr + row * 216;
            for (int nxy = 0; nxy < 9; ++nxy)
            {
                const int n = nxy + 9 * s;
                if (!((pm >> n) & 1u)) continue;
                const int4 ja = *reinterpret_cast<const int4*>(jr + 8 * n);
                const int4 jb = *reinterpret_cast<const int4*>(jr + 8 * n + 4);
                const int jj[8] = {ja.x, ja.y, ja.z, ja.w, jb.x, jb.y, jb.z, jb.w};
                cx<R> sv[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) sv[q] = __ldg(Sf + (size_t)jj[q] * NC);
                toeplitz_parent<R, F>(Gt + (size_t)nxy * 27 * F + lane, sv, A);
            }
        }
        if (s < 2) __syncthreads();  // coefficients consumed before the next build
    }
    if (active && f < NC)
    {
        cx<R> y[8];
        toeplitz_combine<R>(A, y);
#pragma unroll
        for (int c = 0; c < 8; ++c)
        {
            const int t = grp_tgt[(size_t)g * 8 + c];
            if (t >= 0) ACC[(size_t)t * NC + f] = y[c];
        }
    }
}

template<class R, int NB>
void launch_toeplitz(Ctx& c, const FmmPlan& p, const void* S, void* acc)
{
    constexpr bool f32 = std::is_same<R, float>::value;
    constexpr int F = f32 ? 32 : 16, NG = 16;
    using SM = ToeplitzSmem<R, F, NG>;
    auto kfn = toeplitz_mac_kernel<R, F, NG, NB>;
    IBLGF_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM::total));
    dim3 grid(p.n_tiles, (unsigned)((c.NC + F - 1) / F), kGroupTileCap / NG);
    kfn<<<grid, NG * F, SM::total, c.stream>>>((const cx<R>*)c.d_spec.p, (const cx<R>*)S, p.tile_gptr.p,
                                              p.tile_jr.p, p.tile_tab.p, p.tile_coarse.p, p.spec_u.p,
                                              p.grp_pm.p, p.grp_tgt.p, (cx<R>*)acc, c.d_status.p);
    c.launches += 1;
}
}  // namespace

bool toeplitz_mac(Ctx& c, const FmmPlan& p, const void* S, void* acc)
{
    if (!p.n_tiles || p.adj_only) return false;
    if (c.NC != (long long)c.Nb * c.P * c.P) throw Error(IBLGF_EINTERNAL, "spectrum row length differs");
    const bool fp32 = c.cfg.precision == IBLGF_FP32;
#define IBLGF_TOEP(NBV)                                           \
    case NBV:                                                     \
        if (fp32) launch_toeplitz<float, NBV>(c, p, S, acc);      \
        else launch_toeplitz<double, NBV>(c, p, S, acc);          \
        return true;
    switch (c.Nb)
    {
        IBLGF_TOEP(6)
        IBLGF_TOEP(8)
        IBLGF_TOEP(10)
        IBLGF_TOEP(12)
        IBLGF_TOEP(16)
        IBLGF_TOEP(18)
        default: return false;
    }
#undef IBLGF_TOEP
}

}  // namespace iblgf_b200
