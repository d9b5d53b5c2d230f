// Batched per-block FFT convolution of the LGF-FMM sweep, hand-written for
// sm_100a (no cuFFT). Contract: include/iblgf/utilities/convolution.hpp:225-304
// and src/utilities/convolution.cpp — a zero-padded Nb^3 source and a
// (2Nb-1)^3 LGF block in a P^3 = (2Nb-1)^3 box, r2c, pointwise product
// accumulated per target, c2r, window [Nb-1, 2Nb-2]^3 added into the target
// block, scaled by dx^2 / P^3.
//
// B200 structure (one sweep = all blocks of all tree levels at once):
//   fwd_xy_rows  one CTA per source block: thread (z, y) transforms row y
//                along x (real, Nb -> Nb half frequencies), thread (z, kx)
//                then column kx along y (Nb -> P)
//   fwd_z        one thread per (ky,kx) pencil: z transform (Nb -> P)
//                Each source block is transformed once per sweep; the
//                reference transforms it once per (source, target) pair.
//   group_mac    sibling-group spectral multiply-accumulate (mac_kernel:
//                general pair-list fallback)
//   inv_fused    one CTA per (target, half of the output planes): z inverse,
//                y inverse and c2r along x of the extraction window, in
//                shared memory, added into the FP64 target block
// The half spectrum is laid out [kz][ky][kx], kx < Nb (= P/2 + 1), as in the
// reference's r2c output. Transforms are direct pruned DFTs (half of the
// inputs zero, half of the outputs discarded). The forward loops are unrolled
// over frequency and sample index so each twiddle is a compile-time constant
// operand; the FP64 inverse reads a per-CTA twiddle table instead.
#include <cmath>
#include <mutex>
#include <set>
#include <type_traits>
#include <vector>

#include <cuda_pipeline.h>

#include "cplx.cuh"
#include "ctx.hpp"
#include "lgf_dev.cuh"

namespace iblgf_b200
{
namespace
{
enum InMode { kFromLgf = 1, kFromDense = 2 };

template<class R>
__device__ __forceinline__ void load_tw(cx<R>* s_tw, const R* tw, int P)
{
    for (int j = threadIdx.x; j < P; j += blockDim.x) s_tw[j] = mk<R>(tw[2 * j], tw[2 * j + 1]);
}

// Twiddles e^{-2 pi i j / P} of every supported P (Nb = 6, 8, 10, 12, 16, 18)
// in constant memory. The transform loops below are unrolled over both the
// frequency and the sample index, so (k * j) mod P is a compile-time constant
// and every twiddle is an immediate FMA operand: no shared-memory loads.
constexpr int kTwTotal = 11 + 15 + 19 + 23 + 31 + 35;
__host__ __device__ constexpr int tw_base(int P)
{
    return P == 11 ? 0 : P == 15 ? 11 : P == 19 ? 26 : P == 23 ? 45 : P == 31 ? 68 : 99;
}
__constant__ double c_tw64[2 * kTwTotal];
__constant__ float c_tw32[2 * kTwTotal];

template<class R, int P>
__device__ __forceinline__ cx<R> ctw(int j)
{
    if constexpr (std::is_same<R, double>::value)
        return mk<R>(c_tw64[2 * (tw_base(P) + j)], c_tw64[2 * (tw_base(P) + j) + 1]);
    else
        return mk<R>(c_tw32[2 * (tw_base(P) + j)], c_tw32[2 * (tw_base(P) + j) + 1]);
}

// Fully unrolled FP64 transforms at Nb = 18 exceed the register budget (the
// scheduler hoists the loads of every term), so there the output loop stays
// rolled and the twiddle index is carried in per-term counters; the twiddle
// load is then one uniform constant-cache read.
template<class R, int NB>
constexpr bool kRollOutputs = std::is_same<R, double>::value && NB >= 18;

// x and y transforms of a whole field block: thread (z, y) takes row y of
// plane z along x (real NB -> NB half frequencies) into shared memory, then
// thread (z, kx) takes column kx of plane z along y (NB -> P) and writes
// W[item][z][ky][kx]. One CTA (NB^2 threads) per block; shared rows have an
// odd stride (NB + 1 complex), so both passes are free of bank conflicts.
template<class R, int NB>
__global__ void __launch_bounds__(NB * NB) fwd_xy_rows_kernel(const double* __restrict__ field,
                                                              const int* __restrict__ item_oct,
                                                              cx<R>* __restrict__ W)
{
    constexpr int P = 2 * NB - 1, S = NB + 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<R>* s_x1 = reinterpret_cast<cx<R>*>(smraw);  // [z][y][kx]
    const int item = blockIdx.x;
    const int z = threadIdx.x / NB, r = threadIdx.x % NB;
    {
        const double* row = field + (size_t)item_oct[item] * (NB * NB * NB) + (size_t)threadIdx.x * NB;
        R in[NB];
#pragma unroll
        for (int x = 0; x < NB; ++x) in[x] = (R)row[x];
        cx<R>* dst = s_x1 + (size_t)threadIdx.x * S;
        if constexpr (kRollOutputs<R, NB>)
        {
            int j[NB];  // j[x] = kx * x mod P
#pragma unroll
            for (int x = 0; x < NB; ++x) j[x] = 0;
#pragma unroll 1
            for (int kx = 0; kx < NB; ++kx)
            {
                cx<R> s = mk<R>(0, 0);
#pragma unroll
                for (int x = 0; x < NB; ++x)
                {
                    rmac<R>(s, in[x], ctw<R, P>(j[x]));
                    j[x] = j[x] + x >= P ? j[x] + x - P : j[x] + x;
                }
                dst[kx] = s;
            }
        }
        else
        {
#pragma unroll
            for (int kx = 0; kx < NB; ++kx)
            {
                cx<R> s = mk<R>(0, 0);
#pragma unroll
                for (int x = 0; x < NB; ++x) rmac<R>(s, in[x], ctw<R, P>((kx * x) % P));
                dst[kx] = s;
            }
        }
    }
    __syncthreads();
    cx<R> v[NB];
#pragma unroll
    for (int y = 0; y < NB; ++y) v[y] = s_x1[(z * NB + y) * S + r];
    cx<R>* out = W + ((size_t)item * NB + z) * (P * NB) + r;
    if constexpr (kRollOutputs<R, NB>)
    {
        int j[NB];  // j[y] = ky * y mod P
#pragma unroll
        for (int y = 0; y < NB; ++y) j[y] = 0;
#pragma unroll 1
        for (int ky = 0; ky < P; ++ky)
        {
            cx<R> s = mk<R>(0, 0);
#pragma unroll
            for (int y = 0; y < NB; ++y)
            {
                cmac<R>(s, v[y], ctw<R, P>(j[y]));
                j[y] = j[y] + y >= P ? j[y] + y - P : j[y] + y;
            }
            out[(size_t)ky * NB] = s;
        }
    }
    else
    {
#pragma unroll
        for (int ky = 0; ky < P; ++ky)
        {
            cx<R> s = mk<R>(0, 0);
#pragma unroll
            for (int y = 0; y < NB; ++y) cmac<R>(s, v[y], ctw<R, P>((ky * y) % P));
            out[(size_t)ky * NB] = s;
        }
    }
}

// fwd_xy: x and y transforms of one z plane of one block.
//   kFromLgf:   G((b + i) * 2^ld), desc[4*item] = {ld, bx, by, bz}  (NIN = P)
//   kFromDense: dense[item * P^3]                                  (NIN = P)
// W: [item][z < NIN][ky < P][kx < NB]
template<class R, int NB, int NIN, int MODE>
__global__ void __launch_bounds__(256) fwd_xy_kernel(const double* __restrict__ field,
                                                     const int* __restrict__ item_oct,
                                                     const int* __restrict__ desc,
                                                     const double* __restrict__ table,
                                                     const R* __restrict__ tw, cx<R>* __restrict__ W,
                                                     const double* __restrict__ ge, int ge_stride)
{
    constexpr int P = 2 * NB - 1;
    __shared__ cx<R> s_tw[P];
    __shared__ R s_in[NIN * NIN];
    __shared__ cx<R> s_x1[NIN * NB];
    const int item = blockIdx.x;
    const int z = blockIdx.y;
    load_tw<R>(s_tw, tw, P);
    if (MODE == kFromLgf)
    {
        // desc[0] >= 0: LGF_GL at stride 2^level_diff (lgf.hpp:222-262);
        // desc[0] < 0: LGF_GE table -desc[0]-1, E(n) = f[|n1|] f[|n2|] f[|n3|]
        const int ld = desc[4 * item];
        const int bx = desc[4 * item + 1], by = desc[4 * item + 2], bz = desc[4 * item + 3];
        if (ld >= 0)
        {
            const int st = 1 << ld;
            for (int i = threadIdx.x; i < NIN * NIN; i += blockDim.x)
            {
                const int x = i % NIN, y = i / NIN;
                s_in[i] = (R)lgf_get_dev((bx + x) * st, (by + y) * st, (bz + z) * st, table);
            }
        }
        else
        {
            const double* f = ge + (size_t)(-ld - 1) * ge_stride;
            const double fz = f[abs(bz + z)];
            for (int i = threadIdx.x; i < NIN * NIN; i += blockDim.x)
            {
                const int x = i % NIN, y = i / NIN;
                s_in[i] = (R)(f[abs(bx + x)] * f[abs(by + y)] * fz);
            }
        }
    }
    else
    {
        const double* blk = field + (size_t)item * P * P * P + (size_t)z * P * P;
        for (int i = threadIdx.x; i < NIN * NIN; i += blockDim.x) s_in[i] = (R)blk[i];
    }
    __syncthreads();
    // x: real NIN -> NB half frequencies
    for (int i = threadIdx.x; i < NIN * NB; i += blockDim.x)
    {
        const int y = i / NB, kx = i % NB;
        cx<R> s = mk<R>(0, 0);
        int j = 0;
#pragma unroll 6
        for (int x = 0; x < NIN; ++x)
        {
            rmac<R>(s, s_in[y * NIN + x], s_tw[j]);
            j += kx;
            if (j >= P) j -= P;
        }
        s_x1[y * NB + kx] = s;
    }
    __syncthreads();
    // y: NIN -> P
    cx<R>* out = W + ((size_t)item * NIN + z) * (P * NB);
    for (int i = threadIdx.x; i < P * NB; i += blockDim.x)
    {
        const int ky = i / NB, kx = i % NB;
        cx<R> s = mk<R>(0, 0);
        int j = 0;
#pragma unroll 6
        for (int y = 0; y < NIN; ++y)
        {
            cmac<R>(s, s_x1[y * NB + kx], s_tw[j]);
            j += ky;
            if (j >= P) j -= P;
        }
        out[i] = s;
    }
}

// fwd_z: per (ky,kx) pencil, NIN -> P; spectrum slot = item_slot[item] (or item)
template<class R, class RO, int NB, int NIN>
__global__ void __launch_bounds__(128) fwd_z_kernel(const cx<R>* __restrict__ W, const int* __restrict__ item_slot,
                                                    cx<RO>* __restrict__ spec)
{
    constexpr int P = 2 * NB - 1;
    constexpr int NP = P * NB;
    const int item = blockIdx.x;
    const int p = blockIdx.y * blockDim.x + threadIdx.x;
    if (p >= NP) return;
    const cx<R>* w = W + (size_t)item * NIN * NP + p;
    cx<R> v[NIN];
#pragma unroll
    for (int z = 0; z < NIN; ++z) v[z] = w[(size_t)z * NP];
    const int slot = item_slot ? item_slot[item] : item;
    cx<RO>* out = spec + (size_t)slot * P * NP + p;
    if constexpr (NIN > NB)
    {
        // dense P-point input (LGF spectra, cache fill only): kz rolled
#pragma unroll 1
        for (int kz = 0; kz < P; ++kz)
        {
            cx<R> s = mk<R>(0, 0);
            int j = 0;
#pragma unroll
            for (int z = 0; z < NIN; ++z)
            {
                cmac<R>(s, v[z], ctw<R, P>(j));
                j += kz;
                if (j >= P) j -= P;
            }
            out[(size_t)kz * NP] = mk<RO>((RO)s.x, (RO)s.y);
        }
    }
    else
    {
#pragma unroll
        for (int kz = 0; kz < P; ++kz)
        {
            cx<R> s = mk<R>(0, 0);
#pragma unroll
            for (int z = 0; z < NIN; ++z) cmac<R>(s, v[z], ctw<R, P>((kz * z) % P));
            out[(size_t)kz * NP] = mk<RO>((RO)s.x, (RO)s.y);
        }
    }
}

// mac: ACC[t][f] = sum_pairs G[spec][f] * S[src][f]
template<class R>
__global__ void __launch_bounds__(128) mac_kernel(const cx<R>* __restrict__ G, const cx<R>* __restrict__ S,
                                                  const int* __restrict__ pair_ptr,
                                                  const int* __restrict__ pair_src,
                                                  const int* __restrict__ pair_spec, long long NC,
                                                  cx<R>* __restrict__ ACC)
{
    const long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int t = blockIdx.y;
    if (f >= NC) return;
    cx<R> acc = mk<R>(0, 0);
    const int j0 = pair_ptr[t], j1 = pair_ptr[t + 1];
    for (int j = j0; j < j1; ++j)
    {
        const cx<R> g = G[(size_t)pair_spec[j] * NC + f];
        const cx<R> s = S[(size_t)pair_src[j] * NC + f];
        cmac<R>(acc, g, s);
    }
    ACC[(size_t)t * NC + f] = acc;
}

// Sibling-group MAC. At a sweep's base level the neighbours and the influence
// list of a target together are exactly the children of its parent's 27
// neighbours; coarser targets see the non-adjacent ones. The 8 siblings of a
// parent therefore share one candidate source set (216 = 27 x 8 candidates
// k = (n, c')), and the offset of (child c, candidate (n, c')) is
// u = c - c' - 2n in [-3,3]^3 (343 LGF spectra per tile).
// For one neighbour parent n the 64 (c, c') pairs use only the 27 offsets
// u = d - 2n, d = c - c' in [-1,1]^3; the kernel walks n and, per dz = cz - c'z,
// keeps the 9 spectra of that z-offset (shared by the slabs (c'z, cz) = (0, 0)
// and (1, 1) at dz = 0) in registers for 16 or 32 complex MACs.
// Adjacency filtering (coarse targets take only non-adjacent sources, the
// integrating factor only adjacent ones) depends on u alone, so it is applied
// once when the tile's spectra are staged: excluded offsets become zero rows.
// Tiles that take all or the non-adjacent pairs then run every pair (an
// excluded pair adds exactly zero); tiles of adjacent pairs only (the
// integrating factor, 27 of 216) skip the others.
// One CTA = (tile of up to 32 sibling groups, chunk of F frequencies); each warp
// takes one group at 32 consecutive frequencies, so a source load is one
// contiguous 256-byte (FP32) or 512-byte (FP64) row segment. The tile's
// spectra and the groups' candidate rows (precomputed with the plan, tile_jr)
// are copied asynchronously into shared memory; source spectra are read
// through L1/L2. Candidates that do not exist read a zero spectrum row (zrow),
// and parents without any candidate are skipped via the group's 27-bit mask
// (grp_pm).
template<class R, int F, bool ADJ_ONLY>
__device__ __forceinline__ void group_mac_parent(const cx<R>* gn, const cx<R> (&sv)[8], cx<R> (&acc)[8], int nx,
                                                 int ny, int nz)
{
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
    {
        if (ADJ_ONLY && abs(dz - 2 * nz) > 1) continue;
        cx<R> gv[9];
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx)
                gv[(dy + 1) * 3 + dx + 1] = gn[(dx + 7 * dy + 49 * dz) * F];
#pragma unroll
        for (int cpz = 0; cpz < 2; ++cpz)
        {
            const int cz = cpz + dz;
            if (cz < 0 || cz > 1) continue;
#pragma unroll
            for (int q = 0; q < 4; ++q)  // c' = 4 cpz + q
#pragma unroll
                for (int r = 0; r < 4; ++r)  // c = 4 cz + r
                {
                    const int dx = (r & 1) - (q & 1), dy = (r >> 1) - (q >> 1);
                    if (ADJ_ONLY && (abs(dx - 2 * nx) > 1 || abs(dy - 2 * ny) > 1)) continue;
                    cmac<R>(acc[4 * cz + r], gv[(dy + 1) * 3 + dx + 1], sv[4 * cpz + q]);
                }
        }
    }
}

template<class R, int F, int NT, int MINB, int NB>
__global__ void __launch_bounds__(NT, MINB) group_mac_kernel(
    const cx<R>* __restrict__ G, const cx<R>* __restrict__ S, int zrow,
    const int* __restrict__ tile_gptr, const int* __restrict__ tile_jr,
    const int* __restrict__ tile_tab, const int* __restrict__ tile_coarse, const int* __restrict__ spec_u,
    const unsigned* __restrict__ grp_pm,
    const int* __restrict__ grp_tgt, cx<R>* __restrict__ ACC)
{
    constexpr int RW = NT / F;      // thread rows, one group each per pass
    constexpr int P = 2 * NB - 1;
    constexpr long long NC = (long long)(P / 2 + 1) * P * P;  // spectrum row length
    constexpr int per = 16 / sizeof(cx<R>);
    constexpr int parts = F / per;  // 16-byte pieces of a staged row
    static_assert(F % 32 == 0 && NT % F == 0, "a warp covers one row");
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<R>* Gs = reinterpret_cast<cx<R>*>(smraw);                      // [343][F]
    int* Jr = reinterpret_cast<int*>(Gs + 343 * F);                  // [tile groups][216] source rows
    const int tile = blockIdx.x;
    const long long f0 = (long long)blockIdx.y * F;
    const int lane = threadIdx.x % F, row = threadIdx.x / F;
    const int mode = tile_coarse[tile];  // 0 all, 1 non-adjacent only, 2 adjacent only
    const int* su = spec_u + 343 * tile_tab[tile];
    const int g0 = tile_gptr[tile], g1 = tile_gptr[tile + 1];
    const cx<R> zero = mk<R>(0, 0);
    const bool full = f0 + F <= NC;
    {
        // the tile's candidate rows, one 16-byte copy per 4 entries
        const int* jsrc = tile_jr + (size_t)tile * kGroupTileCap * 216;
        for (int i = threadIdx.x; i < kGroupTileCap * 216 / 4; i += blockDim.x)
            __pipeline_memcpy_async(Jr + 4 * i, jsrc + 4 * i, 16);
    }
    // spectrum slot of each offset row (-1: excluded by the tile's mode),
    // evaluated once per row
    int* Sl = Jr + kGroupTileCap * 216;
    for (int r = threadIdx.x; r < 343; r += blockDim.x)
    {
        const int ux = r % 7 - 3, uy = (r / 7) % 7 - 3, uz = r / 49 - 3;
        const bool adj = ux >= -1 && ux <= 1 && uy >= -1 && uy <= 1 && uz >= -1 && uz <= 1;
        Sl[r] = (mode == 1 && adj) || (mode == 2 && !adj) ? -1 : su[r];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 343 * parts; q += blockDim.x)
    {
        const int r = q / parts, part = q % parts;
        const int slot = Sl[r];
        cx<R>* dst = Gs + r * F + part * per;
        const cx<R>* src = slot >= 0 ? G + (size_t)slot * NC + f0 + part * per : nullptr;
        if (src && full) __pipeline_memcpy_async(dst, src, 16);
        else
            for (int e = 0; e < per; ++e)
                dst[e] = (src && f0 + part * per + e < NC) ? src[e] : zero;
    }
    __pipeline_commit();
    __pipeline_wait_prior(0);
    __syncthreads();
    const long long f = f0 + lane;
    const long long fc = f < NC ? f : NC - 1;  // clamped column for the tail chunk
    const cx<R>* Sf = S + fc;
    for (int g = g0 + row; g < g1; g += RW)
    {
        const int* jr = Jr + (g - g0) * 216;
        const unsigned pm = grp_pm[g];
        cx<R> acc[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[c] = zero;
        // neighbour parents n = (nx, ny, nz): the x-offset unrolled, so that the
        // LGF row of u = -2n (d = (dx, dy, dz) adds dx + 7 dy + 49 dz) sits at
        // a compile-time offset from the (ny, nz) base
        for (int nzy = 0; nzy < 9; ++nzy)
        {
            const int ny = nzy % 3 - 1, nz = nzy / 3 - 1;
            const cx<R>* gzy = Gs + (7 * (3 - 2 * ny) + 49 * (3 - 2 * nz)) * F + lane;
#pragma unroll
            for (int nxi = 0; nxi < 3; ++nxi)
            {
                const int n = 3 * nzy + nxi, nx = nxi - 1;
                if (!((pm >> n) & 1u)) continue;
                const int4 ja = *reinterpret_cast<const int4*>(jr + 8 * n);
                const int4 jb = *reinterpret_cast<const int4*>(jr + 8 * n + 4);
                const int jj[8] = {ja.x, ja.y, ja.z, ja.w, jb.x, jb.y, jb.z, jb.w};
                cx<R> sv[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) sv[q] = __ldg(Sf + (size_t)jj[q] * NC);
                const cx<R>* gn = gzy + (3 - 2 * nx) * F;
                if (mode == 2) group_mac_parent<R, F, true>(gn, sv, acc, nx, ny, nz);
                else group_mac_parent<R, F, false>(gn, sv, acc, nx, ny, nz);
            }
        }
        if (f < NC)
        {
#pragma unroll
            for (int c = 0; c < 8; ++c)
            {
                const int t = grp_tgt[(size_t)g * 8 + c];
                if (t >= 0) ACC[(size_t)t * NC + f] = acc[c];
            }
        }
    }
}

// Fused inverse of one target block: z inverse, y inverse, c2r along x and
// target[oct] += scale * window, with every intermediate in shared memory.
// One CTA per (target, half of the NB output z-planes), NB^2 threads:
//   z  thread per pencil (ky, kx): the P accumulators (working precision RA,
//      widened to FP64) -> the NB/2 output planes of this half, into sV
//   y  thread (kx, plane, half of yo): P -> NB/2 outputs yo
//   x  thread (yo, plane, half of xo): c2r NB -> NB/2 outputs xo
// All three passes use one FP64 table sT[k][o] = e^{-2 pi i k (o + NB - 1) / P}
// (conjugated): each pass loops over its input index k and reads row k of
// the table at compile-time offsets, a uniform broadcast read. The inverse
// runs in FP64 on both paths: cancellation in the c2r amplifies FP32
// rounding of the twiddled sums far more than in the forward transforms.
// The summation order per output is the reference order k = 0, 1, ...
template<class RA, int NB>
__global__ void __launch_bounds__(NB * NB, 2) inv_fused_kernel(const cx<RA>* __restrict__ ACC,
                                                               const int* __restrict__ tgt_oct, double scale,
                                                               double* __restrict__ target)
{
    constexpr int P = 2 * NB - 1, NP = P * NB, ZH = NB / 2, S = NB + 1;
    static_assert(NB % 2 == 0, "the block splits into two halves of output planes");
    extern __shared__ __align__(16) unsigned char smraw[];
    double2* sT = reinterpret_cast<double2*>(smraw);  // [k < P][o < NB]
    double2* sV = sT + P * NB;                        // [plane][ky][kx], then [plane][yo][kx] (stride S)
    const int t = blockIdx.x, h = blockIdx.y;
    for (int i = threadIdx.x; i < P * NB; i += blockDim.x)
        sT[i] = ctw<double, P>(((i / NB) * (i % NB + NB - 1)) % P);
    __syncthreads();
    // z: P -> the ZH planes zo = h ZH + i
    const cx<RA>* a = ACC + (size_t)t * P * NP;
    for (int p = threadIdx.x; p < NP; p += blockDim.x)
    {
        double2 acc[ZH];
#pragma unroll
        for (int i = 0; i < ZH; ++i) acc[i] = mk<double>(0, 0);
#pragma unroll 5
        for (int kz = 0; kz < P; ++kz)
        {
            const cx<RA> x0 = a[(size_t)kz * NP + p];
            const double2 x = mk<double>((double)x0.x, (double)x0.y);
            const double2* tr = sT + kz * NB + h * ZH;
#pragma unroll
            for (int i = 0; i < ZH; ++i) cmac_conj<double>(acc[i], x, tr[i]);
        }
#pragma unroll
        for (int i = 0; i < ZH; ++i) sV[i * NP + p] = acc[i];
    }
    __syncthreads();
    // y: thread (kx, plane zl, half yh of the outputs yo)
    const int kx = threadIdx.x % NB, rest = threadIdx.x / NB, zl = rest % ZH, yh = rest / ZH;
    double2 acc[ZH];
#pragma unroll
    for (int i = 0; i < ZH; ++i) acc[i] = mk<double>(0, 0);
#pragma unroll 5
    for (int ky = 0; ky < P; ++ky)
    {
        const double2 x = sV[zl * NP + ky * NB + kx];
        const double2* tr = sT + ky * NB + yh * ZH;
#pragma unroll
        for (int i = 0; i < ZH; ++i) cmac_conj<double>(acc[i], x, tr[i]);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < ZH; ++i) sV[(zl * NB + yh * ZH + i) * S + kx] = acc[i];
    __syncthreads();
    // x: thread (yo, plane zl2, half xh of the outputs xo); c2r of the half
    // spectrum: v = Re y_0 + 2 sum_{k >= 1} Re(y_k e^{+2 pi i k (xo + NB - 1) / P})
    const int xh = threadIdx.x / (ZH * NB), r2 = threadIdx.x % (ZH * NB), zl2 = r2 / NB, yo = r2 % NB;
    const double2* yrow = sV + (size_t)(zl2 * NB + yo) * S;
    double sx[ZH];
#pragma unroll
    for (int i = 0; i < ZH; ++i) sx[i] = 0;
#pragma unroll 6
    for (int k = 1; k < NB; ++k)
    {
        const double2 y = yrow[k];
        const double2* tr = sT + k * NB + xh * ZH;
#pragma unroll
        for (int i = 0; i < ZH; ++i) sx[i] = fma(y.x, tr[i].x, fma(y.y, tr[i].y, sx[i]));
    }
    const double y0 = yrow[0].x;
    double* out = target + (size_t)tgt_oct[t] * NB * NB * NB + ((size_t)(h * ZH + zl2) * NB + yo) * NB + xh * ZH;
#pragma unroll
    for (int i = 0; i < ZH; ++i) out[i] += scale * (y0 + 2.0 * sx[i]);
}

template<class R, int NB>
struct Conv
{
    using Real = R;
    static constexpr int Nb = NB;
    static constexpr int P = 2 * NB - 1;
    static constexpr int NP = P * NB;

    static void launch_fwd_xy_rows(Ctx& c, const double* field, const int* d_item_oct, int n, cx<R>* W)
    {
        const int smem = NB * NB * (NB + 1) * (int)sizeof(cx<R>);
        auto kfn = fwd_xy_rows_kernel<R, NB>;
        IBLGF_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        kfn<<<n, NB * NB, smem, c.stream>>>(field, d_item_oct, W);
    }

    static void launch_inverse(Ctx& c, const cx<R>* acc, const int* d_tgt_oct, int n, double scale, double* target)
    {
        const int smem = (P * NB + NB / 2 * NP) * (int)sizeof(double2);
        auto kfn = inv_fused_kernel<R, NB>;
        IBLGF_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        kfn<<<dim3(n, 2), NB * NB, smem, c.stream>>>(acc, d_tgt_oct, scale, target);
    }

    static void forward_field(Ctx& c, const double* field, const int* d_item_oct, int n, void* spec)
    {
        if (!n) return;
        cx<R>* W = (cx<R>*)c.d_w.p;
        launch_fwd_xy_rows(c, field, d_item_oct, n, W);
        fwd_z_kernel<R, R, NB, NB><<<dim3(n, (NP + 127) / 128), 128, 0, c.stream>>>(W, nullptr, (cx<R>*)spec);
        c.launches += 2;
    }

    // LGF blocks (or a dense kernel) are transformed in FP64 and stored in R
    static void forward_lgf(Ctx& c, const int* d_desc, const double* dense, const int* d_slot, int n,
                            void* spec)
    {
        if (!n) return;
        double2* W = (double2*)c.d_w.p;
        if (dense)
            fwd_xy_kernel<double, NB, P, kFromDense><<<dim3(n, P), 256, 0, c.stream>>>(
                dense, nullptr, nullptr, nullptr, c.d_tw64.p, W, nullptr, 0);
        else
            fwd_xy_kernel<double, NB, P, kFromLgf><<<dim3(n, P), 256, 0, c.stream>>>(
                nullptr, nullptr, d_desc, c.d_lgf_table.p, c.d_tw64.p, W, c.d_ge.p, c.ge_stride);
        fwd_z_kernel<double, R, NB, P><<<dim3(n, (NP + 127) / 128), 128, 0, c.stream>>>(W, d_slot,
                                                                                      (cx<R>*)spec);
        c.launches += 2;
    }

    static void mac(Ctx& c, const void* G, const void* S, const int* ptr, const int* src, const int* spec,
                    int n_tgt, void* acc)
    {
        if (!n_tgt) return;
        dim3 grid((unsigned)((c.NC + 127) / 128), n_tgt);
        mac_kernel<R><<<grid, 128, 0, c.stream>>>((const cx<R>*)G, (const cx<R>*)S, ptr, src, spec, c.NC,
                                                  (cx<R>*)acc);
        c.launches += 1;
    }

    static constexpr bool kF32 = std::is_same<R, float>::value;

    // S holds p.n_src source spectra followed by one zero row. Two tile
    // shapes per precision (frequencies per CTA GF, threads GNT), chosen per
    // plan by the MAC autotuner: variant 0 = (64, 768) FP32 / (32, 512)
    // FP64, variant 1 = (32, 512) / (32, 256)
    template<int GF, int GNT>
    static void group_mac_shape(Ctx& c, const FmmPlan& p, const void* S, void* acc)
    {
        const size_t smem = (size_t)343 * GF * sizeof(cx<R>) + (size_t)(kGroupTileCap * 216 + 344) * sizeof(int);
        auto kfn = group_mac_kernel<R, GF, GNT, 1, NB>;
        IBLGF_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        dim3 grid(p.n_tiles, (unsigned)((c.NC + GF - 1) / GF));
        kfn<<<grid, GNT, smem, c.stream>>>((const cx<R>*)c.d_spec.p, (const cx<R>*)S, p.n_src,
                                            p.tile_gptr.p, p.tile_jr.p, p.tile_tab.p,
                                            p.tile_coarse.p, p.spec_u.p, p.grp_pm.p, p.grp_tgt.p,
                                            (cx<R>*)acc);
        c.launches += 1;
    }

    static void group_mac(Ctx& c, const FmmPlan& p, const void* S, void* acc, int variant)
    {
        if (!p.n_tiles) return;
        if (c.NC != (long long)NB * (2 * NB - 1) * (2 * NB - 1))
            throw Error(IBLGF_EINTERNAL, "spectrum row length differs from the kernel's");
        if (variant == 1)
        {
            if constexpr (kF32) group_mac_shape<32, 512>(c, p, S, acc);
            else group_mac_shape<32, 256>(c, p, S, acc);
        }
        else
        {
            if constexpr (kF32) group_mac_shape<64, 768>(c, p, S, acc);
            else group_mac_shape<32, 512>(c, p, S, acc);
        }
    }

    static void inverse(Ctx& c, const void* acc, const int* d_tgt_oct, int n_tgt, double scale, double* target)
    {
        if (!n_tgt) return;
        if (inverse_pfa(c, acc, d_tgt_oct, n_tgt, scale, target, inverse_fp32_passes(c))) return;
        launch_inverse(c, (const cx<R>*)acc, d_tgt_oct, n_tgt, scale, target);
        c.launches += 1;
    }
};

template<class F>
void dispatch(Ctx& c, F&& f)
{
    const bool fp32 = c.cfg.precision == IBLGF_FP32;
#define IBLGF_CASE(NBV)                                  \
    case NBV:                                            \
        if (fp32) f(Conv<float, NBV>{});                 \
        else f(Conv<double, NBV>{});                     \
        return;
    switch (c.Nb)
    {
        IBLGF_CASE(6)
        IBLGF_CASE(8)
        IBLGF_CASE(10)
        IBLGF_CASE(12)
        IBLGF_CASE(16)
        IBLGF_CASE(18)
        default: throw Error(IBLGF_EINVAL, "unsupported block_extent (supported: 4,6,8,10,14,16)");
    }
#undef IBLGF_CASE
}

void ensure(DevBuf<char>& b, size_t bytes)
{
    if (b.n < bytes) b.alloc(bytes);
}
}  // namespace

bool nb_supported(int Nb) { return Nb == 6 || Nb == 8 || Nb == 10 || Nb == 12 || Nb == 16 || Nb == 18; }

void init_twiddle_constants(int device)
{
    static std::mutex m;
    static std::set<int> done;
    std::lock_guard<std::mutex> lock(m);
    if (done.count(device)) return;
    std::vector<double> t64(2 * kTwTotal);
    std::vector<float> t32(2 * kTwTotal);
    for (int P : {11, 15, 19, 23, 31, 35})
        for (int j = 0; j < P; ++j)
        {
            const double a = 2.0 * M_PI * j / P;
            const int k = 2 * (tw_base(P) + j);
            t64[k] = std::cos(a);
            t64[k + 1] = -std::sin(a);
            t32[k] = (float)t64[k];
            t32[k + 1] = (float)t64[k + 1];
        }
    IBLGF_CUDA(cudaMemcpyToSymbol(c_tw64, t64.data(), t64.size() * sizeof(double)));
    IBLGF_CUDA(cudaMemcpyToSymbol(c_tw32, t32.data(), t32.size() * sizeof(float)));
    done.insert(device);
}

void launch_spectra(Ctx& c, const std::vector<std::array<int, 5>>& new_slots)
{
    // new_slots: {slot, ld, bx, by, bz}; processed in batches of 64
    const int P = c.P;
    const size_t wbytes = (size_t)64 * P * P * c.Nb * 16;
    ensure(c.d_w, wbytes);
    for (size_t b0 = 0; b0 < new_slots.size(); b0 += 64)
    {
        const size_t nb = std::min<size_t>(64, new_slots.size() - b0);
        std::vector<int> desc(4 * nb), slot(nb);
        for (size_t i = 0; i < nb; ++i)
        {
            const auto& s = new_slots[b0 + i];
            slot[i] = s[0];
            desc[4 * i] = s[1];
            desc[4 * i + 1] = s[2];
            desc[4 * i + 2] = s[3];
            desc[4 * i + 3] = s[4];
        }
        DevBuf<int> d_desc, d_slot;
        d_desc.upload(desc, c.stream);
        d_slot.upload(slot, c.stream);
        dispatch(c, [&](auto cv) {
            using CV = decltype(cv);
            CV::forward_lgf(c, d_desc.p, nullptr, d_slot.p, (int)nb, c.d_spec.p);
        });
        IBLGF_CUDA(cudaGetLastError());
        IBLGF_CUDA(cudaStreamSynchronize(c.stream));  // d_desc / d_slot go out of scope
    }
}

void launch_forward_sources(Ctx& c, const double* fmm_s, const int* d_src_oct, int n_src, void* src_spec)
{
    ensure(c.d_w, (size_t)n_src * c.Nb * c.P * c.Nb * c.cplx_bytes());
    dispatch(c, [&](auto cv) {
        using CV = decltype(cv);
        CV::forward_field(c, fmm_s, d_src_oct, n_src, src_spec);
    });
    IBLGF_CUDA(cudaGetLastError());
}

// one run of the sibling-group MAC in the given variant: 0, 1 the direct
// kernel in its two tile shapes, 2 the block-Toeplitz kernel, 3 the
// tensor-core kernel
void group_mac_variant(Ctx& c, const FmmPlan& p, const void* src_spec, void* acc, int variant)
{
    if (variant == 2 && toeplitz_mac(c, p, src_spec, acc)) return;
    if (variant == 3 && tc_mac(c, p, src_spec, acc)) return;
    dispatch(c, [&](auto cv) {
        using CV = decltype(cv);
        CV::group_mac(c, p, src_spec, acc, variant);
    });
}

// The MAC autotuner: on a plan's first sweep (outside stream capture) every
// applicable group-MAC variant runs twice on the sweep's real data, the
// second run timed with CUDA events on the context stream; the fastest one
// is kept for the plan (and run last, so that the accumulators hold its
// result). A plan rebuilt for the same (level, mask index) sweep, after an
// adaptation, takes the choice made for its predecessor without re-timing.
// iblgf_mac_variant() can pin a variant instead; a pinned variant that does
// not apply to a plan runs variant 0.
void launch_mac(Ctx& c, const FmmPlan& p, const void* src_spec, void* acc)
{
    dispatch(c, [&](auto cv) {
        using CV = decltype(cv);
        // targets outside sibling groups: general pair-list MAC
        CV::mac(c, c.d_spec.p, src_spec, p.pair_ptr.p, p.pair_src.p, p.pair_spec.p, p.n_csr_tgt, acc);
    });
    if (p.n_tiles)
    {
        const bool ok[4] = {true, true, !p.adj_only && p.tile_combo.p && c.cfg.precision == IBLGF_FP32,
                            tc_mac_ok(c, p)};
        int v = c.mac_variant_forced;
        if (v >= 0 && !ok[v]) v = 0;
        if (v < 0) v = p.mac_variant;
        if (v < 0)
        {
            auto it = c.mac_choice.find({p.level, p.mask_idx});
            if (it != c.mac_choice.end() && ok[it->second]) v = p.mac_variant = it->second;
        }
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        IBLGF_CUDA(cudaStreamIsCapturing(c.stream, &cs));
        if (v < 0 && cs != cudaStreamCaptureStatusNone) v = 0;
        if (v < 0)
        {
            constexpr int nv = 4;
            double ms[nv] = {-1.0, -1.0, -1.0, -1.0};
            cudaEvent_t e0, e1;
            IBLGF_CUDA(cudaEventCreate(&e0));
            IBLGF_CUDA(cudaEventCreate(&e1));
            for (int k = 0; k < nv; ++k)
            {
                if (!ok[k]) continue;
                group_mac_variant(c, p, src_spec, acc, k);
                IBLGF_CUDA(cudaEventRecord(e0, c.stream));
                group_mac_variant(c, p, src_spec, acc, k);
                IBLGF_CUDA(cudaEventRecord(e1, c.stream));
                IBLGF_CUDA(cudaEventSynchronize(e1));
                float t = 0.0f;
                IBLGF_CUDA(cudaEventElapsedTime(&t, e0, e1));
                ms[k] = t;
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            int best = 0;
            for (int k = 1; k < nv; ++k)
                if (ok[k] && ms[k] < ms[best]) best = k;
            p.mac_variant = best;
            c.mac_choice[{p.level, p.mask_idx}] = best;
            c.mac_tuning.push_back({(double)p.level, (double)p.mask_idx, (double)p.n_tgt, ms[0], ms[1], ms[2], ms[3],
                                    (double)best});
            v = best;
        }
        group_mac_variant(c, p, src_spec, acc, v);
    }
    IBLGF_CUDA(cudaGetLastError());
}

void launch_inverse_add(Ctx& c, const FmmPlan& p, const void* acc, double* fmm_t, double scale)
{
    dispatch(c, [&](auto cv) {
        using CV = decltype(cv);
        CV::inverse(c, acc, p.tgt_oct.p, p.n_tgt, scale, fmm_t);
    });
    IBLGF_CUDA(cudaGetLastError());
}

void launch_conv_block(Ctx& c, const double* src, const double* kernel, double* out, double scale)
{
    const size_t cb = c.cplx_bytes();
    DevBuf<char> gspec, sspec, acc;
    gspec.alloc(c.NC * cb);
    sspec.alloc(c.NC * cb);
    acc.alloc(c.NC * cb);
    ensure(c.d_w, (size_t)c.P * c.P * c.Nb * 16);
    std::vector<int> zero{0}, ptr{0, 1};  // the FP64 inverse of one block fits: Nb*P*Nb <= P*P*Nb
    DevBuf<int> d_zero, d_ptr;
    d_zero.upload(zero, c.stream);
    d_ptr.upload(ptr, c.stream);
    const double s = scale / ((double)c.P * c.P * c.P);
    dispatch(c, [&](auto cv) {
        using CV = decltype(cv);
        CV::forward_lgf(c, nullptr, kernel, nullptr, 1, gspec.p);
        CV::forward_field(c, src, d_zero.p, 1, sspec.p);
        CV::mac(c, gspec.p, sspec.p, d_ptr.p, d_zero.p, d_zero.p, 1, acc.p);
        CV::inverse(c, acc.p, d_zero.p, 1, s, out);
    });
    IBLGF_CUDA(cudaGetLastError());
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
}

// ---------------------------------------------------------------------------
// Single-block convolution without any device allocation. The per-call
// temporaries of launch_conv_block (LGF, source and product spectra, the
// transform work array, two index arrays) live instead in one file-scope
// device array of kNoAllocScratchBytes (2 MiB). At the largest supported
// block (Nb = 18, FP64) a call needs 1.41 MB of it.
//
// Who needs it: a host application that has already reserved the device
// memory for its own block pool, or that calls the solve from a section in
// which it must not allocate — cudaMalloc can fail there, and cudaFree
// synchronises the whole device, which stalls every other stream the
// application keeps busy. The context (twiddles) is created beforehand as
// usual; this call itself performs no cudaMalloc, cudaFree or library
// allocation, and it enqueues on the context stream without synchronising.
//
// Limits: the scratch is one array per device, shared by every context and
// stream of that device, so calls that overlap in time on different streams
// race on it; serialise them (one stream, or a host lock). The first call on a
// device performs the one-time set-up (symbol address, index arrays), so make
// it before any stream capture begins. No scratch byte needs to start at zero:
// every byte a kernel reads is written earlier in the same call, and the two
// index arrays are written once at set-up.
constexpr size_t kNoAllocScratchBytes = size_t(2) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace
{
constexpr int kNoAllocMaxDevices = 64;
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {};
std::mutex g_noalloc_mutex;

// index arrays of the one-block pair list: zero = {0}, ptr = {0, 1}
__global__ void noalloc_index_kernel(int* idx)
{
    if (threadIdx.x == 0)
    {
        idx[0] = 0;
        idx[1] = 0;
        idx[2] = 1;
    }
}

size_t round256(size_t b) { return (b + 255) / 256 * 256; }

// Makes the context's device current for the scope of a call and restores
// the caller's current device on every way out (return or exception).
struct DeviceScope
{
    int prev = -1;
    explicit DeviceScope(int device)
    {
        IBLGF_CUDA(cudaGetDevice(&prev));
        if (prev != device) IBLGF_CUDA(cudaSetDevice(device));
    }
    ~DeviceScope()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// the static scratch's device address on the current device (set up once
// per device); the caller holds a DeviceScope for the context's device
unsigned char* noalloc_scratch(Ctx& c)
{
    int dev = -1;
    IBLGF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) throw Error(IBLGF_EINVAL, "device ordinal beyond the scratch table");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev])
    {
        void* ptr = nullptr;
        IBLGF_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        if (!ptr) throw Error(IBLGF_ECUDA, "cudaGetSymbolAddress returned a null scratch address");
        noalloc_index_kernel<<<1, 32, 0, c.stream>>>(static_cast<int*>(ptr));
        IBLGF_CUDA(cudaGetLastError());
        IBLGF_CUDA(cudaStreamSynchronize(c.stream));
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(ptr);
    }
    return g_noalloc_ptr[dev];
}
}  // namespace

void launch_conv_block_noalloc(Ctx& c, const double* src, const double* kernel, double* out, double scale)
{
    // scratch layout: [index ints | LGF spectrum | source spectrum | product | work]
    const size_t spec = round256((size_t)c.NC * 16);  // sized for FP64 spectra
    const size_t work = round256((size_t)c.P * c.P * c.Nb * 16);
    const size_t need = 256 + 3 * spec + work;
    if (need > kNoAllocScratchBytes)
        throw Error(IBLGF_EINVAL, "block too large for the static convolution scratch (needs " +
                                      std::to_string(need) + " bytes, limit " +
                                      std::to_string(kNoAllocScratchBytes) + ")");
    DeviceScope on_device(c.cfg.device);
    unsigned char* base = noalloc_scratch(c);
    const int* d_zero = reinterpret_cast<const int*>(base);
    const int* d_ptr = d_zero + 1;
    unsigned char* gspec = base + 256;
    unsigned char* sspec = gspec + spec;
    unsigned char* acc = sspec + spec;
    unsigned char* W = acc + spec;
    const double s = scale / ((double)c.P * c.P * c.P);
    dispatch(c, [&](auto cv) {
        using CV = decltype(cv);
        using R = typename CV::Real;
        constexpr int NB = CV::Nb, P = CV::P, NP = CV::NP;
        fwd_xy_kernel<double, NB, P, kFromDense><<<dim3(1, P), 256, 0, c.stream>>>(
            kernel, nullptr, nullptr, nullptr, c.d_tw64.p, (double2*)W, nullptr, 0);
        fwd_z_kernel<double, R, NB, P><<<dim3(1, (NP + 127) / 128), 128, 0, c.stream>>>(
            (const double2*)W, nullptr, (cx<R>*)gspec);
        CV::launch_fwd_xy_rows(c, src, d_zero, 1, (cx<R>*)W);
        fwd_z_kernel<R, R, NB, NB><<<dim3(1, (NP + 127) / 128), 128, 0, c.stream>>>(
            (const cx<R>*)W, nullptr, (cx<R>*)sspec);
        mac_kernel<R><<<dim3((unsigned)((c.NC + 127) / 128), 1), 128, 0, c.stream>>>(
            (const cx<R>*)gspec, (const cx<R>*)sspec, d_ptr, d_zero, d_zero, c.NC, (cx<R>*)acc);
        CV::launch_inverse(c, (const cx<R>*)acc, d_zero, 1, s, out);
        c.launches += 6;
    });
    IBLGF_CUDA(cudaGetLastError());
}

}  // namespace iblgf_b200
