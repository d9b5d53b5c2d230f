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
#include <cuda.h>

#include <algorithm>
#include <string>
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

// the 27 products of one neighbour parent for GPT groups at once: gt =
// coefficient rows of the parent (27 rows of F, this thread's frequency),
// shared by the groups; s[k] = group k's 8 source values of the parent's
// children (c' = x + 2y + 4z)
template<class R, int F, int GPT>
__device__ __forceinline__ void toeplitz_parent(const cx<R>* gt, const cx<R> (&s)[GPT][8], cx<R> (&A)[GPT][27])
{
#pragma unroll
    for (int tz = 0; tz < 3; ++tz)
    {
        // along z: m = x0 + x1, p = x1, q = x0 (x0 / x1: c'z = 0 / 1)
        cx<R> v[GPT][4];
#pragma unroll
        for (int k = 0; k < GPT; ++k)
#pragma unroll
            for (int q = 0; q < 4; ++q)
                v[k][q] = tz == 0 ? cadd<R>(s[k][q], s[k][q + 4]) : (tz == 1 ? s[k][q + 4] : s[k][q]);
#pragma unroll
        for (int ty = 0; ty < 3; ++ty)
        {
            cx<R> w0[GPT], w1[GPT];  // c'x = 0, 1
#pragma unroll
            for (int k = 0; k < GPT; ++k)
            {
                if (ty == 0)
                {
                    w0[k] = cadd<R>(v[k][0], v[k][2]);
                    w1[k] = cadd<R>(v[k][1], v[k][3]);
                }
                else if (ty == 1)
                {
                    w0[k] = v[k][2];
                    w1[k] = v[k][3];
                }
                else
                {
                    w0[k] = v[k][0];
                    w1[k] = v[k][1];
                }
            }
            const int t0 = 3 * ty + 9 * tz;
            const cx<R> c0 = gt[t0 * F], c1 = gt[(t0 + 1) * F], c2 = gt[(t0 + 2) * F];
#pragma unroll
            for (int k = 0; k < GPT; ++k)
            {
                cmac<R>(A[k][t0], c0, cadd<R>(w0[k], w1[k]));
                cmac<R>(A[k][t0 + 1], c1, w1[k]);
                cmac<R>(A[k][t0 + 2], c2, w0[k]);
            }
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

// Coefficient rows of the block-Toeplitz product ("combo" spectra), one
// table per level difference: row n * 27 + t (neighbour parent n, product
// t = tx + 3 ty + 9 tz) at frequency f is
//     C = sum over the axes' stencils of +-G_hat(d - 2n)(f),
// per axis m: {d = 0: +1}, p: {d = -1: +1, d = 0: -1}, q: {d = +1: +1,
// d = 0: -1}, G_hat(u) the cached LGF spectrum of offset u (slot table, 343
// entries; offsets excluded by the table's mode contribute zero). Formed in
// FP64 from the cached spectra and stored in the working precision.
template<class R>
__global__ void combo_table_kernel(const cx<R>* __restrict__ G, const int* __restrict__ slots, int exclude_adjacent,
                                   long long NC, cx<R>* __restrict__ out)
{
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y;  // n * 27 + t
    if (f >= NC) return;
    const int n = row / 27, t = row % 27;
    const int nn[3] = {n % 3 - 1, (n / 3) % 3 - 1, n / 9 - 1};
    const int tt[3] = {t % 3, (t / 3) % 3, t / 9};
    double sx = 0.0, sy = 0.0;
    for (int az = 0; az < (tt[2] ? 2 : 1); ++az)
    {
        const int dz = az ? 0 : (tt[2] == 0 ? 0 : (tt[2] == 1 ? -1 : 1));
        const double wz = az ? -1.0 : 1.0;
        for (int ay = 0; ay < (tt[1] ? 2 : 1); ++ay)
        {
            const int dy = ay ? 0 : (tt[1] == 0 ? 0 : (tt[1] == 1 ? -1 : 1));
            const double wy = ay ? -wz : wz;
            for (int ax = 0; ax < (tt[0] ? 2 : 1); ++ax)
            {
                const int dx = ax ? 0 : (tt[0] == 0 ? 0 : (tt[0] == 1 ? -1 : 1));
                const double w = ax ? -wy : wy;
                const int ux = dx - 2 * nn[0], uy = dy - 2 * nn[1], uz = dz - 2 * nn[2];
                const bool adj = ux >= -1 && ux <= 1 && uy >= -1 && uy <= 1 && uz >= -1 && uz <= 1;
                const int slot = slots[(ux + 3) + 7 * (uy + 3) + 49 * (uz + 3)];
                if (slot < 0 || (exclude_adjacent && adj)) continue;
                const cx<R> g = G[(size_t)slot * NC + f];
                sx = fma(w, (double)g.x, sx);
                sy = fma(w, (double)g.y, sy);
            }
        }
    }
    out[(size_t)row * NC + f] = mk<R>((R)sx, (R)sy);
}

// 2-D tiled TMA load (no multicast): box of the tensor map at (x, y) into
// shared memory, completion counted on the mbarrier
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// shared memory: three slab buffers of coefficient rows [243][F] (slab s
// always in buffer s), two buffers of candidate rows [NG][216], mbarriers
template<class R, int F, int NG>
struct ToeplitzSmem
{
    static constexpr size_t slab = (size_t)243 * F * sizeof(cx<R>);
    static constexpr size_t jr = (size_t)NG * 216 * sizeof(int);
    static constexpr size_t bars = 10 * sizeof(unsigned long long);
    static constexpr size_t total = 3 * slab + 2 * jr + bars;
};

// Persistent, warp-specialised pipeline. A work item is (tile part: up to NG
// groups of one tile, chunk of F frequencies); CTA b takes items b, b + grid,
// ... . Warp CW (the producer) issues, per item, one bulk copy of the
// groups' candidate rows and three 2-D TMA tiles of coefficient rows (slab s
// = neighbour parents nz = s - 1, rows 243 s .. 243 s + 242 of the tile's
// table; rows past the end of the spectrum are zero-filled by the TMA unit).
// Warps 0 .. CW-1 (the consumers) each take GPT groups at F consecutive
// frequencies, wait for a slab, run its 9 parents and release the buffer; the
// producer refills a buffer with the next item's slab as soon as every
// consumer has released it, so the copies overlap the other slabs' work and
// no block-wide barrier is taken. Every wait is bounded: one that runs out
// sets the status word and the CTA stops taking items.
template<class R, int F, int NG, int GPT, int NB>
__global__ void __launch_bounds__((NG / GPT + 1) * F, 1)
    toeplitz_mac_kernel(const __grid_constant__ CUtensorMap combo, const cx<R>* __restrict__ S,
                        const int* __restrict__ parts, int n_parts, int n_chunks,
                        const int* __restrict__ tile_gptr, const int* __restrict__ tile_jr,
                        const int* __restrict__ tile_combo, const unsigned* __restrict__ grp_pm,
                        const int* __restrict__ grp_tgt, cx<R>* __restrict__ ACC, int* __restrict__ status)
{
    constexpr int P = 2 * NB - 1;
    constexpr long long NC = (long long)(P / 2 + 1) * P * P;
    constexpr int UNITS = sizeof(cx<R>) / 8;  // 8-byte tensor-map elements per complex value
    constexpr int CW = NG / GPT;              // consumer warps (one row of F lanes each)
    static_assert(F == 32, "one consumer warp per row of groups");
    using SM = ToeplitzSmem<R, F, NG>;
    extern __shared__ __align__(128) unsigned char smraw[];
    int* Jr0 = reinterpret_cast<int*>(smraw + 3 * SM::slab);
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smraw + 3 * SM::slab + 2 * SM::jr);
    unsigned long long* full = bar;         // [3] slab s landed
    unsigned long long* empty = bar + 3;    // [3] slab s consumed by all CW consumers
    unsigned long long* jfull = bar + 6;    // [2] candidate rows landed
    unsigned long long* jempty = bar + 8;   // [2] candidate rows consumed
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const long long n_items = (long long)n_parts * n_chunks;
    const unsigned slab_bytes = (unsigned)SM::slab, jr_bytes = (unsigned)SM::jr;

    if (threadIdx.x == 0)
    {
        for (int i = 0; i < 3; ++i)
        {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], CW);
        }
        for (int i = 0; i < 2; ++i)
        {
            mbar_init(&jfull[i], 1);
            mbar_init(&jempty[i], CW);
        }
    }
    __syncthreads();

    if (warp == CW)
    {
        // producer
        if (lane == 0)
        {
            int k = 0;
            for (long long it = blockIdx.x; it < n_items; it += gridDim.x, ++k)
            {
                const int th = (int)(it % n_parts), chunk = (int)(it / n_parts);
                const int tile = parts[th] >> 2, part = parts[th] & 3;
                const int jb = k & 1;
                if (k >= 2 && !mbar_wait(&jempty[jb], (unsigned)(((k >> 1) - 1) & 1)))
                {
                    atomicOr(status, kStatusTimeout);
                    break;
                }
                mbar_arrive_expect_tx(&jfull[jb], jr_bytes);
                bulk_g2s(Jr0 + jb * (NG * 216), tile_jr + ((size_t)tile * kGroupTileCap + part * NG) * 216, jr_bytes,
                         &jfull[jb]);
                const int x = (int)((long long)chunk * F * UNITS), y = tile_combo[tile] * 729;
                bool ok = true;
                for (int s = 0; s < 3 && ok; ++s)
                {
                    if (k >= 1 && !mbar_wait(&empty[s], (unsigned)((k - 1) & 1))) ok = false;
                    else
                    {
                        fence_proxy_async_smem();
                        mbar_arrive_expect_tx(&full[s], slab_bytes);
                        tma_load_2d(smraw + s * SM::slab, &combo, x, y + 243 * s, &full[s]);
                    }
                }
                if (!ok)
                {
                    atomicOr(status, kStatusTimeout);
                    break;
                }
            }
        }
        return;
    }

    // consumers: warp = row of GPT groups
    const cx<R> zero = mk<R>(0, 0);
    int k = 0;
    for (long long it = blockIdx.x; it < n_items; it += gridDim.x, ++k)
    {
        const int th = (int)(it % n_parts), chunk = (int)(it / n_parts);
        const int tile = parts[th] >> 2, part = parts[th] & 3;
        const int g0 = tile_gptr[tile] + part * NG, g1 = min(tile_gptr[tile + 1], g0 + NG);
        const int gb = g0 + GPT * warp;
        const bool active = gb < g1;
        unsigned pm = 0;
#pragma unroll
        for (int q = 0; q < GPT; ++q) pm |= gb + q < g1 ? grp_pm[gb + q] : 0u;
        const long long f = (long long)chunk * F + lane;
        const cx<R>* Sf = S + (f < NC ? f : NC - 1);  // clamped column for the tail chunk
        const int jb = k & 1;
        bool ok = mbar_wait(&jfull[jb], (unsigned)((k >> 1) & 1));
        const int* jr = Jr0 + jb * (NG * 216) + GPT * warp * 216;
        cx<R> A[GPT][27];
#pragma unroll
        for (int q = 0; q < GPT; ++q)
#pragma unroll
            for (int t = 0; t < 27; ++t) A[q][t] = zero;
        for (int s = 0; s < 3 && ok; ++s)
        {
            ok = mbar_wait(&full[s], (unsigned)(k & 1));
            if (!ok) break;
            if (active)
            {
                const cx<R>* gs = reinterpret_cast<const cx<R>*>(smraw + s * SM::slab) + lane;
                for (int nxy = 0; nxy < 9; ++nxy)
                {
                    const int n = nxy + 9 * s;
                    if (!((pm >> n) & 1u)) continue;
                    cx<R> sv[GPT][8];
#pragma unroll
                    for (int q = 0; q < GPT; ++q)
                    {
                        const int4 ja = *reinterpret_cast<const int4*>(jr + q * 216 + 8 * n);
                        const int4 jc = *reinterpret_cast<const int4*>(jr + q * 216 + 8 * n + 4);
                        const int jj[8] = {ja.x, ja.y, ja.z, ja.w, jc.x, jc.y, jc.z, jc.w};
#pragma unroll
                        for (int c = 0; c < 8; ++c) sv[q][c] = __ldg(Sf + (size_t)jj[c] * NC);
                    }
                    toeplitz_parent<R, F, GPT>(gs + (size_t)nxy * 27 * F, sv, A);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&jempty[jb]);
        if (!ok)
        {
            if (lane == 0) atomicOr(status, kStatusTimeout);
            return;
        }
        if (active && f < NC)
        {
#pragma unroll
            for (int q = 0; q < GPT; ++q)
            {
                if (gb + q >= g1) continue;
                cx<R> y[8];
                toeplitz_combine<R>(A[q], y);
#pragma unroll
                for (int c = 0; c < 8; ++c)
                {
                    const int t = grp_tgt[(size_t)(gb + q) * 8 + c];
                    if (t >= 0) ACC[(size_t)t * NC + f] = y[c];
                }
            }
        }
    }
}

template<class R, int NB>
void launch_toeplitz(Ctx& c, const FmmPlan& p, const void* S, void* acc)
{
    static_assert(std::is_same<R, float>::value, "FP32 path");
    // 7 consumer warps of 2 groups + the producer warp: 8 warps, so that the
    // register file allows the 2 x 27 complex accumulators per thread
    constexpr int F = 32, NG = kToeplitzPart, GPT = 2;
    using SM = ToeplitzSmem<R, F, NG>;
    auto kfn = toeplitz_mac_kernel<R, F, NG, GPT, NB>;
    IBLGF_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM::total));
    const int n_chunks = (int)((c.NC + F - 1) / F);
    const long long items = (long long)p.n_parts * n_chunks;
    int sms = 0;
    IBLGF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.cfg.device));
    const unsigned grid = (unsigned)std::min<long long>(items, sms);
    kfn<<<grid, (NG / GPT + 1) * F, SM::total, c.stream>>>(*reinterpret_cast<const CUtensorMap*>(c.combo_map),
                                                           (const cx<R>*)S, p.tile_parts.p, p.n_parts, n_chunks,
                                                           p.tile_gptr.p, p.tile_jr.p, p.tile_combo.p, p.grp_pm.p,
                                                           p.grp_tgt.p, (cx<R>*)acc, c.d_status.p);
    c.launches += 1;
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// the tensor map over all combo tables: [tables x 729 rows][NC complex] as
// 8-byte elements, box = one slab (243 rows) of one frequency chunk
void encode_combo_map(Ctx& c)
{
    static EncodeTiled encode = nullptr;
    if (!encode)
    {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        IBLGF_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn)
            throw Error(IBLGF_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
        encode = reinterpret_cast<EncodeTiled>(fn);
    }
    const bool f32 = c.cfg.precision == IBLGF_FP32;
    const cuuint64_t units = (cuuint64_t)c.NC * (f32 ? 1 : 2);
    const cuuint64_t dims[2] = {units, (cuuint64_t)c.combo_tables * 729};
    const cuuint64_t strides[1] = {units * 8};
    const cuuint32_t box[2] = {(cuuint32_t)(f32 ? 32 : 32), 243};  // F = 32 (FP32) / 16 complex (FP64)
    const cuuint32_t estr[2] = {1, 1};
    CUtensorMap* map = reinterpret_cast<CUtensorMap*>(c.combo_map);
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, c.d_combo.p, dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(IBLGF_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}
}  // namespace

int combo_table(Ctx& c, int ld, const std::vector<int>& slots)
{
    auto it = c.combo_of_ld.find(ld);
    if (it != c.combo_of_ld.end()) return it->second;
    const size_t tbytes = (size_t)729 * c.NC * c.cplx_bytes();
    const int idx = c.combo_tables;
    if (idx + 1 > c.combo_cap)
    {
        const int cap = std::max(idx + 1, 2 * c.combo_cap);
        DevBuf<char> nb;
        nb.alloc((size_t)cap * tbytes);
        if (idx) IBLGF_CUDA(cudaMemcpyAsync(nb.p, c.d_combo.p, (size_t)idx * tbytes, cudaMemcpyDeviceToDevice, c.stream));
        IBLGF_CUDA(cudaStreamSynchronize(c.stream));
        c.d_combo = std::move(nb);
        c.combo_cap = cap;
    }
    DevBuf<int> d_slots;
    d_slots.upload(slots, c.stream);
    dim3 grid((unsigned)((c.NC + 255) / 256), 729);
    char* out = c.d_combo.p + (size_t)idx * tbytes;
    if (c.cfg.precision != IBLGF_FP32) throw Error(IBLGF_EINTERNAL, "block-Toeplitz tables are FP32-path only");
    combo_table_kernel<float><<<grid, 256, 0, c.stream>>>((const float2*)c.d_spec.p, d_slots.p, ld > 0 ? 1 : 0,
                                                          c.NC, (float2*)out);
    IBLGF_CUDA(cudaGetLastError());
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    c.combo_tables = idx + 1;
    c.combo_of_ld.emplace(ld, idx);
    encode_combo_map(c);
    return idx;
}

bool toeplitz_mac(Ctx& c, const FmmPlan& p, const void* S, void* acc)
{
    if (!p.n_tiles || p.adj_only || !p.tile_combo.p || c.cfg.precision != IBLGF_FP32) return false;
    if (c.NC != (long long)c.Nb * c.P * c.P) throw Error(IBLGF_EINTERNAL, "spectrum row length differs");
#define IBLGF_TOEP(NBV)                                 \
    case NBV:                                           \
        launch_toeplitz<float, NBV>(c, p, S, acc);      \
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
