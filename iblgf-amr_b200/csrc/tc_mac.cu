// Sibling-group spectral MAC on the tensor cores (tcgen05, TF32 with a
// 3-product split, FP32 accumulation in tensor memory).
//
// Contract (include/iblgf/utilities/convolution.hpp:204-221, per pair
// acc += G_hat(u) * S_hat, summed over a target's neighbour and influence
// lists, fmm.hpp:907-1027): for a sibling group (the 8 children c of one
// parent) and a frequency f,
//     acc[c] = sum_n sum_c' G(c - c' - 2n) * s_n[c'],
// n over the parent's 27 neighbour parents, c' over their children. All
// groups of one level distance share G, so per frequency this is a matrix
// product over groups. With complex numbers embedded as real 2 x 2 blocks
// (re, im of each child):
//     D[group][2c + i] += sum_(n, c', j) A[group][(n, 2c' + j)] B_n[2c + i][2c' + j]
// A = the group's candidate sources (16 reals per neighbour parent), B_n =
// the 16 x 16 real form of the 8 x 8 matrix G(c - c' - 2n):
//     B[2c][2c'] = B[2c+1][2c'+1] = Re G,  B[2c][2c'+1] = -Im G,  B[2c+1][2c'] = Im G.
// M = 128 groups, N = 16, K = 16 per neighbour parent.
//
// CTA = (tile of up to 128 groups of one level distance and one pair mode,
// 2 consecutive frequencies), 9 warps:
//   producer warps 0-7: thread (m, h) = group m of the tile (its tensor-memory
//   lane), children h*4 .. h*4+3 of each neighbour parent. Per neighbour parent
//   present in the tile it loads its 4 candidate source values (16 bytes =
//   both frequencies; absent candidates read the zero row; loads run two
//   parents ahead), splits them into TF32 hi + lo, stores them to its lane of
//   the stage's A columns, and writes its share of the stage's B_n (both
//   frequencies, hi and lo) from the tile's 343 LGF rows staged once per CTA;
//   then it arrives on the stage's "full" mbarrier;
//   MMA warp 8: one thread waits for "full", issues per frequency 2 K-steps x
//   3 MMAs (Ahi Bhi, Alo Bhi, Ahi Blo; M = 128, N = 16, K = 8) accumulating
//   into D in tensor memory, and commits to the stage's "empty" mbarrier,
//   which frees the stage when those MMAs have completed.
// Stages form a ring of kTcStages (A in tensor memory, B in shared memory),
// so the producers run up to kTcStages parents ahead of the tensor cores and
// no block-wide barrier sits in the loop. After the last parent the MMA
// thread commits to "dfull"; the producers read D from tensor memory and
// write the accumulators of their 4 children. Excluded offsets of a tile's
// mode (coarse targets take only non-adjacent sources; the integrating
// factor only adjacent ones) are zero rows of the staged LGF spectra, as in
// the CUDA-core kernels. Every mbarrier wait is bounded and records
// IBLGF_ETIMEOUT in the context's status word.
#include <algorithm>
#include <vector>

#include "cplx.cuh"
#include "ctx.hpp"
#include "tcgen05.cuh"

namespace iblgf_b200
{
namespace
{
constexpr int kTcGroups = 128;  // M: groups per tile, one per tensor-memory lane
constexpr int kTcF = 2;         // frequencies per CTA
constexpr int kTcStages = 3;
constexpr int kTcProducers = 256;  // 8 warps: 128 lanes x 2 halves of the children
constexpr int kTcThreads = kTcProducers + 32;
constexpr unsigned kTcCols = 256;
// tensor-memory columns: D of frequency f at 16 f; stage s of A at 32 + 64 s,
// frequency f at + 32 f, hi at + 0, lo at + 16 (children half h at + 8 h)
constexpr unsigned kColA = 32;
static_assert(kColA + 64 * kTcStages <= kTcCols, "tensor-memory columns");

// float offset of element (row nn, column k) of a 16 x 16 K-major B tile in
// the no-swizzle core-matrix layout (K-step k / 8 at + 128 floats)
__device__ __forceinline__ int b_off(int nn, int k)
{
    return (k >> 3) * 128 + (nn >> 3) * (int)(tc::kSbo / 4) + ((k & 7) >> 2) * (int)(tc::kLbo / 4) + (nn & 7) * 4 +
           (k & 3);
}

struct TcSmem
{
    float b[kTcStages][kTcF][2][256];  // [stage][frequency][hi, lo][16 x 16 tile]
    float2 g[343][kTcF];               // LGF spectra of the tile's offsets
    unsigned long long full[kTcStages], empty[kTcStages], dfull;
    unsigned tmem;
    int npar;
    int plist[27];
};

template<int NB>
__global__ void __launch_bounds__(kTcThreads, 2)
    tc_mac_kernel(const float2* __restrict__ G, const float2* __restrict__ S, int zrow,
                  const int* __restrict__ tc_gptr, const int* __restrict__ tc_tab, const int* __restrict__ tc_mode,
                  const unsigned* __restrict__ tc_pm, const int* __restrict__ spec_u, const int* __restrict__ grp_jr,
                  const int* __restrict__ grp_tgt, float2* __restrict__ ACC, int* __restrict__ status)
{
    constexpr int P = 2 * NB - 1;
    constexpr long long NC = (long long)(P / 2 + 1) * P * P;
    static_assert(NC % kTcF == 0, "frequency pairs cover the row");
    __shared__ __align__(1024) TcSmem sm;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int tile = blockIdx.x;
    const long long f0 = (long long)blockIdx.y * kTcF;
    const int g0 = tc_gptr[tile], ng = tc_gptr[tile + 1] - g0;
    const int mode = tc_mode[tile];  // 0 all, 1 non-adjacent only, 2 adjacent only
    const int* su = spec_u + 343 * tc_tab[tile];
    if (warp == 8) tc::alloc(&sm.tmem, kTcCols);
    if (tid == 0)
    {
        for (int s = 0; s < kTcStages; ++s)
        {
            mbar_init(&sm.full[s], kTcProducers);
            mbar_init(&sm.empty[s], 1);
        }
        mbar_init(&sm.dfull, 1);
        const unsigned pm = tc_pm[tile];
        int k = 0;
        for (int n = 0; n < 27; ++n)
            if (pm >> n & 1u) sm.plist[k++] = n;
        sm.npar = k;
    }
    for (int r = tid; r < 343; r += kTcThreads)
    {
        const int ux = r % 7 - 3, uy = (r / 7) % 7 - 3, uz = r / 49 - 3;
        const bool adj = ux >= -1 && ux <= 1 && uy >= -1 && uy <= 1 && uz >= -1 && uz <= 1;
        const int slot = (mode == 1 && adj) || (mode == 2 && !adj) ? -1 : su[r];
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (slot >= 0) v = __ldg(reinterpret_cast<const float4*>(G + (size_t)slot * NC + f0));
        sm.g[r][0] = make_float2(v.x, v.y);
        sm.g[r][1] = make_float2(v.z, v.w);
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const unsigned tb = sm.tmem;
    const int npar = sm.npar;
    bool timed_out = false;
    if (warp == 8)
    {
        // MMA issue
        if (tid == 8 * 32)
        {
            constexpr unsigned idesc = tc::idesc_tf32(kTcGroups, 16);
            for (int it = 0; it < npar; ++it)
            {
                const int s = it % kTcStages;
                if (!mbar_wait(&sm.full[s], (it / kTcStages) & 1)) timed_out = true;
                tc::fence_after();
#pragma unroll
                for (int f = 0; f < kTcF; ++f)
#pragma unroll
                    for (int ks = 0; ks < 2; ++ks)
#pragma unroll
                        for (int term = 0; term < 3; ++term)
                        {
                            const unsigned a = tb + kColA + 64u * s + 32u * f + (term == 1 ? 16u : 0u) + 8u * ks;
                            const unsigned long long bd = tc::smem_desc(&sm.b[s][f][term == 2 ? 1 : 0][128 * ks]);
                            tc::mma_tf32(tb + 16u * f, a, bd, idesc, it > 0 || ks > 0 || term > 0);
                        }
                tc::commit(&sm.empty[s]);
            }
            if (npar > 0) tc::commit(&sm.dfull);
        }
        __syncwarp();
    }
    else
    {
        // producers
        const int m = tid & 127, h = tid >> 7;
        const unsigned lane = (unsigned)(32 * (warp & 3)) << 16;
        const bool valid = m < ng;
        const int* jr = grp_jr + (size_t)(g0 + (valid ? m : 0)) * 216 + 4 * h;
        // this thread's B work: frequency bf, child pair (bc, bcp), rows 2 bc + h
        const int bf = m >> 6, bc = (m >> 3) & 7, bcp = m & 7;
        const int bdx = (bc & 1) - (bcp & 1), bdy = ((bc >> 1) & 1) - ((bcp >> 1) & 1), bdz = (bc >> 2) - (bcp >> 2);
        const int o0 = b_off(2 * bc + h, 2 * bcp), o1 = b_off(2 * bc + h, 2 * bcp + 1);
        float4 sv[2][4];
        auto load_parent = [&](int n, float4 (&v)[4]) {
            int j[4] = {zrow, zrow, zrow, zrow};
            if (valid)
            {
                const int4 ja = *reinterpret_cast<const int4*>(jr + 8 * n);
                j[0] = ja.x, j[1] = ja.y, j[2] = ja.z, j[3] = ja.w;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) v[q] = __ldg(reinterpret_cast<const float4*>(S + (size_t)j[q] * NC + f0));
        };
        if (npar > 0) load_parent(sm.plist[0], sv[0]);
        if (npar > 1) load_parent(sm.plist[1], sv[1]);
        auto stage = [&](int it, float4 (&v)[4]) {
            const int n = sm.plist[it], s = it % kTcStages;
            if (it >= kTcStages && !mbar_wait(&sm.empty[s], (it / kTcStages - 1) & 1)) timed_out = true;
            tc::fence_after();
            const unsigned abuf = tb + lane + kColA + 64u * s + 8u * h;
#pragma unroll
            for (int f = 0; f < kTcF; ++f)
            {
                unsigned hi[8], lo[8];
#pragma unroll
                for (int q = 0; q < 4; ++q)
                {
                    tc::split(f ? v[q].z : v[q].x, hi[2 * q], lo[2 * q]);
                    tc::split(f ? v[q].w : v[q].y, hi[2 * q + 1], lo[2 * q + 1]);
                }
                tc::st8(abuf + 32u * f, hi);
                tc::st8(abuf + 32u * f + 16u, lo);
            }
            if (it + 2 < npar) load_parent(sm.plist[it + 2], v);
            // B_n row 2 bc + h, columns 2 bcp (+1): (Re G, -Im G) for h = 0,
            // (Im G, Re G) for h = 1, G = G(c - c' - 2n) at frequency bf
            const int nx = n % 3 - 1, ny = (n / 3) % 3 - 1, nz = n / 9 - 1;
            const int r = (bdx - 2 * nx + 3) + 7 * (bdy - 2 * ny + 3) + 49 * (bdz - 2 * nz + 3);
            const float2 gv = sm.g[r][bf];
            unsigned ah, al, bh, bl;
            tc::split(h ? gv.y : gv.x, ah, al);
            tc::split(h ? gv.x : -gv.y, bh, bl);
            float* th = sm.b[s][bf][0];
            float* tl = sm.b[s][bf][1];
            th[o0] = __uint_as_float(ah), tl[o0] = __uint_as_float(al);
            th[o1] = __uint_as_float(bh), tl[o1] = __uint_as_float(bl);
            tc::wait_st();
            fence_proxy_async_smem();
            tc::fence_before();
            mbar_arrive(&sm.full[s]);
        };
        int it = 0;
        for (; it + 1 < npar; it += 2)
        {
            stage(it, sv[0]);
            stage(it + 1, sv[1]);
        }
        if (it < npar) stage(it, sv[0]);
        unsigned d[kTcF][8];
        if (npar > 0)
        {
            if (!mbar_wait(&sm.dfull, 0)) timed_out = true;
            tc::fence_after();
#pragma unroll
            for (int f = 0; f < kTcF; ++f) tc::ld8(tb + lane + 16u * f + 8u * h, d[f]);
            tc::wait_ld();
        }
        if (valid)
        {
            const int g = g0 + m;
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
                const int t = grp_tgt[(size_t)g * 8 + 4 * h + q];
                if (t < 0) continue;
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (npar > 0)
                    v = make_float4(__uint_as_float(d[0][2 * q]), __uint_as_float(d[0][2 * q + 1]),
                                    __uint_as_float(d[1][2 * q]), __uint_as_float(d[1][2 * q + 1]));
                *reinterpret_cast<float4*>(ACC + (size_t)t * NC + f0) = v;
            }
        }
    }
    if (timed_out) atomicOr(status, kStatusTimeout);
    tc::fence_before();
    __syncthreads();
    if (warp == 8)
    {
        tc::fence_after();
        tc::dealloc(tb, kTcCols);
    }
}

template<int NB>
void launch_tc(Ctx& c, const FmmPlan& p, const void* S, void* acc)
{
    dim3 grid((unsigned)p.n_tc, (unsigned)(c.NC / kTcF));
    tc_mac_kernel<NB><<<grid, kTcThreads, 0, c.stream>>>(
        (const float2*)c.d_spec.p, (const float2*)S, p.n_src, p.tc_gptr.p, p.tc_tab.p, p.tc_mode.p, p.tc_pm.p,
        p.spec_u.p, p.grp_jr.p, p.grp_tgt.p, (float2*)acc, c.d_status.p);
    c.launches += 1;
}
}  // namespace

bool tc_mac_ok(const Ctx& c, const FmmPlan& p)
{
    return p.n_tc > 0 && c.cfg.precision == IBLGF_FP32 && c.NC % kTcF == 0;
}

bool tc_mac(Ctx& c, const FmmPlan& p, const void* S, void* acc)
{
    if (!tc_mac_ok(c, p)) return false;
    if (c.NC != (long long)c.Nb * c.P * c.P) throw Error(IBLGF_EINTERNAL, "spectrum row length differs");
#define IBLGF_TC(NBV)                   \
    case NBV:                           \
        launch_tc<NBV>(c, p, S, acc);   \
        return true;
    switch (c.Nb)
    {
        IBLGF_TC(6)
        IBLGF_TC(8)
        IBLGF_TC(10)
        IBLGF_TC(12)
        IBLGF_TC(16)
        IBLGF_TC(18)
        default: return false;
    }
#undef IBLGF_TC
}

void build_tc_tiles(const std::vector<int>& tgptr, const std::vector<int>& ttab, const std::vector<int>& tmode,
                    const std::vector<unsigned>& gpm, std::vector<int>& gptr, std::vector<int>& tab,
                    std::vector<int>& mode, std::vector<unsigned>& pm)
{
    gptr.clear(), tab.clear(), mode.clear(), pm.clear();
    for (size_t t = 0; t + 1 < tgptr.size(); ++t)
    {
        const int a = tgptr[t], e = tgptr[t + 1];
        for (int g = a; g < e; ++g)
        {
            const bool open = !tab.empty() && tab.back() == ttab[t] && mode.back() == tmode[t] &&
                              g - gptr.back() < kTcGroups;
            if (!open)
            {
                gptr.push_back(g);
                tab.push_back(ttab[t]);
                mode.push_back(tmode[t]);
                pm.push_back(0u);
            }
            pm.back() |= gpm[g];
        }
    }
    if (!tab.empty()) gptr.push_back(tgptr.back());
}
}  // namespace iblgf_b200
