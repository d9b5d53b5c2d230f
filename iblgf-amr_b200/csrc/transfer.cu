// Inter-level transfers and block field operations of the FMM sweep and the
// Poisson level loop, FP64 (fields stay FP64 in every precision mode).
//
//   tp_kernel     tensor-product Lagrange transfers on Nb^3 blocks:
//                 FMM anterpolation / interpolation (include/iblgf/fmm/
//                 fmm_nli.hpp:101-247) and cell-centred interpolation /
//                 coarsification (interpolation/cell_center_nli_intrp.hpp:
//                 310-420, 557-674). One CTA per receiving block; the sending
//                 blocks of a group are applied in child order, so sums are
//                 deterministic without atomics.
//   halo_kernel   same-level buffer exchange (domain/mpi/haloCommunicator.hpp:
//                 63-107): each buffer cell takes the value of the neighbour
//                 interior cell that overlaps it
//   correction    add_source_correction (cell_center_nli_intrp.hpp:171-238)
//   zero / copy_interior / axpy over block lists (fmm.hpp:1029-1106,
//                 poisson.hpp:921-1013)
#include <algorithm>
#include <cstring>

#include "ctx.hpp"

namespace iblgf_b200
{
namespace
{
// The Nb x Nb matrices of a transfer per axis and child bit, passed by
// value: they sit in the constant bank, and with the passes fully unrolled
// every matrix entry is an FMA operand at a fixed offset (no shared-memory
// loads). Face and edge components use different matrices per axis.
// lo: for the banded passes (W > 0), first column of row m's band of width W
// in summation order (the row's nonzeros all lie in [lo, lo + W))
template<int NB, class T>
struct TpMats
{
    T m[3][2][NB * NB];
    unsigned char lo[3][2][NB];
};

template<int NB>
constexpr int tp_threads()
{
    return (NB * NB + 31) / 32 * 32;
}

// One pass along the fastest axis of `in`: thread p owns the pencil
// in[p*NB + n] and writes out[m*NB^2 + p] = sum_n T(m,n) in[p*NB + n] with
// T(m,n) = M_K(m,n) (anterpolation) or M_K(n,m) (interpolation). Writing the
// result with the axes rotated ([z][y][x] -> [x][z][y]) makes the next axis
// the fastest one, so all three passes read contiguous pencils; after three
// passes the layout is back to [z][y][x]. The last pass adds into the
// thread's accumulators instead of writing shared memory.
// W > 0: only the W entries of row m's band [lo, lo + W) are summed, in
// the same order; the skipped entries are zeros, whose FMAs leave the running
// sum unchanged, so the result equals the full row's
// T: arithmetic and shared-memory type of the passes (the accumulators acc,
// which start from and end in the FP64 target block, stay FP64)
template<int NB, int A, int K, bool TR, bool LAST, int W, class T>
__device__ __forceinline__ void tp_pass(const T* __restrict__ in, T* __restrict__ out,
                                        const TpMats<NB, T>& mt, int p, double* acc)
{
    if constexpr (W == 0)
    {
        T v[NB];
#pragma unroll
        for (int n = 0; n < NB; ++n) v[n] = in[p * NB + n];
#pragma unroll
        for (int m = 0; m < NB; ++m)
        {
            T s = 0;
#pragma unroll
            for (int n = 0; n < NB; ++n) s = fma(TR ? mt.m[A][K][n * NB + m] : mt.m[A][K][m * NB + n], v[n], s);
            if (LAST) acc[m] += s;
            else out[m * NB * NB + p] = s;
        }
    }
    else
    {
        const T* row = in + p * NB;
#pragma unroll
        for (int m = 0; m < NB; ++m)
        {
            const int lo = mt.lo[A][K][m];
            T s = 0;
#pragma unroll
            for (int j = 0; j < W; ++j)
            {
                const int n = lo + j;
                s = fma(TR ? mt.m[A][K][n * NB + m] : mt.m[A][K][m * NB + n], row[n], s);
            }
            if (LAST) acc[m] += s;
            else out[m * NB * NB + p] = s;
        }
    }
}

template<int NB, int A, bool TR, bool LAST, int W, class T>
__device__ __forceinline__ void tp_pass_bit(int bit, const T* in, T* out, const TpMats<NB, T>& mt, int p, double* acc)
{
    if (bit) tp_pass<NB, A, 1, TR, LAST, W, T>(in, out, mt, p, acc);
    else tp_pass<NB, A, 0, TR, LAST, W, T>(in, out, mt, p, acc);
}

// mode 0: dst[group] += sum_tasks A(src)        (anterpolation / coarsify)
// mode 1: dst[group] += I(src)                  (FMM interpolation)
// mode 2: dst[group]  = I(src)                  (cell-centred interpolation)
// One CTA per receiving block, one thread per pencil; the sending blocks of
// a group are applied in child order into per-thread accumulators.
template<int NB, bool TR, int W, class T>
__global__ void __launch_bounds__(tp_threads<NB>(), 2) tp_kernel(
    const int* __restrict__ gptr, const int* __restrict__ gdst, const int* __restrict__ tsrc,
    const int* __restrict__ tcid, const double* __restrict__ src, double* __restrict__ dst,
    const __grid_constant__ TpMats<NB, T> mt, int mode)
{
    constexpr int N3 = NB * NB * NB;
    extern __shared__ __align__(16) unsigned char tp_smem[];
    T* a = reinterpret_cast<T*>(tp_smem);
    T* b = a + N3;
    const int g = blockIdx.x;
    const int p = threadIdx.x;
    const bool active = p < NB * NB;
    // accumulate onto the receiving block in task order (dst += r_0, += r_1, ...)
    double* d = dst + (size_t)gdst[g] * N3 + p;
    double acc[NB];
#pragma unroll
    for (int m = 0; m < NB; ++m) acc[m] = (active && mode != 2) ? d[m * NB * NB] : 0.0;
    for (int t = gptr[g]; t < gptr[g + 1]; ++t)
    {
        const double2* s2 = reinterpret_cast<const double2*>(src + (size_t)tsrc[t] * N3);
        const int cid = tcid[t];
        for (int i = threadIdx.x; i < N3 / 2; i += blockDim.x)
        {
            const double2 v = s2[i];
            a[2 * i] = (T)v.x;
            a[2 * i + 1] = (T)v.y;
        }
        __syncthreads();
        if (active) tp_pass_bit<NB, 0, TR, false, W, T>(cid & 1, a, b, mt, p, acc);
        __syncthreads();
        if (active) tp_pass_bit<NB, 1, TR, false, W, T>((cid >> 1) & 1, b, a, mt, p, acc);
        __syncthreads();
        if (active) tp_pass_bit<NB, 2, TR, true, W, T>((cid >> 2) & 1, a, (T*)nullptr, mt, p, acc);
        __syncthreads();
    }
    if (!active) return;
#pragma unroll
    for (int m = 0; m < NB; ++m) d[m * NB * NB] = acc[m];
}

// Width-2 band, sending-side form (mode 0, coarsening): thread p = (x', y')
// owns the receiving z-pencil, as in the last pass of tp_kernel, and forms
// the three passes' values it needs straight from the sending block in
// registers, in the passes' order (x band, then y band, then z band, the
// band entries in summation order): the same FMAs as tp_kernel<NB, false, 2>
// without the shared-memory staging and its barriers. Sending blocks whose x
// or y band is zero for the thread (they feed other octants of the
// receiving block) are skipped: their sums would add exact zeros.
template<int NB, class T>
__global__ void __launch_bounds__(tp_threads<NB>(), 2) tp_band2_kernel(
    const int* __restrict__ gptr, const int* __restrict__ gdst, const int* __restrict__ tsrc,
    const int* __restrict__ tcid, const double* __restrict__ src, double* __restrict__ dst,
    const __grid_constant__ TpMats<NB, T> mt)
{
    constexpr int N3 = NB * NB * NB;
    const int g = blockIdx.x;
    const int p = threadIdx.x;
    if (p >= NB * NB) return;
    const int xo = p % NB, yo = p / NB;
    double* d = dst + (size_t)gdst[g] * N3 + p;
    double acc[NB];
#pragma unroll
    for (int m = 0; m < NB; ++m) acc[m] = d[m * NB * NB];
    for (int t = gptr[g]; t < gptr[g + 1]; ++t)
    {
        const int cid = tcid[t];
        const int kx = cid & 1, ky = (cid >> 1) & 1, kz = (cid >> 2) & 1;
        const int lx = mt.lo[0][kx][xo], ly = mt.lo[1][ky][yo];
        const T wx0 = mt.m[0][kx][xo * NB + lx], wx1 = mt.m[0][kx][xo * NB + lx + 1];
        const T wy0 = mt.m[1][ky][yo * NB + ly], wy1 = mt.m[1][ky][yo * NB + ly + 1];
        if ((wx0 == (T)0 && wx1 == (T)0) || (wy0 == (T)0 && wy1 == (T)0)) continue;
        const double* blk = src + (size_t)tsrc[t] * N3;
        T cz[NB];
#pragma unroll
        for (int nz = 0; nz < NB; ++nz)
        {
            const double* r0 = blk + (size_t)(nz * NB + ly) * NB + lx;
            const double* r1 = r0 + NB;
            T b0 = 0, b1 = 0;
            b0 = fma(wx0, (T)__ldg(r0), b0);
            b0 = fma(wx1, (T)__ldg(r0 + 1), b0);
            b1 = fma(wx0, (T)__ldg(r1), b1);
            b1 = fma(wx1, (T)__ldg(r1 + 1), b1);
            T c = 0;
            c = fma(wy0, b0, c);
            c = fma(wy1, b1, c);
            cz[nz] = c;
        }
#pragma unroll
        for (int m = 0; m < NB; ++m)
        {
            const int lz = mt.lo[2][kz][m];
            T s = 0;
            s = fma(mt.m[2][kz][m * NB + lz], cz[lz], s);
            s = fma(mt.m[2][kz][m * NB + lz + 1], cz[lz + 1], s);
            acc[m] += s;
        }
    }
#pragma unroll
    for (int m = 0; m < NB; ++m) d[m * NB * NB] = acc[m];
}

// threads walk the buffer shell only: the two z = 0, NB-1 planes, then per
// inner z plane its ring (rows y = 0, NB-1, columns x = 0, NB-1)
template<int NB>
__global__ void halo_kernel(double* __restrict__ f, const int* __restrict__ list, const int* __restrict__ nbr,
                            const int* __restrict__ bbase, int e)
{
    constexpr int N3 = NB * NB * NB;
    constexpr int P2 = NB * NB, RING = 4 * NB - 4, SHELL = 2 * P2 + (NB - 2) * RING;
    const int o = list[blockIdx.x];
    double* blk = f + (size_t)o * N3;
    for (int t = threadIdx.x; t < SHELL; t += blockDim.x)
    {
        int x, y, z;
        if (t < 2 * P2)
        {
            z = t < P2 ? 0 : NB - 1;
            x = (t % P2) % NB;
            y = (t % P2) / NB;
        }
        else
        {
            const int u = t - 2 * P2, r = u % RING;
            z = 1 + u / RING;
            if (r < 2 * NB)
            {
                y = r < NB ? 0 : NB - 1;
                x = r % NB;
            }
            else
            {
                const int w = r - 2 * NB;
                x = (w & 1) ? NB - 1 : 0;
                y = 1 + w / 2;
            }
        }
        const int i = x + NB * (y + NB * z);
        const int dx = x == 0 ? -1 : (x == NB - 1 ? 1 : 0);
        const int dy = y == 0 ? -1 : (y == NB - 1 ? 1 : 0);
        const int dz = z == 0 ? -1 : (z == NB - 1 ? 1 : 0);
        const int q = nbr[27 * o + (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)];
        if (q < 0) continue;
        // global cell of this buffer node and its position in q's interior
        const int lx = bbase[3 * o] - 1 + x - bbase[3 * q];
        const int ly = bbase[3 * o + 1] - 1 + y - bbase[3 * q + 1];
        const int lz = bbase[3 * o + 2] - 1 + z - bbase[3 * q + 2];
        if (lx < 0 || ly < 0 || lz < 0 || lx >= e || ly >= e || lz >= e) continue;
        blk[i] = f[(size_t)q * N3 + (lx + 1) + NB * ((ly + 1) + NB * (lz + 1))];
    }
}

template<int NB>
__global__ void correction_kernel(const double* __restrict__ tt, double* __restrict__ corr,
                                  const int* __restrict__ list, double r)
{
    constexpr int N3 = NB * NB * NB;
    const int o = list[blockIdx.x];
    const double* t = tt + (size_t)o * N3;
    double* c = corr + (size_t)o * N3;
    for (int i = threadIdx.x; i < N3; i += blockDim.x)
    {
        const int x = i % NB, y = (i / NB) % NB, z = i / (NB * NB);
        if (x == 0 || y == 0 || z == 0 || x == NB - 1 || y == NB - 1 || z == NB - 1) continue;
        double v = c[i];
        v += 6.0 * t[i] * r;
        v -= t[i - NB * NB] * r;
        v -= t[i + NB * NB] * r;
        v -= t[i - NB] * r;
        v -= t[i + NB] * r;
        v -= t[i + 1] * r;
        v -= t[i - 1] * r;
        c[i] = v;
    }
}

__global__ void zero_kernel(double* __restrict__ f, const int* __restrict__ list, int n3)
{
    double* b = f + (size_t)list[blockIdx.x] * n3;
    for (int i = threadIdx.x; i < n3; i += blockDim.x) b[i] = 0.0;
}

__global__ void copy_interior_kernel(const double* __restrict__ s, double* __restrict__ d,
                                     const int* __restrict__ list, int NB)
{
    const int n3 = NB * NB * NB;
    const size_t off = (size_t)list[blockIdx.x] * n3;
    for (int i = threadIdx.x; i < n3; i += blockDim.x)
    {
        const int x = i % NB, y = (i / NB) % NB, z = i / (NB * NB);
        if (x == 0 || y == 0 || z == 0 || x == NB - 1 || y == NB - 1 || z == NB - 1) continue;
        d[off + i] = s[off + i];
    }
}

__global__ void axpy_kernel(const double* __restrict__ s, double* __restrict__ d, const int* __restrict__ list,
                            int n3, double a, int assign)
{
    const size_t off = (size_t)list[blockIdx.x] * n3;
    for (int i = threadIdx.x; i < n3; i += blockDim.x)
    {
        if (assign) d[off + i] = a * s[off + i];
        else d[off + i] += s[off + i] * a;
    }
}

template<class F>
void nb_dispatch(int Nb, F&& f)
{
    switch (Nb)
    {
        case 6: f(std::integral_constant<int, 6>{}); return;
        case 8: f(std::integral_constant<int, 8>{}); return;
        case 10: f(std::integral_constant<int, 10>{}); return;
        case 12: f(std::integral_constant<int, 12>{}); return;
        case 16: f(std::integral_constant<int, 16>{}); return;
        case 18: f(std::integral_constant<int, 18>{}); return;
        default: throw Error(IBLGF_EINVAL, "unsupported block size");
    }
}
}  // namespace

void launch_tp(Ctx& c, const TpTasks& t, const double* src, double* dst, int mat_base, int mode, bool fp32)
{
    const int bases[3] = {mat_base, mat_base, mat_base};
    launch_tp_axes(c, t, src, dst, bases, mode, fp32);
}

namespace
{
template<int NB, class T>
void launch_tp_typed(Ctx& c, const TpTasks& t, const double* src, double* dst, const int* mat_base, int mode)
{
    static_assert((NB * NB * NB) % 2 == 0, "blocks are copied as double2");
    TpMats<NB, T> mt;
    const bool tr = mode != 0;
    int width = 0;  // widest band of any row, in summation order
    for (int a = 0; a < 3; ++a)
    {
        const size_t off = (size_t)mat_base[a] * NB * NB;
        if (c.h_mats.size() < off + 2 * NB * NB) throw Error(IBLGF_EINTERNAL, "transfer matrices missing");
        for (int k = 0; k < 2; ++k)
            for (int i = 0; i < NB * NB; ++i) mt.m[a][k][i] = (T)c.h_mats[off + (size_t)k * NB * NB + i];
        for (int k = 0; k < 2; ++k)
            for (int m = 0; m < NB; ++m)
            {
                int lo = NB, hi = 0;
                for (int n = 0; n < NB; ++n)
                    if ((tr ? mt.m[a][k][n * NB + m] : mt.m[a][k][m * NB + n]) != (T)0)
                    {
                        lo = std::min(lo, n);
                        hi = n + 1;
                    }
                mt.lo[a][k][m] = (unsigned char)(lo < hi ? lo : 0);
                width = std::max(width, lo < hi ? hi - lo : 0);
            }
    }
    const int W = width <= 2 ? 2 : (width <= 5 ? 5 : 0);
    if (W)
        for (int a = 0; a < 3; ++a)
            for (int k = 0; k < 2; ++k)
                for (int m = 0; m < NB; ++m) mt.lo[a][k][m] = (unsigned char)std::min<int>(mt.lo[a][k][m], NB - W);
    const size_t smem = 2 * (size_t)NB * NB * NB * sizeof(T);
    auto launch = [&](auto kfn) {
        IBLGF_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kfn<<<t.n_groups, tp_threads<NB>(), smem, c.stream>>>(t.group_ptr.p, t.group_dst.p, t.task_src.p,
                                                              t.task_cid.p, src, dst, mt, mode);
    };
    if (mode == 0)
    {
        if (W == 2)
        {
            auto kfn = tp_band2_kernel<NB, T>;
            kfn<<<t.n_groups, tp_threads<NB>(), 0, c.stream>>>(t.group_ptr.p, t.group_dst.p, t.task_src.p,
                                                              t.task_cid.p, src, dst, mt);
        }
        else if (W == 5) launch(tp_kernel<NB, false, 5, T>);
        else launch(tp_kernel<NB, false, 0, T>);
    }
    else
    {
        if (W == 2) launch(tp_kernel<NB, true, 2, T>);
        else if (W == 5) launch(tp_kernel<NB, true, 5, T>);
        else launch(tp_kernel<NB, true, 0, T>);
    }
}
}  // namespace

// fp32: the passes in FP32 (matrices rounded to FP32), the sums into the
// FP64 receiving blocks in FP64
void launch_tp_axes(Ctx& c, const TpTasks& t, const double* src, double* dst, const int* mat_base, int mode, bool fp32)
{
    if (!t.n_groups) return;
    nb_dispatch(c.Nb, [&](auto nbc) {
        constexpr int NB = decltype(nbc)::value;
        if (fp32) launch_tp_typed<NB, float>(c, t, src, dst, mat_base, mode);
        else launch_tp_typed<NB, double>(c, t, src, dst, mat_base, mode);
    });
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_halo(Ctx& c, double* f, const int* list, int n)
{
    if (!n) return;
    nb_dispatch(c.Nb, [&](auto nbc) {
        constexpr int NB = decltype(nbc)::value;
        halo_kernel<NB><<<n, 256, 0, c.stream>>>(f, list, c.d_nbr.p, c.d_bbase.p, c.cfg.block_extent);
    });
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_source_correction(Ctx& c, const double* target_tmp, double* corr, const int* list, int n,
                              double inv_dx2)
{
    if (!n) return;
    nb_dispatch(c.Nb, [&](auto nbc) {
        constexpr int NB = decltype(nbc)::value;
        correction_kernel<NB><<<n, 256, 0, c.stream>>>(target_tmp, corr, list, inv_dx2);
    });
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

namespace
{
// n doubles from p set to zero (16-byte stores where p is aligned)
__global__ void fill_zero_kernel(double* __restrict__ p, size_t n)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if ((reinterpret_cast<uintptr_t>(p) & 15) == 0)
    {
        double2* q = reinterpret_cast<double2*>(p);
        const double2 z = make_double2(0.0, 0.0);
        for (size_t j = i; j < n / 2; j += stride) q[j] = z;
        if (i == 0 && (n & 1)) p[n - 1] = 0.0;
    }
    else
        for (size_t j = i; j < n; j += stride) p[j] = 0.0;
}
// smallest index of a non-finite value (NaN or +-inf); *first starts at ~0
__global__ void nonfinite_kernel(const double* __restrict__ p, size_t n, unsigned long long* first)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride)
        if (!isfinite(p[j]))
        {
            atomicMin(first, (unsigned long long)j);
            return;  // later indices of this thread are larger
        }
}
}  // namespace

long long first_nonfinite(Ctx& c, const double* p, size_t n)
{
    DevBuf<unsigned long long> d;
    d.alloc(1);
    IBLGF_CUDA(cudaMemsetAsync(d.p, 0xFF, sizeof(unsigned long long), c.stream));
    if (n)
    {
        const size_t blocks = std::min<size_t>((n + 255) / 256, 148 * 8);
        nonfinite_kernel<<<(unsigned)blocks, 256, 0, c.stream>>>(p, n, d.p);
        c.launches += 1;
        IBLGF_CUDA(cudaGetLastError());
    }
    unsigned long long h = 0;
    IBLGF_CUDA(cudaMemcpyAsync(&h, d.p, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    return h == ~0ull ? -1 : (long long)h;
}

// a plain kernel (not cudaMemsetAsync), so that the zeroing can sit in the
// body of a conditional graph node
void launch_fill_zero(Ctx& c, double* p, size_t n)
{
    if (!n) return;
    const size_t blocks = std::min<size_t>((n / 2 + 255) / 256, 148 * 8);
    fill_zero_kernel<<<(unsigned)std::max<size_t>(blocks, 1), 256, 0, c.stream>>>(p, n);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_zero_blocks(Ctx& c, double* f, const int* list, int n)
{
    if (!n) return;
    zero_kernel<<<n, 256, 0, c.stream>>>(f, list, (int)c.block_elems());
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

// one CTA per leaf; host order: leaf i's interior e^3 values, x fastest
__global__ void leaves_scatter_kernel(const double* __restrict__ stage, double* __restrict__ f,
                                      const int* __restrict__ list, int e, int NB)
{
    const int e3 = e * e * e;
    const double* s = stage + (size_t)blockIdx.x * e3;
    double* b = f + (size_t)list[blockIdx.x] * NB * NB * NB;
    for (int i = threadIdx.x; i < e3; i += blockDim.x)
    {
        const int x = i % e, y = (i / e) % e, z = i / (e * e);
        b[((z + 1) * NB + y + 1) * NB + x + 1] = s[i];
    }
}

__global__ void leaves_gather_kernel(const double* __restrict__ f, double* __restrict__ stage,
                                     const int* __restrict__ list, int e, int NB)
{
    const int e3 = e * e * e;
    double* s = stage + (size_t)blockIdx.x * e3;
    const double* b = f + (size_t)list[blockIdx.x] * NB * NB * NB;
    for (int i = threadIdx.x; i < e3; i += blockDim.x)
    {
        const int x = i % e, y = (i / e) % e, z = i / (e * e);
        s[i] = b[((z + 1) * NB + y + 1) * NB + x + 1];
    }
}

void launch_leaves_scatter(Ctx& c, const double* stage, double* field, const int* list, int n)
{
    if (!n) return;
    leaves_scatter_kernel<<<n, 256, 0, c.stream>>>(stage, field, list, c.Nb - 2, c.Nb);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

namespace
{
// one CTA per listed block: field block <-> buf[i]
__global__ void blocks_copy_kernel(const double* __restrict__ from, double* __restrict__ to,
                                   const int* __restrict__ list, int b3, int gather)
{
    const size_t o = (size_t)list[blockIdx.x] * b3, i0 = (size_t)blockIdx.x * b3;
    for (int i = threadIdx.x; i < b3; i += blockDim.x)
    {
        if (gather) to[i0 + i] = from[o + i];
        else to[o + i] = from[i0 + i];
    }
}
}  // namespace

void launch_blocks_gather(Ctx& c, const double* field, double* buf, const int* list, int n)
{
    if (!n) return;
    blocks_copy_kernel<<<n, 256, 0, c.stream>>>(field, buf, list, (int)c.block_elems(), 1);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_blocks_scatter(Ctx& c, const double* buf, double* field, const int* list, int n)
{
    if (!n) return;
    blocks_copy_kernel<<<n, 256, 0, c.stream>>>(buf, field, list, (int)c.block_elems(), 0);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_leaves_gather(Ctx& c, const double* field, double* stage, const int* list, int n)
{
    if (!n) return;
    leaves_gather_kernel<<<n, 256, 0, c.stream>>>(field, stage, list, c.Nb - 2, c.Nb);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

namespace
{
// the leaf blocks (flag bit 0) in canonical order and a staging buffer for
// their interiors, built on first use after each domain (re)build
int leaf_blocks(Ctx& c)
{
    if (c.n_leaf_blocks < 0)
    {
        std::vector<int> l;
        for (int o = 0; o < c.n_oct; ++o)
            if (c.flags[o] & 1) l.push_back(o);
        c.d_leaf_blocks.upload(l, c.stream);
        c.n_leaf_blocks = (int)l.size();
        const size_t e = (size_t)c.Nb - 2;
        c.leaf_stage.alloc(std::max<size_t>(1, l.size() * e * e * e), c.cfg.device, c.stream);
    }
    return c.n_leaf_blocks;
}
}  // namespace

// DataField::update_device / update_host (datafield.hpp:211-226) restricted to
// the values a solve reads and produces: the interiors of the leaf blocks.
// The upload zeroes the whole field first (buffers and non-leaf blocks).
void field_upload_leaves(Ctx& c, int f, const double* host, size_t count)
{
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    const int n = leaf_blocks(c);
    const size_t e = (size_t)c.Nb - 2;
    if (!host || count != (size_t)n * e * e * e) throw Error(IBLGF_EINVAL, "leaf field size mismatch");
    IBLGF_CUDA(cudaMemcpyAsync(c.leaf_stage.p, host, count * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    IBLGF_CUDA(cudaMemsetAsync(c.field(f), 0, c.field_elems() * sizeof(double), c.stream));
    launch_leaves_scatter(c, c.leaf_stage.p, c.field(f), c.d_leaf_blocks.p, n);
}

void field_download_leaves(Ctx& c, int f, double* host, size_t count)
{
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    const int n = leaf_blocks(c);
    const size_t e = (size_t)c.Nb - 2;
    if (!host || count != (size_t)n * e * e * e) throw Error(IBLGF_EINVAL, "leaf field size mismatch");
    launch_leaves_gather(c, c.field(f), c.leaf_stage.p, c.d_leaf_blocks.p, n);
    IBLGF_CUDA(cudaMemcpyAsync(host, c.leaf_stage.p, count * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
}

namespace
{
void ensure_copy_stream(Ctx& c)
{
    if (c.copy_stream) return;
    IBLGF_CUDA(cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking));
    IBLGF_CUDA(cudaEventCreateWithFlags(&c.ev_gathered, cudaEventDisableTiming));
    IBLGF_CUDA(cudaEventCreateWithFlags(&c.ev_copied, cudaEventDisableTiming));
    IBLGF_CUDA(cudaEventCreateWithFlags(&c.ev_in_copied, cudaEventDisableTiming));
    IBLGF_CUDA(cudaEventCreateWithFlags(&c.ev_scattered, cudaEventDisableTiming));
    IBLGF_CUDA(cudaEventRecord(c.ev_copied, c.copy_stream));
    IBLGF_CUDA(cudaEventRecord(c.ev_scattered, c.stream));
}
}  // namespace

// Gather on the context stream, host copy on a second stream, so that the
// copy overlaps whatever the context stream runs next (the next upload, the
// next solve). The gather waits for the previous asynchronous copy out of
// leaf_out; iblgf_synchronize waits for both streams.
void field_download_leaves_async(Ctx& c, int f, double* host, size_t count)
{
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    const int n = leaf_blocks(c);
    const size_t e = (size_t)c.Nb - 2, vals = (size_t)n * e * e * e;
    if (!host || count != vals) throw Error(IBLGF_EINVAL, "leaf field size mismatch");
    ensure_copy_stream(c);
    IBLGF_CUDA(cudaStreamWaitEvent(c.stream, c.ev_copied, 0));
    if (c.leaf_out.n != std::max<size_t>(1, vals)) c.leaf_out.alloc(std::max<size_t>(1, vals), c.cfg.device, c.stream);
    launch_leaves_gather(c, c.field(f), c.leaf_out.p, c.d_leaf_blocks.p, n);
    IBLGF_CUDA(cudaEventRecord(c.ev_gathered, c.stream));
    IBLGF_CUDA(cudaStreamWaitEvent(c.copy_stream, c.ev_gathered, 0));
    IBLGF_CUDA(cudaMemcpyAsync(host, c.leaf_out.p, vals * sizeof(double), cudaMemcpyDeviceToHost, c.copy_stream));
    IBLGF_CUDA(cudaEventRecord(c.ev_copied, c.copy_stream));
}

// Host copy on the copy stream into leaf_in, then zeroing and scatter into
// the field on the context stream, which waits for the copy; the copy waits
// for the previous upload's scatter out of leaf_in. Issued right after a
// solve, the copy of the next input runs under that solve.
void field_upload_leaves_async(Ctx& c, int f, const double* host, size_t count)
{
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    const int n = leaf_blocks(c);
    const size_t e = (size_t)c.Nb - 2, vals = (size_t)n * e * e * e;
    if (!host || count != vals) throw Error(IBLGF_EINVAL, "leaf field size mismatch");
    ensure_copy_stream(c);
    if (c.leaf_in.n != std::max<size_t>(1, vals))
    {
        // stream-ordered on the context stream; the copy stream waits for it
        IBLGF_CUDA(cudaStreamSynchronize(c.copy_stream));
        c.leaf_in.alloc(std::max<size_t>(1, vals), c.cfg.device, c.stream);
        IBLGF_CUDA(cudaEventRecord(c.ev_scattered, c.stream));
    }
    IBLGF_CUDA(cudaStreamWaitEvent(c.copy_stream, c.ev_scattered, 0));
    IBLGF_CUDA(cudaMemcpyAsync(c.leaf_in.p, host, vals * sizeof(double), cudaMemcpyHostToDevice, c.copy_stream));
    IBLGF_CUDA(cudaEventRecord(c.ev_in_copied, c.copy_stream));
    IBLGF_CUDA(cudaStreamWaitEvent(c.stream, c.ev_in_copied, 0));
    IBLGF_CUDA(cudaMemsetAsync(c.field(f), 0, c.field_elems() * sizeof(double), c.stream));
    launch_leaves_scatter(c, c.leaf_in.p, c.field(f), c.d_leaf_blocks.p, n);
    IBLGF_CUDA(cudaEventRecord(c.ev_scattered, c.stream));
}

void copy_stream_release(Ctx& c)
{
    if (!c.copy_stream) return;
    cudaStreamSynchronize(c.copy_stream);
    cudaStreamSynchronize(c.stream);
    c.leaf_out.release();
    c.leaf_in.release();
    cudaEventDestroy(c.ev_gathered);
    cudaEventDestroy(c.ev_copied);
    cudaEventDestroy(c.ev_in_copied);
    cudaEventDestroy(c.ev_scattered);
    cudaStreamDestroy(c.copy_stream);
    c.copy_stream = nullptr;
    c.ev_gathered = c.ev_copied = c.ev_in_copied = c.ev_scattered = nullptr;
}

void launch_copy_interior(Ctx& c, const double* src, double* dst, const int* list, int n)
{
    if (!n) return;
    copy_interior_kernel<<<n, 256, 0, c.stream>>>(src, dst, list, c.Nb);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_axpy_blocks(Ctx& c, const double* src, double* dst, const int* list, int n, double a, bool assign)
{
    if (!n) return;
    axpy_kernel<<<n, 256, 0, c.stream>>>(src, dst, list, (int)c.block_elems(), a, assign ? 1 : 0);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

// Adaptation: new block b takes old block src[b] (or zeros when src[b] < 0)
__global__ void remap_blocks_kernel(const double2* __restrict__ old, double2* __restrict__ nw,
                                    const int* __restrict__ src, int half_block)
{
    const int b = blockIdx.x;
    const int s = src[b];
    double2* d = nw + (size_t)b * half_block;
    if (s < 0)
        for (int i = threadIdx.x; i < half_block; i += blockDim.x) d[i] = make_double2(0.0, 0.0);
    else
    {
        const double2* o = old + (size_t)s * half_block;
        for (int i = threadIdx.x; i < half_block; i += blockDim.x) d[i] = o[i];
    }
}

void launch_remap_blocks(Ctx& c, const double* old, double* nw, const int* d_src, int n_new)
{
    if (!n_new) return;
    const int half = (int)(c.block_elems() / 2);  // Nb even: Nb^3 / 2 double2
    remap_blocks_kernel<<<n_new, 256, 0, c.stream>>>(reinterpret_cast<const double2*>(old),
                                                     reinterpret_cast<double2*>(nw), d_src, half);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

// Operator::maxnorm / blockRootMeanSquare (operators.hpp:1149-1211) over the
// block's interior nodes: max over nodes of sqrt(sum_c v_c^2) and
// sqrt(sum_nodes sum_c v_c^2 / nodes)
__global__ void block_norms_kernel(const double* __restrict__ f0, const double* __restrict__ f1,
                                   const double* __restrict__ f2, int n_comp, int NB, double* __restrict__ out_max,
                                   double* __restrict__ out_rms)
{
    const int b = blockIdx.x;
    const int e = NB - 2;
    const size_t base = (size_t)b * NB * NB * NB;
    double mx = 0.0, sum = 0.0;
    for (int i = threadIdx.x; i < e * e * e; i += blockDim.x)
    {
        const int x = i % e + 1, y = (i / e) % e + 1, z = i / (e * e) + 1;
        const size_t at = base + x + (size_t)NB * (y + (size_t)NB * z);
        double v = f0[at] * f0[at];
        if (n_comp > 1) v += f1[at] * f1[at];
        if (n_comp > 2) v += f2[at] * f2[at];
        sum += v;
        mx = fmax(mx, sqrt(v));
    }
    __shared__ double smx[256], ssum[256];
    smx[threadIdx.x] = mx;
    ssum[threadIdx.x] = sum;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1)
    {
        if ((int)threadIdx.x < o)
        {
            smx[threadIdx.x] = fmax(smx[threadIdx.x], smx[threadIdx.x + o]);
            ssum[threadIdx.x] += ssum[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        out_max[b] = smx[0];
        out_rms[b] = sqrt(ssum[0] / ((double)e * e * e));
    }
}

void launch_block_norms(Ctx& c, const double* const* comps, int n_comp, double* d_max, double* d_rms)
{
    if (!c.n_oct) return;
    block_norms_kernel<<<c.n_oct, 256, 0, c.stream>>>(comps[0], n_comp > 1 ? comps[1] : comps[0],
                                                      n_comp > 2 ? comps[2] : comps[0], n_comp, c.Nb, d_max, d_rms);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

}  // namespace iblgf_b200
