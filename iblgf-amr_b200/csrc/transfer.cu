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
#include "ctx.hpp"

namespace iblgf_b200
{
namespace
{
// One pass of a separable transfer along axis d: out[..m..] = sum_n T(m,n) in[..n..]
// with T(m,n) = M(m,n) (anterpolation) or M(n,m) (interpolation).
template<int NB>
__device__ __forceinline__ void tp_pass(const double* __restrict__ in, double* __restrict__ out,
                                        const double* __restrict__ M, int axis, bool transpose)
{
    constexpr int N3 = NB * NB * NB;
    const int stride = axis == 0 ? 1 : (axis == 1 ? NB : NB * NB);
    for (int i = threadIdx.x; i < N3; i += blockDim.x)
    {
        const int m = (i / stride) % NB;
        const int base = i - m * stride;
        double s = 0.0;
#pragma unroll 6
        for (int n = 0; n < NB; ++n)
        {
            const double t = transpose ? M[n * NB + m] : M[m * NB + n];
            s = fma(t, in[base + n * stride], s);
        }
        out[i] = s;
    }
}

// mode 0: dst[group] += sum_tasks A(src)        (anterpolation / coarsify)
// mode 1: dst[group] += I(src)                  (FMM interpolation)
// mode 2: dst[group]  = I(src)                  (cell-centred interpolation)
template<int NB>
__global__ void __launch_bounds__(256) tp_kernel(const int* __restrict__ gptr, const int* __restrict__ gdst,
                                                 const int* __restrict__ tsrc, const int* __restrict__ tcid,
                                                 const double* __restrict__ src, double* __restrict__ dst,
                                                 const double* __restrict__ mats, int mode)
{
    constexpr int N3 = NB * NB * NB;
    extern __shared__ double sm[];
    double* a = sm;
    double* b = a + N3;
    double* acc = b + N3;
    double* mat = acc + N3;  // 2 matrices
    const int g = blockIdx.x;
    for (int i = threadIdx.x; i < 2 * NB * NB; i += blockDim.x) mat[i] = mats[i];
    for (int i = threadIdx.x; i < N3; i += blockDim.x) acc[i] = 0.0;
    const bool tr = mode != 0;
    for (int t = gptr[g]; t < gptr[g + 1]; ++t)
    {
        const double* s = src + (size_t)tsrc[t] * N3;
        const int cid = tcid[t];
        __syncthreads();
        for (int i = threadIdx.x; i < N3; i += blockDim.x) a[i] = s[i];
        __syncthreads();
        tp_pass<NB>(a, b, mat + ((cid >> 0) & 1) * NB * NB, 0, tr);
        __syncthreads();
        tp_pass<NB>(b, a, mat + ((cid >> 1) & 1) * NB * NB, 1, tr);
        __syncthreads();
        tp_pass<NB>(a, b, mat + ((cid >> 2) & 1) * NB * NB, 2, tr);
        __syncthreads();
        for (int i = threadIdx.x; i < N3; i += blockDim.x) acc[i] += b[i];
    }
    __syncthreads();
    double* d = dst + (size_t)gdst[g] * N3;
    if (mode == 2)
        for (int i = threadIdx.x; i < N3; i += blockDim.x) d[i] = acc[i];
    else
        for (int i = threadIdx.x; i < N3; i += blockDim.x) d[i] += acc[i];
}

template<int NB>
__global__ void halo_kernel(double* __restrict__ f, const int* __restrict__ list, const int* __restrict__ nbr,
                            const int* __restrict__ bbase, int e)
{
    constexpr int N3 = NB * NB * NB;
    const int o = list[blockIdx.x];
    double* blk = f + (size_t)o * N3;
    for (int i = threadIdx.x; i < N3; i += blockDim.x)
    {
        const int x = i % NB, y = (i / NB) % NB, z = i / (NB * NB);
        const int dx = x == 0 ? -1 : (x == NB - 1 ? 1 : 0);
        const int dy = y == 0 ? -1 : (y == NB - 1 ? 1 : 0);
        const int dz = z == 0 ? -1 : (z == NB - 1 ? 1 : 0);
        if (!dx && !dy && !dz) continue;
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

void launch_tp(Ctx& c, const TpTasks& t, const double* src, double* dst, int mat_base, int mode)
{
    if (!t.n_groups) return;
    nb_dispatch(c.Nb, [&](auto nbc) {
        constexpr int NB = decltype(nbc)::value;
        const size_t smem = (3 * (size_t)NB * NB * NB + 2 * NB * NB) * sizeof(double);
        static bool attr = false;
        if (!attr)
        {
            IBLGF_CUDA(cudaFuncSetAttribute(tp_kernel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
            attr = true;
        }
        tp_kernel<NB><<<t.n_groups, 256, smem, c.stream>>>(t.group_ptr.p, t.group_dst.p, t.task_src.p,
                                                           t.task_cid.p, src, dst,
                                                           c.d_mats.p + (size_t)mat_base * NB * NB, mode);
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

void launch_zero_blocks(Ctx& c, double* f, const int* list, int n)
{
    if (!n) return;
    zero_kernel<<<n, 256, 0, c.stream>>>(f, list, (int)c.block_elems());
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
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

}  // namespace iblgf_b200
