// Field kernels of the IF-HERK time step (FP64, whole component fields):
//   clean_kernel     Ifherk::clean (ifherk.hpp:1309-1352): zero whole blocks,
//                    or with non_leaf_only only the outer `width` planes of
//                    leaves and all of every other block
//   axpby_kernel     Ifherk::copy / add (ifherk.hpp:1878-1960) and in-place
//                    scaling, over every node including buffers
//   smooth_kernel    Operator::smooth2zero (operators.hpp:653-760) as called
//                    by clean_leaf_correction_boundary (ifherk.hpp:1383-1404):
//                    each listed (block, neighbour direction) multiplies the
//                    block by the tanh taper towards that face / edge / corner,
//                    `reps` times in a row (once per component of the field)
#include <algorithm>

#include "ctx.hpp"

namespace iblgf_b200
{
namespace
{
template<int NB>
__global__ void clean_kernel(double* __restrict__ f, const int* __restrict__ leaf, int non_leaf_only, int w)
{
    constexpr int N3 = NB * NB * NB;
    const int o = blockIdx.x;
    double* b = f + (size_t)o * N3;
    const bool shell = non_leaf_only && leaf[o];
    for (int i = threadIdx.x; i < N3; i += blockDim.x)
    {
        if (shell)
        {
            const int x = i % NB, y = (i / NB) % NB, z = i / (NB * NB);
            if (x >= w && y >= w && z >= w && x < NB - w && y < NB - w && z < NB - w) continue;
        }
        b[i] = 0.0;
    }
}

// up to three component fields per launch (blockIdx.y = component)
struct Fields3
{
    double* to[3];
    const double* from[3];
};

template<int NB>
__global__ void clean3_kernel(Fields3 f, const int* __restrict__ leaf, int non_leaf_only, int w)
{
    constexpr int N3 = NB * NB * NB;
    const int o = blockIdx.x;
    double* b = f.to[blockIdx.y] + (size_t)o * N3;
    const bool shell = non_leaf_only && leaf[o];
    for (int i = threadIdx.x; i < N3; i += blockDim.x)
    {
        if (shell)
        {
            const int x = i % NB, y = (i / NB) % NB, z = i / (NB * NB);
            if (x >= w && y >= w && z >= w && x < NB - w && y < NB - w && z < NB - w) continue;
        }
        b[i] = 0.0;
    }
}

// mode 0: to = a * from; 1: to += a * from; 2: to *= a (per component)
__global__ void axpby3_kernel(Fields3 f, double a, size_t n, int mode)
{
    double* __restrict__ to = f.to[blockIdx.y];
    const double* __restrict__ from = f.from[blockIdx.y];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    {
        if (mode == 0) to[i] = from[i] * a;
        else if (mode == 1) to[i] += from[i] * a;
        else to[i] *= a;
    }
}

// mode 0: to = a * from; 1: to += a * from; 2: to *= a; 3: to += a
__global__ void axpby_kernel(double* __restrict__ to, const double* __restrict__ from, double a, size_t n, int mode)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    {
        if (mode == 0) to[i] = from[i] * a;
        else if (mode == 1) to[i] += from[i] * a;
        else if (mode == 2) to[i] *= a;
        else to[i] += a;
    }
}

__device__ __forceinline__ double taper(double x)
{
    const double fac = 10.0, shift = 0.2;
    const double c = 1.0 - (0.5 + 0.5 * tanh(fac * (1.0 - shift)));
    return (0.5 + 0.5 * tanh(fac * (x - shift))) + c;
}

// entries [ptr[b], ptr[b+1]) of block list[b]: neighbour directions (0..26).
// The taper takes 2 NB distinct values (node index i from the low or the high
// side); the CTA evaluates them once into shared memory.
template<int NB>
__global__ void smooth_kernel(double* __restrict__ f, const int* __restrict__ list, const int* __restrict__ ptr,
                              const int* __restrict__ dirs, int reps)
{
    constexpr int N3 = NB * NB * NB;
    __shared__ double tlo[NB], thi[NB];  // taper(i / (NB-1)), taper(1 - i / (NB-1))
    if (threadIdx.x < NB)
    {
        // local_pct over the block with its buffer (node.hpp:121-124)
        const double pc = (double)threadIdx.x / (NB - 1);
        tlo[threadIdx.x] = taper(pc);
        thi[threadIdx.x] = taper(1.0 - pc);
    }
    __syncthreads();
    double* b = f + (size_t)list[blockIdx.x] * N3;
    const int e0 = ptr[blockIdx.x], e1 = ptr[blockIdx.x + 1];
    for (int i = threadIdx.x; i < N3; i += blockDim.x)
    {
        const int ix = i % NB, iy = (i / NB) % NB, iz = i / (NB * NB);
        double v = b[i];
        for (int e = e0; e < e1; ++e)
        {
            const int d = dirs[e], x = d % 3, y = (d / 3) % 3, z = d / 9;
            double sq = 0.0;
            int cnt = 0;
            if (z == 0) sq = fmax(sq, tlo[iz]), ++cnt;
            else if (z == 2) sq = fmax(sq, thi[iz]), ++cnt;
            if (y == 0) sq = fmax(sq, tlo[iy]), ++cnt;
            else if (y == 2) sq = fmax(sq, thi[iy]), ++cnt;
            if (x == 0) sq = fmax(sq, tlo[ix]), ++cnt;
            else if (x == 2) sq = fmax(sq, thi[ix]), ++cnt;
            if (cnt > 0)
                for (int r = 0; r < reps; ++r) v *= sq;
        }
        b[i] = v;
    }
}

template<class F>
void nb_switch(int Nb, F&& f)
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

void launch_clean(Ctx& c, double* f, const int* d_leaf, bool non_leaf_only, int width)
{
    if (!c.n_oct) return;
    nb_switch(c.Nb, [&](auto nbc) {
        constexpr int NB = decltype(nbc)::value;
        clean_kernel<NB><<<c.n_oct, 256, 0, c.stream>>>(f, d_leaf, non_leaf_only ? 1 : 0, width);
    });
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

// the component fields of one vector field in one launch
void launch_clean_vf(Ctx& c, double* const* f, int n, const int* d_leaf, bool non_leaf_only, int width)
{
    if (!c.n_oct || n < 1 || n > 3) return;
    Fields3 p{};
    for (int k = 0; k < n; ++k) p.to[k] = f[k];
    nb_switch(c.Nb, [&](auto nbc) {
        constexpr int NB = decltype(nbc)::value;
        clean3_kernel<NB><<<dim3(c.n_oct, n), 256, 0, c.stream>>>(p, d_leaf, non_leaf_only ? 1 : 0, width);
    });
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_axpby_vf(Ctx& c, double* const* to, const double* const* from, int n, double a, int mode)
{
    const size_t elems = c.field_elems();
    if (!elems || n < 1 || n > 3) return;
    Fields3 p{};
    for (int k = 0; k < n; ++k)
    {
        p.to[k] = to[k];
        p.from[k] = from ? from[k] : nullptr;
    }
    const unsigned grid = (unsigned)std::min<size_t>((elems + 255) / 256, 148 * 16 / n);
    axpby3_kernel<<<dim3(grid, n), 256, 0, c.stream>>>(p, a, elems, mode);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_axpby(Ctx& c, double* to, const double* from, double a, int mode)
{
    const size_t n = c.field_elems();
    if (!n) return;
    const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16);
    axpby_kernel<<<grid, 256, 0, c.stream>>>(to, from, a, n, mode);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_smooth(Ctx& c, double* f, const int* list, const int* ptr, const int* dirs, int n, int reps)
{
    if (!n) return;
    nb_switch(c.Nb, [&](auto nbc) {
        constexpr int NB = decltype(nbc)::value;
        smooth_kernel<NB><<<n, 256, 0, c.stream>>>(f, list, ptr, dirs, reps);
    });
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

}  // namespace iblgf_b200
