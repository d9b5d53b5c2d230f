// Inverse transform of the accumulated spectra of one FMM sweep, added into
// the targets (Convolution::apply_backward + dfft_c2r::execute + add_solution,
// include/iblgf/utilities/convolution.hpp:232-304, src/utilities/
// convolution.cpp:151-238): per target, c2r of the P^3 half spectrum,
// window [Nb-1, 2Nb-2]^3 scaled and added into the Nb^3 target block.
//
// B200 structure: a cluster of two CTAs per target. CTA h owns the kx half
// [h Nb/2, (h+1) Nb/2) of the half spectrum, so every accumulated value is
// read from HBM once:
//   z  thread per (ky, kx) pencil: P frequencies -> the Nb window planes
//   y  thread per (plane, kx) column: P -> the Nb window rows
//   x  thread per (plane, row): this CTA's kx half of the c2r sum, all Nb
//      outputs (a partial sum)
// then each CTA adds its half of the planes, own partial plus the peer's
// read through distributed shared memory (always rank 0's partial first, so
// the result does not depend on timing), into the target.
// The z and y passes use the prime-factor (Good-Thomas) algorithm for
// P = N1 N2 with coprime N1, N2 (35 = 5 x 7, 15 = 3 x 5): with input
// n = (N2 n1 + N1 n2) mod P and output k, e^{2 pi i n k / P} =
// e^{2 pi i n1 (k mod N1) / N1} e^{2 pi i n2 (k mod N2) / N2}, so
//     X[k] = sum_n2 W_N2^{n2 (k mod N2)} T_n2[k mod N1],
//     T_n2[k1] = sum_n1 W_N1^{n1 k1} x[N2 n1 + N1 n2 mod P],
// N2 short DFTs of length N1 plus Nb sums of N2 terms per pencil, with no
// twiddle multiplications: 301 complex multiply-adds per 35-point pencil and
// window instead of the direct 630, and error growth over 5- and 7-term sums
// instead of 35-term ones. All loops are unrolled, so every root of unity is
// a compile-time-indexed constant-bank operand.
#include <cooperative_groups.h>

#include <type_traits>

#include "cplx.cuh"
#include "ctx.hpp"

namespace cg = cooperative_groups;

namespace iblgf_b200
{
namespace
{
// roots of unity e^{+2 pi i j / N} for N in {3, 5, 7} and the c2r roots
// e^{+2 pi i j / P} for P in {15, 35}
constexpr int kPfaTw = 3 + 5 + 7;
__constant__ double c_pfa64[2 * kPfaTw];
__constant__ float c_pfa32[2 * kPfaTw];
__constant__ double c_c2r64[2 * (15 + 35)];

__host__ __device__ constexpr int pfa_base(int N) { return N == 3 ? 0 : (N == 5 ? 3 : 8); }
__host__ __device__ constexpr int c2r_base(int P) { return P == 15 ? 0 : 15; }

template<class R, int N>
__device__ __forceinline__ cx<R> wroot(int j)
{
    if constexpr (std::is_same<R, double>::value)
        return mk<R>(c_pfa64[2 * (pfa_base(N) + j)], c_pfa64[2 * (pfa_base(N) + j) + 1]);
    else
        return mk<R>(c_pfa32[2 * (pfa_base(N) + j)], c_pfa32[2 * (pfa_base(N) + j) + 1]);
}

template<int NB>
struct Pfa
{
    static constexpr int P = 2 * NB - 1;
    static constexpr int N1 = P == 35 ? 5 : 3;
    static constexpr int N2 = P == 35 ? 7 : 5;
    static_assert(P == 35 || P == 15, "prime-factor split of 15 or 35");
};

// One PFA pass over a pencil of P values: x(i) loads input i (i < P), the
// window outputs (k = o + NB - 1) accumulate into out[o]. N2 range [A, B).
template<class R, int NB, int A, int B, class Load>
__device__ __forceinline__ void pfa_pencil(Load&& x, cx<R> (&out)[NB])
{
    using PF = Pfa<NB>;
    constexpr int P = PF::P, N1 = PF::N1, N2 = PF::N2;
#pragma unroll
    for (int n2 = A; n2 < B; ++n2)
    {
        cx<R> v[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) v[n1] = x((N2 * n1 + N1 * n2) % P);
        cx<R> T[N1];
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1)
        {
            T[k1] = v[0];
#pragma unroll
            for (int n1 = 1; n1 < N1; ++n1)
            {
                const int j = (n1 * k1) % N1;
                if (j == 0)
                {
                    T[k1].x += v[n1].x;
                    T[k1].y += v[n1].y;
                }
                else
                    cmac<R>(T[k1], v[n1], wroot<R, N1>(j));
            }
        }
#pragma unroll
        for (int o = 0; o < NB; ++o)
        {
            const int k = o + NB - 1;
            const int j = (n2 * (k % N2)) % N2;
            if (j == 0)
            {
                out[o].x += T[k % N1].x;
                out[o].y += T[k % N1].y;
            }
            else
                cmac<R>(out[o], T[k % N1], wroot<R, N2>(j));
        }
    }
}

// x pass of CTA half H: partial c2r over kx in [H NB/2, (H+1) NB/2) of one
// row y[kx] (local index), v(xo) = sum w_kx Re(y e^{+2 pi i kx (xo+NB-1)/P}),
// w = 1 for kx = 0, 2 otherwise
template<class R, int NB, int H>
__device__ __forceinline__ void c2r_half(const cx<R>* yrow, double (&out)[NB])
{
    constexpr int P = 2 * NB - 1, KH = NB / 2;
#pragma unroll
    for (int o = 0; o < NB; ++o) out[o] = 0.0;
#pragma unroll
    for (int j = 0; j < KH; ++j)
    {
        const int kx = H * KH + j;
        const cx<R> yv = yrow[j];
        const double yr = (double)yv.x * (kx ? 2.0 : 1.0), yi = (double)yv.y * (kx ? 2.0 : 1.0);
#pragma unroll
        for (int o = 0; o < NB; ++o)
        {
            const int idx = (kx * (o + NB - 1)) % P;
            const double c = c_c2r64[2 * (c2r_base(P) + idx)], s = c_c2r64[2 * (c2r_base(P) + idx) + 1];
            out[o] = fma(yr, c, fma(-yi, s, out[o]));
        }
    }
}

// shared memory: V [NB planes][P][KH] complex (z output, then y output in
// the first NB rows of each plane) and the x-pass partials [NB][NB][NB]
template<class RZ, int NB>
struct InvSmem
{
    static constexpr int P = 2 * NB - 1, KH = NB / 2;
    static constexpr size_t v = (size_t)NB * P * KH * sizeof(cx<RZ>);
    static constexpr size_t part = (size_t)NB * NB * NB * sizeof(double);
    static constexpr size_t total = v + part;
};

template<class RZ, class RA, int NB>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(NB* NB)
    inv_pfa_kernel(const cx<RA>* __restrict__ ACC, const int* __restrict__ tgt_oct, double scale,
                   double* __restrict__ target)
{
    constexpr int P = 2 * NB - 1, KH = NB / 2, NP = P * NB;
    using SM = InvSmem<RZ, NB>;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<RZ>* V = reinterpret_cast<cx<RZ>*>(smraw);                  // [zo][ky][kxl]
    double* part = reinterpret_cast<double*>(smraw + SM::v);         // [zo][yo][xo]
    cg::cluster_group cluster = cg::this_cluster();
    const int h = (int)cluster.block_rank();
    const int t = blockIdx.x / 2;
    const cx<RZ> zero = mk<RZ>(0, 0);

    // z: pencil (ky, kxl); the accumulator is [kz][ky][kx]
    {
        const int p = threadIdx.x;
        if (p < P * KH)
        {
            const int ky = p / KH, kxl = p % KH;
            const cx<RA>* a = ACC + (size_t)t * P * NP + (size_t)ky * NB + h * KH + kxl;
            cx<RZ> out[NB];
#pragma unroll
            for (int o = 0; o < NB; ++o) out[o] = zero;
            pfa_pencil<RZ, NB, 0, Pfa<NB>::N2>(
                [&](int kz) {
                    const cx<RA> v = a[(size_t)kz * NP];
                    return mk<RZ>((RZ)v.x, (RZ)v.y);
                },
                out);
#pragma unroll
            for (int o = 0; o < NB; ++o) V[(o * P + ky) * KH + kxl] = out[o];
        }
    }
    __syncthreads();
    // y: column (zo, kxl), outputs written over the column's first NB rows
    {
        const int q = threadIdx.x;
        if (q < NB * KH)
        {
            const int zo = q / KH, kxl = q % KH;
            cx<RZ>* col = V + (size_t)zo * P * KH + kxl;
            cx<RZ> out[NB];
#pragma unroll
            for (int o = 0; o < NB; ++o) out[o] = zero;
            pfa_pencil<RZ, NB, 0, Pfa<NB>::N2>([&](int ky) { return col[(size_t)ky * KH]; }, out);
#pragma unroll
            for (int o = 0; o < NB; ++o) col[(size_t)o * KH] = out[o];
        }
    }
    __syncthreads();
    // x: row (zo, yo), partial c2r over this CTA's kx half
    {
        const int zo = threadIdx.x / NB, yo = threadIdx.x % NB;
        const cx<RZ>* yrow = V + ((size_t)zo * P + yo) * KH;
        double out[NB];
        if (h == 0) c2r_half<RZ, NB, 0>(yrow, out);
        else c2r_half<RZ, NB, 1>(yrow, out);
        double* prow = part + ((size_t)zo * NB + yo) * NB;
#pragma unroll
        for (int o = 0; o < NB; ++o) prow[o] = out[o];
    }
    cluster.sync();  // both partials complete
    {
        const double* p0 = h == 0 ? part : cluster.map_shared_rank(part, 0);
        const double* p1 = h == 1 ? part : cluster.map_shared_rank(part, 1);
        double* out = target + (size_t)tgt_oct[t] * NB * NB * NB;
        const int base = h * (NB / 2) * NB * NB;
        for (int i = threadIdx.x; i < (NB / 2) * NB * NB; i += blockDim.x)
            out[base + i] += scale * (p0[base + i] + p1[base + i]);
    }
    cluster.sync();  // the peer has read this CTA's partials
}

template<class RZ, class RA, int NB>
void launch_inv_pfa(Ctx& c, const void* acc, const int* d_tgt_oct, int n, double scale, double* target)
{
    using SM = InvSmem<RZ, NB>;
    auto kfn = inv_pfa_kernel<RZ, RA, NB>;
    IBLGF_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM::total));
    kfn<<<2 * n, NB * NB, SM::total, c.stream>>>((const cx<RA>*)acc, d_tgt_oct, scale, target);
    c.launches += 1;
}
}  // namespace

void init_pfa_constants(int device)
{
    (void)device;
    double t64[2 * kPfaTw];
    float t32[2 * kPfaTw];
    for (int N : {3, 5, 7})
        for (int j = 0; j < N; ++j)
        {
            const double a = 2.0 * M_PI * j / N;
            t64[2 * (pfa_base(N) + j)] = std::cos(a);
            t64[2 * (pfa_base(N) + j) + 1] = std::sin(a);
        }
    for (int i = 0; i < 2 * kPfaTw; ++i) t32[i] = (float)t64[i];
    double c2r[2 * (15 + 35)];
    for (int P : {15, 35})
        for (int j = 0; j < P; ++j)
        {
            const double a = 2.0 * M_PI * j / P;
            c2r[2 * (c2r_base(P) + j)] = std::cos(a);
            c2r[2 * (c2r_base(P) + j) + 1] = std::sin(a);
        }
    IBLGF_CUDA(cudaMemcpyToSymbol(c_pfa64, t64, sizeof(t64)));
    IBLGF_CUDA(cudaMemcpyToSymbol(c_pfa32, t32, sizeof(t32)));
    IBLGF_CUDA(cudaMemcpyToSymbol(c_c2r64, c2r, sizeof(c2r)));
}

// true if the prime-factor inverse handles this block size; the FP32 path
// runs its z and y passes in FP32 when fp32_passes is set
bool inverse_pfa(Ctx& c, const void* acc, const int* d_tgt_oct, int n, double scale, double* target,
                 bool fp32_passes)
{
    if (!n) return true;
    const bool f32 = c.cfg.precision == IBLGF_FP32;
    switch (c.Nb)
    {
        case 18:
            if (!f32) launch_inv_pfa<double, double, 18>(c, acc, d_tgt_oct, n, scale, target);
            else if (fp32_passes) launch_inv_pfa<float, float, 18>(c, acc, d_tgt_oct, n, scale, target);
            else launch_inv_pfa<double, float, 18>(c, acc, d_tgt_oct, n, scale, target);
            return true;
        case 8:
            if (!f32) launch_inv_pfa<double, double, 8>(c, acc, d_tgt_oct, n, scale, target);
            else if (fp32_passes) launch_inv_pfa<float, float, 8>(c, acc, d_tgt_oct, n, scale, target);
            else launch_inv_pfa<double, float, 8>(c, acc, d_tgt_oct, n, scale, target);
            return true;
        default: return false;
    }
}

}  // namespace iblgf_b200
