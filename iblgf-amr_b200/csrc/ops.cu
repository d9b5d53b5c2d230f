// Staggered mimetic block operators on the device, FP64:
//   include/iblgf/operators/operators.hpp:1386-1419 laplace (cell -> cell),
//   :1421-1446 gradient (cell -> face), :1448-1477 divergence (face -> cell),
//   :1479-1513 curl (face -> edge), :2416-2453 curl_transpose (edge -> face),
//   :2455-2531 nonlinear (face x edge -> face, the u x omega term).
// One CTA per block; each writes the block's interior nodes and reads the
// one-cell buffer (filled by iblgf_buffer_exchange beforehand, as the
// reference's level wrappers call buffer_exchange first). Vector fields are
// three component fields.
#include "ctx.hpp"

namespace iblgf_b200
{
namespace
{
struct OpArgs
{
    const double* in[6];
    double* out[3];
    const int* list;
    const double* dx;      // per listed block: dx_level
    double scale;
};

template<int NB, int OP>
__global__ void __launch_bounds__(256) op_kernel(OpArgs a)
{
    constexpr int N3 = NB * NB * NB;
    constexpr int SY = NB, SZ = NB * NB;
    const int o = a.list[blockIdx.x];
    const double dx = a.dx[blockIdx.x];
    const double fac = 1.0 / dx;
    const size_t base = (size_t)o * N3;
    for (int i = threadIdx.x; i < N3; i += blockDim.x)
    {
        const int x = i % NB, y = (i / NB) % NB, z = i / SZ;
        if (x == 0 || y == 0 || z == 0 || x == NB - 1 || y == NB - 1 || z == NB - 1) continue;
        const size_t p = base + i;
        auto F = [&](int c, int off) { return a.in[c][p + off]; };
        if (OP == 0)
        {
            const double v = -6.0 * F(0, 0) + F(0, -SZ) + F(0, SZ) + F(0, -SY) + F(0, SY) + F(0, -1) + F(0, 1);
            a.out[0][p] = v * (1.0 / (dx * dx));
        }
        else if (OP == 1)
        {
            const double s = F(0, 0);
            a.out[0][p] = fac * (s - F(0, -1));
            a.out[1][p] = fac * (s - F(0, -SY));
            a.out[2][p] = fac * (s - F(0, -SZ));
        }
        else if (OP == 2)
        {
            const double v = -F(0, 0) - F(1, 0) - F(2, 0) + F(0, 1) + F(1, SY) + F(2, SZ);
            a.out[0][p] = v * fac;
        }
        else if (OP == 3)
        {
            a.out[0][p] = fac * (F(2, 0) - F(2, -SY) - F(1, 0) + F(1, -SZ));
            a.out[1][p] = fac * (F(0, 0) - F(0, -SZ) - F(2, 0) + F(2, -1));
            a.out[2][p] = fac * (F(1, 0) - F(1, -1) - F(0, 0) + F(0, -SY));
        }
        else if (OP == 4)
        {
            const double f = fac * a.scale;
            a.out[0][p] = f * (F(1, 0) - F(1, SZ) + F(2, SY) - F(2, 0));
            a.out[1][p] = f * (F(2, 0) - F(2, 1) + F(0, SZ) - F(0, 0));
            a.out[2][p] = f * (F(0, 0) - F(0, SY) + F(1, 1) - F(1, 0));
        }
        else
        {
            // in[0..2] face u, in[3..5] edge omega
            a.out[0][p] = 0.25 * (F(4, 0) * (F(2, 0) + F(2, -1)) + F(4, SZ) * (F(2, SZ) + F(2, SZ - 1)) -
                                  F(5, 0) * (F(1, 0) + F(1, -1)) - F(5, SY) * (F(1, SY) + F(1, SY - 1)));
            a.out[1][p] = 0.25 * (F(5, 0) * (F(0, 0) + F(0, -SY)) + F(5, 1) * (F(0, 1) + F(0, 1 - SY)) -
                                  F(3, 0) * (F(2, 0) + F(2, -SY)) - F(3, SZ) * (F(2, SZ) + F(2, SZ - SY)));
            a.out[2][p] = 0.25 * (F(3, 0) * (F(1, 0) + F(1, -SZ)) + F(3, SY) * (F(1, SY) + F(1, SY - SZ)) -
                                  F(4, 0) * (F(0, 0) + F(0, -SZ)) - F(4, 1) * (F(0, 1) + F(0, 1 - SZ)));
        }
    }
}

template<int NB>
void launch_nb(Ctx& c, int op, const OpArgs& a, int n)
{
    switch (op)
    {
        case 0: op_kernel<NB, 0><<<n, 256, 0, c.stream>>>(a); break;
        case 1: op_kernel<NB, 1><<<n, 256, 0, c.stream>>>(a); break;
        case 2: op_kernel<NB, 2><<<n, 256, 0, c.stream>>>(a); break;
        case 3: op_kernel<NB, 3><<<n, 256, 0, c.stream>>>(a); break;
        case 4: op_kernel<NB, 4><<<n, 256, 0, c.stream>>>(a); break;
        default: op_kernel<NB, 5><<<n, 256, 0, c.stream>>>(a); break;
    }
}
}  // namespace

void launch_op(Ctx& c, int op, const double* const* in, int n_in, double* const* out, int n_out, const int* list,
               const double* dx, int n, double scale)
{
    if (!n) return;
    OpArgs a{};
    for (int i = 0; i < n_in && i < 6; ++i) a.in[i] = in[i];
    for (int i = 0; i < n_out && i < 3; ++i) a.out[i] = out[i];
    a.list = list;
    a.dx = dx;
    a.scale = scale;
    switch (c.Nb)
    {
        case 6: launch_nb<6>(c, op, a, n); break;
        case 8: launch_nb<8>(c, op, a, n); break;
        case 10: launch_nb<10>(c, op, a, n); break;
        case 12: launch_nb<12>(c, op, a, n); break;
        case 16: launch_nb<16>(c, op, a, n); break;
        case 18: launch_nb<18>(c, op, a, n); break;
        default: throw Error(IBLGF_EINVAL, "unsupported block size");
    }
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

}  // namespace iblgf_b200
