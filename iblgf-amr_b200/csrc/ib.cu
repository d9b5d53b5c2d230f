// Immersed-boundary transfer kernels (FP64):
//   ib_projection_kernel  Operator::ib_projection (operators.hpp:841-861):
//                         one thread per (point, component) sums u_c(node) *
//                         delta over the point's influence nodes in list order
//   ib_smearing_kernel    Operator::ib_smearing (operators.hpp:996-1013) as a
//                         gather: one thread per (node, component) adds
//                         f_c(point) * delta over the points that reach the
//                         node, in point order (deterministic, no atomics)
//   face_planes_kernel    clean_ib_region_boundary / Operator::
//                         clean_leaf_correction_boundary (operators.hpp:73-170,
//                         329-517): zero the outer planes of listed faces
// The delta weights (yang3 x yang3 x yang3 at the component's face offset)
// are computed once on the host when the points are set.
#include "ctx.hpp"

namespace iblgf_b200
{
namespace
{
// entries e in [ptr[i], ptr[i+1]) of point i: field offset at[e], weight w[3e + c]
__global__ void ib_projection_kernel(const double* __restrict__ u0, const double* __restrict__ u1,
                                     const double* __restrict__ u2, const int* __restrict__ ptr,
                                     const long long* __restrict__ at, const double* __restrict__ w, int n,
                                     double* __restrict__ f)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * n) return;
    const int i = t / 3, c = t % 3;
    const double* u = c == 0 ? u0 : (c == 1 ? u1 : u2);
    double s = 0.0;
    for (int e = ptr[i]; e < ptr[i + 1]; ++e) s += u[at[e]] * w[3 * e + c];
    f[3 * i + c] = s;
}

// nodes k: field offset node_at[k]; entries [nptr[k], nptr[k+1]) of node k
// give (point nidx[j], entry weight row nw[j]) in increasing point order
__global__ void ib_smearing_kernel(double* __restrict__ u0, double* __restrict__ u1, double* __restrict__ u2,
                                   const long long* __restrict__ node_at, const int* __restrict__ nptr,
                                   const int* __restrict__ npt, const int* __restrict__ nent,
                                   const double* __restrict__ w, int n_nodes, const double* __restrict__ f)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * n_nodes) return;
    const int k = t / 3, c = t % 3;
    double* u = c == 0 ? u0 : (c == 1 ? u1 : u2);
    double v = u[node_at[k]];
    for (int j = nptr[k]; j < nptr[k + 1]; ++j) v += f[3 * npt[j] + c] * w[3 * nent[j] + c];
    u[node_at[k]] = v;
}

// list[b]: octant, faces[b]: bit q set = zero the planes towards face q
// (q: 0 z-, 1 y-, 2 x-, 3 x+, 4 y+, 5 z+)
template<int NB>
__global__ void face_planes_kernel(double* __restrict__ f, const int* __restrict__ list,
                                   const unsigned char* __restrict__ faces, int width)
{
    constexpr int N3 = NB * NB * NB;
    double* b = f + (size_t)list[blockIdx.x] * N3;
    const unsigned m = faces[blockIdx.x];
    for (int i = threadIdx.x; i < N3; i += blockDim.x)
    {
        const int x = i % NB, y = (i / NB) % NB, z = i / (NB * NB);
        const bool zero = ((m & 1) && z < width) || ((m & 2) && y < width) || ((m & 4) && x < width) ||
                          ((m & 8) && x >= NB - width) || ((m & 16) && y >= NB - width) ||
                          ((m & 32) && z >= NB - width);
        if (zero) b[i] = 0.0;
    }
}
}  // namespace

void launch_ib_projection(Ctx& c, const double* const* u, const int* ptr, const long long* at, const double* w,
                          int n, double* f)
{
    if (!n) return;
    ib_projection_kernel<<<(3 * n + 127) / 128, 128, 0, c.stream>>>(u[0], u[1], u[2], ptr, at, w, n, f);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_ib_smearing(Ctx& c, double* const* u, const long long* node_at, const int* nptr, const int* npt,
                        const int* nent, const double* w, int n_nodes, const double* f)
{
    if (!n_nodes) return;
    ib_smearing_kernel<<<(3 * n_nodes + 127) / 128, 128, 0, c.stream>>>(u[0], u[1], u[2], node_at, nptr, npt, nent,
                                                                         w, n_nodes, f);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_face_planes(Ctx& c, double* f, const int* list, const unsigned char* faces, int n, int width)
{
    if (!n) return;
    switch (c.Nb)
    {
        case 6: face_planes_kernel<6><<<n, 256, 0, c.stream>>>(f, list, faces, width); break;
        case 8: face_planes_kernel<8><<<n, 256, 0, c.stream>>>(f, list, faces, width); break;
        case 10: face_planes_kernel<10><<<n, 256, 0, c.stream>>>(f, list, faces, width); break;
        case 12: face_planes_kernel<12><<<n, 256, 0, c.stream>>>(f, list, faces, width); break;
        case 16: face_planes_kernel<16><<<n, 256, 0, c.stream>>>(f, list, faces, width); break;
        case 18: face_planes_kernel<18><<<n, 256, 0, c.stream>>>(f, list, faces, width); break;
        default: throw Error(IBLGF_EINVAL, "unsupported block size");
    }
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

}  // namespace iblgf_b200
