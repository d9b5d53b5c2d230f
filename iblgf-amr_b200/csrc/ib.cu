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


// ---------------------------------------------------------------------------
// Force CG of LinSysSolver::CG_solve (linsys.hpp:171-230) on the device. The
// iterates and residuals stay in device memory; the scalars (FP64 dot
// products, linsys.hpp:501-517) are reduced by one CTA in a fixed order, so a
// solve is bit-reproducible. sc: [0] rsold, [1] p.Ap, [2] rsnew, [3] f.f;
// ctl: [0] done, [1] iterations, [2] stopped at max_iter without converging.
namespace
{
constexpr int kDotThreads = 1024;

// sum over i < n of a[i] * b[i] (and of c[i] * d[i] when c is given): each
// thread sums its strided elements in order, then a fixed tree over threads
__global__ void __launch_bounds__(kDotThreads) cg_dot_kernel(const double* __restrict__ a,
                                                             const double* __restrict__ b,
                                                             const double* __restrict__ c,
                                                             const double* __restrict__ d, int n,
                                                             double* __restrict__ out0, double* __restrict__ out1,
                                                             const int* __restrict__ ctl)
{
    __shared__ double s0[kDotThreads], s1[kDotThreads];
    if (ctl && ctl[0]) return;
    double t0 = 0.0, t1 = 0.0;
    for (int i = threadIdx.x; i < n; i += kDotThreads)
    {
        t0 = fma(a[i], b[i], t0);
        if (c) t1 = fma(c[i], d[i], t1);
    }
    s0[threadIdx.x] = t0;
    s1[threadIdx.x] = t1;
    __syncthreads();
    for (int h = kDotThreads / 2; h > 0; h >>= 1)
    {
        if ((int)threadIdx.x < h)
        {
            s0[threadIdx.x] += s0[threadIdx.x + h];
            s1[threadIdx.x] += s1[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        *out0 = s0[0];
        if (c) *out1 = s1[0];
    }
}

// r = uc - Ax, p = r; the controls reset (done when max_iter <= 0)
__global__ void cg_init_kernel(const double* __restrict__ uc, const double* __restrict__ Ax, double* __restrict__ r,
                               double* __restrict__ p, int n, int* __restrict__ ctl, int max_iter)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        const double v = uc[i] - Ax[i];
        r[i] = v;
        p[i] = v;
    }
    if (i == 0)
    {
        ctl[0] = max_iter <= 0 ? 1 : 0;
        ctl[1] = 0;
        ctl[2] = 0;
    }
}

// after Ap and p.Ap: one more iteration counted; p.Ap = 0 stops the solve;
// otherwise f += a p, r -= a Ap with a = rsold / p.Ap
__global__ void cg_update_kernel(double* __restrict__ f, double* __restrict__ r, const double* __restrict__ p,
                                 const double* __restrict__ Ap, int n, const double* __restrict__ sc,
                                 int* __restrict__ ctl)
{
    if (ctl[0]) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double pAp = sc[1];
    if (pAp == 0.0) return;
    const double a = sc[0] / pAp;
    if (i < n)
    {
        f[i] = f[i] + p[i] * a;
        r[i] = r[i] + Ap[i] * -a;
    }
}

// direction update p = r + (rsnew / rsold) p unless this iteration stops
// the solve (p.Ap = 0, or sqrt(rsnew / f.f) < threshold)
__global__ void cg_direction_kernel(double* __restrict__ p, const double* __restrict__ r, int n,
                                    const double* __restrict__ sc, const int* __restrict__ ctl, double threshold)
{
    if (ctl[0]) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (sc[1] == 0.0 || sqrt(sc[2] / sc[3]) < threshold) return;
    if (i < n) p[i] = r[i] + p[i] * (sc[2] / sc[0]);
}

// the scalar side of the iteration (one thread, after the direction update
// has read rsold): iteration count, stop decision, rsold = rsnew; inside a
// graph the loop's condition is set from it
__global__ void cg_advance_kernel(double* __restrict__ sc, int* __restrict__ ctl, double threshold, int max_iter,
                                  cudaGraphConditionalHandle cond, int set_cond)
{
    if (!ctl[0])
    {
        const int it = ctl[1] + 1;
        ctl[1] = it;
        const bool stop_zero = sc[1] == 0.0;
        const bool conv = !stop_zero && sqrt(sc[2] / sc[3]) < threshold;
        if (stop_zero || conv) ctl[0] = 1;
        else
        {
            sc[0] = sc[2];
            if (it >= max_iter)
            {
                ctl[0] = 1;
                ctl[2] = 1;
            }
        }
    }
    if (set_cond) cudaGraphSetConditional(cond, ctl[0] ? 0u : 1u);
}

// per-stage record of a finished solve: [iterations, not converged]
__global__ void cg_record_kernel(const int* __restrict__ ctl, int* __restrict__ rec)
{
    rec[0] = ctl[1];
    rec[1] = ctl[2];
}
}  // namespace

void launch_cg_dot(Ctx& c, const double* a, const double* b, const double* a2, const double* b2, int n,
                   double* out0, double* out1, const int* ctl)
{
    cg_dot_kernel<<<1, kDotThreads, 0, c.stream>>>(a, b, a2, b2, n, out0, out1, ctl);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_cg_init(Ctx& c, const double* uc, const double* Ax, double* r, double* p, int n, int* ctl, int max_iter)
{
    cg_init_kernel<<<(n + 255) / 256 + (n == 0), 256, 0, c.stream>>>(uc, Ax, r, p, n, ctl, max_iter);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_cg_update(Ctx& c, double* f, double* r, const double* p, const double* Ap, int n, const double* sc,
                      int* ctl)
{
    if (!n) return;
    cg_update_kernel<<<(n + 255) / 256, 256, 0, c.stream>>>(f, r, p, Ap, n, sc, ctl);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_cg_direction(Ctx& c, double* p, const double* r, int n, const double* sc, const int* ctl,
                         double threshold)
{
    if (!n) return;
    cg_direction_kernel<<<(n + 255) / 256, 256, 0, c.stream>>>(p, r, n, sc, ctl, threshold);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_cg_advance(Ctx& c, double* sc, int* ctl, double threshold, int max_iter,
                       unsigned long long cond, bool set_cond)
{
    cg_advance_kernel<<<1, 1, 0, c.stream>>>(sc, ctl, threshold, max_iter, (cudaGraphConditionalHandle)cond,
                                             set_cond ? 1 : 0);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_cg_record(Ctx& c, const int* ctl, int* rec)
{
    cg_record_kernel<<<1, 1, 0, c.stream>>>(ctl, rec);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}


// ---------------------------------------------------------------------------
// Warm start of a stage's force CG: f0 = the stage's previous force, or its
// linear extrapolation 2 f_prev - f_prev2 once two forces are recorded
// (count >= 2); record: f_prev2 = f_prev, f_prev = f, count + 1. The count
// lives on the device so that a captured time step extrapolates exactly when
// a direct one would.
namespace
{
__global__ void ws_base_kernel(double* __restrict__ f0, const double* __restrict__ fp, const double* __restrict__ fp2,
                               int n, const int* __restrict__ count, int extrapolate)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f0[i] = (extrapolate && *count >= 2) ? 2.0 * fp[i] - fp2[i] : fp[i];
}

__global__ void ws_record_kernel(double* __restrict__ fp2, double* __restrict__ fp, const double* __restrict__ f, int n,
                                 int* __restrict__ count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        fp2[i] = fp[i];
        fp[i] = f[i];
    }
    if (i == 0) *count += 1;
}
}  // namespace

void launch_ws_base(Ctx& c, double* f0, const double* fp, const double* fp2, int n, const int* count, bool extrapolate)
{
    if (!n) return;
    ws_base_kernel<<<(n + 255) / 256, 256, 0, c.stream>>>(f0, fp, fp2, n, count, extrapolate ? 1 : 0);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_ws_record(Ctx& c, double* fp2, double* fp, const double* f, int n, int* count)
{
    if (!n) return;
    ws_record_kernel<<<(n + 255) / 256, 256, 0, c.stream>>>(fp2, fp, f, n, count);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

}  // namespace iblgf_b200
