// Neighbour and influence lists built on the device, bit-identical to
// Tree::neighbor_list_build / influence_list_build
// (include/iblgf/domain/octree/tree.hpp:571-603) with Key::get_neighbor_keys /
// get_infl_keys (key.hpp:200-250): 27 neighbours z-slowest, self at 13;
// influence = children of the parent's 27 neighbours that are not adjacent,
// in (parent-neighbour, child id) order, compacted over octants that exist.
// Lookup is a binary search in the sorted key array of all octants that hold
// data (an octant without data counts as absent, as in the reference).
#include "ctx.hpp"

namespace iblgf_b200
{
namespace
{
__device__ int find_key(const u64* __restrict__ keys, const int* __restrict__ idx, int n, u64 k)
{
    int lo = 0, hi = n - 1;
    while (lo <= hi)
    {
        const int mid = (lo + hi) >> 1;
        const u64 v = keys[mid];
        if (v == k) return idx[mid];
        if (v < k) lo = mid + 1;
        else hi = mid - 1;
    }
    return -1;
}

__global__ void build_lists_kernel(const u64* __restrict__ skeys, const int* __restrict__ sidx, int ns,
                                   const u64* __restrict__ keys, int n, int* __restrict__ nbr,
                                   int* __restrict__ infl, int* __restrict__ ninfl)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const u64 k = keys[o];
    int m = 0;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
                nbr[27 * o + (m++)] = find_key(skeys, sidx, ns, key_neighbor(k, dx, dy, dz));
    int cnt = 0;
    const int lvl = key_level(k);
    if (lvl > 0)
    {
        int c[3];
        key_coord(k, c);
        const u64 pk = key_parent(k);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                {
                    const u64 pn = key_neighbor(pk, dx, dy, dz);
                    if (key_is_end(pn)) continue;
                    for (int id = 0; id < 8; ++id)
                    {
                        const u64 ck = key_child(pn, id);
                        int cc[3];
                        key_coord(ck, cc);
                        if (abs(cc[0] - c[0]) > 1 || abs(cc[1] - c[1]) > 1 || abs(cc[2] - c[2]) > 1)
                        {
                            const int f = find_key(skeys, sidx, ns, ck);
                            if (f >= 0 && cnt < 189) infl[189 * o + (cnt++)] = f;
                        }
                    }
                }
    }
    for (int j = cnt; j < 189; ++j) infl[189 * o + j] = -1;
    ninfl[o] = cnt;
}
}  // namespace

void launch_build_lists(Ctx& c, const u64* d_sorted_keys, const int* d_sorted_idx, int n_sorted,
                        const u64* d_keys, int n, int* d_nbr, int* d_infl, int* d_ninfl)
{
    if (!n) return;
    build_lists_kernel<<<(n + 127) / 128, 128, 0, c.stream>>>(d_sorted_keys, d_sorted_idx, n_sorted, d_keys, n,
                                                              d_nbr, d_infl, d_ninfl);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

}  // namespace iblgf_b200
