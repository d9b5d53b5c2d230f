// Morton keys of the reference octree (include/iblgf/domain/octree/key.hpp,
// bitmasks.hpp, Dim = 3): 57 coordinate bits interleaved x,y,z from bit 63
// down, 5 level bits at [2,7), flag bit 0 set. max_level 19. Coordinates wrap
// modulo 2^level exactly as the reference's unsigned arithmetic does, so keys
// of out-of-range neighbours alias in-range ones the same way.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define IBLGF_HD __host__ __device__ __forceinline__
#else
#define IBLGF_HD inline
#endif

namespace iblgf_b200
{
using u64 = std::uint64_t;
constexpr int kMaxLevel = 19;
constexpr int kShiftToCoord = 7;

IBLGF_HD u64 split3(u64 w)
{
    w &= 0x00000000001fffffull;
    w = (w | w << 32) & 0x001f00000000ffffull;
    w = (w | w << 16) & 0x001f0000ff0000ffull;
    w = (w | w << 8) & 0x010f00f00f00f00full;
    w = (w | w << 4) & 0x10c30c30c30c30c3ull;
    w = (w | w << 2) & 0x1249249249249249ull;
    return w;
}
IBLGF_HD int compress3(u64 w)
{
    w &= 0x1249249249249249ull;
    w = (w ^ (w >> 2)) & 0x30c30c30c30c30c3ull;
    w = (w ^ (w >> 4)) & 0xf00f00f00f00f00full;
    w = (w ^ (w >> 8)) & 0x00ff0000ff0000ffull;
    w = (w ^ (w >> 16)) & 0x00ff00000000ffffull;
    w = (w ^ (w >> 32)) & 0x00000000001fffffull;
    return (int)w;
}
IBLGF_HD u64 key_make(int x, int y, int z, int level)
{
    u64 idx = split3((u64)(long long)x) | (split3((u64)(long long)y) << 1) |
              (split3((u64)(long long)z) << 2);
    idx <<= kShiftToCoord;
    idx <<= (kMaxLevel - level) * 3;
    return idx | ((u64)level << 2) | 1ull;
}
IBLGF_HD int key_level(u64 k) { return (int)((k & 0x7Cull) >> 2); }
IBLGF_HD void key_coord(u64 k, int* c)
{
    const int sh = kShiftToCoord + (kMaxLevel - key_level(k)) * 3;
    c[0] = compress3(k >> sh);
    c[1] = compress3(k >> (sh + 1));
    c[2] = compress3(k >> (sh + 2));
}
IBLGF_HD u64 coord_mask_arr(int i) { return i <= 0 ? 0ull : (((1ull << (3 * i)) - 1ull) << (64 - 3 * i)); }
IBLGF_HD u64 key_parent(u64 k)
{
    const int l = key_level(k);
    if (l == 0) return k;
    return ((coord_mask_arr(l - 1) & k) | ((u64)(l - 1) << 2)) + 1ull;
}
IBLGF_HD u64 key_child(u64 k, int i)
{
    const int l = key_level(k);
    if (l == kMaxLevel) return k;
    return ((coord_mask_arr(l) & k) | ((u64)i << ((kMaxLevel - (l + 1)) * 3 + kShiftToCoord)) |
            ((u64)(l + 1) << 2)) + 1ull;
}
IBLGF_HD int key_child_number(u64 k, int level)
{
    if (level == 0) return -1;
    return (int)(((7ull << (64 - 3 * level)) & k) >> (kShiftToCoord + 3 * (kMaxLevel - level)));
}
IBLGF_HD bool key_is_end(u64 k)
{
    const u64 end = ((((u64)key_level(k) << 2) | 1ull) | (~0ull << kShiftToCoord)) + 1ull;
    return k >= end;
}
IBLGF_HD u64 key_neighbor(u64 k, int dx, int dy, int dz)
{
    int c[3];
    key_coord(k, c);
    return key_make(c[0] + dx, c[1] + dy, c[2] + dz, key_level(k));
}

}  // namespace iblgf_b200
