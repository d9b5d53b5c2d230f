// ORACLE (test infrastructure): Morton keys, pointer octree and domain
// construction, restating
//   include/iblgf/domain/octree/key.hpp:64-275,447-457 (keys, split bits),
//   include/iblgf/domain/octree/bitmasks.hpp (Dim 3 masks),
//   include/iblgf/domain/octree/tree.hpp:385-453 (refine), :336-383 (try_2to1),
//     :571-603 (neighbour / influence lists), :765-824 (level and leaf maps),
//   include/iblgf/domain/octree/iterators.hpp:265-282 (depth-first order),
//   include/iblgf/domain/domain.hpp:107-212,405-488 (base mesh),
//     :617-736 (mark_correction), :878-939 (init_refine), :1092-1106 (refine).
// Single process: every octant is "locally owned".
#include <algorithm>
#include <functional>
#include <set>
#include <cmath>
#include <stack>
#include <stdexcept>

#include "orc.hpp"

namespace orc
{
namespace
{
u64 split3(u64 w)
{
    w &= 0x00000000001fffffull;
    w = (w | w << 32) & 0x001f00000000ffffull;
    w = (w | w << 16) & 0x001f0000ff0000ffull;
    w = (w | w << 8) & 0x010f00f00f00f00full;
    w = (w | w << 4) & 0x10c30c30c30c30c3ull;
    w = (w | w << 2) & 0x1249249249249249ull;
    return w;
}
int compress3(u64 w)
{
    w &= 0x1249249249249249ull;
    w = (w ^ (w >> 2)) & 0x30c30c30c30c30c3ull;
    w = (w ^ (w >> 4)) & 0xf00f00f00f00f00full;
    w = (w ^ (w >> 8)) & 0x00ff0000ff0000ffull;
    w = (w ^ (w >> 16)) & 0x00ff00000000ffffull;
    w = (w ^ (w >> 32)) & 0x00000000001fffffull;
    return (int)w;
}
constexpr int kShiftToCoord = 7;  // 5 level bits + 2 flag bits
u64 coord_mask_arr(int i)
{
    if (i <= 0) return 0ull;
    return ((1ull << (3 * i)) - 1ull) << (64 - 3 * i);
}
u64 level_coord_mask_arr(int i) { return 7ull << (64 - 3 * i); }
const u64 kCoordMask = ~0ull << kShiftToCoord;
}  // namespace

u64 key_make(int x, int y, int z, int level)
{
    u64 idx = split3((u64)(long long)x);
    idx |= split3((u64)(long long)y) << 1;
    idx |= split3((u64)(long long)z) << 2;
    idx <<= kShiftToCoord;
    idx <<= (kMaxLevel - level) * 3;
    idx |= (u64)level << 2;
    idx |= 1ull;
    return idx;
}
int key_level(u64 k) { return (int)((k & 0x7Cull) >> 2); }
std::array<int, 3> key_coord(u64 k)
{
    const int l = key_level(k);
    std::array<int, 3> c{};
    for (int d = 0; d < 3; ++d) c[d] = compress3(k >> (d + kShiftToCoord + (kMaxLevel - l) * 3));
    return c;
}
u64 key_parent(u64 k)
{
    const int l = key_level(k);
    if (l == 0) return k;
    return ((coord_mask_arr(l - 1) & k) | ((u64)(l - 1) << 2)) + 1ull;
}
u64 key_child(u64 k, int i)
{
    const int l = key_level(k);
    if (l == kMaxLevel) return k;
    return ((coord_mask_arr(l) & k) | ((u64)i << ((kMaxLevel - (l + 1)) * 3 + kShiftToCoord)) |
            ((u64)(l + 1) << 2)) +
           1ull;
}
int key_child_number(u64 k, int level)
{
    if (level == 0) return -1;
    return (int)((level_coord_mask_arr(level) & k) >> (kShiftToCoord + 3 * (kMaxLevel - level)));
}
bool key_is_end(u64 k)
{
    const int l = key_level(k);
    const u64 end = ((((u64)l << 2) | 1ull) | kCoordMask) + 1ull;
    return k >= end;
}
u64 key_neighbor(u64 k, int dx, int dy, int dz)
{
    auto c = key_coord(k);
    return key_make(c[0] + dx, c[1] + dy, c[2] + dz, key_level(k));
}
std::vector<u64> key_neighbor_keys(u64 k)
{
    std::vector<u64> r;
    r.reserve(27);
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) r.push_back(key_neighbor(k, dx, dy, dz));
    return r;
}
std::vector<u64> key_infl_keys(u64 k)
{
    std::vector<u64> r;
    if (key_level(k) == 0) return r;
    const u64 p = key_parent(k);
    const auto c = key_coord(k);
    for (u64 pn : key_neighbor_keys(p))
    {
        if (key_is_end(pn)) continue;
        for (int id = 0; id < 8; ++id)
        {
            const u64 ck = key_child(pn, id);
            const auto cc = key_coord(ck);
            if (std::abs(cc[0] - c[0]) > 1 || std::abs(cc[1] - c[1]) > 1 ||
                std::abs(cc[2] - c[2]) > 1)
                r.push_back(ck);
        }
    }
    return r;
}

// ------------------------------------------------------------------ Domain
Octant* Domain::find(u64 k) const
{
    Octant* n = root.get();
    const int l = key_level(k);
    for (int i = 1; i <= l; ++i)
    {
        Octant* c = n->child[key_child_number(k, i)].get();
        if (!c) return nullptr;
        n = c;
    }
    return n;
}

Octant* Domain::refine_child(Octant* o, int i)
{
    if (!o->child[i])
    {
        o->child[i] = std::make_unique<Octant>();
        o->child[i]->key = key_child(o->key, i);
        o->child[i]->level = o->level + 1;
        o->child[i]->parent = o;
    }
    return o->child[i].get();
}

Octant* Domain::insert(u64 k)
{
    Octant* n = root.get();
    const int l = key_level(k);
    for (int i = 1; i <= l; ++i) n = refine_child(n, key_child_number(k, i));
    if (l + 1 > depth) depth = l + 1;
    return n;
}

void Domain::alloc(Octant* o, int data_level)
{
    // octant_to_level_coordinate: (coord + base * 2^level) * block_extent
    const auto c = key_coord(o->key);
    const int s = 1 << std::max(data_level, 0);
    for (int d = 0; d < 3; ++d) o->bbase[d] = (c[d] + base_shift[d] * s) * e;
    o->data_level = data_level;
    o->has_data = true;
}

namespace
{
// Depth-first traversal with the reference iterator's semantics: a node's
// children are pushed when the node becomes current.
template<class F>
void dfs(Octant* root, F&& f)
{
    std::stack<Octant*> st;
    st.push(root);
    while (!st.empty())
    {
        Octant* cur = st.top();
        st.pop();
        for (int i = 7; i >= 0; --i)
            if (cur->child[i]) st.push(cur->child[i].get());
        if (cur->level == 0) continue;
        f(cur);
    }
}
}  // namespace

void Domain::construct_level_maps()
{
    level_maps.assign(kMaxLevel, {});
    // the root is visited first by the reference iterator
    if (root->has_data) level_maps[0][root->key] = root.get();
    dfs(root.get(), [&](Octant* o) {
        if (o->has_data) level_maps[o->level][o->key] = o;
    });
}

void Domain::construct_leaf_flags_from_search()
{
    auto f = [](Octant* o) {
        if (!o->has_data) return;
        bool leaf = true;
        for (auto& c : o->child)
            if (c) leaf = false;
        o->leaf = leaf;
    };
    f(root.get());
    dfs(root.get(), f);
}

void Domain::construct_lists()
{
    auto build = [&](Octant* o) {
        if (!o->has_data) return;
        const auto nk = key_neighbor_keys(o->key);
        for (int i = 0; i < 27; ++i)
        {
            Octant* n = find(nk[i]);
            o->neighbor[i] = (n && n->has_data) ? n : nullptr;
        }
        o->n_infl = 0;
        o->influence.fill(nullptr);
        if (!o->parent) return;
        for (u64 ik : key_infl_keys(o->key))
        {
            Octant* n = find(ik);
            if (n && n->has_data)
            {
                if (o->n_infl >= 189) throw std::runtime_error("influence list overflow");
                o->influence[o->n_infl++] = n;
            }
        }
    };
    build(root.get());
    dfs(root.get(), build);
}

std::vector<u64> Domain::unfound_neighbors(Octant* o, bool correction_as_neighbors)
{
    std::vector<u64> keys;
    for (u64 nk : key_neighbor_keys(o->key))
    {
        if (key_is_end(nk)) continue;
        if (nk == o->key) continue;
        Octant* n = find(nk);
        if (!n || !n->has_data) keys.push_back(nk);
        else if (!correction_as_neighbors && n->correction)
            keys.push_back(nk);
    }
    return keys;
}

bool Domain::try_2to1(u64 k, std::map<u64, bool>& checklist)
{
    auto it = checklist.find(k);
    if (it != checklist.end()) return it->second;
    const int rf = key_level(k) - base_level;
    if (rf == 0)
    {
        for (u64 nk : key_neighbor_keys(k))
        {
            if (nk == k) continue;
            auto c = key_coord(nk);
            for (int d = 0; d < 3; ++d)
            {
                if (c[d] < 0 || c[d] > key_bd_extent[d] - 1)
                {
                    checklist.emplace(k, false);
                    return false;
                }
            }
        }
        checklist.emplace(k, true);
        return true;
    }
    else if (rf > 0)
    {
        for (u64 nk : key_neighbor_keys(k))
        {
            if (nk == k) continue;
            if (!try_2to1(key_parent(nk), checklist))
            {
                checklist.emplace(k, false);
                return false;
            }
        }
        checklist.emplace(k, true);
        return true;
    }
    return false;
}

void Domain::refine(Octant* l, bool ratio_2to1)
{
    auto f = [&](Octant* o) { alloc(o, o->level - base_level); };
    if (ratio_2to1)
    {
        for (int i = 0; i < 27; ++i)
            if (l->neighbor[i] && l->neighbor[i]->has_data) l->neighbor[i]->aim_deletion = false;
        if (refinement_level(l) >= 0)
        {
            for (u64 k : unfound_neighbors(l, false))
            {
                if (key_is_end(k)) continue;
                if (refinement_level(l) == 0)
                {
                    Octant* oct = insert(k);
                    if (!oct->has_data) f(oct);
                    oct->leaf = true;
                    oct->correction = false;
                    oct->aim_deletion = false;
                }
                else
                {
                    const u64 pk = key_parent(k);
                    Octant* pa = find(pk);
                    if (!pa)
                    {
                        pa = insert(pk);
                        f(pa);
                    }
                    refine(pa, ratio_2to1);
                }
            }
        }
    }
    for (int i = 0; i < 8; ++i)
    {
        if (l->child[i] && l->child[i]->has_data) continue;
        Octant* c = refine_child(l, i);
        if (!c->has_data) f(c);
    }
    for (int i = 0; i < 8; ++i)
    {
        Octant* c = l->child[i].get();
        c->leaf = true;
        c->correction = false;
        c->aim_deletion = false;
    }
    l->leaf = false;
    l->correction = false;
    l->aim_deletion = false;
    if (l->level + 2 > depth) depth = l->level + 2;
}

void Domain::init_refine(int nRef, int level_up_max, RefinePred pred, void* user)
{
    construct_leaf_flags_from_search();
    std::map<u64, bool> checklist;
    for (int l = 0; l < nRef; ++l)
    {
        std::vector<Octant*> dummy;
        // iterate with the reference's depth-first semantics while refining
        std::stack<Octant*> st;
        st.push(root.get());
        while (!st.empty())
        {
            Octant* cur = st.top();
            st.pop();
            for (int i = 7; i >= 0; --i)
                if (cur->child[i]) st.push(cur->child[i].get());
            if (cur->level == 0) continue;
            if (refinement_level(cur) != l) continue;
            int ext[3] = {e, e, e};
            if (pred && pred(user, cur->bbase, ext, refinement_level(cur), nRef - l))
            {
                if (try_2to1(cur->key, checklist)) refine(cur, true);
            }
        }
    }
    construct_level_maps();
    for (int g = 0; g < level_up_max; ++g)
    {
        for (int l = depth - 1; l >= base_level; --l)
        {
            std::vector<Octant*> lv;
            for (auto& kv : level_maps[l]) lv.push_back(kv.second);
            for (Octant* o : lv)
                if (o->leaf) refine(o, false);
        }
        construct_level_maps();
        construct_lists();
    }
    mark_correction();
}

void Domain::mark_correction()
{
    // physical flags, finest level first
    auto clear_phys = [](Octant* o) { o->physical = false; };
    clear_phys(root.get());
    dfs(root.get(), clear_phys);
    construct_level_maps();
    for (int l = depth - 1; l >= base_level; --l)
    {
        for (auto& kv : level_maps[l])
        {
            Octant* o = kv.second;
            o->physical = o->leaf && !o->aim_deletion;
            if (!o->physical)
                for (auto& c : o->child)
                    if (c && c->has_data) o->physical = o->physical || c->physical;
        }
    }
    // correction buffers around physical octants of refined levels
    for (int l = base_level + 1; l < depth; ++l)
    {
        std::vector<Octant*> lv;
        for (auto& kv : level_maps[l]) lv.push_back(kv.second);
        for (Octant* o : lv)
        {
            if (!o->physical) continue;
            for (u64 k : unfound_neighbors(o, true))
            {
                Octant* n = insert(k);
                if (!n->has_data) alloc(n, n->level - base_level);
            }
        }
    }
    construct_lists();
    construct_level_maps();
    for (int l = base_level + 1; l < depth; ++l)
    {
        for (auto& kv : level_maps[l])
        {
            Octant* o = kv.second;
            if (!o->physical) continue;
            for (int i = 0; i < 27; ++i)
            {
                Octant* n = o->neighbor[i];
                if (!n || !n->has_data || n->physical) continue;
                n->aim_deletion = false;
                n->correction = true;
            }
        }
    }
    construct_level_maps();
    construct_lists();
    for (auto& kv : level_maps[base_level])
    {
        Octant* o = kv.second;
        if (!o->physical) continue;
        bool all = true;
        for (int i = 0; i < 27; ++i)
            if (!o->neighbor[i] || !o->neighbor[i]->has_data) all = false;
        if (!all)
        {
            o->correction = true;
            o->aim_deletion = false;
            o->leaf = true;
        }
        else
        {
            o->correction = false;
            o->aim_deletion = false;
        }
    }
    construct_level_maps();
    construct_lists();
}

bool Domain::leaf_search(const Octant* o, bool require_data) const
{
    for (auto& c : o->child)
        if (c && (!require_data || c->has_data)) return false;
    return true;
}

// octree/tree.hpp:455-466: data dropped; an octant without children leaves
// its parent (and is freed)
void Domain::delete_oct(Octant* o)
{
    o->has_data = false;
    o->leaf = o->correction = false;
    o->idx = -1;
    if (leaf_search(o, false) && o->parent)
    {
        Octant* p = o->parent;
        for (auto& c : p->child)
            if (c.get() == o) c.reset();
    }
}

// Decomposition::adapt_decoposition, server part (domain/decomposition/
// decomposition.hpp:182-470) for one client; Tree::deletionReset_2to1
// (octree/tree.hpp:304-327); Domain::delete_all_children (domain.hpp:512-569);
// baseBlockBufferNumber_ = 2 (domain.hpp:1336)
std::vector<Octant*> Domain::adapt(const std::vector<std::pair<u64, int>>& attempts, bool& base_mesh_update)
{
    base_mesh_update = false;
    auto all_octants = [&]() {
        std::vector<Octant*> v{root.get()};
        dfs(root.get(), [&](Octant* o) { v.push_back(o); });
        return v;
    };
    auto ordered = [](std::vector<Octant*> v) {
        std::sort(v.begin(), v.end(), [](const Octant* a, const Octant* b) {
            return a->level != b->level ? a->level < b->level : a->key < b->key;
        });
        return v;
    };
    auto leaves = [&]() {
        std::vector<Octant*> v;
        for (Octant* o : all_octants())
            if (o->has_data && o->leaf) v.push_back(o);
        return ordered(v);
    };
    auto at_level = [&](int l) {
        std::vector<Octant*> v;
        for (Octant* o : all_octants())
            if (o->has_data && o->level == l) v.push_back(o);
        return ordered(v);
    };
    std::set<u64> old_leaves;
    for (Octant* o : all_octants())
    {
        if (o->has_data && o->leaf) old_leaves.insert(o->key);
        o->aim_deletion = o->correction && !o->ib;
        // time_march (ifherk.hpp:247-258): old_correction = correction on the base level
        o->old_correction = o->has_data && o->level == base_level && o->correction;
    }
    std::map<Octant*, int> change;
    for (auto& a : attempts)
    {
        if (!a.second) continue;
        Octant* o = find(a.first);
        if (!o || !o->has_data) throw std::runtime_error("oracle: adaptation attempt for an octant without data");
        change[o] = a.second;
    }
    std::map<u64, bool> checklist;
    std::vector<Octant*> to_refine;
    for (Octant* o : leaves())
    {
        auto it = change.find(o);
        if (it == change.end()) continue;
        if (it->second < 0) o->aim_deletion = true;
        else if (o->ib || try_2to1(o->key, checklist))
            to_refine.push_back(o);
    }
    for (Octant* o : leaves())
        if (o->ib || o->ext_ib) o->aim_deletion = false;
    // base blocks within two blocks of every kept base block
    std::set<u64> away;
    for (Octant* o : at_level(base_level))
    {
        if (o->aim_deletion || o->correction) continue;
        const auto c = key_coord(o->key);
        for (int dz = -2; dz <= 2; ++dz)
            for (int dy = -2; dy <= 2; ++dy)
                for (int dx = -2; dx <= 2; ++dx)
                {
                    const int x = c[0] + dx, y = c[1] + dy, z = c[2] + dz;
                    const int lim = 1 << o->level;
                    if (x < 0 || y < 0 || z < 0 || x >= lim || y >= lim || z >= lim) continue;
                    away.insert(key_make(x, y, z, o->level));
                }
    }
    for (u64 nk : away)
    {
        const auto c = key_coord(nk);
        bool inside = true;
        for (int d = 0; d < 3; ++d)
            if (c[d] < 0 || c[d] > key_bd_extent[d] - 1) inside = false;
        if (!inside) continue;
        Octant* n = find(nk);
        if (!n || !n->has_data)
        {
            n = insert(nk);
            alloc(n, n->level - base_level);
            n->leaf = true;
            n->correction = false;
            base_mesh_update = true;
        }
        n->aim_deletion = false;
    }
    construct_level_maps();
    for (Octant* o : to_refine)
        if (o->leaf) refine(o, true);
    // deletionReset_2to1 from the parents of refined leaves
    std::set<Octant*> done;
    std::function<void(Octant*)> reset = [&](Octant* l) {
        if (done.count(l)) return;
        if (l->level - base_level < 0) return;
        for (u64 nk : key_neighbor_keys(l->key))
        {
            if (key_is_end(nk)) continue;
            Octant* n = find(nk);
            if (!n || !n->has_data) continue;
            n->aim_deletion = false;
            reset(n->parent);
        }
        done.insert(l);
    };
    for (Octant* o : leaves())
        if (o->level - base_level > 0) reset(o->parent);
    for (Octant* o : at_level(base_level))
        if (o->aim_deletion && o->leaf) delete_oct(o);
    construct_level_maps();
    // sibling groups whose children all go: the parent becomes the leaf
    for (int l = depth - 2; l >= base_level; --l)
        for (Octant* o : at_level(l))
        {
            if (leaf_search(o, true)) continue;
            bool all = true;
            for (auto& c : o->child)
            {
                if (!c || !c->has_data) continue;
                if (!c->aim_deletion || (!c->leaf && !c->correction))
                {
                    all = false;
                    break;
                }
            }
            for (auto& c : o->child)
            {
                if (!c) continue;
                if (all)
                {
                    c->leaf = c->correction = false;
                    c->aim_deletion = true;
                }
                else
                    c->aim_deletion = false;
            }
            if (all)
            {
                o->leaf = true;
                o->correction = false;
                o->aim_deletion = false;
            }
        }
    construct_level_maps();
    mark_correction();
    for (Octant* o : all_octants())
        if (o->has_data && o->aim_deletion && o->level - base_level > 0) delete_oct(o);
    for (int l = base_level - 1; l > 0; --l)
        for (Octant* o : all_octants())
            if (o->level == l && leaf_search(o, false)) delete_oct(o);
    // ancestors of new octants get data
    for (Octant* o : all_octants())
    {
        if (!o->has_data || o->idx >= 0) continue;
        for (Octant* p = o->parent; p && !p->has_data; p = p->parent) alloc(p, p->level - base_level);
    }
    depth = 0;
    for (Octant* o : all_octants())
        if (o->has_data) depth = std::max(depth, o->level + 1);
    construct_level_maps();
    construct_lists();
    std::vector<Octant*> parents;
    for (Octant* o : leaves())
        if (o->level - base_level > 0 && !old_leaves.count(o->key)) parents.push_back(o->parent);
    parents = ordered(parents);
    parents.erase(std::unique(parents.begin(), parents.end()), parents.end());
    return parents;
}

void Domain::finalize()
{
    octs.clear();
    for (int l = 0; l < (int)level_maps.size(); ++l)
        for (auto& kv : level_maps[l]) octs.push_back(kv.second);
    for (int i = 0; i < (int)octs.size(); ++i) octs[i]->idx = i;
}

std::unique_ptr<Domain> domain_create(const int* bd_base, const int* bd_extent,
    int block_extent, double dx_base, int n_blocks, const int* block_base,
    const int* block_ext)
{
    auto d = std::make_unique<Domain>();
    d->e = block_extent;
    d->Nb = block_extent + 2;
    d->dx_base = dx_base;
    for (int i = 0; i < 3; ++i)
    {
        d->bd_base[i] = bd_base[i];
        d->bd_extent[i] = bd_extent[i];
        d->base_shift[i] = bd_base[i] / block_extent;
        d->key_bd_extent[i] = bd_extent[i] / block_extent;
    }
    // construct_basemesh_blocks: divide each configured block into e^3 blocks
    std::vector<std::array<int, 3>> bases;
    for (int b = 0; b < n_blocks; ++b)
    {
        for (int i = 0; i < 3; ++i)
        {
            if (block_ext[3 * b + i] % block_extent)
                throw std::runtime_error("Domain: Extent of blocks are not evenly divisible");
            if (std::abs(block_base[3 * b + i]) % block_extent)
                throw std::runtime_error("Domain: Base of blocks are not evenly divisible");
        }
        const int nx = block_ext[3 * b] / block_extent, ny = block_ext[3 * b + 1] / block_extent,
                  nz = block_ext[3 * b + 2] / block_extent;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                    bases.push_back({block_base[3 * b] / block_extent + i,
                                     block_base[3 * b + 1] / block_extent + j,
                                     block_base[3 * b + 2] / block_extent + k});
    }
    // construct_tree
    int mx = 0;
    for (int i = 0; i < 3; ++i) mx = std::max(mx, d->key_bd_extent[i]);
    int bl = 0;
    while (mx >= (1 << bl)) ++bl;
    d->base_level = bl;
    d->depth = bl + 1;
    d->root = std::make_unique<Octant>();
    d->root->key = key_make(0, 0, 0, 0);
    d->root->level = 0;
    for (auto& b : bases)
        d->insert(key_make(b[0] - d->base_shift[0], b[1] - d->base_shift[1],
                           b[2] - d->base_shift[2], bl));
    // every octant of the initial tree gets a block at level 0
    d->alloc(d->root.get(), 0);
    dfs(d->root.get(), [&](Octant* o) { d->alloc(o, 0); });
    d->construct_level_maps();
    d->construct_lists();
    return d;
}

}  // namespace orc
