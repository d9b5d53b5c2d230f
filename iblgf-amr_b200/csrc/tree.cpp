// Host octree construction with the reference's semantics, in an index-based
// layout (one vector of octants, children by index):
//   base mesh  include/iblgf/domain/domain.hpp:405-488, construct_tree :190-230
//   refine     include/iblgf/domain/octree/tree.hpp:385-453 (2:1 balance),
//              try_2to1 :336-383, insert/find :270-300
//   init_refine domain.hpp:878-939 — refinement candidates are visited in the
//              reference iterator's depth-first order (iterators.hpp:265-282),
//              so octants created by 2:1 balancing during a pass are visited
//              exactly when the reference would visit them
//   mark_correction domain.hpp:617-736.
// The neighbour and influence lists of the finished tree are built on the
// device (lists.cu). Only one process owns the tree, so "locally owned" is
// always true.
#include <algorithm>
#include <cmath>
#include <functional>
#include <set>
#include <stack>

#include "ctx.hpp"

namespace iblgf_b200
{
void HostTree::init(int block_extent, const int* bd_base, const int* bd_extent)
{
    e = block_extent;
    int mx = 0;
    for (int d = 0; d < 3; ++d)
    {
        base_shift[d] = bd_base[d] / block_extent;
        key_bd_extent[d] = bd_extent[d] / block_extent;
        mx = std::max(mx, key_bd_extent[d]);
    }
    base_level = 0;
    while (mx >= (1 << base_level)) ++base_level;  // Key::minimum_level
    depth = base_level + 1;
    o.clear();
    HOct root;
    root.key = key_make(0, 0, 0, 0);
    root.level = 0;
    o.push_back(root);
}

void HostTree::add_base_blocks(const std::vector<std::array<int, 3>>& nb)
{
    for (auto& b : nb)
        insert(key_make(b[0] - base_shift[0], b[1] - base_shift[1], b[2] - base_shift[2], base_level));
    // every octant of the initial tree gets a block at level 0
    for (int i : dfs_order()) alloc(i, 0);
}

int HostTree::find(u64 k) const
{
    int n = 0;
    const int l = key_level(k);
    for (int i = 1; i <= l; ++i)
    {
        n = o[n].child[key_child_number(k, i)];
        if (n < 0) return -1;
    }
    return n;
}

int HostTree::refine_child(int p, int i)
{
    if (o[p].child[i] < 0)
    {
        HOct c;
        c.key = key_child(o[p].key, i);
        c.level = o[p].level + 1;
        c.parent = p;
        o.push_back(c);
        o[p].child[i] = (int)o.size() - 1;
    }
    return o[p].child[i];
}

int HostTree::insert(u64 k)
{
    int n = 0;
    const int l = key_level(k);
    for (int i = 1; i <= l; ++i) n = refine_child(n, key_child_number(k, i));
    depth = std::max(depth, l + 1);
    return n;
}

void HostTree::alloc(int i, int data_level)
{
    int c[3];
    key_coord(o[i].key, c);
    const int s = 1 << std::max(data_level, 0);
    for (int d = 0; d < 3; ++d) o[i].bbase[d] = (c[d] + base_shift[d] * s) * e;
    o[i].has_data = true;
}

std::vector<int> HostTree::dfs_order() const
{
    std::vector<int> out;
    std::vector<int> st{0};
    out.push_back(0);
    while (!st.empty())
    {
        const int cur = st.back();
        st.pop_back();
        for (int i = 7; i >= 0; --i)
            if (o[cur].child[i] >= 0) st.push_back(o[cur].child[i]);
        if (o[cur].level == 0) continue;
        out.push_back(cur);
    }
    return out;
}

std::vector<u64> HostTree::unfound_neighbors(int i, bool correction_as_neighbors) const
{
    std::vector<u64> keys;
    const u64 k = o[i].key;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
            {
                const u64 nk = key_neighbor(k, dx, dy, dz);
                if (key_is_end(nk) || nk == k) continue;
                const int n = find(nk);
                if (n < 0 || !o[n].has_data) keys.push_back(nk);
                else if (!correction_as_neighbors && o[n].correction)
                    keys.push_back(nk);
            }
    return keys;
}

bool HostTree::try_2to1(u64 k, std::map<u64, bool>& checklist) const
{
    auto it = checklist.find(k);
    if (it != checklist.end()) return it->second;
    const int rf = key_level(k) - base_level;
    bool ok = true;
    if (rf < 0) return false;
    for (int dz = -1; dz <= 1 && ok; ++dz)
        for (int dy = -1; dy <= 1 && ok; ++dy)
            for (int dx = -1; dx <= 1 && ok; ++dx)
            {
                const u64 nk = key_neighbor(k, dx, dy, dz);
                if (nk == k) continue;
                if (rf == 0)
                {
                    int c[3];
                    key_coord(nk, c);
                    for (int d = 0; d < 3; ++d)
                        if (c[d] < 0 || c[d] > key_bd_extent[d] - 1) ok = false;
                }
                else if (!try_2to1(key_parent(nk), checklist))
                    ok = false;
            }
    checklist.emplace(k, ok);
    return ok;
}

void HostTree::refine(int l, bool ratio_2to1)
{
    auto f = [&](int x) { alloc(x, o[x].level - base_level); };
    if (ratio_2to1 && o[l].level - base_level >= 0)
    {
        for (u64 k : unfound_neighbors(l, false))
        {
            if (key_is_end(k)) continue;
            if (o[l].level - base_level == 0)
            {
                const int n = insert(k);
                if (!o[n].has_data) f(n);
                o[n].leaf = true;
                o[n].correction = false;
            }
            else
            {
                const u64 pk = key_parent(k);
                int pa = find(pk);
                if (pa < 0)
                {
                    pa = insert(pk);
                    f(pa);
                }
                refine(pa, ratio_2to1);
            }
        }
    }
    for (int i = 0; i < 8; ++i)
    {
        const int ci = o[l].child[i];
        if (ci >= 0 && o[ci].has_data) continue;
        const int c = refine_child(l, i);
        if (!o[c].has_data) f(c);
    }
    for (int i = 0; i < 8; ++i)
    {
        HOct& c = o[o[l].child[i]];
        c.leaf = true;
        c.correction = false;
    }
    o[l].leaf = false;
    o[l].correction = false;
    depth = std::max(depth, o[l].level + 2);
}

void HostTree::init_refine(int n_ref, int level_up_max, iblgf_refine_fn pred, void* user)
{
    // construct_leaf_maps(): leaf = no children at all
    for (int i : dfs_order())
    {
        if (!o[i].has_data) continue;
        bool leaf = true;
        for (int c : o[i].child)
            if (c >= 0) leaf = false;
        o[i].leaf = leaf;
    }
    std::map<u64, bool> checklist;
    for (int l = 0; l < n_ref; ++l)
    {
        std::vector<int> st{0};
        while (!st.empty())
        {
            const int cur = st.back();
            st.pop_back();
            for (int i = 7; i >= 0; --i)
                if (o[cur].child[i] >= 0) st.push_back(o[cur].child[i]);
            if (o[cur].level == 0 || o[cur].level - base_level != l) continue;
            int ext[3] = {e, e, e};
            if (pred && pred(user, o[cur].bbase, ext, l, n_ref - l))
                if (try_2to1(o[cur].key, checklist)) refine(cur, true);
        }
    }
    for (int g = 0; g < level_up_max; ++g)
    {
        for (int l = depth - 1; l >= base_level; --l)
        {
            std::vector<std::pair<u64, int>> lv;
            for (int i = 0; i < (int)o.size(); ++i)
                if (o[i].has_data && o[i].level == l) lv.push_back({o[i].key, i});
            std::sort(lv.begin(), lv.end());
            for (auto& kv : lv)
                if (o[kv.second].leaf) refine(kv.second, false);
        }
    }
    mark_correction();
}

void HostTree::mark_correction(std::vector<char>* aim_del)
{
    auto del = [&](int i) { return aim_del && i < (int)aim_del->size() && (*aim_del)[i]; };
    auto keep = [&](int i) {
        if (!aim_del) return;
        if ((int)aim_del->size() <= i) aim_del->resize(o.size(), 0);
        (*aim_del)[i] = 0;
    };
    for (auto& x : o) x.physical = false;
    for (int l = depth - 1; l >= base_level; --l)
        for (int i = 0; i < (int)o.size(); ++i)
        {
            if (!o[i].has_data || o[i].level != l) continue;
            o[i].physical = o[i].leaf && !del(i);
            if (!o[i].physical)
                for (int c : o[i].child)
                    if (c >= 0 && o[c].has_data) o[i].physical = o[i].physical || o[c].physical;
        }
    // correction buffers around physical octants of refined levels
    for (int l = base_level + 1; l < depth; ++l)
    {
        std::vector<int> lv;
        for (int i = 0; i < (int)o.size(); ++i)
            if (o[i].has_data && o[i].level == l) lv.push_back(i);
        for (int i : lv)
        {
            if (!o[i].physical) continue;
            for (u64 k : unfound_neighbors(i, true))
            {
                const int n = insert(k);
                if (!o[n].has_data) alloc(n, o[n].level - base_level);
            }
        }
    }
    auto neighbors_of = [&](int i, int* out) {
        int m = 0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                {
                    const int n = find(key_neighbor(o[i].key, dx, dy, dz));
                    out[m++] = (n >= 0 && o[n].has_data) ? n : -1;
                }
    };
    int nb[27];
    for (int l = base_level + 1; l < depth; ++l)
        for (int i = 0; i < (int)o.size(); ++i)
        {
            if (!o[i].has_data || o[i].level != l || !o[i].physical) continue;
            neighbors_of(i, nb);
            for (int n : nb)
            {
                if (n < 0 || o[n].physical) continue;
                keep(n);
                o[n].correction = true;
            }
        }
    for (int i = 0; i < (int)o.size(); ++i)
    {
        if (!o[i].has_data || o[i].level != base_level || !o[i].physical) continue;
        neighbors_of(i, nb);
        bool all = true;
        for (int n : nb)
            if (n < 0) all = false;
        if (!all)
        {
            o[i].correction = true;
            o[i].leaf = true;
        }
        else
            o[i].correction = false;
        keep(i);
    }
}

bool HostTree::leaf_search(int i, bool require_data) const
{
    for (int c : o[i].child)
        if (c >= 0 && (!require_data || o[c].has_data)) return false;
    return true;
}

// Tree::delete_oct (tree.hpp:455-466): the octant loses its data and, without
// children, its place in the parent
void HostTree::delete_oct(int i)
{
    o[i].has_data = false;
    o[i].leaf = false;
    o[i].correction = false;
    o[i].idx = -1;
    if (leaf_search(i, false) && o[i].parent >= 0)
    {
        HOct& p = o[o[i].parent];
        for (int& c : p.child)
            if (c == i) c = -1;
    }
}

// Domain::adapt / Decomposition::adapt_decoposition, server part
// (domain/decomposition/decomposition.hpp:182-470) for one process, with
// Tree::deletionReset_2to1 (octree/tree.hpp:304-327) and
// Domain::delete_all_children (domain.hpp:512-569); baseBlockBufferNumber_ = 2
std::vector<int> HostTree::adapt(const std::vector<std::pair<u64, int>>& attempts, const std::vector<char>& ib,
                                 bool& base_mesh_update)
{
    base_mesh_update = false;
    std::vector<char> del(o.size(), 0);
    std::vector<int> lchange(o.size(), 0);
    auto grow = [&]() {
        if (del.size() < o.size()) del.resize(o.size(), 0);
        if (lchange.size() < o.size()) lchange.resize(o.size(), 0);
    };
    auto is_ib = [&](int i) { return i < (int)ib.size() && (ib[i] & 1); };
    auto is_ext = [&](int i) { return i < (int)ib.size() && (ib[i] & 2); };
    auto by_level_key = [&](std::vector<int> v) {
        std::sort(v.begin(), v.end(), [&](int a, int b) {
            return o[a].level != o[b].level ? o[a].level < o[b].level : o[a].key < o[b].key;
        });
        return v;
    };
    auto leaves = [&]() {
        std::vector<int> v;
        for (int i = 0; i < (int)o.size(); ++i)
            if (o[i].has_data && o[i].leaf) v.push_back(i);
        return by_level_key(v);
    };
    auto level_list = [&](int l) {
        std::vector<int> v;
        for (int i = 0; i < (int)o.size(); ++i)
            if (o[i].has_data && o[i].level == l) v.push_back(i);
        return by_level_key(v);
    };
    std::set<u64> old_leaves;
    for (int i = 0; i < (int)o.size(); ++i)
    {
        if (o[i].has_data && o[i].leaf) old_leaves.insert(o[i].key);
        del[i] = o[i].correction && !is_ib(i);
    }
    for (auto& a : attempts)
    {
        if (a.second == 0) continue;
        const int i = find(a.first);
        if (i < 0 || !o[i].has_data) throw Error(IBLGF_EINVAL, "adaptation attempt for an octant without data");
        lchange[i] = a.second;
    }
    std::map<u64, bool> checklist;
    std::vector<int> refine_list;
    for (int i : leaves())
    {
        if (lchange[i] == 0) continue;
        if (lchange[i] < 0) del[i] = 1;
        else if (is_ib(i) || try_2to1(o[i].key, checklist))
            refine_list.push_back(i);
    }
    for (int i : leaves())
        if (is_ib(i) || is_ext(i)) del[i] = 0;
    // base-level blocks within two blocks of a kept base block
    std::set<u64> away;
    for (int i : level_list(base_level))
    {
        if (del[i] || o[i].correction) continue;
        int c[3];
        key_coord(o[i].key, c);
        const int lim = 1 << o[i].level;
        for (int dz = -2; dz <= 2; ++dz)
            for (int dy = -2; dy <= 2; ++dy)
                for (int dx = -2; dx <= 2; ++dx)
                {
                    const int x = c[0] + dx, y = c[1] + dy, z = c[2] + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= lim || y >= lim || z >= lim) continue;
                    away.insert(key_make(x, y, z, o[i].level));
                }
    }
    for (u64 nk : away)
    {
        int c[3];
        key_coord(nk, c);
        bool inside = true;
        for (int d = 0; d < 3; ++d)
            if (c[d] < 0 || c[d] > key_bd_extent[d] - 1) inside = false;
        if (!inside) continue;
        int n = find(nk);
        if (n < 0 || !o[n].has_data)
        {
            n = insert(nk);
            alloc(n, o[n].level - base_level);
            o[n].leaf = true;
            o[n].correction = false;
            base_mesh_update = true;
            grow();
        }
        del[n] = 0;
    }
    for (int i : refine_list)
    {
        if (!o[i].leaf) continue;
        refine(i, true);
        grow();
    }
    // deletionReset_2to1 from the parents of refined leaves
    std::set<int> reset_done;
    std::function<void(int)> reset = [&](int l) {
        if (reset_done.count(l)) return;
        if (o[l].level - base_level < 0) return;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                {
                    const u64 nk = key_neighbor(o[l].key, dx, dy, dz);
                    if (key_is_end(nk)) continue;
                    const int n = find(nk);
                    if (n < 0 || !o[n].has_data) continue;
                    del[n] = 0;
                    reset(o[n].parent);
                }
        reset_done.insert(l);
    };
    for (int i : leaves())
        if (o[i].level - base_level > 0) reset(o[i].parent);
    // base-level deletions, then collapse of fully deleted sibling groups
    for (int i : level_list(base_level))
        if (del[i] && o[i].leaf) delete_oct(i);
    for (int l = depth - 2; l >= base_level; --l)
        for (int i : level_list(l))
        {
            if (leaf_search(i, true)) continue;
            bool all = true;
            for (int ch : o[i].child)
            {
                if (ch < 0 || !o[ch].has_data) continue;
                if (!del[ch] || (!o[ch].leaf && !o[ch].correction))
                {
                    all = false;
                    break;
                }
            }
            if (all)
            {
                for (int ch : o[i].child)
                {
                    if (ch < 0) continue;
                    o[ch].leaf = false;
                    o[ch].correction = false;
                    del[ch] = 1;
                }
                o[i].leaf = true;
                o[i].correction = false;
                del[i] = 0;
            }
            else
                for (int ch : o[i].child)
                    if (ch >= 0) del[ch] = 0;
        }
    mark_correction(&del);
    grow();
    for (int i = 0; i < (int)o.size(); ++i)
        if (o[i].has_data && del[i] && o[i].level - base_level > 0) delete_oct(i);
    for (int l = base_level - 1; l > 0; --l)
        for (int i = 0; i < (int)o.size(); ++i)
            if (o[i].level == l && leaf_search(i, false)) delete_oct(i);
    // new octants' ancestors get data
    for (int i = 0; i < (int)o.size(); ++i)
    {
        if (!o[i].has_data || o[i].idx >= 0) continue;
        for (int pa = o[i].parent; pa >= 0 && !o[pa].has_data; pa = o[pa].parent) alloc(pa, o[pa].level - base_level);
    }
    depth = 0;
    for (auto& x : o)
        if (x.has_data) depth = std::max(depth, x.level + 1);
    // parents of new leaves above the base level
    std::vector<int> parents;
    for (int i : leaves())
        if (o[i].level - base_level > 0 && !old_leaves.count(o[i].key)) parents.push_back(o[i].parent);
    parents = by_level_key(parents);
    parents.erase(std::unique(parents.begin(), parents.end()), parents.end());
    return parents;
}

void HostTree::import_octants(int n, const u64* keys, const int* flags)
{
    if (o.size() != 1 || o[0].has_data) throw Error(IBLGF_EINVAL, "import needs an empty tree");
    for (int i = 0; i < n; ++i)
    {
        const int lv = key_level(keys[i]);
        if (lv > kMaxLevel) throw Error(IBLGF_EINVAL, "key level out of range");
        const int x = insert(keys[i]);
        if (o[x].key != keys[i]) throw Error(IBLGF_EINVAL, "malformed key");
        alloc(x, lv - base_level);
        o[x].leaf = (flags[i] & 1) != 0;
        o[x].correction = (flags[i] & 2) != 0;
    }
}

// Domain restart (domain.hpp:235-290 with restart_list_construct, :839-849):
// the keys Tree::write stored (every octant with data but the root) with
// their leaf flags; ancestors get data as in the run that wrote them, then
// mark_correction derives the correction flags.
void HostTree::restart(int n, const u64* keys, const unsigned char* leaf)
{
    std::vector<int> flags(n);
    for (int i = 0; i < n; ++i) flags[i] = leaf[i] ? 1 : 0;
    import_octants(n, keys, flags.data());
    for (int i = 0; i < (int)o.size(); ++i)
        if (o[i].has_data)
            for (int pa = o[i].parent; pa >= 0 && !o[pa].has_data; pa = o[pa].parent) alloc(pa, o[pa].level - base_level);
    mark_correction();
}

std::vector<int> HostTree::canonical() const
{
    std::vector<std::pair<std::pair<int, u64>, int>> v;
    for (int i = 0; i < (int)o.size(); ++i)
        if (o[i].has_data) v.push_back({{o[i].level, o[i].key}, i});
    std::sort(v.begin(), v.end());
    std::vector<int> out;
    for (auto& x : v) out.push_back(x.second);
    return out;
}

}  // namespace iblgf_b200
