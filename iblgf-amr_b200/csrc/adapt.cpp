// Mesh adaptation on one GPU: Ifherk::adapt (include/iblgf/solver/
// time_integration/ifherk.hpp:1018-1076) with the server side of
// Domain::adapt / Decomposition::adapt_decoposition (domain/decomposition/
// decomposition.hpp:182-470; the tree part is HostTree::adapt). Field data
// follows its octant: every field is gathered into the new canonical order on
// the device (kept octants copy, new octants start at zero); the fields the
// caller lists are then interpolated from each interpolation parent into all
// its children with data (cell_center_nli_intrp.hpp:310-420, assignment),
// parents in (level, key) order. Plans, lists and masks are rebuilt; the LGF
// spectrum cache depends only on block offsets and is kept.
//
// Also the per-block norms of the adaptation criterion: Operator::maxnorm and
// blockRootMeanSquare (operators/operators.hpp:1149-1211).
#include <algorithm>
#include <set>

#include "ctx.hpp"

namespace iblgf_b200
{
void poisson_release(Ctx& c);

namespace
{
// relative positions of a component (cell_center_nli_intrp.hpp:349-365):
// mesh 0 cell, 1 face, 2 edge
void component_relpos(int mesh, int comp, int rp[3])
{
    for (int a = 0; a < 3; ++a) rp[a] = 1;
    if (mesh == 1) rp[comp] = 0;
    else if (mesh == 2)
    {
        for (int a = 0; a < 3; ++a) rp[a] = 0;
        rp[comp] = 1;
    }
}
}  // namespace

void domain_adapt(Ctx& c, int n_att, const u64* keys, const int* lchange, int n_interp, const int* interp_fields,
                  const int* interp_mesh, int* base_mesh_update)
{
    need_single(c);
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    if (n_att < 0 || (n_att && (!keys || !lchange)) || n_interp < 0 || (n_interp && (!interp_fields || !interp_mesh)))
        throw Error(IBLGF_EINVAL, "bad adaptation arguments");
    const int nf = (int)c.fields.size();
    for (int i = 0; i < n_interp; ++i)
    {
        if (interp_mesh[i] < 0 || interp_mesh[i] > 2) throw Error(IBLGF_EINVAL, "mesh must be 0 cell, 1 face, 2 edge");
        const int nc = interp_mesh[i] == 0 ? 1 : 3;
        for (int k = 0; k < nc; ++k)
            if (interp_fields[3 * i + k] < 0 || interp_fields[3 * i + k] >= nf)
                throw Error(IBLGF_EINVAL, "bad interpolation field id");
    }
    HostTree& t = c.tree;
    // IB flags per tree position (is_ib blocks are refined regardless of 2:1
    // and never deleted, decomposition.hpp:243-268)
    std::vector<char> ib(t.o.size(), 0);
    const std::vector<int> of = ib_octant_flags(c);
    for (size_t i = 0; i < t.o.size(); ++i)
        if (t.o[i].has_data && t.o[i].idx >= 0 && !of.empty()) ib[i] = (char)of[t.o[i].idx];
    std::vector<std::pair<u64, int>> att(n_att);
    for (int i = 0; i < n_att; ++i) att[i] = {keys[i], lchange[i]};
    // base-level correction blocks before the change (Octant::old_correction)
    std::set<u64> old_corr_keys;
    for (int o = 0; o < c.n_oct; ++o)
        if (c.levels[o] == t.base_level && (c.flags[o] & 2)) old_corr_keys.insert(c.keys[o]);
    bool bmu = false;
    const std::vector<int> parents = t.adapt(att, ib, bmu);
    // old canonical index of every tree position that keeps its data
    std::vector<int> old_idx(t.o.size(), -1);
    for (size_t i = 0; i < t.o.size(); ++i)
        if (t.o[i].has_data) old_idx[i] = t.o[i].idx;
    std::vector<std::tuple<int, int, int>> plan_keys;
    for (const auto& kv : c.plans) plan_keys.push_back(kv.first);
    c.plans.clear();
    poisson_release(c);
    domain_rebuild(c);
    // gather every field into the new order
    std::vector<int> src(c.n_oct, -1);
    for (size_t i = 0; i < t.o.size(); ++i)
        if (t.o[i].has_data) src[t.o[i].idx] = old_idx[i];
    DevBuf<int> d_src;
    d_src.upload(src, c.stream);
    for (auto& f : c.fields)
    {
        PoolBuf nw;
        nw.alloc(c.field_elems(), c.cfg.device, c.stream);
        launch_remap_blocks(c, f->d.p, nw.p, d_src.p, c.n_oct);
        f->d = std::move(nw);  // the old buffer is freed in stream order after the remap
    }
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    // interpolation parents -> all their children with data, one level at a time
    if (n_interp && !parents.empty())
    {
        std::vector<int> levels;
        for (int p : parents) levels.push_back(t.o[p].level);
        std::sort(levels.begin(), levels.end());
        levels.erase(std::unique(levels.begin(), levels.end()), levels.end());
        for (int lv : levels)
        {
            std::vector<int> dst;
            std::vector<std::vector<std::pair<int, int>>> tasks;
            for (int p : parents)
            {
                if (t.o[p].level != lv) continue;
                for (int k = 0; k < 8; ++k)
                {
                    const int ch = t.o[p].child[k];
                    if (ch < 0 || !t.o[ch].has_data) continue;
                    dst.push_back(t.o[ch].idx);
                    tasks.push_back({{t.o[p].idx, k}});
                }
            }
            HostTasks ht;
            host_tasks(ht, dst, tasks);
            TpTasks tt;
            upload_host_tasks(c, tt, ht);
            for (int i = 0; i < n_interp; ++i)
            {
                const int nc = interp_mesh[i] == 0 ? 1 : 3;
                for (int k = 0; k < nc; ++k)
                {
                    int rp[3], m[3];
                    component_relpos(interp_mesh[i], k, rp);
                    for (int a = 0; a < 3; ++a) m[a] = rp[a] ? 2 : 6;
                    double* f = c.field(interp_fields[3 * i + k]);
                    launch_tp_axes(c, tt, f, f, m, 2);
                }
            }
            IBLGF_CUDA(cudaStreamSynchronize(c.stream));  // tt goes out of scope
        }
    }
    std::vector<char> old_corr(c.n_oct, 0);
    for (int o = 0; o < c.n_oct; ++o) old_corr[o] = c.levels[o] == t.base_level && old_corr_keys.count(c.keys[o]);
    ns_on_adapt(c, bmu, old_corr);
    ib_on_adapt(c);
    // the sweeps of the next steps: their plans built now, in parallel
    prebuild_plans(c, plan_keys);
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    if (base_mesh_update) *base_mesh_update = bmu ? 1 : 0;
}

void block_norms(Ctx& c, const int* fields, int n_comp, double* host_max, double* host_rms)
{
    need_single(c);
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    if (n_comp < 1 || n_comp > 3 || !fields || !host_max || !host_rms) throw Error(IBLGF_EINVAL, "bad arguments");
    const double* comps[3];
    for (int k = 0; k < n_comp; ++k)
    {
        if (fields[k] < 0 || fields[k] >= (int)c.fields.size()) throw Error(IBLGF_EINVAL, "bad field id");
        comps[k] = c.field(fields[k]);
    }
    DevBuf<double> mx, rms;
    mx.alloc(c.n_oct);
    rms.alloc(c.n_oct);
    launch_block_norms(c, comps, n_comp, mx.p, rms.p);
    IBLGF_CUDA(cudaMemcpyAsync(host_max, mx.p, c.n_oct * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaMemcpyAsync(host_rms, rms.p, c.n_oct * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
}

}  // namespace iblgf_b200
