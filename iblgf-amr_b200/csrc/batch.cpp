// Batches of independent unbounded Poisson problems of uneven size, solved in
// one pass of the LGF-FMM level loop (PoissonSolver::apply_lgf,
// include/iblgf/solver/poisson/poisson.hpp:587-894, per problem).
//
// Every problem keeps its own octree, neighbour / influence lists and masks
// (a topology-only sub-context built exactly as a single-problem context).
// The batch context owns the fields, with the problems' octants back to back,
// and one LGF spectra cache shared by all problems. The sweep plans of all
// problems at the same level relative to their base level are concatenated
// (octant indices, source / target slots and spectrum tables offset), so each
// stage of a sweep -- anterpolation per tree level, forward transforms, the
// spectral MAC, inverse transforms, interpolation -- is one launch for the
// whole batch. Problems never interact: every list entry stays inside its
// own problem, and the LGF spectra are keyed by (level difference, block
// offset) only, so equal keys mean equal kernels.
//
// Requirements: one block_extent, dx_base and precision for the batch (the
// context's configuration); each problem has its own bounding box, blocks and
// refinement.
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>

#include "ctx.hpp"

namespace iblgf_b200
{
void ctx_init(Ctx& c);

namespace
{
struct BatchState
{
    int rmax = 0;                    // largest number of mesh levels over the problems
    std::vector<int> depth_rel;      // mesh levels per problem
    DevBuf<int> leaves;
    // per relative level r
    std::vector<DevBuf<int>> level_leaves, corr_all, corr_next, corr_children;
    std::vector<TpTasks> coarsify, cc_intrp, corr_intrp;
    std::map<std::pair<int, int>, std::unique_ptr<FmmPlan>> plans;  // (r, non_leaf_as_source)
};

int no_refine(void*, const int*, const int*, int, int) { return 0; }

void append_tasks(HostTasks& m, const HostTasks& h, int off)
{
    const int base = (int)m.src.size();
    for (size_t g = 0; g < h.dst.size(); ++g)
    {
        m.dst.push_back(h.dst[g] + off);
        m.ptr.push_back(base + h.ptr[g + 1]);
    }
    for (size_t t = 0; t < h.src.size(); ++t)
    {
        m.src.push_back(h.src[t] + off);
        m.cid.push_back(h.cid[t]);
    }
}

void append_off(std::vector<int>& m, const std::vector<int>& v, int off)
{
    for (int x : v) m.push_back(x + off);
}

// Concatenates the plans of independent problems (plan, first octant of the
// problem in the batch). Anterpolation passes are aligned at the sweep level
// (first pass = one level up), interpolation passes at the sweep level too
// (last pass = parents one level up), so every problem keeps its own order.
HostPlan merge_plans(const std::vector<std::pair<HostPlan, int>>& parts)
{
    HostPlan m;
    size_t na = 0, ni = 0;
    for (auto& pp : parts)
    {
        na = std::max(na, pp.first.antrp.size());
        ni = std::max(ni, pp.first.intrp.size());
    }
    m.antrp.resize(na);
    m.intrp.resize(ni);
    std::vector<int> srcb(parts.size()), csrb(parts.size()), grpb(parts.size());
    for (size_t i = 0; i < parts.size(); ++i)
    {
        const HostPlan& h = parts[i].first;
        const int off = parts[i].second;
        append_off(m.zs, h.zs, off);
        append_off(m.zt, h.zt, off);
        append_off(m.cs, h.cs, off);
        append_off(m.at, h.at, off);
        srcb[i] = (int)m.srcs.size();
        append_off(m.srcs, h.srcs, off);
        for (size_t j = 0; j < h.antrp.size(); ++j) append_tasks(m.antrp[j], h.antrp[j], off);
        for (size_t j = 0; j < h.intrp.size(); ++j) append_tasks(m.intrp[ni - h.intrp.size() + j], h.intrp[j], off);
        csrb[i] = (int)m.tgt_list.size();
        for (int t = 0; t < h.n_csr_tgt; ++t) m.tgt_list.push_back(h.tgt_list[t] + off);
        const int pb = (int)m.psrc.size();
        for (size_t k = 1; k < h.ptr.size(); ++k) m.ptr.push_back(pb + h.ptr[k]);
        append_off(m.psrc, h.psrc, srcb[i]);
        m.pkey.insert(m.pkey.end(), h.pkey.begin(), h.pkey.end());
        m.all_keys.insert(m.all_keys.end(), h.all_keys.begin(), h.all_keys.end());
        m.n_pairs += h.n_pairs;
        m.n_exec += h.n_exec;
    }
    m.n_csr_tgt = (int)m.tgt_list.size();
    for (size_t i = 0; i < parts.size(); ++i)
    {
        const HostPlan& h = parts[i].first;
        const int off = parts[i].second;
        grpb[i] = (int)m.tgt_list.size();
        for (size_t t = h.n_csr_tgt; t < h.tgt_list.size(); ++t) m.tgt_list.push_back(h.tgt_list[t] + off);
        const int tab_base = (int)(m.tab_keys.size() / 343);
        m.tab_keys.insert(m.tab_keys.end(), h.tab_keys.begin(), h.tab_keys.end());
        const int gbase = (int)(m.gtgt.size() / 8), sbase = (int)m.tsrc.size();
        for (size_t k = 1; k < h.tgptr.size(); ++k) m.tgptr.push_back(gbase + h.tgptr[k]);
        for (size_t k = 1; k < h.tsptr.size(); ++k) m.tsptr.push_back(sbase + h.tsptr[k]);
        append_off(m.tsrc, h.tsrc, srcb[i]);
        append_off(m.ttab, h.ttab, tab_base);
        m.tcoarse.insert(m.tcoarse.end(), h.tcoarse.begin(), h.tcoarse.end());
        m.gsrc.insert(m.gsrc.end(), h.gsrc.begin(), h.gsrc.end());
        m.gpm.insert(m.gpm.end(), h.gpm.begin(), h.gpm.end());
        for (int x : h.gtgt)
            m.gtgt.push_back(x < 0 ? -1 : (x < h.n_csr_tgt ? csrb[i] + x : grpb[i] + x - h.n_csr_tgt));
        m.n_groups += h.n_groups;
        m.max_tile_src = std::max(m.max_tile_src, h.max_tile_src);
    }
    std::vector<std::array<int, 4>> u = m.all_keys;
    std::sort(u.begin(), u.end());
    m.n_spec_unique = (int)(std::unique(u.begin(), u.end()) - u.begin());
    return m;
}

BatchState& batch_state(Ctx& c)
{
    if (auto* have = c.ext_get<BatchState>(Ctx::kExtBatch)) return *have;
    auto b = std::make_unique<BatchState>();
    const int np = (int)c.sub.size();
    b->depth_rel.resize(np);
    for (int i = 0; i < np; ++i)
    {
        b->depth_rel[i] = c.sub[i]->tree.depth - c.sub[i]->tree.base_level;
        b->rmax = std::max(b->rmax, b->depth_rel[i]);
    }
    const int R = b->rmax;
    b->level_leaves.resize(R);
    b->corr_all.resize(R);
    b->corr_next.resize(R);
    b->corr_children.resize(R);
    b->coarsify.resize(R);
    b->cc_intrp.resize(R);
    b->corr_intrp.resize(R);
    std::vector<int> leaves;
    std::vector<std::vector<int>> lleaves(R), call(R), cnext(R), cchild(R);
    std::vector<HostTasks> hco(R), hcc(R), hci(R);
    for (int i = 0; i < np; ++i)
    {
        const Ctx& s = *c.sub[i];
        const int off = c.sub_off[i], bl = s.tree.base_level, dr = b->depth_rel[i];
        for (int o = 0; o < s.n_oct; ++o)
            if (s.flags[o] & 1) leaves.push_back(o + off);
        for (int r = 0; r < dr; ++r)
        {
            const int l = bl + r;
            std::vector<int> cdst, idst, kdst, ch;
            std::vector<std::vector<std::pair<int, int>>> ct, it_, kt;
            for (int o : s.level_octs[l])
            {
                if (s.flags[o] & 1) lleaves[r].push_back(o + off);
                cdst.push_back(o);
                ct.emplace_back();
                for (int k = 0; k < 8; ++k)
                {
                    const int x = s.child[8 * o + k];
                    if (x < 0) continue;
                    ct.back().push_back({x, k});
                    idst.push_back(x);
                    it_.push_back({{o, k}});
                    ch.push_back(x);
                    if (s.flags[x] & 2)
                    {
                        kdst.push_back(x);
                        kt.push_back({{o, k}});
                    }
                }
            }
            HostTasks t;
            if (r <= dr - 2)
            {
                host_tasks(t, cdst, ct);
                append_tasks(hco[r], t, off);
            }
            t = HostTasks();
            host_tasks(t, idst, it_);
            append_tasks(hcc[r], t, off);
            // source correction only below the problem's finest level
            if (r < dr - 1)
            {
                t = HostTasks();
                host_tasks(t, kdst, kt);
                append_tasks(hci[r], t, off);
                for (int o : s.level_octs[l]) call[r].push_back(o + off);
                for (int o : s.level_octs[l + 1]) cnext[r].push_back(o + off);
                append_off(cchild[r], ch, off);
            }
        }
    }
    b->leaves.upload(leaves, c.stream);
    for (int r = 0; r < R; ++r)
    {
        b->level_leaves[r].upload(lleaves[r], c.stream);
        b->corr_all[r].upload(call[r], c.stream);
        b->corr_next[r].upload(cnext[r], c.stream);
        b->corr_children[r].upload(cchild[r], c.stream);
        upload_host_tasks(c, b->coarsify[r], hco[r]);
        upload_host_tasks(c, b->cc_intrp[r], hcc[r]);
        upload_host_tasks(c, b->corr_intrp[r], hci[r]);
    }
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    auto& ref = *b;
    c.ext[Ctx::kExtBatch] = std::shared_ptr<BatchState>(std::move(b));
    return ref;
}

FmmPlan& batch_plan(Ctx& c, BatchState& b, int r, bool nlas)
{
    auto key = std::make_pair(r, nlas ? 1 : 0);
    auto it = b.plans.find(key);
    if (it != b.plans.end()) return *it->second;
    std::vector<std::pair<HostPlan, int>> parts;
    for (size_t i = 0; i < c.sub.size(); ++i)
    {
        if (b.depth_rel[i] <= r) continue;
        const Ctx& s = *c.sub[i];
        parts.emplace_back(build_host_plan(s, s.tree.base_level + r, mask_idx_gen(IBLGF_AMR2AMR, r, nlas ? 1 : 0), -1),
                           c.sub_off[i]);
    }
    auto plan = upload_plan(c, merge_plans(parts));
    auto& ref = *plan;
    b.plans.emplace(key, std::move(plan));
    return ref;
}
}  // namespace

int batch_add_problem(Ctx& c, const int* bd_base, const int* bd_extent, int n, const int* base, const int* extent,
                      int n_ref, iblgf_refine_fn pred, void* user)
{
    if (c.finalized) throw Error(IBLGF_EINVAL, "batch already finalized");
    if (c.has_blocks) throw Error(IBLGF_EINVAL, "the context already holds a single-problem domain");
    if (!bd_base || !bd_extent) throw Error(IBLGF_EINVAL, "null bounding box");
    if (n_ref < 0) throw Error(IBLGF_EINVAL, "negative refinement");
    if (n_ref > 0 && !pred) throw Error(IBLGF_EINVAL, "refinement needs a predicate");
    auto s = std::make_unique<Ctx>();
    s->cfg = c.cfg;
    for (int d = 0; d < 3; ++d)
    {
        s->cfg.bd_base[d] = bd_base[d];
        s->cfg.bd_extent[d] = bd_extent[d];
    }
    s->cfg.stream = c.stream;
    s->topology_only = true;
    ctx_init(*s);
    add_blocks(*s, n, base, extent);
    s->tree.init_refine(n_ref, 0, pred ? pred : no_refine, user);
    c.batch = true;
    c.sub.push_back(std::move(s));
    return (int)c.sub.size() - 1;
}

void batch_finalize(Ctx& c)
{
    if (!c.batch || c.sub.empty()) throw Error(IBLGF_EINVAL, "no problems in the batch");
    if (c.finalized) throw Error(IBLGF_EINVAL, "batch already finalized");
    c.sub_off.clear();
    int total = 0;
    for (auto& s : c.sub)
    {
        s->subtract_non_leaf = c.subtract_non_leaf;
        domain_finalize(*s);
        c.sub_off.push_back(total);
        total += s->n_oct;
    }
    c.n_oct = total;
    c.flags.clear();
    c.bbase.clear();
    c.levels.clear();
    std::vector<int> nbr;
    for (size_t i = 0; i < c.sub.size(); ++i)
    {
        const Ctx& s = *c.sub[i];
        const int off = c.sub_off[i];
        c.flags.insert(c.flags.end(), s.flags.begin(), s.flags.end());
        c.levels.insert(c.levels.end(), s.levels.begin(), s.levels.end());
        c.bbase.insert(c.bbase.end(), s.bbase.begin(), s.bbase.end());
        for (int q : s.nbr) nbr.push_back(q < 0 ? -1 : q + off);
    }
    c.d_nbr.upload(nbr, c.stream);
    c.d_bbase.upload(c.bbase, c.stream);
    c.f_source_tmp = field_create(c);
    c.f_target_tmp = field_create(c);
    c.f_correction_tmp = field_create(c);
    c.f_fmm_s = field_create(c);
    c.f_fmm_t = field_create(c);
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    c.finalized = true;
}

void batch_apply_lgf(Ctx& c, int src, int tgt)
{
    if (!c.batch || !c.finalized) throw Error(IBLGF_EINVAL, "batch not finalized");
    const int nf = (int)c.fields.size();
    if (src < 0 || src >= nf || tgt < 0 || tgt >= nf) throw Error(IBLGF_EINVAL, "bad field id");
    BatchState& b = batch_state(c);
    double* st = c.field(c.f_source_tmp);
    double* tt = c.field(c.f_target_tmp);
    double* ct = c.field(c.f_correction_tmp);
    const size_t bytes = c.field_elems() * sizeof(double);
    launch_fill_zero(c, st, bytes / sizeof(double));
    launch_fill_zero(c, tt, bytes / sizeof(double));
    launch_fill_zero(c, ct, bytes / sizeof(double));
    launch_axpy_blocks(c, c.field(src), st, b.leaves.p, (int)b.leaves.n, 1.0, true);
    for (int r = b.rmax - 2; r >= 0; --r) launch_tp(c, b.coarsify[r], st, st, 4, 0);
    for (int r = 0; r < b.rmax; ++r)
    {
        const double dx_level = c.cfg.dx_base / std::pow(2.0, r);
        if (!c.subtract_non_leaf)
        {
            run_sweep(c, batch_plan(c, b, r, true), c.f_source_tmp, c.f_target_tmp, dx_level, 1.0, -1);
            launch_tp(c, b.cc_intrp[r], tt, tt, 2, 2);
            run_sweep(c, batch_plan(c, b, r, false), c.f_source_tmp, c.f_target_tmp, dx_level, 1.0, -1);
            launch_axpy_blocks(c, tt, c.field(tgt), b.level_leaves[r].p, (int)b.level_leaves[r].n, 1.0, true);
        }
        if (!c.use_correction || !b.corr_all[r].n) continue;
        launch_halo(c, st, b.corr_all[r].p, (int)b.corr_all[r].n);
        launch_tp(c, b.corr_intrp[r], st, ct, 2, 2);
        const double dx = dx_level / 2.0;
        launch_source_correction(c, tt, ct, b.corr_children[r].p, (int)b.corr_children[r].n, 1.0 / (dx * dx));
        launch_axpy_blocks(c, ct, st, b.corr_next[r].p, (int)b.corr_next[r].n, 1.0, false);
    }
}

void batch_release(Ctx& c) { c.ext[Ctx::kExtBatch].reset(); }

}  // namespace iblgf_b200
