// IF-HERK time step of the incompressible Navier-Stokes solver on the device,
// Ifherk::time_step (include/iblgf/solver/time_integration/ifherk.hpp:
// 1078-1200) with its helpers: up_and_down (:992-1015), clean (:1309-1352),
// clean_leaf_correction_boundary (:1355-1405), lin_sys_with_ib_solve
// (:1451-1517), nonlinear (:1638-1692), divergence (:1738-1763), gradient
// (:1766-1795), add / copy (:1878-1960). Every stage runs on the context
// stream from device-resident component fields: the Poisson and integrating-
// factor solves, the mimetic operators, buffer exchanges and level transfers
// are the library's own kernels, with no host round trip inside a step.
//
// Steps without an immersed boundary replay a CUDA graph of one captured step
// once a direct step with the same fields, dt and Re has run.
// Scope: optional immersed boundary (lin_sys_with_ib_solve), constant frame
// velocity, no adaptation, no body force. The velocity refresh (pad_velocity
// + adapt_corr_time_step, taken once (T - T_last_refresh) 3.3 / (Re dx_base^2)
// > 7, ifherk.hpp:1093-1111) runs with direct launches.
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>

#include "ctx.hpp"

namespace iblgf_b200
{
void launch_clean(Ctx& c, double* f, const int* d_leaf, bool non_leaf_only, int width = 1);
void launch_axpby(Ctx& c, double* to, const double* from, double a, int mode);
void launch_clean_vf(Ctx& c, double* const* f, int n, const int* d_leaf, bool non_leaf_only, int width = 1);
void launch_axpby_vf(Ctx& c, double* const* to, const double* const* from, int n, double a, int mode);
void launch_smooth(Ctx& c, double* f, const int* list, const int* ptr, const int* dirs, int n, int reps);

namespace
{
enum Mesh { kCell = 0, kFace = 1, kEdge = 2 };

// component field ids of a cell (1) or face / edge (3) field
struct VF
{
    int mesh = kCell;
    int n = 1;
    int id[3] = {-1, -1, -1};
};

// relative positions of a component (cell_center_nli_intrp.hpp:349-365)
void relpos(int mesh, int comp, int rp[3])
{
    for (int a = 0; a < 3; ++a) rp[a] = 1;
    if (mesh == kFace) rp[comp] = 0;
    else if (mesh == kEdge)
    {
        for (int a = 0; a < 3; ++a) rp[a] = 0;
        rp[comp] = 1;
    }
}

// What a captured time step depends on besides the device data: the field
// ids, dt, Re, the frame velocity (a launch argument, and whether the
// frame-velocity update launches at all) and the Poisson solver's switches
// (which launches a solve makes)
struct StepKey
{
    int u[3] = {-1, -1, -1}, p = -1;
    double dt = 0.0, Re = 0.0, fv[3] = {0.0, 0.0, 0.0};
    bool corr = true, snl = false;
    bool operator==(const StepKey& o) const
    {
        return u[0] == o.u[0] && u[1] == o.u[1] && u[2] == o.u[2] && p == o.p && dt == o.dt && Re == o.Re &&
               fv[0] == o.fv[0] && fv[1] == o.fv[1] && fv[2] == o.fv[2] && corr == o.corr && snl == o.snl;
    }
};

struct NsState
{
    VF q_i, g_i, d_i, r_i, u_i, w_1, w_2, cell_aux, face_aux, edge_aux;
    VF stream_f;                     // velocity refresh only, created on first use
    DevBuf<int> leaf;                // 1 for leaves, per octant
    std::vector<DevBuf<int>> corr;   // per level: correction blocks
    std::vector<DevBuf<int>> nc;     // per level: blocks that are not correction blocks
    std::vector<DevBuf<double>> nc_dx;
    // Octant::old_correction (ifherk.hpp:247-258): base-level correction flags
    // from before the last adaptation, in force for the step that follows it
    std::vector<char> old_corr;
    // smooth2zero lists of the base level for leaf_only_boundary false / true
    DevBuf<int> sm_list[2], sm_ptr[2], sm_dirs[2];
    int sm_n[2] = {0, 0};
    double T_last_vel_refresh = 0.0;  // ifherk.hpp:1980
    bool force_refresh = false;       // base_mesh_update of the last adaptation
    // one captured time step (steps without an immersed boundary): replayed
    // while everything the capture baked in stays the same (g_key)
    cudaGraphExec_t graph = nullptr;
    StepKey g_key;
    bool graph_failed = false;
    int steps_done = 0;
    long long graph_launches = 0;
    // the key of the last step run with direct launches: a capture needs one
    // such step first, so that every plan, table and buffer the step uses
    // exists before capturing
    StepKey w_key;
};

long long st_launches(const NsState& s) { return s.graph_launches; }
// per context: constant frame velocity and IB CG settings (set any time)
struct NsOptions
{
    double frame_vel[3] = {0.0, 0.0, 0.0};
    double cg_threshold = 1e-3;
    int cg_max_iter = 40;
};
// an adaptation before the context's first time step: its old-correction
// flags and base-mesh update wait for the time step's state
struct NsPending
{
    std::vector<char> old_corr;
    bool base_mesh_update = false;
};

NsOptions& ns_opt(Ctx& c)
{
    if (!c.ext[Ctx::kExtNsOpt]) c.ext[Ctx::kExtNsOpt] = std::make_shared<NsOptions>();
    return *c.ext_get<NsOptions>(Ctx::kExtNsOpt);
}

VF make_vf(Ctx& c, int mesh)
{
    VF f;
    f.mesh = mesh;
    f.n = mesh == kCell ? 1 : 3;
    for (int k = 0; k < f.n; ++k) f.id[k] = field_create(c);
    return f;
}

void ns_build_lists(Ctx& c, NsState& st);

// the loop's next iteration copies the correction flags into the old ones
// (ifherk.hpp:247-258): without an adaptation in between they add nothing
void drop_old_correction(Ctx& c, NsState& s)
{
    if (s.old_corr.empty()) return;
    s.old_corr.clear();
    ns_build_lists(c, s);
}

NsState& ns_state(Ctx& c)
{
    if (auto* have = c.ext_get<NsState>(Ctx::kExtNs)) return *have;
    auto s = std::make_unique<NsState>();
    s->q_i = make_vf(c, kFace);
    s->g_i = make_vf(c, kFace);
    s->d_i = make_vf(c, kCell);
    s->r_i = make_vf(c, kFace);
    s->u_i = make_vf(c, kFace);
    s->w_1 = make_vf(c, kFace);
    s->w_2 = make_vf(c, kFace);
    s->cell_aux = make_vf(c, kCell);
    s->face_aux = make_vf(c, kFace);
    s->edge_aux = make_vf(c, kEdge);
    if (const NsPending* pend = c.ext_get<NsPending>(Ctx::kExtNsPending))
    {
        s->old_corr = pend->old_corr;
        s->force_refresh = pend->base_mesh_update;
        c.ext[Ctx::kExtNsPending].reset();
    }
    ns_build_lists(c, *s);
    auto& ref = *s;
    c.ext[Ctx::kExtNs] = std::shared_ptr<NsState>(s.release(), [](NsState* p) {
        if (p->graph) cudaGraphExecDestroy(p->graph);
        delete p;
    });
    return ref;
}

// the step's per-tree lists: leaves, correction / other blocks per level,
// smooth2zero directions of the base level
void ns_build_lists(Ctx& c, NsState& st)
{
    NsState* s = &st;
    std::vector<int> leaf(c.n_oct);
    for (int i = 0; i < c.n_oct; ++i) leaf[i] = c.flags[i] & 1;
    s->leaf.upload(leaf, c.stream);
    s->corr.resize(c.level_octs.size());
    s->nc.resize(c.level_octs.size());
    s->nc_dx.resize(c.level_octs.size());
    auto old = [&](int o) { return o < (int)s->old_corr.size() && s->old_corr[o]; };
    for (size_t l = 0; l < c.level_octs.size(); ++l)
    {
        std::vector<int> v, w;
        for (int o : c.level_octs[l])
            (c.flags[o] & 2 ? v : w).push_back(o);
        // clean_leaf_correction_boundary zeroes correction or old-correction blocks
        std::vector<int> vz = v;
        for (int o : w)
            if (old(o)) vz.push_back(o);
        std::sort(vz.begin(), vz.end());
        s->corr[l].upload(vz, c.stream);
        s->nc[l].upload(w, c.stream);
        s->nc_dx[l].upload(std::vector<double>(w.size(), c.cfg.dx_base / std::pow(2.0, (int)l - c.tree.base_level)),
                           c.stream);
    }
    const int bl = c.tree.base_level;
    for (int lo = 0; lo < 2; ++lo)
    {
        std::vector<int> list, ptr{0}, dirs;
        for (int o : c.level_octs[bl])
        {
            const size_t d0 = dirs.size();
            for (int i = 0; i < 27; ++i)
            {
                const int q = c.nbr[27 * (size_t)o + i];
                if (q < 0 || (lo && ((c.flags[q] & 2) || old(q)))) dirs.push_back(i);
            }
            if (dirs.size() == d0) continue;
            list.push_back(o);
            ptr.push_back((int)dirs.size());
        }
        s->sm_n[lo] = (int)list.size();
        s->sm_list[lo].upload(list, c.stream);
        s->sm_ptr[lo].upload(ptr, c.stream);
        s->sm_dirs[lo].upload(dirs, c.stream);
    }
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
}

class Step
{
  public:
    Step(Ctx& c_, NsState& s_, double dt_, double Re_)
    : c(c_), s(s_), pl(poisson_lists(c_)), ol(op_lists(c_)), dt(dt_), Re(Re_), opt(ns_opt(c_))
    {
        bl = c.tree.base_level;
        depth = c.tree.depth;
        // ifherk.hpp:164-173
        const double tmp = Re * c.cfg.dx_base * c.cfg.dx_base / dt;
        for (int k = 0; k < 3; ++k) alpha[k] = (cc[k + 1] - cc[k]) / tmp;
    }

    // refresh: ifherk.hpp:1093-1111, the velocity refresh (pad_velocity and
    // adapt_corr_time_step) takes the place of up_and_down(u)
    void time_step(const VF& u, const VF& p, bool refresh)
    {
        if (refresh)
        {
            pad_velocity(u);
            adapt_corr_time_step(u, p);
        }
        else
            up_and_down(u);
        copy(u, s.q_i, 1.0);
        // stage 1
        clean(s.g_i, false);
        clean(s.d_i, false);
        clean(s.cell_aux, false);
        clean(s.face_aux, false);
        nonlinear(u, s.g_i, coeff_a(1, 1) * (-dt));
        copy(s.q_i, s.r_i, 1.0);
        add(s.g_i, s.r_i, 1.0);
        stage = 1;
        lin_sys(alpha[0]);
        // stage 2
        clean(s.r_i, false);
        clean(s.d_i, false);
        clean(s.cell_aux, false);
        add(s.g_i, s.face_aux, -1.0);
        copy(s.face_aux, s.w_1, -1.0 / dt / coeff_a(1, 1));
        apply_if(s.q_i, s.q_i, alpha[0]);
        apply_if(s.w_1, s.w_1, alpha[0]);
        add(s.q_i, s.r_i, 1.0);
        add(s.w_1, s.r_i, dt * coeff_a(2, 1));
        up_and_down(s.u_i);
        nonlinear(s.u_i, s.g_i, coeff_a(2, 2) * (-dt));
        add(s.g_i, s.r_i, 1.0);
        stage = 2;
        lin_sys(alpha[1]);
        // stage 3
        clean(s.d_i, false);
        clean(s.cell_aux, false);
        clean(s.w_2, false);
        add(s.g_i, s.face_aux, -1.0);
        copy(s.face_aux, s.w_2, -1.0 / dt / coeff_a(2, 2));
        copy(s.q_i, s.r_i, 1.0);
        add(s.w_1, s.r_i, dt * coeff_a(3, 1));
        add(s.w_2, s.r_i, dt * coeff_a(3, 2));
        apply_if(s.r_i, s.r_i, alpha[1]);
        up_and_down(s.u_i);
        nonlinear(s.u_i, s.g_i, coeff_a(3, 3) * (-dt));
        add(s.g_i, s.r_i, 1.0);
        stage = 3;
        lin_sys(alpha[2]);
        copy(s.u_i, u, 1.0);
        copy(s.d_i, p, 1.0 / coeff_a(3, 3) / dt);
    }

    // pad_velocity<u, u>(true) (ifherk.hpp:1522-1573): u rebuilt from its
    // vorticity through the stream function on the base level
    void pad_velocity(const VF& u)
    {
        if (s.stream_f.id[0] < 0) s.stream_f = make_vf(c, kEdge);
        clean(u, true);
        up(u);
        clean(s.edge_aux, false);
        clean(s.stream_f, false);
        for (int l = bl; l < depth; ++l)
        {
            exchange(u, l);
            // curl on the blocks that are not correction blocks
            const double* pin[3] = {F(u.id[0]), F(u.id[1]), F(u.id[2])};
            double* pout[3] = {F(s.edge_aux.id[0]), F(s.edge_aux.id[1]), F(s.edge_aux.id[2])};
            launch_op(c, 3, pin, 3, pout, 3, s.nc[l].p, s.nc_dx[l].p, (int)s.nc[l].n, 1.0);
        }
        clean_leaf_correction_boundary(s.edge_aux, bl, true);
        for (int k = 0; k < 3; ++k) poisson_apply_lgf(c, s.edge_aux.id[k], s.stream_f.id[k], IBLGF_STREAM);
        // refresh_correction_only: curl_transpose on the base level only
        op(4, {&s.stream_f}, u, bl, -1.0);
        down_to_correction(u);
    }
    // adapt_corr_time_step (ifherk.hpp:1206-1303): three projection stages
    // with alpha = 0 and no nonlinear term; the IB solves read but do not
    // replace the stages' previous forces
    void adapt_corr_time_step(const VF& u, const VF& p)
    {
        up_and_down(u);
        copy(u, s.q_i, 1.0);
        write_prev = false;
        // stage 1
        clean(s.g_i, false);
        clean(s.d_i, false);
        clean(s.cell_aux, false);
        clean(s.face_aux, false);
        copy(s.q_i, s.r_i, 1.0);
        stage = 1;
        lin_sys(0.0);
        // stage 2
        clean(s.r_i, false);
        clean(s.d_i, false);
        clean(s.cell_aux, false);
        add(s.q_i, s.r_i, 1.0);
        up_and_down(s.u_i);
        stage = 2;
        lin_sys(0.0);
        // stage 3
        clean(s.d_i, false);
        clean(s.cell_aux, false);
        clean(s.w_2, false);
        copy(s.q_i, s.r_i, 1.0);
        apply_if(s.r_i, s.r_i, 0.0);
        up_and_down(s.u_i);
        stage = 3;
        lin_sys(0.0);
        write_prev = true;
        copy(s.u_i, u, 1.0);
        copy(s.d_i, p, 0.0);
    }

  private:
    Ctx& c;
    NsState& s;
    PoissonLists& pl;
    OpLists& ol;
    double dt, Re;
    NsOptions opt;
    int bl = 0, depth = 0, stage = 0;
    bool write_prev = true;
    // ifherk.hpp:2010-2011
    const double a[6] = {1.0 / 3, -1.0, 2.0, 0.0, 0.75, 0.25};
    const double cc[4] = {0.0, 1.0 / 3, 1.0, 1.0};
    double alpha[3] = {0.0, 0.0, 0.0};

    double coeff_a(int i, int j) const { return a[i * (i - 1) / 2 + j - 1]; }
    double* F(int id) { return c.field(id); }

    // the components of a vector field in one launch each
    void clean(const VF& f, bool non_leaf_only)
    {
        double* p[3] = {F(f.id[0]), f.n > 1 ? F(f.id[1]) : nullptr, f.n > 2 ? F(f.id[2]) : nullptr};
        launch_clean_vf(c, p, f.n, s.leaf.p, non_leaf_only);
    }
    void copy(const VF& from, const VF& to, double a_)
    {
        double* t[3];
        const double* fr[3];
        for (int k = 0; k < from.n; ++k) t[k] = F(to.id[k]), fr[k] = F(from.id[k]);
        launch_axpby_vf(c, t, fr, from.n, a_, 0);
    }
    void add(const VF& from, const VF& to, double a_)
    {
        double* t[3];
        const double* fr[3];
        for (int k = 0; k < from.n; ++k) t[k] = F(to.id[k]), fr[k] = F(from.id[k]);
        launch_axpby_vf(c, t, fr, from.n, a_, 1);
    }
    void scale(const VF& f, double a_)
    {
        double* t[3];
        for (int k = 0; k < f.n; ++k) t[k] = F(f.id[k]);
        launch_axpby_vf(c, t, nullptr, f.n, a_, 2);
    }
    void exchange(const VF& f, int l)
    {
        for (int k = 0; k < f.n; ++k) launch_halo(c, F(f.id[k]), ol.list[l].p, (int)ol.list[l].n);
    }
    // source_coarsify (poisson.hpp:1136-1194) into the field itself
    void up(const VF& f)
    {
        for (int k = 0; k < f.n; ++k)
        {
            int rp[3], m[3];
            relpos(f.mesh, k, rp);
            for (int a_ = 0; a_ < 3; ++a_) m[a_] = rp[a_] ? 4 : 8;
            for (int ls = depth - 2; ls >= bl; --ls) launch_tp_axes(c, pl.coarsify[ls], F(f.id[k]), F(f.id[k]), m, 0);
        }
    }
    // intrp_to_correction_buffer (poisson.hpp:1015-1069), correction children only
    void down_to_correction(const VF& f)
    {
        for (int k = 0; k < f.n; ++k)
        {
            int rp[3], m[3];
            relpos(f.mesh, k, rp);
            for (int a_ = 0; a_ < 3; ++a_) m[a_] = rp[a_] ? 2 : 6;
            for (int l = depth - 2; l >= bl; --l)
            {
                launch_halo(c, F(f.id[k]), ol.list[l].p, (int)ol.list[l].n);
                launch_tp_axes(c, pl.corr_intrp[l], F(f.id[k]), F(f.id[k]), m, 2);
            }
        }
    }
    void up_and_down(const VF& f)
    {
        clean(f, true);
        up(f);
        down_to_correction(f);
    }
    void op(int o, std::initializer_list<const VF*> in, const VF& out, int l, double sc)
    {
        const double* pin[6] = {};
        double* pout[3] = {};
        int n_in = 0;
        for (const VF* v : in)
            for (int k = 0; k < v->n; ++k) pin[n_in++] = F(v->id[k]);
        for (int k = 0; k < out.n; ++k) pout[k] = F(out.id[k]);
        launch_op(c, o, pin, n_in, pout, out.n, ol.list[l].p, ol.dx[l].p, (int)ol.list[l].n, sc);
    }
    void clean_leaf_correction_boundary(const VF& f, int l, bool leaf_only_boundary)
    {
        if (leaf_only_boundary)
            for (int k = 0; k < f.n; ++k) launch_zero_blocks(c, F(f.id[k]), s.corr[l].p, (int)s.corr[l].n);
        if (l != bl) return;
        const int v = leaf_only_boundary ? 1 : 0;
        // smooth2zero scales every component; the reference calls it once per component
        for (int k = 0; k < f.n; ++k)
            launch_smooth(c, F(f.id[k]), s.sm_list[v].p, s.sm_ptr[v].p, s.sm_dirs[v].p, s.sm_n[v], f.n);
    }
    void nonlinear(const VF& src, const VF& tgt, double sc)
    {
        clean(s.edge_aux, false);
        clean(tgt, false);
        clean(s.face_aux, false);
        for (int l = bl; l < depth; ++l)
        {
            exchange(src, l);
            op(3, {&src}, s.edge_aux, l, 1.0);
        }
        copy(src, s.face_aux, 1.0);
        // add_field_expression(frame_vel, -1): a constant frame velocity
        for (int k = 0; k < 3; ++k)
            if (opt.frame_vel[k] != 0.0) launch_axpby(c, F(s.face_aux.id[k]), nullptr, -opt.frame_vel[k], 3);
        for (int l = bl; l < depth; ++l)
        {
            exchange(s.edge_aux, l);
            clean_leaf_correction_boundary(s.edge_aux, l, false);
            op(5, {&s.face_aux, &s.edge_aux}, tgt, l, 1.0);
        }
        scale(tgt, sc);
    }
    void divergence(const VF& src, const VF& tgt)
    {
        up_and_down(src);
        for (int l = bl; l < depth; ++l)
        {
            exchange(src, l);
            op(2, {&src}, tgt, l, 1.0);
            clean_leaf_correction_boundary(tgt, l, true);
        }
    }
    void gradient(const VF& src, const VF& tgt)
    {
        clean(tgt, false);
        for (int l = bl; l < depth; ++l)
        {
            op(1, {&src}, tgt, l, 1.0);
            exchange(tgt, l);
        }
    }
    void apply_if(const VF& src, const VF& tgt, double alpha_base)
    {
        for (int k = 0; k < src.n; ++k)
        {
            int rp[3];
            relpos(src.mesh, k, rp);
            iblgf_b200::apply_if(c, src.id[k], tgt.id[k], alpha_base, IBLGF_AMR2AMR, rp);
        }
    }
    void lin_sys(double alpha_k)
    {
        divergence(s.r_i, s.cell_aux);
        poisson_apply_lgf(c, s.cell_aux.id[0], s.d_i.id[0], IBLGF_AMR2AMR);
        if (ib_active(c))
        {
            // lin_sys_with_ib_solve (ifherk.hpp:1451-1517)
            VF fa2;
            fa2.mesh = kFace;
            fa2.n = 3;
            for (int k = 0; k < 3; ++k) fa2.id[k] = ib_face_aux2(c)[k];
            copy(s.r_i, fa2, 1.0);
            gradient(s.d_i, s.face_aux);
            add(s.face_aux, fa2, -1.0);
            if (std::fabs(alpha_k) > 1e-14)
                for (int k = 0; k < 3; ++k)
                {
                    int rp[3];
                    relpos(kFace, k, rp);
                    iblgf_b200::apply_if(c, fa2.id[k], fa2.id[k], alpha_k, IBLGF_IB2xIB, rp);
                }
            ns_ib_stage(c, stage, alpha_k, opt.cg_threshold, opt.cg_max_iter, s.d_i.id[0], s.face_aux.id,
                        [&]() { gradient(s.d_i, s.face_aux); }, write_prev);
            add(s.face_aux, s.r_i, -1.0);
            if (std::fabs(alpha_k) > 1e-14) apply_if(s.r_i, s.u_i, alpha_k);
            else copy(s.r_i, s.u_i, 1.0);
            return;
        }
        gradient(s.d_i, s.face_aux);
        add(s.face_aux, s.r_i, -1.0);
        if (std::fabs(alpha_k) > 1e-14) apply_if(s.r_i, s.u_i, alpha_k);
        else copy(s.r_i, s.u_i, 1.0);
    }
};
}  // namespace

void ns_step(Ctx& c, const int* u, int p, double dt, double Re, double* T, int n_steps)
{
    need_single(c);
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    if (!(dt > 0.0) || !(Re > 0.0)) throw Error(IBLGF_EINVAL, "dt and Re must be positive");
    const int nf = (int)c.fields.size();
    for (int k = 0; k < 3; ++k)
        if (u[k] < 0 || u[k] >= nf) throw Error(IBLGF_EINVAL, "bad velocity field id");
    if (p < 0 || p >= nf) throw Error(IBLGF_EINVAL, "bad pressure field id");
    NsState& s = ns_state(c);
    VF uf, pf;
    uf.mesh = kFace;
    uf.n = 3;
    for (int k = 0; k < 3; ++k) uf.id[k] = u[k];
    pf.id[0] = p;
    Step st(c, s, dt, Re);
    const double dx = c.cfg.dx_base;
    for (int i = 0; i < n_steps; ++i)
    {
        if (s.force_refresh || (*T - s.T_last_vel_refresh) / (Re * dx * dx) * 3.3 > 7)
        {
            s.force_refresh = false;
            // velocity refresh step (ifherk.hpp:1093-1104): direct launches
            s.T_last_vel_refresh = *T;
            st.time_step(uf, pf, true);
            ++s.steps_done;
            *T += dt;
            drop_old_correction(c, s);
            continue;
        }
        // steps with the immersed boundary are captured too: their force CG
        // is a conditional while-node of the graph (not with the learned
        // warm start, which assembles its inputs on the host)
        // (a sharded context's sweeps call its host-side exchange: direct launches)
        const bool graphable =
            (!ib_active(c) || ib_graphable(c)) && !c.profile && !s.graph_failed && c.owner.empty();
        StepKey key;
        for (int k = 0; k < 3; ++k) key.u[k] = u[k];
        key.p = p;
        key.dt = dt;
        key.Re = Re;
        const NsOptions& opt = ns_opt(c);
        for (int k = 0; k < 3; ++k) key.fv[k] = opt.frame_vel[k];
        key.corr = c.use_correction;
        key.snl = c.subtract_non_leaf;
        const bool same = s.graph && s.g_key == key;
        if (graphable && same)
        {
            IBLGF_CUDA(cudaGraphLaunch(s.graph, c.stream));
            c.launches += st_launches(s);
        }
        else if (graphable && s.w_key == key)
        {
            // capture after a first direct step has built every plan and sized
            // every buffer, so the step makes no host synchronisation
            if (s.graph)
            {
                cudaGraphExecDestroy(s.graph);
                s.graph = nullptr;
            }
            const long long l0 = c.launches;
            cudaGraph_t g = nullptr;
            IBLGF_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeRelaxed));
            bool ok = true;
            try
            {
                st.time_step(uf, pf, false);
            }
            catch (const Error&)
            {
                ok = false;
            }
            const cudaError_t e = cudaStreamEndCapture(c.stream, &g);
            if (!ok || e != cudaSuccess || !g || cudaGraphInstantiate(&s.graph, g, 0) != cudaSuccess)
            {
                cudaGetLastError();
                if (g) cudaGraphDestroy(g);
                s.graph = nullptr;
                s.graph_failed = true;
                c.launches = l0;
                st.time_step(uf, pf, false);  // nothing of the failed capture ran
            }
            else
            {
                cudaGraphDestroy(g);
                s.graph_launches = c.launches - l0;
                s.g_key = key;
                IBLGF_CUDA(cudaGraphLaunch(s.graph, c.stream));
            }
        }
        else
        {
            st.time_step(uf, pf, false);
            s.w_key = key;
        }
        ++s.steps_done;
        *T += dt;
        drop_old_correction(c, s);
    }
    IBLGF_CUDA(cudaGetLastError());
}

void ns_fields(Ctx& c, int* ids)
{
    need_single(c);
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    NsState& s = ns_state(c);
    ids[0] = s.cell_aux.id[0];
    for (int k = 0; k < 3; ++k) ids[1 + k] = s.edge_aux.id[k];
    ids[4] = c.f_correction_tmp;
}

void ns_clean(Ctx& c, int field, bool non_leaf_only, int width)
{
    need_single(c);
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    if (field < 0 || field >= (int)c.fields.size() || width < 1 || width > c.Nb / 2)
        throw Error(IBLGF_EINVAL, "bad clean arguments");
    NsState& s = ns_state(c);
    launch_clean(c, c.field(field), s.leaf.p, non_leaf_only, width);
}

void ns_clean_leaf_correction_boundary(Ctx& c, const int* fields, int n, int level, bool leaf_only_boundary)
{
    need_single(c);
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    if (n < 1 || n > 3 || level < 0 || level > kMaxLevel) throw Error(IBLGF_EINVAL, "bad arguments");
    for (int k = 0; k < n; ++k)
        if (fields[k] < 0 || fields[k] >= (int)c.fields.size()) throw Error(IBLGF_EINVAL, "bad field id");
    NsState& s = ns_state(c);
    if (leaf_only_boundary && level < (int)s.corr.size())
        for (int k = 0; k < n; ++k) launch_zero_blocks(c, c.field(fields[k]), s.corr[level].p, (int)s.corr[level].n);
    if (level != c.tree.base_level) return;
    const int v = leaf_only_boundary ? 1 : 0;
    for (int k = 0; k < n; ++k)
        launch_smooth(c, c.field(fields[k]), s.sm_list[v].p, s.sm_ptr[v].p, s.sm_dirs[v].p, s.sm_n[v], n);
}

void ns_options(Ctx& c, const double* frame_vel, double cg_threshold, int cg_max_iter)
{
    if (!(cg_threshold > 0) || cg_max_iter < 0) throw Error(IBLGF_EINVAL, "bad CG settings");
    NsOptions& o = ns_opt(c);
    for (int k = 0; k < 3; ++k) o.frame_vel[k] = frame_vel ? frame_vel[k] : 0.0;
    o.cg_threshold = cg_threshold;
    o.cg_max_iter = cg_max_iter;
}

void ns_on_adapt(Ctx& c, bool base_mesh_update, const std::vector<char>& old_corr)
{
    NsState* sp = c.ext_get<NsState>(Ctx::kExtNs);
    if (!sp)
    {
        if (!c.ext[Ctx::kExtNsPending]) c.ext[Ctx::kExtNsPending] = std::make_shared<NsPending>();
        NsPending& pend = *c.ext_get<NsPending>(Ctx::kExtNsPending);
        pend.old_corr = old_corr;
        pend.base_mesh_update = pend.base_mesh_update || base_mesh_update;
        return;
    }
    NsState& s = *sp;
    s.old_corr = old_corr;
    if (s.graph) cudaGraphExecDestroy(s.graph);
    s.graph = nullptr;
    s.graph_failed = false;
    s.g_key = s.w_key = StepKey{};
    ns_build_lists(c, s);
    // ifherk.hpp:1093-1096: a grown base mesh refreshes the velocity
    s.force_refresh = s.force_refresh || base_mesh_update;
}

void ns_release(Ctx& c)
{
    c.ext[Ctx::kExtNs].reset();
    c.ext[Ctx::kExtNsOpt].reset();
    c.ext[Ctx::kExtNsPending].reset();
}

}  // namespace iblgf_b200
